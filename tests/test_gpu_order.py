"""Design order of accuracy of the CUDA path on the 2-D isentropic vortex
(Euler, quads, Gauss points, c_dg correction, Rusanov, RK45).

The vortex (strength 5, free stream rho=1, u=1, v=0, p=1) is advected for
t = 1 on periodic [-10, 10]^2 meshes of n^2 elements; the domain is wide
enough that the vortex's tail at the boundary (~e^-49) does not limit the
error.  The exact solution is the initial field shifted by (t, 0).  The L2
density error, integrated with the tensor Gauss weights and the Jacobian,
falls between the DG rates P + 1/2 (proven) and P + 1 (design): measured on
the two finest meshes, 2.3 for P=1, 2.5 for P=2 and 4.5 for P=3 -- the CPU
oracle, which repeats the reference's arithmetic, gives the same errors to
four digits, so these are the scheme's rates.  The check is slope > P + 0.4
on the two finest meshes."""
import numpy as np
import pytest

import hifiles_b200 as H
import oracle as O

pytestmark = pytest.mark.gpu

T_END, DT = 1.0, 1e-3
MESHES = {1: (16, 32, 64), 2: (16, 32, 64), 3: (16, 32, 64)}


def _l2_density_error(P, n):
    s = H.Solver.box(2, P, (n, n), (-10.0, -10.0), (10.0, 10.0), viscous=False, vcjh_scheme=1, gamma=1.4)
    g = s.geometry()
    pos = g["pos_upts"]
    s.set_state(np.asfortranarray(O.ic_vortex(pos)))
    s.advance(int(round(T_END / DT)), DT)
    u = s.get_state()
    exact = O.ic_vortex(pos, t=T_END)
    w1 = np.polynomial.legendre.leggauss(P + 1)[1]
    w = np.outer(w1, w1).T.ravel()              # point u = a + (P+1) b  ->  w[a] w[b]
    err2 = (w[:, None] * g["detjac_upts"] * (u[:, :, 0] - exact[..., 0]) ** 2).sum()
    return float(np.sqrt(err2))


@pytest.mark.parametrize("P", [1, 2, 3])
def test_vortex_converges_at_design_order(P):
    ns = MESHES[P]
    errs = [_l2_density_error(P, n) for n in ns]
    slopes = [np.log(errs[i] / errs[i + 1]) / np.log(ns[i + 1] / ns[i]) for i in range(len(ns) - 1)]
    print("P=%d errors %s slopes %s" % (P, ["%.3e" % e for e in errs], ["%.2f" % s for s in slopes]))
    assert all(np.isfinite(errs))
    assert slopes[-1] > P + 0.4, (errs, slopes)
