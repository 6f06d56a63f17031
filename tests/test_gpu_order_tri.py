"""Order of accuracy of the fused mixed-mesh stage on triangles: the 2-D
isentropic vortex (Euler, Rusanov, DG correction, RK45, dt 1e-3, t = 1) on
periodic meshes of [-5, 5]^2, each of n x n squares split along its
(0,0)-(1,1) diagonal into two triangles, n = 10, 20, 40, 80, P = 1, 2, 3;
operators, metrics and wiring from the library's own set-up
(hifiles_b200.mixed), the stage from fr_mixed_stage_* (FusedMixedMesh).

The error is the density at the solution points against the exact solution
(the initial field shifted by (t, 0)), in the discrete L2 norm weighted by
each element's area.  Measured rates (n = 10 -> 20 -> 40 -> 80): 2.20, 2.36,
2.12 (P = 1); 2.72, 2.62, 2.72 (P = 2); 3.90, 4.37, 4.31 (P = 3): the
quadrilateral path's pattern (design order at P = 1 and 3, about P + 0.6 at
P = 2, as the reference gives on quads)."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

T_END, DT = 1.0, 1e-3
NS = (10, 20, 40, 80)
EULER = {"gamma": 1.4, "prandtl": 0.72, "mu_inf": 0.0, "rt_inf": 1.0, "c_sth": 1.0, "fix_vis": 1.0, "tau": 0.0,
         "pen_fact": 0.5}


def tri_box(n, lo=-5.0, hi=5.0):
    """Vertices and counter-clockwise triangles of a periodic n x n box."""
    g = np.linspace(lo, hi, n + 1)
    X, Y = np.meshgrid(g, g, indexing="xy")
    xv = np.stack([X.ravel(), Y.ravel()], axis=1)
    c = lambda i, j: i + (n + 1) * j  # noqa: E731
    cells = []
    for j in range(n):
        for i in range(n):
            cells.append([c(i, j), c(i + 1, j), c(i + 1, j + 1)])
            cells.append([c(i, j), c(i + 1, j + 1), c(i, j + 1)])
    return xv, cells


def _run(P, n):
    from hifiles_b200 import mixed as X
    from hifiles_b200 import seam
    xv, tris = tri_box(n)
    M = X.MixedMesh(P, xv, [(X.TRI, t) for t in tris], [10.0, 10.0], [],
                    X.ElementOpts(upts_type_tri=0, vcjh_scheme_tri=1))
    ty = M.types[X.TRI]
    pos = ty["pos_upts"]
    types, ints, bdys = M.operator_inputs({X.TRI: np.asfortranarray(O.ic_vortex(pos))})
    m = seam.FusedMixedMesh(types, ints, EULER, bdys, viscous=False)
    m.advance(int(round(T_END / DT)), DT)
    u = m.get_state(X.TRI)
    exact = O.ic_vortex(pos, t=T_END)
    w = np.asarray(ty["detjac_upts"])
    err = np.sqrt(np.sum(w * (u[..., 0] - exact[..., 0]) ** 2) / np.sum(w))
    return err


@pytest.mark.parametrize("P", [1, 2, 3])
def test_vortex_convergence_rate_on_triangles(P):
    errs = [_run(P, n) for n in NS]
    rates = [np.log(errs[i] / errs[i + 1]) / np.log(NS[i + 1] / NS[i]) for i in range(len(NS) - 1)]
    print("triangles P=%d errors %s rates %s" % (P, ["%.3e" % e for e in errs], ["%.2f" % r for r in rates]))
    assert all(np.isfinite(errs))
    assert rates[-1] > P + 0.4, (errs, rates)
