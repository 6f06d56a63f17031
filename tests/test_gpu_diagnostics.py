"""Integral diagnostics on the device (fr_solver_integral_quantities,
fr_solver_kinetic_energy): the quantities of eles::CalcIntegralQuantities
(src/eles.cpp:6503-6641) on the reference's volume cubature, against the
values the reference itself computed on the same mesh and state
(tests/golden/iq_*.npz), and against the numpy restatement on the solver's
own gradient.  Tolerance 1e-12 relative to the integral of each quantity's
absolute value (the pressure dilatation is a cancelling sum)."""
import numpy as np
import pytest

import hifiles_b200 as H
import oracle as O
from golden_util import IQ_CASES, integral_quantities_numpy, load

pytestmark = pytest.mark.gpu

NAMES = ("kineticenergy", "vorticity", "pressuredilatation", "straincolonproduct", "devstraincolonproduct")


def _solver(meta):
    ph = meta["physics"]
    return H.Solver.box(meta["dims"], meta["order"], meta["n"], meta["lo"], meta["hi"], jitter=meta["jitter"],
                        seed=meta["seed"], viscous=True, vcjh_scheme=meta["vcjh"], **ph)


@pytest.mark.parametrize("case", IQ_CASES)
def test_integral_quantities_match_reference(case):
    meta, a = load(case)
    s = _solver(meta)
    s.set_volume_cubature(a["loc"], a["weight"])
    s.set_state(a["u0"])
    iq = s.integral_quantities()
    _, mags = integral_quantities_numpy(a["u0"], a["grad"], a["opp"], a["weight"], a["detjac"], meta["dims"],
                                        meta["physics"]["gamma"])
    for k, want, m in zip(NAMES, a["iq"], mags):
        assert abs(iq[k] - want) <= 1e-12 * m, (k, iq[k], want)
    assert abs(s.kinetic_energy() - a["iq"][0]) <= 1e-12 * abs(a["iq"][0])


@pytest.mark.parametrize("dims,P,n,jit,rule", [(3, 3, (4, 3, 3), 0.1, 3), (3, 2, (3, 3, 3), 0.0, 4),
                                               (2, 4, (4, 5), 0.1, 6)])
def test_integral_quantities_match_numpy(dims, P, n, jit, rule):
    lo, hi = [0.0] * dims, [2 * np.pi] * dims
    s = H.Solver.box(dims, P, n, lo, hi, jitter=jit, seed=3, viscous=True, gamma=1.4, prandtl=0.71,
                     mu_inf=1e-3, tau=1.0, pen_fact=0.5)
    pos = s.geometry()["pos_upts"]
    u = O.ic_tgv(pos) if dims == 3 else O.ic_vortex(pos * (10 / (2 * np.pi)) - 5)
    u = np.asfortranarray(u + 0.02 * np.random.default_rng(2).standard_normal(u.shape) * (np.arange(u.shape[2]) > 0))
    s.set_state(u)
    loc, w = H.volume_cubature(dims, rule)
    if rule != 3:
        s.set_volume_cubature(loc, w)
    iq = s.integral_quantities()
    # the interpolation rows and Jacobians at the cubature points, restated
    x1 = H.line_operators(P)["loc"]
    nl = len(x1)

    def lag(x, m):
        return np.prod([(x - x1[i]) / (x1[m] - x1[i]) for i in range(nl) if i != m], axis=0)
    nu = nl ** dims
    opp = np.ones((w.size, nu))
    for k in range(nu):
        for d in range(dims):
            opp[:, k] *= lag(loc[d], (k // nl ** d) % nl)
    vals, mags = integral_quantities_numpy(u, s.gradient(), opp, w, _detj_cub(s, loc), dims, 1.4)
    for k, v, m in zip(NAMES, vals, mags):
        assert abs(iq[k] - v) <= 1e-12 * m, (k, iq[k], v)
    assert abs(iq["kineticenergy"] - s.kinetic_energy()) <= 1e-13 * abs(iq["kineticenergy"])


def _detj_cub(s, loc):
    """Jacobian determinant of each element's bi/tri-linear map at the cubature points."""
    D = s.dims
    g = s.geometry()
    # corner positions from the solution-point positions: the map is (bi/tri)linear,
    # so fit it exactly from the element's points
    pos = g["pos_upts"]                                   # (nu, E, D)
    x1 = H.line_operators(s.order)["loc"]
    nl = len(x1)
    nu = nl ** D
    R = np.array([[x1[(k // nl ** d) % nl] for d in range(D)] for k in range(nu)])
    cols = [np.ones(nu)] + [R[:, d] for d in range(D)]
    if D == 2:
        cols += [R[:, 0] * R[:, 1]]
    else:
        cols += [R[:, 0] * R[:, 1], R[:, 0] * R[:, 2], R[:, 1] * R[:, 2], R[:, 0] * R[:, 1] * R[:, 2]]
    M = np.stack(cols, axis=1)
    coef = np.linalg.lstsq(M, pos.reshape(nu, -1), rcond=None)[0].reshape(M.shape[1], pos.shape[1], D)
    out = np.zeros((loc.shape[1], pos.shape[1]))
    for j in range(loc.shape[1]):
        r = loc[:, j]
        if D == 2:
            dM = np.array([[0, 1, 0, r[1]], [0, 0, 1, r[0]]])
        else:
            dM = np.array([[0, 1, 0, 0, r[1], r[2], 0, r[1] * r[2]],
                           [0, 0, 1, 0, r[0], 0, r[2], r[0] * r[2]],
                           [0, 0, 0, 1, 0, r[0], r[1], r[0] * r[1]]])
        J = np.einsum("ck,kei->eic", dM, coef)            # J[e, i, c] = d x_i / d r_c
        out[j] = np.linalg.det(J)
    return out


def test_integral_quantities_need_the_viscous_path():
    s = H.Solver.box(2, 3, (3, 3), (-5, -5), (5, 5), viscous=False)
    with pytest.raises(H.FrError):
        s.integral_quantities()


def test_solver_vtu_matches_host_writer(tmp_path):
    s = H.Solver.box(3, 2, (2, 2, 3), (0, 0, 0), (2 * np.pi,) * 3, viscous=True, gamma=1.4, mu_inf=1e-3)
    pos = s.geometry()["pos_upts"]
    s.set_state(np.asfortranarray(O.ic_tgv(pos)))
    s.advance(2, 1e-3)
    s.write_vtu(tmp_path / "a.vtu")
    H.vtu_write(tmp_path / "b.vtu", 3, 2, pos, s.get_state())
    assert (tmp_path / "a.vtu").read_bytes() == (tmp_path / "b.vtu").read_bytes()
