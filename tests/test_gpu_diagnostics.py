"""Integral diagnostics on the device (fr_solver_integral_quantities): the
quantities of eles::CalcIntegralQuantities (src/eles.cpp:6503-6641) from the
state and its corrected gradient, against the same formulas evaluated in
numpy on the solver's own gradient, at 1e-12 relative."""
import numpy as np
import pytest

import hifiles_b200 as H
import oracle as O

pytestmark = pytest.mark.gpu


def _numpy_quantities(u, g, detj, w1, dims, gamma):
    F = dims + 2
    q = u.reshape(-1, F, order="F")
    gg = g.reshape(-1, F, dims, order="F")
    nu = len(w1) ** dims
    W = np.ones(nu)
    for d in range(dims):
        W = W * np.asarray(w1)[(np.arange(nu) // len(w1) ** d) % len(w1)]
    wj = np.tile(W, q.shape[0] // nu) * detj.reshape(-1, order="F")
    irho = 1.0 / q[:, 0]
    A = irho[:, None, None] * (gg[:, 1:1 + dims, :] - q[:, 1:1 + dims, None] * irho[:, None, None] * gg[:, 0:1, :])
    tke = 0.5 * (q[:, 1:1 + dims] ** 2).sum(axis=1)
    ke = irho * tke
    wz = A[:, 1, 0] - A[:, 0, 1]
    en = wz * wz
    if dims == 3:
        en = en + (A[:, 2, 1] - A[:, 1, 2]) ** 2 + (A[:, 0, 2] - A[:, 2, 0]) ** 2
    en = en * 0.5 / irho
    p = (gamma - 1.0) * (q[:, -1] - irho * tke)
    pd = p * np.trace(A, axis1=1, axis2=2)
    S = 0.5 * (A + A.transpose(0, 2, 1))
    sc = (S * S).sum(axis=(1, 2))
    Sd = S - np.eye(dims)[None] * (np.trace(S, axis1=1, axis2=2) / 3.0)[:, None, None]
    dsc = (Sd * Sd).sum(axis=(1, 2))
    return [float((x * wj).sum()) for x in (ke, en, pd, sc, dsc)]


@pytest.mark.parametrize("dims,P,n,jit", [(3, 3, (4, 3, 3), 0.1), (3, 2, (3, 3, 3), 0.0), (2, 4, (4, 5), 0.1)])
def test_integral_quantities_match_numpy(dims, P, n, jit):
    lo, hi = [0.0] * dims, [2 * np.pi] * dims
    s = H.Solver.box(dims, P, n, lo, hi, jitter=jit, seed=3, viscous=True, gamma=1.4, prandtl=0.71,
                     mu_inf=1e-3, tau=1.0, pen_fact=0.5)
    g = s.geometry()
    pos = g["pos_upts"]
    u = O.ic_tgv(pos) if dims == 3 else O.ic_vortex(pos * (10 / (2 * np.pi)) - 5)
    u = np.asfortranarray(u + 0.02 * np.random.default_rng(2).standard_normal(u.shape) * (np.arange(u.shape[2]) > 0))
    s.set_state(u)
    iq = s.integral_quantities()
    want = _numpy_quantities(u, s.gradient(), g["detjac_upts"], np.polynomial.legendre.leggauss(P + 1)[1], dims, 1.4)
    for (k, v), w in zip(iq.items(), want):
        assert abs(v - w) <= 1e-12 * max(abs(w), 1e-30) + 1e-14, (k, v, w)
    assert abs(iq["kineticenergy"] - s.kinetic_energy()) <= 1e-13 * abs(iq["kineticenergy"])


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
