"""Parity of the CUDA path (fused sm_100a kernels through the C ABI) with the
reference: against the golden fixtures made by running the reference itself,
against the reference's regression known-answer values, and against the CPU
oracle on states the fixtures do not cover.

Tolerance: normwise relative error ||x - x_ref||_2 / ||x_ref||_2 <= 1e-12 for
one residual evaluation in FP64.  The inviscid fluxes, their extrapolation,
divergence and correction round as the reference does; the viscous terms
(damped by 1/Re) contract products into FMAs, so the path is close to, but
not, bit-identical."""
import json
import os

import numpy as np
import pytest

import hifiles_b200 as H
import oracle as O
from golden_util import BC_CASES, CASES, GOLDEN, load, rel

pytestmark = pytest.mark.gpu

TOL_RES = 1e-12


def _solver(meta, precision=0):
    ph = meta["physics"]
    return H.Solver.box(meta["dims"], meta["order"], meta["n"], meta["lo"], meta["hi"], jitter=meta["jitter"],
                        seed=meta["seed"], viscous=bool(meta["viscous"]), vcjh_scheme=meta["vcjh"],
                        precision=precision, side_bc=meta.get("side_bc"), **ph)


@pytest.mark.parametrize("case", CASES + BC_CASES)
def test_residual_matches_reference(case):
    meta, a = load(case)
    s = _solver(meta)
    s.set_state(a["u0"])
    div = s.residual()
    assert rel(div, a["div0"]) <= TOL_RES


@pytest.mark.parametrize("case", CASES + BC_CASES)
def test_rk45_steps_match_reference(case):
    meta, a = load(case)
    s = _solver(meta)
    s.set_state(a["u0"])
    nrm = s.advance(meta["steps"], meta["dt"], norms=True)
    u = s.get_state()
    tol = 1e-11 if meta["steps"] > 100 else 1e-12
    assert rel(u, a["uN"]) <= tol
    assert np.all(np.abs(nrm - a["norms"][:, -1]) <= 1e-10 * np.abs(a["norms"][:, -1]) + 1e-14)


def test_stage_loop_equals_graph_replay():
    meta, a = load("hex_tgv_p3_n3")
    s1, s2 = _solver(meta), _solver(meta)
    s1.set_state(a["u0"])
    s2.set_state(a["u0"])
    s1.advance(3, 1e-3)
    for _ in range(3):
        for k in range(5):
            s2.rk_stage(k, 1e-3)
    assert np.array_equal(s1.get_state(), s2.get_state())


def test_reference_regression_kat_tgv():
    """testcases/regression_tests.py:300-310: TGV 15^3 hex P=3 SD, iter 25 L1 residuals, abs tol 1e-5."""
    kat = json.load(open(os.path.join(GOLDEN, "kat_tgv.json")))
    ph = O.tgv_kat_physics()
    s = H.Solver.box(3, 3, (15, 15, 15), (0, 0, 0), (2 * np.pi,) * 3, viscous=True, vcjh_scheme=2,
                     gamma=ph.gamma, prandtl=ph.prandtl, mu_inf=ph.mu_inf, rt_inf=ph.rt_inf, c_sth=ph.c_sth,
                     fix_vis=ph.fix_vis, tau=ph.tau, pen_fact=ph.pen_fact)
    s.set_state(O.ic_tgv(s.geometry()["pos_upts"], p0=100.0))
    nrm = s.advance(kat["test_iter"], 1e-3, norms=True)
    assert np.all(np.abs(nrm - np.array(kat["test_vals"])) < kat["tol"])
    assert np.all(np.abs(nrm - np.array(kat["oracle_vals"])) <= 1e-10 * np.abs(kat["oracle_vals"]))


def _perturbed(u, seed, amp=0.02):
    r = np.random.default_rng(seed).standard_normal(u.shape)
    v = np.array(u, copy=True, order="F")
    v[:, :, 1:-1] += amp * r[:, :, 1:-1]
    v[:, :, 0] *= 1.0 + 0.1 * amp * r[:, :, 0]
    return v


@pytest.mark.parametrize("dims,P,n,visc,scheme,jit", [
    (2, 1, (5, 4), 0, 1, 0.1), (2, 2, (3, 5), 1, 2, 0.2), (2, 4, (3, 3), 0, 3, 0.1), (2, 5, (2, 3), 1, 1, 0.0),
    (3, 1, (3, 4, 2), 1, 1, 0.1), (3, 2, (2, 3, 2), 1, 4, 0.15), (3, 3, (3, 2, 3), 1, 2, 0.1),
    (3, 4, (2, 2, 3), 1, 1, 0.1), (3, 3, (1, 1, 1), 1, 1, 0.0), (3, 3, (4, 3, 2), 0, 1, 0.12)])
def test_residual_matches_oracle_on_perturbed_states(dims, P, n, visc, scheme, jit):
    lo, hi = [0.0] * dims, [2 * np.pi] * dims
    kw = dict(viscous=bool(visc), gamma=1.4, prandtl=0.71, mu_inf=1e-2, tau=1.0, pen_fact=0.5)
    s = H.Solver.box(dims, P, n, lo, hi, jitter=jit, seed=3, vcjh_scheme=scheme, **kw)
    m = O.Mesh.box(dims, P, n, lo, hi, jitter=jit, seed=3, vcjh_scheme=scheme)
    pos = m.geometry()["pos_upts"]
    if dims == 3:
        u = O.ic_tgv(pos)
    else:
        u = O.ic_vortex(pos * (10.0 / (2 * np.pi)) - 5.0)
    u = _perturbed(u, seed=P * 10 + dims)
    s.set_state(u)
    ph = O.physics(viscous=visc, gamma=1.4, prandtl=0.71, mu_inf=1e-2, tau=1.0, pen_fact=0.5)
    assert rel(s.residual(), m.residual(ph, u)) <= TOL_RES


def test_fp32_form_error_is_small_and_stated():
    """FP32 traces/fluxes/operators, FP64 state, RK register and reductions:
    the L2 error of the solution against the FP64 path stays below 1e-6
    relative (the residual itself is only good to ~1e-4 at Mach 0.1, where
    the flux terms are ~1e3 times larger than the residual)."""
    meta, a = load("hex_tgv_p3_n3")
    s64, s32 = _solver(meta, 0), _solver(meta, 1)
    s64.set_state(a["u0"])
    s32.set_state(a["u0"])
    e_res = rel(s32.residual(), s64.residual())
    s64.advance(20, 1e-3)
    s32.advance(20, 1e-3)
    e_state = rel(s32.get_state(), s64.get_state())
    print("fp32 form: residual rel %.3e, state rel after 20 steps %.3e" % (e_res, e_state))
    assert e_res < 1e-3
    assert e_state < 1e-6


@pytest.mark.parametrize("n", [8, 16])
def test_tgv_residual_at_scale_matches_oracle(n):
    """TGV at Mach 0.1, P=3: the flux terms are 1e3-1e4 times larger than the
    residual, so parity at 1e-12 needs the reference's rounding, not just FP64."""
    kw = dict(viscous=True, gamma=1.4, prandtl=0.71, mu_inf=1.0 / 1600.0, tau=1.0, pen_fact=0.5)
    s = H.Solver.box(3, 3, (n, n, n), (0, 0, 0), (2 * np.pi,) * 3, vcjh_scheme=1, **kw)
    m = O.Mesh.box(3, 3, (n, n, n), (0, 0, 0), (2 * np.pi,) * 3, vcjh_scheme=1)
    u = O.ic_tgv(m.geometry()["pos_upts"])
    s.set_state(u)
    ph = O.physics(viscous=1, gamma=1.4, prandtl=0.71, mu_inf=1.0 / 1600.0, tau=1.0, pen_fact=0.5)
    assert rel(s.residual(), m.residual(ph, u)) <= TOL_RES


def test_errors_are_reported():
    meta, a = load("quad_vortex_p3_n6")
    s = _solver(meta)
    bad = np.array(a["u0"], copy=True, order="F")
    bad[0, 0, 0] = np.nan
    with pytest.raises(H.FrError) as ei:
        s.set_state(bad)
    assert ei.value.status == 3
    with pytest.raises(ValueError):
        s.set_state(bad[:, :-1])
    with pytest.raises(H.FrError) as ei:
        s.rk_stage(7, 1e-3)
    assert ei.value.status == 1
    with pytest.raises(H.FrError) as ei:
        s.advance(1, -1.0)
    assert ei.value.status == 1
    with pytest.raises(H.FrError) as ei:
        H.Solver.box(3, 5, (2, 2, 2), (0, 0, 0), (1, 1, 1))
    assert ei.value.status == 5
    # a state that blows up is reported at the next monitored step
    s.set_state(a["u0"])
    with pytest.raises(H.FrError) as ei:
        s.advance(200, 5.0, norms=True)
    assert ei.value.status == 3


def test_autotuned_tiles_give_identical_states():
    """Tile choice (elements and threads per CTA) changes nothing per element."""
    meta, a = load("hex_tgv_p3_n3")
    s1, s2 = _solver(meta), _solver(meta)
    s1.set_state(a["u0"])
    s2.set_state(a["u0"])
    before = s2.get_state()
    tiles = s2.autotune(2)
    assert np.array_equal(s2.get_state(), before)
    assert all(t > 0 for t in tiles)
    s1.advance(3, 1e-3)
    s2.advance(3, 1e-3)
    assert np.array_equal(s1.get_state(), s2.get_state())


def test_solver_restart_round_trip_with_reference_file(tmp_path):
    """Solver state from the reference's own restart file, stepped on, and
    written back in the same format."""
    meta, a = load("quad_vortex_p3_n6")
    s = _solver(meta)
    t = s.read_restart(os.path.join(GOLDEN, "rest_quad_vortex_p3_n6.dat"))
    assert abs(t - 0.02) < 1e-12
    assert rel(s.get_state(), a["uN"]) <= 1e-14
    out = tmp_path / "Rest.dat"
    s.write_restart(out, t)
    assert out.read_bytes() == open(os.path.join(GOLDEN, "rest_quad_vortex_p3_n6.dat"), "rb").read()
