"""The CPU oracle (oracle/fr_oracle.c) against the reference's own outputs.

The fixtures were produced by running the unmodified reference (oracle/_ref)
on the same meshes and states; the oracle repeats the reference's operation
order, so agreement is expected to the last bit."""
import json
import os

import numpy as np
import pytest

import oracle as O
from golden_util import (BC_CASES, CASES, GOLDEN, IQ_CASES, LES_CASES, ROE_CASES, integral_quantities_numpy, load,
                         over_integrated_density_error, rel)


def _mesh(meta):
    return O.Mesh.box(meta["dims"], meta["order"], meta["n"], meta["lo"], meta["hi"], jitter=meta["jitter"],
                      seed=meta["seed"], vcjh_scheme=meta["vcjh"], side_bc=meta.get("side_bc"))


def _phys(meta):
    return O.physics(viscous=meta["viscous"], **meta["physics"])


def test_point_tables_match_reference():
    tab = json.load(open(os.path.join(GOLDEN, "points_1d.json")))
    for kind, rows in tab.items():
        for p, vals in rows.items():
            assert O.points_1d(int(p), 0 if kind == "gauss" else 1).tolist() == vals, (kind, p)


@pytest.mark.parametrize("case", CASES + BC_CASES)
def test_oracle_residual_matches_reference(case):
    meta, a = load(case)
    m = _mesh(meta)
    div = m.residual(_phys(meta), a["u0"])
    assert rel(div, a["div0"]) <= 1e-14


@pytest.mark.parametrize("case", [c for c in CASES if c != "quad_vortex_p3_n20"] + BC_CASES)
def test_oracle_steps_match_reference(case):
    meta, a = load(case)
    m = _mesh(meta)
    u, _, nrm = m.rk45(_phys(meta), a["u0"], meta["dt"], meta["steps"])
    assert rel(u, a["uN"]) <= 1e-14
    assert rel(nrm, a["norms"]) <= 1e-12


@pytest.mark.parametrize("case", ["quad_vortex_p3_n6", "hex_tgv_p3_n3", "hex_tgv_p2_n3_jit"] + LES_CASES + ROE_CASES + BC_CASES)
def test_oracle_stage_arrays_match_reference(case):
    meta, a = load(case)
    m = _mesh(meta)
    _, st = m.residual(_phys(meta), a["u0"], stages=True)
    assert rel(st["disu_fpts"], a["disu_fpts0"]) <= 1e-14
    assert rel(st["tdisf_upts"], a["tdisf_upts0"]) <= 1e-14
    assert rel(st["norm_tdisf_fpts"], a["norm_tdisf_fpts0"]) <= 1e-14
    assert rel(st["norm_tconf_fpts"], a["norm_tconf_fpts0"]) <= 1e-14
    if meta["viscous"]:
        assert rel(st["grad_disu_upts"], a["grad_disu_upts0"]) <= 1e-14
        assert rel(st["grad_disu_fpts"], a["grad_disu_fpts0"]) <= 1e-14
        assert rel(st["delta_disu_fpts"], a["delta_disu_fpts0"]) <= 1e-14
    if meta["physics"].get("les"):
        assert rel(st["sgsf_upts"], a["sgsf_upts0"]) <= 1e-14


@pytest.mark.slow
def test_oracle_vortex_1000_steps_matches_reference():
    """The 2-D isentropic vortex workload (20x20 quads, P=3, c_dg, Rusanov, RK45, dt 1e-3, 1000 steps)."""
    meta, a = load("quad_vortex_p3_n20")
    m = _mesh(meta)
    u, _, nrm = m.rk45(_phys(meta), a["u0"], meta["dt"], meta["steps"])
    assert rel(u, a["uN"]) <= 1e-13
    assert rel(nrm, a["norms"]) <= 1e-10


@pytest.mark.slow
def test_oracle_reproduces_reference_regression_kat():
    """testcases/regression_tests.py:300-310: TGV 15^3 hex P=3 SD, iter 25 L1 residuals, abs tol 1e-5."""
    kat = json.load(open(os.path.join(GOLDEN, "kat_tgv.json")))
    m = O.Mesh.box(3, 3, (15, 15, 15), (0, 0, 0), (2 * np.pi,) * 3, vcjh_scheme=2)
    u0 = O.ic_tgv(m.geometry()["pos_upts"], p0=100.0)
    _, _, nrm = m.rk45(O.tgv_kat_physics(), u0, 1e-3, kat["test_iter"])
    assert np.all(np.abs(nrm[:, -1] - np.array(kat["test_vals"])) < kat["tol"])


@pytest.mark.parametrize("case", IQ_CASES)
def test_integral_quantity_restatement_matches_reference(case):
    """The numpy restatement of eles::CalcIntegralQuantities (golden_util) on the
    reference's own state, gradient and cubature gives the reference's values."""
    meta, a = load(case)
    vals, mags = integral_quantities_numpy(a["u0"], a["grad"], a["opp"], a["weight"], a["detjac"], meta["dims"],
                                           meta["physics"]["gamma"])
    for v, w, m in zip(vals, a["iq"], mags):
        assert abs(v - w) <= 1e-13 * m


def test_reference_convergence_rate_at_p2():
    """The reference's own P = 2 vortex runs (10^2, 20^2, 40^2 to t = 1, over-integrated
    density error): rates 2.64 and 2.59 -- the rate the CUDA path is held to at P = 2."""
    errs = []
    for n in (10, 20, 40):
        meta, a = load("order_vortex_p2_n%d" % n)
        errs.append(over_integrated_density_error(a["uN"], a["pos"], 2, 10.0 / n, 1.0))
    rates = [np.log(errs[i] / errs[i + 1]) / np.log(2.0) for i in range(2)]
    assert 2.5 < rates[0] < 2.8 and 2.5 < rates[1] < 2.8, rates
