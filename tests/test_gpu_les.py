"""Eddy-viscosity LES on the CUDA path (input keys LES 1, SGS_model 0/1):
the SGS flux of eles::calc_sgsf_upts (src/eles.cpp:2456-2778) inside the
gradient kernel, its flux-point extrapolation (evaluate_sgsFlux,
src/eles.cpp:3294-3368) and its share of the common viscous flux
(src/int_inters.cpp:415-427), checked against the oracle, which matches the
reference's own LES runs to the last bit (tests/golden/*wale*, *smag*).

Tolerance: the residual parity bar of the other FP64 tests, 1e-12 normwise
relative.  Every case also checks that the SGS flux moves the residual by far
more than that bar, so the comparison is not won by a path that drops it."""
import numpy as np
import pytest

import hifiles_b200 as H
import oracle as O
from golden_util import load, rel

pytestmark = pytest.mark.gpu

TOL_RES = 1e-12
KW = dict(gamma=1.4, prandtl=0.71, mu_inf=1e-3, tau=1.0, pen_fact=0.5)


def _state(m, dims, seed):
    pos = m.geometry()["pos_upts"]
    u = O.ic_tgv(pos) if dims == 3 else O.ic_vortex(pos * (10.0 / (2 * np.pi)) - 5.0)
    r = np.random.default_rng(seed).standard_normal(u.shape)
    v = np.array(u, copy=True, order="F")
    v[:, :, 1:-1] += 0.05 * r[:, :, 1:-1]
    return v


@pytest.mark.parametrize("dims,P,n,sgs,jit,fr", [
    (3, 3, (3, 2, 3), 1, 0.1, 1.0), (3, 2, (2, 3, 2), 0, 0.15, 2.0), (3, 4, (2, 2, 2), 1, 0.1, 1.0),
    (3, 1, (3, 3, 2), 1, 0.1, 1.0), (2, 3, (4, 3), 1, 0.1, 1.0), (2, 5, (2, 3), 0, 0.0, 1.5),
    (2, 2, (3, 3), 1, 0.2, 0.5)])
def test_les_residual_matches_oracle(dims, P, n, sgs, jit, fr):
    lo, hi = [0.0] * dims, [2 * np.pi] * dims
    s = H.Solver.box(dims, P, n, lo, hi, jitter=jit, seed=7, viscous=True, vcjh_scheme=1, les=1, sgs_model=sgs,
                     filter_ratio=fr, **KW)
    m = O.Mesh.box(dims, P, n, lo, hi, jitter=jit, seed=7, vcjh_scheme=1)
    u = _state(m, dims, seed=P + 10 * dims + sgs)
    s.set_state(u)
    want = m.residual(O.physics(viscous=1, les=1, sgs_model=sgs, filter_ratio=fr, **KW), u)
    plain = m.residual(O.physics(viscous=1, **KW), u)
    assert rel(plain, want) > 1e3 * TOL_RES        # the SGS flux matters at this bar
    assert rel(s.residual(), want) <= TOL_RES


def test_les_tgv_8_cubed_steps_match_oracle():
    """WALE on the Mach 0.1 Taylor-Green vortex, 8^3 hexes P=3, three RK45 steps."""
    kw = dict(KW, mu_inf=1.0 / 1600.0)
    s = H.Solver.box(3, 3, (8, 8, 8), (0, 0, 0), (2 * np.pi,) * 3, viscous=True, les=1, sgs_model=1, **kw)
    m = O.Mesh.box(3, 3, (8, 8, 8), (0, 0, 0), (2 * np.pi,) * 3)
    u = O.ic_tgv(m.geometry()["pos_upts"])
    ph = O.physics(viscous=1, les=1, sgs_model=1, **kw)
    s.set_state(u)
    assert rel(s.residual(), m.residual(ph, u)) <= TOL_RES
    uN, _, nrm = m.rk45(ph, u, 1e-3, 3)
    got = s.advance(3, 1e-3, norms=True)
    assert rel(s.get_state(), uN) <= TOL_RES
    assert np.all(np.abs(got - nrm[:, -1]) <= 1e-10 * np.abs(nrm[:, -1]) + 1e-14)


def test_les_fp32_form_error_is_small():
    meta, a = load("hex_wale_p3_n3_jit")
    mk = lambda prec: H.Solver.box(3, 3, meta["n"], meta["lo"], meta["hi"], jitter=meta["jitter"],
                                   seed=meta["seed"], viscous=True, vcjh_scheme=meta["vcjh"], precision=prec,
                                   **meta["physics"])
    s64, s32 = mk(0), mk(1)
    s64.set_state(a["u0"])
    s32.set_state(a["u0"])
    assert rel(s32.residual(), s64.residual()) < 1e-3
    s64.advance(20, 1e-3)
    s32.advance(20, 1e-3)
    assert rel(s32.get_state(), s64.get_state()) < 1e-6


def test_les_autotuned_tiles_give_identical_states():
    meta, a = load("hex_wale_p3_n3_jit")
    mk = lambda: H.Solver.box(3, 3, meta["n"], meta["lo"], meta["hi"], jitter=meta["jitter"], seed=meta["seed"],
                              viscous=True, vcjh_scheme=meta["vcjh"], **meta["physics"])
    s1, s2 = mk(), mk()
    s1.set_state(a["u0"])
    s2.set_state(a["u0"])
    s2.autotune(2)
    s1.advance(3, 1e-3)
    s2.advance(3, 1e-3)
    assert np.array_equal(s1.get_state(), s2.get_state())


def test_les_options_are_checked():
    box = dict(dims=3, order=2, n=(2, 2, 2), lo=(0, 0, 0), hi=(1, 1, 1))
    with pytest.raises(H.FrError) as ei:            # LES needs the viscous equations
        H.Solver.box(**box, viscous=False, les=1)
    assert ei.value.status == 1
    for model in (2, 3, 4):                         # filter-based models are not built
        with pytest.raises(H.FrError) as ei:
            H.Solver.box(**box, viscous=True, les=1, sgs_model=model)
        assert ei.value.status == 5
    with pytest.raises(H.FrError) as ei:
        H.Solver.box(**box, viscous=True, les=1, sgs_model=1, filter_ratio=0.0)
    assert ei.value.status == 1
