"""The per-operator entry points (the reference's GPU seam, one method at a
time) against the reference's own intermediate arrays of one CalcResidual.

Operators, metrics and interface tables are the ones the reference builds
(taken from the oracle, which reproduces them bit for bit); device memory comes
from torch, pointers cross the C ABI as plain integers."""
import ctypes as C

import numpy as np
import pytest

import hifiles_b200 as H
import oracle as O
from golden_util import load, rel

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _dev(a):
    a = np.asfortranarray(a, dtype=np.float64)
    return torch.from_numpy(a.ravel(order="F").copy()).cuda()


def _host(t, shape):
    return t.cpu().numpy().reshape(shape, order="F")


def _ptr_table(base, offsets):
    """Device array of device pointers base + 8*offset (int_inters-style table)."""
    p = np.asarray(offsets, dtype=np.int64) * 8 + base.data_ptr()
    return torch.from_numpy(np.asfortranarray(p).ravel(order="F").copy()).cuda()


VP = C.c_void_p


def _bind(L):
    dbl, i = C.c_double, C.c_int
    L.fr_op_extrapolate_solution.argtypes = [i, i, i, i, VP, VP, VP, VP]
    L.fr_op_evaluate_invFlux.argtypes = [i, i, i, i, VP, VP, VP, C.c_void_p, VP]
    L.fr_op_calculate_gradient.argtypes = [i, i, i, i, VP, VP, VP, VP]
    L.fr_op_correct_gradient.argtypes = [i, i, i, i, i, VP, VP, VP, VP, VP, VP]
    L.fr_op_extrapolate_corrected_gradient.argtypes = [i, i, i, i, i, VP, VP, VP, VP]
    L.fr_op_evaluate_viscFlux.argtypes = [i, i, i, i, VP, VP, VP, VP, C.c_void_p, VP]
    L.fr_op_extrapolate_totalFlux.argtypes = [i, i, i, i, i, VP, VP, VP, VP]
    L.fr_op_calculate_divergence.argtypes = [i, i, i, i, VP, VP, VP, VP]
    L.fr_op_calculate_corrected_divergence.argtypes = [i, i, i, i, VP, VP, VP, VP, VP]
    L.fr_op_int_inters_common_invFlux.argtypes = [i, i, i, i] + [VP] * 9 + [C.c_void_p, i, i, VP]
    L.fr_op_int_inters_common_viscFlux.argtypes = [i, i, i, i] + [VP] * 9 + [C.c_void_p, VP]
    L.fr_op_advance_rk45.argtypes = [i, i, i, i, dbl, dbl, VP, VP, VP, VP, VP, VP]
    L.fr_op_evaluate_viscFlux_les.argtypes = [i, i, i, i, VP, VP, VP, VP, VP, VP, C.c_void_p, i, dbl, i, VP]
    L.fr_op_evaluate_sgsFlux.argtypes = [i, i, i, i, i, VP, VP, VP, VP]
    L.fr_op_int_inters_common_viscFlux_les.argtypes = [i, i, i, i] + [VP] * 11 + [C.c_void_p, VP]
    return L


class PhysDesc(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("gamma", "prandtl", "mu_inf", "rt_inf", "c_sth", "fix_vis", "tau",
                                          "pen_fact")]


def _ok(st):
    assert st == 0, H.lib().fr_last_error().decode()


@pytest.mark.parametrize("case", ["quad_vortex_p3_n6", "hex_tgv_p3_n3", "hex_tgv_p2_n3_jit", "hex_euler_p3_n3",
                                  "hex_wale_p3_n3_jit", "hex_smag_p2_n3", "quad_wale_p3_n6_jit"])
def test_operator_seam_matches_reference_stage_arrays(case):
    meta, a = load(case)
    L = _bind(H.lib())
    m = O.Mesh.box(meta["dims"], meta["order"], meta["n"], meta["lo"], meta["hi"], jitter=meta["jitter"],
                   seed=meta["seed"], vcjh_scheme=meta["vcjh"])
    E, nu, nf, F, D = m.n_eles, m.n_upts, m.n_fpts, m.n_fields, m.dims
    visc = bool(meta["viscous"])
    g = m.geometry()
    il, ir = m.interfaces()
    nfpi = (meta["order"] + 1) ** (D - 1)
    ni = len(il) // nfpi
    ph = PhysDesc(**{k: meta["physics"][k] for k, _ in PhysDesc._fields_})
    les = bool(meta["physics"].get("les", 0))
    opp = {w: _dev(m.operator(w)) for w in (0, 3)}
    opd = {w: [_dev(m.operator(w, d)) for d in range(D)] for w in (1, 2, 5)}
    arr_ptrs = {w: (C.c_void_p * D)(*[t.data_ptr() for t in opd[w]]) for w in opd}
    u = _dev(a["u0"])
    ufp = torch.zeros(nf * E * F, dtype=torch.float64, device="cuda")
    tf = torch.zeros(nu * E * F * D, dtype=torch.float64, device="cuda")
    gup = torch.zeros(nu * E * F * D, dtype=torch.float64, device="cuda")
    gfp = torch.zeros(nf * E * F * D, dtype=torch.float64, device="cuda")
    ntc = torch.zeros(nf * E * F, dtype=torch.float64, device="cuda")
    ntd = torch.zeros(nf * E * F, dtype=torch.float64, device="cuda")
    ddu = torch.zeros(nf * E * F, dtype=torch.float64, device="cuda")
    div = torch.zeros(nu * E * F, dtype=torch.float64, device="cuda")
    JG, dj, tdA, nrm = (_dev(g[k]) for k in ("JGinv_upts", "detjac_upts", "tdA_fpts", "norm_fpts"))
    fk = np.arange(F)[None, :] * (nf * E)
    tab = dict(ul=_ptr_table(ufp, il[:, None] + fk), ur=_ptr_table(ufp, ir[:, None] + fk),
               tl=_ptr_table(ntc, il[:, None] + fk), tr=_ptr_table(ntc, ir[:, None] + fk),
               dl=_ptr_table(ddu, il[:, None] + fk), dr=_ptr_table(ddu, ir[:, None] + fk),
               al=_ptr_table(tdA, il), ar=_ptr_table(tdA, ir),
               n=_ptr_table(nrm, il[:, None] + np.arange(D)[None, :] * (nf * E)))
    gk = (np.arange(F)[:, None] + F * np.arange(D)[None, :]).ravel(order="F")[None, :] * (nf * E)
    tab["gl"] = _ptr_table(gfp, il[:, None] + gk)
    tab["gr"] = _ptr_table(gfp, ir[:, None] + gk)
    sgu = torch.zeros(nu * E * F * D, dtype=torch.float64, device="cuda")
    sgf = torch.zeros(nf * E * F * D, dtype=torch.float64, device="cuda")
    tab["sl"] = _ptr_table(sgf, il[:, None] + gk)
    tab["sr"] = _ptr_table(sgf, ir[:, None] + gk)
    P = lambda t: t.data_ptr()  # noqa: E731

    _ok(L.fr_op_extrapolate_solution(nf, nu, F, E, P(opp[0]), P(u), P(ufp), None))
    if visc:
        _ok(L.fr_op_calculate_gradient(nu, D, F, E, C.cast(arr_ptrs[2], VP), P(u), P(gup), None))
    _ok(L.fr_op_evaluate_invFlux(nu, D, F, E, P(u), P(JG), P(tf), C.byref(ph), None))
    _ok(L.fr_op_int_inters_common_invFlux(nfpi, D, F, ni, P(tab["ul"]), P(tab["ur"]), P(tab["tl"]), P(tab["tr"]),
                                          P(tab["al"]), P(tab["ar"]), P(tab["n"]), P(tab["dl"]), P(tab["dr"]),
                                          C.byref(ph), 0, int(visc), None))
    if visc:
        _ok(L.fr_op_correct_gradient(nu, nf, D, F, E, C.cast(arr_ptrs[5], VP), P(ddu), P(JG), P(dj), P(gup), None))
        _ok(L.fr_op_extrapolate_corrected_gradient(nf, nu, D, F, E, P(opp[0]), P(gup), P(gfp), None))
        if les:
            _ok(L.fr_op_evaluate_viscFlux_les(nu, D, F, E, P(u), P(gup), P(JG), P(dj), P(tf), P(sgu), C.byref(ph),
                                              meta["physics"]["sgs_model"], meta["physics"]["filter_ratio"],
                                              meta["order"], None))
            _ok(L.fr_op_evaluate_sgsFlux(nf, nu, D, F, E, P(opp[0]), P(sgu), P(sgf), None))
        else:
            _ok(L.fr_op_evaluate_viscFlux(nu, D, F, E, P(u), P(gup), P(JG), P(tf), C.byref(ph), None))
    _ok(L.fr_op_extrapolate_totalFlux(nf, nu, D, F, E, C.cast(arr_ptrs[1], VP), P(tf), P(ntd), None))
    _ok(L.fr_op_calculate_divergence(nu, D, F, E, C.cast(arr_ptrs[2], VP), P(tf), P(div), None))
    if visc and les:
        _ok(L.fr_op_int_inters_common_viscFlux_les(nfpi, D, F, ni, P(tab["ul"]), P(tab["ur"]), P(tab["gl"]),
                                                   P(tab["gr"]), P(tab["tl"]), P(tab["tr"]), P(tab["al"]),
                                                   P(tab["ar"]), P(tab["n"]), P(tab["sl"]), P(tab["sr"]),
                                                   C.byref(ph), None))
    elif visc:
        _ok(L.fr_op_int_inters_common_viscFlux(nfpi, D, F, ni, P(tab["ul"]), P(tab["ur"]), P(tab["gl"]),
                                               P(tab["gr"]), P(tab["tl"]), P(tab["tr"]), P(tab["al"]),
                                               P(tab["ar"]), P(tab["n"]), C.byref(ph), None))
    ntc_before = _host(ntc, (nf, E, F))
    _ok(L.fr_op_calculate_corrected_divergence(nu, nf, F, E, P(opp[3]), P(ntd), P(ntc), P(div), None))
    torch.cuda.synchronize()
    tol = 1e-12
    assert rel(_host(ufp, (nf, E, F)), a["disu_fpts0"]) <= tol
    assert rel(_host(tf, (nu, E, F, D)), a["tdisf_upts0"]) <= tol
    assert rel(_host(ntd, (nf, E, F)), a["norm_tdisf_fpts0"]) <= tol
    assert rel(ntc_before, a["norm_tconf_fpts0"]) <= tol
    if les:
        # the SGS flux at the solution points (transformed) and its extrapolation
        assert rel(_host(sgu, (nu, E, F, D)), a["sgsf_upts0"]) <= tol
        want_f = np.einsum("fu,uekd->fekd", m.operator(0), a["sgsf_upts0"])
        assert rel(_host(sgf, (nf, E, F, D)), want_f) <= tol
    if visc:
        assert rel(_host(ddu, (nf, E, F)), a["delta_disu_fpts0"]) <= tol
        assert rel(_host(gup, (nu, E, F, D)), a["grad_disu_upts0"]) <= tol
        assert rel(_host(gfp, (nf, E, F, D)), a["grad_disu_fpts0"]) <= tol
    assert rel(_host(div, (nu, E, F)), a["div0"]) <= tol
    # one RK45 stage on top (eles::AdvanceSolution stage 0)
    reg = torch.zeros_like(u)
    _ok(L.fr_op_advance_rk45(nu, F, E, 0, meta["dt"], 0.0, P(u), P(reg), P(div), P(dj), None, None))
    torch.cuda.synchronize()
    d = a["div0"]
    res = meta["dt"] * (-d / g["detjac_upts"][:, :, None])
    assert rel(_host(u, (nu, E, F)), a["u0"] + 0.149659021999229 * res) <= 1e-14
