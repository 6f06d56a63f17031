"""Mixed-element meshes (tets, prisms, hexes) through the per-operator entry
points, against the reference's own arrays.

The fixtures (tests/golden/mixed_*.npz, made by tests/golden/make_mixed.py
from runs of the reference itself) hold what the reference's per-type classes
pass across the seam: every element type's dense operators opp_0..opp_6
(eles_tets, eles_pris, eles_hexas set-up), its metrics, and the wiring of the
triangular and quadrilateral interfaces, decoded from int_inters' pointer
tables (src/int_inters.cpp:95-178).  The GPU test runs CalcResidual
(src/solver.cpp:65-225) one operator at a time, element type by element type
and interface type by interface type as the reference does, then three RK45
steps, and compares every intermediate array and the final state.

The channel cases put an isothermal and an adiabatic wall on the prisms'
triangular faces; their boundary fluxes go through the boundary entry points
(bdy_inters' tables, src/bdy_inters.cpp:111-203).

The CPU tests check the fixtures themselves: the interior and boundary
wiring covers every flux point exactly once, and the dumped arrays obey the
linear operator relations they are defined by."""
import ctypes as C

import numpy as np
import pytest

from golden_util import load, rel

MIXED = ["mixed_pritet_p3", "mixed_pritet_p2", "mixed_hexpri_p3", "mixed_channel_p2", "mixed_channel_p3",
         "mixed_triquad_p3", "mixed_triquad_p2"]
# 2-D quadrilateral boxes with a boundary on every side: Euler with
# characteristic / subsonic outflow / slip wall / dual-consistent slip wall and
# simple in- and outflow / supersonic in- and outflow, Navier-Stokes with
# characteristic in- and outflow and moving isothermal / adiabatic walls; the
# Roe common flux (riemann_solve_type 2) with boundaries and periodic
SEAM_2D = ["seam_quad_bc_euler_p3", "seam_quad_bc_euler2_p2", "seam_quad_ns_bc_p3", "seam_quad_roe_bc_p3",
           "seam_quad_roe_p3_jit"]
CASES = MIXED + SEAM_2D


def _dims(meta):
    return meta.get("dims", 3)


def _visc(meta):
    return bool(meta.get("viscous", 1))


def _keys(meta):
    """Harness stage arrays of the final transformed flux and common flux."""
    return ("s07_tdisf_upts", "s10_norm_tconf_fpts") if _visc(meta) else ("s03_tdisf_upts", "s04_norm_tconf_fpts")
RK4B = [0.149659021999229, 0.379210312999627, 0.822955029386982, 0.699450455949122, 0.153057247968152]


def _types(meta):
    return {t["index"]: t for t in meta["types"]}


@pytest.mark.parametrize("case", CASES)
def test_mixed_wiring_pairs_every_flux_point_once(case):
    meta, a = load(case)
    ty = _types(meta)
    seen = {i: np.zeros((t["n_fpts"], t["n_eles"]), dtype=np.int64) for i, t in ty.items()}
    for it in meta["inters"]:
        w = a["int_inters_%d" % it["index"]].reshape(6, -1)
        for s in (0, 3):
            for tt, e, f in zip(w[s], w[s + 1], w[s + 2]):
                seen[int(tt)][f, e] += 1
        # both sides of an interface point sit at the same place: same state
        # trace in the reference's extrapolated solution
        for k in range(w.shape[1]):
            tl, el, fl, tr, er, fr = (int(x) for x in w[:, k])
            ul = a["t%d_s01_disu_fpts" % ty[tl]["ele_type"]][fl, el, 0]
            ur = a["t%d_s01_disu_fpts" % ty[tr]["ele_type"]][fr, er, 0]
            assert abs(ul - ur) < 0.05 * abs(ul)
    for it in meta.get("bdy_inters", []):
        w = a["bdy_inters_%d" % it["index"]].reshape(4, -1)
        for tt, e, f in zip(w[0], w[1], w[2]):
            seen[int(tt)][f, e] += 1
        assert set(int(x) for x in w[3]) <= set(meta["side_bc"])
    for i, s in seen.items():
        assert (s == 1).all(), (case, ty[i]["ele_type"])


@pytest.mark.parametrize("case", CASES)
def test_mixed_fixture_operator_relations(case):
    meta, a = load(case)
    tf_key, ntc_key = _keys(meta)
    for t in meta["types"]:
        T = "t%d_" % t["ele_type"]
        u0 = a[T + "disu_upts_init"]
        nu, E, F = u0.shape
        # extrapolation: disu_fpts = opp_0 u
        got = np.einsum("fu,uek->fek", a[T + "opp_0"], u0)
        assert rel(got, a[T + "s01_disu_fpts"]) < 1e-14
        # divergence: div = sum_d opp_2[d] tdisf[d]; corrected: += opp_3 (norm_tconf - norm_tdisf)
        div = sum(np.einsum("vu,uek->vek", a[T + "opp_2_%d" % d], a[T + tf_key][..., d]) for d in range(_dims(meta)))
        assert rel(div, a[T + "s09_div_tconf_upts"]) < 1e-13
        jump = a[T + ntc_key] - a[T + "s08_norm_tdisf_fpts"]
        corr = a[T + "s09_div_tconf_upts"] + np.einsum("uf,fek->uek", a[T + "opp_3"], jump)
        assert rel(corr, a[T + "s11_div_tconf_upts"]) < 1e-12
        # RK45 stage 0 from a zero register: u1 = u0 + b_0 dt (-div / detJ)
        res = meta["dt"] * (-a[T + "s11_div_tconf_upts"] / a[T + "detjac_upts"][:, :, None])
        assert rel(a[T + "s12_disu_upts0"], u0 + RK4B[0] * res) < 1e-15


# ------------------------------------------------------------------ GPU path

def _seam():
    import hifiles_b200 as H
    import test_gpu_ops as T
    L = T._bind(H.lib())
    i, VP = C.c_int, C.c_void_p
    L.fr_op_bdy_inters_common_invFlux.argtypes = [i, i, i, i] + [VP] * 7 + [VP, C.c_double, i, i, VP]
    L.fr_op_bdy_inters_common_viscFlux.argtypes = [i, i, i, i] + [VP] * 7 + [VP, C.c_double, VP]
    return H, T, L


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_mixed_mesh_through_the_operator_seam_matches_the_reference(case):
    torch = pytest.importorskip("torch")
    H, T, L = _seam()
    meta, a = load(case)
    VP = C.c_void_p
    ty = _types(meta)
    ph = T.PhysDesc(**meta["physics"])
    D = _dims(meta)
    F = D + 2
    visc = _visc(meta)
    riemann = int(meta.get("riemann", 0))
    tf_key, ntc_key = _keys(meta)
    P = lambda t: t.data_ptr()  # noqa: E731
    dev = T._dev
    S = {}
    for i, t in ty.items():
        X = "t%d_" % t["ele_type"]
        nu, nf, E = t["n_upts"], t["n_fpts"], t["n_eles"]
        s = dict(nu=nu, nf=nf, E=E, X=X)
        s["opp0"], s["opp3"] = dev(a[X + "opp_0"]), dev(a[X + "opp_3"])
        s["opp6"] = dev(a[X + "opp_6"]) if visc else None
        for w in ((1, 2, 4, 5) if visc else (1, 2)):
            s["opp%d" % w] = [dev(a[X + "opp_%d_%d" % (w, d)]) for d in range(D)]
            s["opp%d_ptrs" % w] = (VP * D)(*[P(x) for x in s["opp%d" % w]])
        s["JG"], s["dj"], s["tdA"], s["nrm"] = (dev(a[X + k]) for k in ("JGinv_upts", "detjac_upts", "tdA_fpts",
                                                                         "norm_fpts"))
        s["u"] = dev(a[X + "disu_upts_init"])
        s["reg"] = torch.zeros_like(s["u"])
        z = lambda n: torch.zeros(n, dtype=torch.float64, device="cuda")  # noqa: E731
        s["ufp"], s["ntc"], s["ntd"], s["ddu"] = z(nf * E * F), z(nf * E * F), z(nf * E * F), z(nf * E * F)
        s["tf"], s["gup"], s["gfp"] = z(nu * E * F * D), z(nu * E * F * D), z(nf * E * F * D)
        s["div"] = z(nu * E * F)
        S[i] = s

    def table(w, side, arr, comps):
        """int_inters-style device table: for every (fpt, inter) of one side and
        every component c, the address of arr[fpt, ele, c] of that side's type."""
        tt, e, f = (w[side + q].reshape(-1, order="F").astype(np.int64) for q in range(3))
        rows = np.zeros((tt.size, comps), dtype=np.int64)
        for i, s in S.items():
            m = tt == i
            if not m.any():
                continue
            base = s[arr].data_ptr()
            slot = f[m] + s["nf"] * e[m]
            rows[m] = base + 8 * (slot[:, None] + s["nf"] * s["E"] * np.arange(comps)[None, :])
        return torch.from_numpy(np.asfortranarray(rows).ravel(order="F").copy()).cuda()

    inters = []
    for it in meta["inters"]:
        w = a["int_inters_%d" % it["index"]]
        tb = dict(nfpi=it["n_fpts"], ni=it["n_inters"])
        for side, sfx in ((0, "l"), (3, "r")):
            tb["u" + sfx] = table(w, side, "ufp", F)
            tb["t" + sfx] = table(w, side, "ntc", F)
            tb["d" + sfx] = table(w, side, "ddu", F)
            tb["g" + sfx] = table(w, side, "gfp", F * D)
            tb["a" + sfx] = table(w, side, "tdA", 1)
        tb["n"] = table(w, 0, "nrm", D)
        inters.append(tb)
    bdys = []
    for it in meta.get("bdy_inters", []):
        w = a["bdy_inters_%d" % it["index"]]
        tb = dict(nfpi=it["n_fpts"], ni=it["n_inters"])
        tb["ul"], tb["tl"], tb["dl"] = table(w, 0, "ufp", F), table(w, 0, "ntc", F), table(w, 0, "ddu", F)
        tb["gl"], tb["al"], tb["n"] = table(w, 0, "gfp", F * D), table(w, 0, "tdA", 1), table(w, 0, "nrm", D)
        tb["type"] = torch.from_numpy(np.ascontiguousarray(w[3, 0, :]).astype(np.int32)).cuda()
        bdys.append(tb)
    bdy_params = torch.tensor(meta["bdy"], dtype=torch.float64, device="cuda")
    R_ref = float(meta["R_ref"])

    def ok(st):
        assert st == 0, H.lib().fr_last_error().decode()

    def residual():
        for s in S.values():
            ok(L.fr_op_extrapolate_solution(s["nf"], s["nu"], F, s["E"], P(s["opp0"]), P(s["u"]), P(s["ufp"]), None))
            if visc:
                ok(L.fr_op_calculate_gradient(s["nu"], D, F, s["E"], C.cast(s["opp4_ptrs"], VP), P(s["u"]),
                                              P(s["gup"]), None))
            ok(L.fr_op_evaluate_invFlux(s["nu"], D, F, s["E"], P(s["u"]), P(s["JG"]), P(s["tf"]), C.byref(ph), None))
        for tb in inters:
            ok(L.fr_op_int_inters_common_invFlux(tb["nfpi"], D, F, tb["ni"], P(tb["ul"]), P(tb["ur"]), P(tb["tl"]),
                                                 P(tb["tr"]), P(tb["al"]), P(tb["ar"]), P(tb["n"]), P(tb["dl"]),
                                                 P(tb["dr"]), C.byref(ph), riemann, int(visc), None))
        for tb in bdys:
            ok(L.fr_op_bdy_inters_common_invFlux(tb["nfpi"], D, F, tb["ni"], P(tb["ul"]), P(tb["tl"]), P(tb["al"]),
                                                 P(tb["n"]), P(tb["type"]), P(bdy_params), P(tb["dl"]), C.byref(ph),
                                                 R_ref, riemann, int(visc), None))
        for s in S.values():
            if not visc:
                break
            ok(L.fr_op_correct_gradient(s["nu"], s["nf"], D, F, s["E"], C.cast(s["opp5_ptrs"], VP), P(s["ddu"]),
                                        P(s["JG"]), P(s["dj"]), P(s["gup"]), None))
            ok(L.fr_op_extrapolate_corrected_gradient(s["nf"], s["nu"], D, F, s["E"], P(s["opp6"]), P(s["gup"]),
                                                      P(s["gfp"]), None))
            ok(L.fr_op_evaluate_viscFlux(s["nu"], D, F, s["E"], P(s["u"]), P(s["gup"]), P(s["JG"]), P(s["tf"]),
                                         C.byref(ph), None))
        for s in S.values():
            ok(L.fr_op_extrapolate_totalFlux(s["nf"], s["nu"], D, F, s["E"], C.cast(s["opp1_ptrs"], VP), P(s["tf"]),
                                             P(s["ntd"]), None))
            ok(L.fr_op_calculate_divergence(s["nu"], D, F, s["E"], C.cast(s["opp2_ptrs"], VP), P(s["tf"]),
                                            P(s["div"]), None))
        for tb in (inters if visc else []):
            ok(L.fr_op_int_inters_common_viscFlux(tb["nfpi"], D, F, tb["ni"], P(tb["ul"]), P(tb["ur"]), P(tb["gl"]),
                                                  P(tb["gr"]), P(tb["tl"]), P(tb["tr"]), P(tb["al"]), P(tb["ar"]),
                                                  P(tb["n"]), C.byref(ph), None))
        for tb in (bdys if visc else []):
            ok(L.fr_op_bdy_inters_common_viscFlux(tb["nfpi"], D, F, tb["ni"], P(tb["ul"]), P(tb["gl"]), P(tb["tl"]),
                                                  P(tb["al"]), P(tb["n"]), P(tb["type"]), P(bdy_params), C.byref(ph),
                                                  R_ref, None))
        snap = {i: T._host(s["ntc"], (s["nf"], s["E"], F)) for i, s in S.items()}
        for s in S.values():
            ok(L.fr_op_calculate_corrected_divergence(s["nu"], s["nf"], F, s["E"], P(s["opp3"]), P(s["ntd"]),
                                                      P(s["ntc"]), P(s["div"]), None))
        return snap

    def advance(stage):
        for s in S.values():
            ok(L.fr_op_advance_rk45(s["nu"], F, s["E"], stage, meta["dt"], 0.0, P(s["u"]), P(s["reg"]), P(s["div"]),
                                    P(s["dj"]), None, None))

    ntc_visc = residual()
    torch.cuda.synchronize()
    tol = 1e-12
    for i, s in S.items():
        X, nu, nf, E = s["X"], s["nu"], s["nf"], s["E"]
        assert rel(T._host(s["ufp"], (nf, E, F)), a[X + "s01_disu_fpts"]) <= tol
        if visc:
            # delta = u_common - u_own is a difference of nearly equal traces
            # (on faces that carry solution points it nearly vanishes): bounded
            # by 1e-12 of itself plus a few ulps of the traces it comes from
            dd = T._host(s["ddu"], (nf, E, F)) - a[X + "s04_delta_disu_fpts"]
            assert np.linalg.norm(dd) <= (tol * np.linalg.norm(a[X + "s04_delta_disu_fpts"])
                                          + 4e-16 * np.linalg.norm(a[X + "s01_disu_fpts"]))
            assert rel(T._host(s["gup"], (nu, E, F, D)), a[X + "s05_grad_disu_upts"]) <= tol
            assert rel(T._host(s["gfp"], (nf, E, F, D)), a[X + "s06_grad_disu_fpts"]) <= tol
        assert rel(T._host(s["tf"], (nu, E, F, D)), a[X + tf_key]) <= tol
        assert rel(T._host(s["ntd"], (nf, E, F)), a[X + "s08_norm_tdisf_fpts"]) <= tol
        assert rel(ntc_visc[i], a[X + ntc_key]) <= tol
        assert rel(T._host(s["div"], (nu, E, F)), a[X + "s11_div_tconf_upts"]) <= tol
    advance(0)
    torch.cuda.synchronize()
    for s in S.values():
        assert rel(T._host(s["u"], (s["nu"], s["E"], F)), a[s["X"] + "s12_disu_upts0"]) <= 1e-14
    # the rest of three RK45 steps (src/HiFiLES.cpp:159-183)
    for step in range(meta["steps"]):
        for stage in range(1 if step == 0 else 0, 5):
            residual()
            advance(stage)
    torch.cuda.synchronize()
    for s in S.values():
        X = s["X"]
        u = T._host(s["u"], (s["nu"], s["E"], F))
        u0 = a[X + "disu_upts_init"]
        assert rel(u, a[X + "final_disu_upts0"]) <= 1e-14
        # the change over three steps, not only the state, agrees
        assert rel(u - u0, a[X + "final_disu_upts0"] - u0) <= 1e-10


@pytest.mark.parametrize("case", ["mixed_channel_p2", "mixed_hexpri_p3"])
def test_tiled_mixed_mesh_wires_each_copy_to_itself(case):
    import hifiles_b200.seam as SM
    meta, a = load(case)
    types, ints, bdys = SM.mixed_mesh_inputs(meta, a)
    K = 3
    tt, ti, tb = SM.tile_mixed_mesh(types, ints, bdys, K)
    for i, ty in types.items():
        E = ty["u"].shape[1]
        assert tt[i]["u"].shape[1] == K * E
        assert np.array_equal(tt[i]["JGinv_upts"][..., E:2 * E], ty["JGinv_upts"])
    for w, w3 in zip(ints + bdys, ti + tb):
        ni = w.shape[2]
        assert w3.shape[2] == K * ni
        for c in range(K):
            blk = w3[:, :, c * ni:(c + 1) * ni]
            for s in ((0, 3) if w.shape[0] == 6 else (0,)):
                assert np.array_equal(blk[s], w[s]) and np.array_equal(blk[s + 2], w[s + 2])
                for i, ty in types.items():
                    m = w[s] == i
                    assert np.array_equal(blk[s + 1][m], w[s + 1][m] + c * ty["u"].shape[1])


@pytest.mark.gpu
def test_mixed_mesh_driver_matches_the_reference_and_its_copies():
    """The package driver used for throughput runs (seam.MixedOperatorMesh):
    the reference's final state of the wall channel, and every copy of a tiled
    mesh bit for bit equal to the single mesh."""
    import hifiles_b200.seam as SM
    meta, a = load("mixed_channel_p2")
    types, ints, bdys = SM.mixed_mesh_inputs(meta, a)
    m = SM.MixedOperatorMesh(types, ints, meta["physics"], bdys, meta["bdy"], meta["R_ref"])
    m.advance(meta["steps"], meta["dt"])
    one = {}
    for t in meta["types"]:
        one[t["index"]] = m.get_state(t["index"])
        assert rel(one[t["index"]], a["t%d_final_disu_upts0" % t["ele_type"]]) <= 1e-14
    K = 3
    tt, ti, tb = SM.tile_mixed_mesh(types, ints, bdys, K)
    m3 = SM.MixedOperatorMesh(tt, ti, meta["physics"], tb, meta["bdy"], meta["R_ref"])
    m3.advance(meta["steps"], meta["dt"])
    for i, u1 in one.items():
        u3 = m3.get_state(i)
        E = u1.shape[1]
        for c in range(K):
            assert np.array_equal(u3[:, c * E:(c + 1) * E], u1)


def test_ellpack_matches_the_reference_layout():
    """seam.ellpack follows array_to_ellpack (src/funcs.cpp:961-1011): entries
    >= 1e-12 in increasing column order, slot s of row i at i + m s, padding
    0 at column 0; the dense operator is recovered from it."""
    import hifiles_b200.seam as SM
    a = np.array([[0.0, 2.0, 0.0, 3.0], [1.0, 0.0, 0.0, 0.0], [4.0, 5.0, 6.0, 1e-13]])
    data, idx, nnz = SM.ellpack(a)
    assert nnz == 3
    m = a.shape[0]
    assert list(idx[0::m]) == [1, 3, 0] and list(data[0::m]) == [2.0, 3.0, 0.0]
    assert list(idx[1::m]) == [0, 0, 0] and list(data[1::m]) == [1.0, 0.0, 0.0]
    assert list(idx[2::m]) == [0, 1, 2] and list(data[2::m]) == [4.0, 5.0, 6.0]
    meta, arr = load("mixed_pritet_p3")
    for t in meta["types"]:
        op = arr["t%d_opp_3" % t["ele_type"]]
        d, ix, nz = SM.ellpack(op)
        back = np.zeros_like(op)
        for s in range(nz):
            for i in range(op.shape[0]):
                back[i, ix[i + op.shape[0] * s]] += d[i + op.shape[0] * s]
        assert np.array_equal(back, np.where(np.abs(op) >= 1e-12, op, 0.0))


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["mixed_pritet_p3", "mixed_hexpri_p3"])
def test_sparse_operator_product_matches_the_reference(case):
    """fr_op_spmv_ell (bespoke_SPMV) on the reference's own operators in ELL
    form: the extrapolation (add_flag 0) and the corrected divergence
    (add_flag 1) of every element type against the reference's stage arrays."""
    torch = pytest.importorskip("torch")
    import hifiles_b200 as H
    import hifiles_b200.seam as SM
    L = SM._bind(H.lib())
    meta, a = load(case)
    dev = lambda x: torch.from_numpy(np.asfortranarray(x).ravel(order="F").copy()).cuda()  # noqa: E731
    for t in meta["types"]:
        X = "t%d_" % t["ele_type"]
        nu, nf, E, F = t["n_upts"], t["n_fpts"], t["n_eles"], 5
        d0, i0, z0 = SM.ellpack(a[X + "opp_0"])
        d3, i3, z3 = SM.ellpack(a[X + "opp_3"])
        # device copies stay referenced until the products have run
        D0, I0, D3, I3 = dev(d0), dev(i0), dev(d3), dev(i3)
        u = dev(a[X + "disu_upts_init"])
        ufp = torch.zeros(nf * E * F, dtype=torch.float64, device="cuda")
        st = L.fr_op_spmv_ell(nf, nu, F, E, D0.data_ptr(), I0.data_ptr(), z0, u.data_ptr(), ufp.data_ptr(),
                              t["ele_type"], meta["order"], 0, None)
        assert st == 0, H.lib().fr_last_error().decode()
        jump = dev(a[X + "s10_norm_tconf_fpts"] - a[X + "s08_norm_tdisf_fpts"])
        div = dev(a[X + "s09_div_tconf_upts"])
        st = L.fr_op_spmv_ell(nu, nf, F, E, D3.data_ptr(), I3.data_ptr(), z3, jump.data_ptr(),
                              div.data_ptr(), t["ele_type"], meta["order"], 1, None)
        assert st == 0, H.lib().fr_last_error().decode()
        torch.cuda.synchronize()
        got0 = ufp.cpu().numpy().reshape((nf, E, F), order="F")
        got3 = div.cpu().numpy().reshape((nu, E, F), order="F")
        assert rel(got0, a[X + "s01_disu_fpts"]) <= 1e-12
        assert rel(got3, a[X + "s11_div_tconf_upts"]) <= 1e-12
