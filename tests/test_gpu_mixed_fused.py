"""The fused mixed-mesh stage (fr_mixed_stage_*, hifiles_b200.seam.FusedMixedMesh):
tets, prisms, hexes, triangles and quads advanced by one gradient kernel and one
interface/update kernel per element type and RK stage, operator products on
the FP64 tensor cores.

GPU tests:
  * on the reference-made fixtures (tests/golden/mixed_*.npz, written by
    tests/golden/make_mixed.py from runs of the reference itself): the
    residual div_tconf_upts of the initial state and the state after the
    fixture's RK45 steps, against the reference's, at 1e-12;
  * on the library's own set-up of the fixture meshes: the same final state;
  * on a small jittered channel built by hifiles_b200.mixed (prism walls, tet
    core): residual and state after three steps against the per-operator
    path (MixedOperatorMesh) at 1e-12.

CPU tests: the create call's argument checks, which run before any device
work."""
import ctypes as C

import numpy as np
import pytest

from golden_util import load, rel

FR_ERR_ARG, FR_ERR_UNSUPPORTED = 1, 5  # fr_status codes of include/fr_b200.h
FUSED = ["mixed_pritet_p3", "mixed_pritet_p2", "mixed_hexpri_p3", "mixed_channel_p2", "mixed_channel_p3",
         "mixed_triquad_p2", "mixed_triquad_p3"]


def _div(m, i):
    s = m.S[i]
    return s["div"].cpu().numpy().reshape((s["nu"], s["E"], m.F), order="F")


# quadrilateral boxes with a boundary on every side, made by the reference:
# Euler with characteristic / subsonic outflow / slip wall / dual-consistent
# slip wall and with simple and supersonic in- and outflow, Navier-Stokes with
# characteristic in- and outflow and moving isothermal and adiabatic walls,
# the Roe flux with boundaries and periodic
SEAM_2D = ["seam_quad_bc_euler_p3", "seam_quad_bc_euler2_p2", "seam_quad_ns_bc_p3", "seam_quad_roe_bc_p3",
           "seam_quad_roe_p3_jit"]


@pytest.mark.gpu
@pytest.mark.parametrize("case", FUSED + SEAM_2D)
def test_fused_stage_matches_the_reference(case):
    torch = pytest.importorskip("torch")
    from hifiles_b200 import seam
    meta, a = load(case)
    types, ints, bdys = seam.mixed_mesh_inputs(meta, a)
    m = seam.FusedMixedMesh(types, ints, meta["physics"], bdys, meta["bdy"], meta["R_ref"],
                            viscous=bool(meta.get("viscous", 1)), riemann=int(meta.get("riemann", 0)))
    assert m.launches_per_stage == 2 * len(types)
    m.residual()
    torch.cuda.synchronize()
    for t in meta["types"]:
        got = _div(m, t["index"])
        assert np.isfinite(got).all()
        assert rel(got, a["t%d_s11_div_tconf_upts" % t["ele_type"]]) <= 1e-12, (case, t["ele_type"])
    for step in range(meta["steps"]):
        # the L1 residual norms of each step, as the reference's CalcNormResidual
        norms = m.advance(1, meta["dt"], norms=True)
        want = a["res_norms"][:, step]
        assert np.all(np.abs(norms - want) <= 1e-12 * np.abs(want)), (case, step, norms, want)
    for t in meta["types"]:
        got = m.get_state(t["index"])
        assert rel(got, a["t%d_final_disu_upts0" % t["ele_type"]]) <= 1e-12, (case, t["ele_type"])


@pytest.mark.gpu
@pytest.mark.parametrize("case", FUSED)
def test_fused_stage_with_own_setup_advances_like_the_reference(case):
    pytest.importorskip("torch")
    from hifiles_b200 import mixed as X
    from hifiles_b200 import seam
    from test_mixed_setup import fixture_mesh
    meta, a = load(case)
    xv, cells, period, bfaces, opts = fixture_mesh(meta)
    M = X.MixedMesh(meta["order"], xv, cells, period, bfaces, opts)
    types, ints, bdys = M.operator_inputs({t: a["t%d_disu_upts_init" % t] for t in M.types})
    m = seam.FusedMixedMesh(types, ints, meta["physics"], bdys, meta["bdy"], meta["R_ref"])
    m.advance(meta["steps"], meta["dt"])
    for t in M.types:
        assert rel(m.get_state(t), a["t%d_final_disu_upts0" % t]) <= 1e-12, (case, t)


CHANNEL_PHYSICS = {"gamma": 1.4, "prandtl": 0.71, "mu_inf": 0.000625, "rt_inf": 69.32142857142854,
                   "c_sth": 0.41215868109222054, "fix_vis": 1.0, "tau": 1.0, "pen_fact": 0.5}
CHANNEL_BDY = [1.0, 1.0, 0.0, 0.0, 71.4285714285714, 0.0, 0.0, 0.0, 1.0, 71.92982267888384, 1.002, 1.0, 0.0, 0.0]


def _channel_state(pos):
    """Mach 0.1 channel flow with a seeded, smooth perturbation."""
    x, y, z = pos[..., 0], pos[..., 1], pos[..., 2]
    rho = 1.0 + 0.01 * np.sin(x) * np.cos(z)
    u = 0.1 * y * (2.0 - y) + 0.01 * np.sin(z) * np.sin(np.pi * y / 2.0)
    v = 0.01 * np.sin(x) * np.sin(np.pi * y / 2.0)
    w = 0.01 * np.cos(x) * y * (2.0 - y)
    p = 71.4285714285714 + 0.01 * np.cos(x + z)
    e = p / 0.4 + 0.5 * rho * (u * u + v * v + w * w)
    return np.stack([rho, rho * u, rho * v, rho * w, e], axis=-1)


@pytest.mark.gpu
@pytest.mark.parametrize("order", [2, 3])
def test_fused_channel_matches_the_operator_path(order):
    """A 6 x 4 x 4 jittered channel (prism walls, tet core, isothermal and
    adiabatic walls) set up by the library: the fused stage and the
    per-operator path give the same residual and the same state after three
    RK45 steps."""
    torch = pytest.importorskip("torch")
    from hifiles_b200 import mixed as X
    from hifiles_b200 import seam
    xv, cells, period, bfaces = X.channel_mesh((6, 4, 4))
    M = X.MixedMesh(order, xv, cells, period, bfaces,
                    X.ElementOpts(vcjh_scheme_tet=2, vcjh_scheme_tri=1, vcjh_scheme_pri_1d=1))
    types, ints, bdys = M.operator_inputs({t: _channel_state(m["pos_upts"]) for t, m in M.types.items()})
    ref = seam.MixedOperatorMesh(types, ints, CHANNEL_PHYSICS, bdys, CHANNEL_BDY, 71.42857142857142)
    fus = seam.FusedMixedMesh(types, ints, CHANNEL_PHYSICS, bdys, CHANNEL_BDY, 71.42857142857142)
    ref.residual()
    fus.residual()
    torch.cuda.synchronize()
    for t in M.types:
        s = ref.S[t]
        want = s["div"].cpu().numpy().reshape((s["nu"], s["E"], 5), order="F")
        assert rel(_div(fus, t), want) <= 1e-12, (order, t)
    ref.advance(3, 2e-4)
    fus.advance(3, 2e-4)
    for t in M.types:
        got, want = fus.get_state(t), ref.get_state(t)
        assert np.isfinite(got).all()
        assert rel(got, want) <= 1e-12, (order, t)


def test_fused_stage_rejects_unsupported_meshes():
    """1-D meshes and element shapes without kernels are refused before any
    device work, with a reason."""
    import hifiles_b200 as H
    from hifiles_b200 import seam
    L = seam._bind_stage(H.lib())
    ph = seam.PhysDesc(**CHANNEL_PHYSICS)
    d = (seam._MixedStageType * 1)()
    h = C.c_void_p()
    st = L.fr_mixed_stage_create(1, 1, d, 0, None, None, None, 0, None, None, None, None, 1.0, C.byref(ph), 1, 0,
                                 C.byref(h))
    assert st == FR_ERR_UNSUPPORTED and "3-D" in H.lib().fr_last_error().decode()
    # a hex of order 4 (125 solution, 150 flux points) has no kernels
    keep = [np.zeros(9 * 125 * 150)]
    p = keep[0].ctypes.data
    d[0].n_upts, d[0].n_fpts, d[0].n_eles = 125, 150, 1
    d[0].opp_0 = d[0].opp_3 = d[0].opp_6 = d[0].JGinv_upts = d[0].detjac_upts = d[0].tdA_fpts = p
    d[0].norm_fpts = d[0].disu_upts = p
    for name in ("opp_1", "opp_2", "opp_4", "opp_5"):
        arr = getattr(d[0], name)
        for q in range(3):
            arr[q] = p
    st = L.fr_mixed_stage_create(3, 1, d, 0, None, None, None, 0, None, None, None, None, 1.0, C.byref(ph), 1, 0,
                                 C.byref(h))
    assert st == FR_ERR_UNSUPPORTED and "125" in H.lib().fr_last_error().decode()
    d[0].n_upts = 0
    st = L.fr_mixed_stage_create(3, 1, d, 0, None, None, None, 0, None, None, None, None, 1.0, C.byref(ph), 1, 0,
                                 C.byref(h))
    assert st == FR_ERR_ARG
    assert not h.value


@pytest.mark.gpu
def test_fused_launch_shapes_give_the_same_bits():
    """Every launch shape of the two stage kernels, and one stream instead of
    side streams per element type, end on the same state bit for bit;
    autotune() leaves the state as it was."""
    torch = pytest.importorskip("torch")
    from hifiles_b200 import seam
    meta, a = load("mixed_channel_p3")
    types, ints, bdys = seam.mixed_mesh_inputs(meta, a)
    out = {}
    for shapes in ((0, 0), (1, 1), (2, 2), (3, 0), (4, 1), (1, 0), (0, 2)):
        m = seam.FusedMixedMesh(types, ints, meta["physics"], bdys, meta["bdy"], meta["R_ref"])
        for i in m.S:
            m.set_launch(i, *shapes)
            assert m.launch(i) == shapes
        m.advance(2, meta["dt"])
        out[shapes] = {i: m.get_state(i) for i in m.S}
    m = seam.FusedMixedMesh(types, ints, meta["physics"], bdys, meta["bdy"], meta["R_ref"])
    m.set_concurrent(False)
    m.advance(2, meta["dt"])
    out["one stream"] = {i: m.get_state(i) for i in m.S}
    for shapes, st in out.items():
        for i in st:
            assert np.array_equal(st[i], out[(0, 0)][i]), shapes
    m = seam.FusedMixedMesh(types, ints, meta["physics"], bdys, meta["bdy"], meta["R_ref"])
    before = {i: m.get_state(i) for i in m.S}
    picked = m.autotune()
    torch.cuda.synchronize()
    for i in m.S:
        assert np.array_equal(m.get_state(i), before[i])
        assert 0 <= picked[i][0] < 5 and 0 <= picked[i][1] < 3


def test_fused_stage_rejects_bad_wiring_before_device_work():
    """Interface and boundary tables are checked on the host before anything
    is allocated: a flux point wired twice or on no interface, entries out of
    range, unknown boundary types."""
    import hifiles_b200 as H
    from hifiles_b200 import seam
    L = seam._bind_stage(H.lib())
    ph = seam.PhysDesc(**CHANNEL_PHYSICS)
    nu, nf, E = 10, 24, 2  # two tets of order 2
    keep = [np.zeros(9 * nu * nf * E)]
    p = keep[0].ctypes.data
    d = (seam._MixedStageType * 1)()
    d[0].n_upts, d[0].n_fpts, d[0].n_eles = nu, nf, E
    d[0].opp_0 = d[0].opp_3 = d[0].opp_6 = d[0].JGinv_upts = d[0].detjac_upts = d[0].tdA_fpts = p
    d[0].norm_fpts = d[0].disu_upts = p
    for name in ("opp_1", "opp_2", "opp_4", "opp_5"):
        arr = getattr(d[0], name)
        for q in range(3):
            arr[q] = p

    def create(ints=(), bdys=()):
        def pack(ws):
            ws = [np.asfortranarray(w, dtype=np.int32) for w in ws]
            keep.extend(ws)
            n = max(len(ws), 1)
            return (len(ws), (C.c_void_p * n)(*[w.ctypes.data for w in ws]),
                    (C.c_int * n)(*[w.shape[1] for w in ws]), (C.c_longlong * n)(*[w.shape[2] for w in ws]))
        ni, ip, inf, inn = pack(ints)
        nb, bp, bnf, bnn = pack(bdys)
        h = C.c_void_p()
        st = L.fr_mixed_stage_create(3, 1, d, ni, ip, inf, inn, nb, bp, bnf, bnn, None, 1.0, C.byref(ph), 1, 0,
                                     C.byref(h))
        assert not h.value
        return st, H.lib().fr_last_error().decode()

    def inter(pairs):
        w = np.zeros((6, 1, len(pairs)), dtype=np.int32)
        for j, (t0, e0, f0, t1, e1, f1) in enumerate(pairs):
            w[:, 0, j] = (t0, e0, f0, t1, e1, f1)
        return w

    full = [(0, 0, f, 0, 1, f) for f in range(nf)]
    st, msg = create([inter(full[:-1] + [full[0]])])
    assert st == 6 and "twice" in msg
    st, msg = create([inter(full[:-1])])
    assert st == 6 and "no interface" in msg
    st, msg = create([inter(full[:-1] + [(0, 2, 0, 0, 1, 23)])])
    assert st == 6 and "out of range" in msg
    st, msg = create([inter(full[:-1] + [(1, 0, 23, 0, 1, 23)])])
    assert st == 6 and "out of range" in msg
    b = np.zeros((4, 1, 2), dtype=np.int32)
    b[:, 0, 0] = (0, 0, 23, 9)
    b[:, 0, 1] = (0, 1, 23, 7)
    st, msg = create([inter(full[:-1])], [b])
    assert st == 5 and "boundary type 9" in msg


def _smooth_state(pos, dims):
    """A smooth Mach-0.1-like state at points pos (n, E, dims)."""
    x, y = pos[..., 0], pos[..., 1]
    z = pos[..., 2] if dims == 3 else 0.0 * x
    rho = 1.0 + 0.05 * np.sin(x) * np.cos(y)
    u, v, w = 1.0 + 0.1 * np.sin(y), 0.1 * np.cos(x), 0.05 * np.sin(x + y + z)
    p = 71.4285714285714 * (1.0 + 0.01 * np.cos(x + y))
    if dims == 2:
        return np.stack([rho, rho * u, rho * v, p / 0.4 + 0.5 * rho * (u * u + v * v)], -1)
    return np.stack([rho, rho * u, rho * v, rho * w, p / 0.4 + 0.5 * rho * (u * u + v * v + w * w)], -1)


@pytest.mark.gpu
@pytest.mark.parametrize("case,order", [("mixed_pritet_p3", 1), ("mixed_pritet_p3", 4), ("mixed_channel_p3", 1),
                                        ("mixed_channel_p3", 4), ("mixed_hexpri_p3", 1), ("mixed_triquad_p3", 1),
                                        ("mixed_triquad_p3", 4)])
def test_fused_orders_1_and_4_match_the_operator_path(case, order):
    """Orders 1 and 4 on the fixture meshes, set up by the library: the fused
    stage's residual and its state after two RK45 steps match the
    per-operator path's (the entry points pinned against the reference at
    orders 2 and 3) at 1e-12."""
    torch = pytest.importorskip("torch")
    from hifiles_b200 import mixed as X
    from hifiles_b200 import seam
    from test_mixed_setup import fixture_mesh
    meta, _ = load(case)
    meta = dict(meta, order=order)
    dims = int(meta.get("dims", 3))
    xv, cells, period, bfaces, opts = fixture_mesh(meta)
    opts.vcjh_scheme_tet = opts.vcjh_scheme_tri = 1  # DG: defined at every order
    M = X.MixedMesh(order, xv, cells, period, bfaces, opts)
    types, ints, bdys = M.operator_inputs({t: _smooth_state(m["pos_upts"], dims) for t, m in M.types.items()})
    ref = seam.MixedOperatorMesh(types, ints, meta["physics"], bdys, meta["bdy"], meta["R_ref"])
    fus = seam.FusedMixedMesh(types, ints, meta["physics"], bdys, meta["bdy"], meta["R_ref"])
    ref.residual()
    fus.residual()
    torch.cuda.synchronize()
    for t in M.types:
        s = ref.S[t]
        want = s["div"].cpu().numpy().reshape((s["nu"], s["E"], dims + 2), order="F")
        assert rel(_div(fus, t), want) <= 1e-12, (case, order, t)
    ref.advance(2, meta["dt"])
    fus.advance(2, meta["dt"])
    for t in M.types:
        got, want = fus.get_state(t), ref.get_state(t)
        assert np.isfinite(got).all()
        assert rel(got, want) <= 1e-12, (case, order, t)
