"""The library's own set-up of tetrahedra, prisms and hexahedra
(fr_element_operators, fr_mixed_*; hifiles_b200.mixed) against what the
reference's element and interface classes computed for the same meshes.

The fixtures tests/golden/mixed_*.npz hold the reference's operators
opp_0 .. opp_6 per element type (eles_tets / eles_pris / eles_hexas set-up),
its metrics and its interface and boundary tables, for jittered periodic and
walled meshes that tests/golden/make_mixed.py wrote (mixed_cells, seed 12345).
Here the same meshes go through the library's host set-up instead:

  * operators: opp_0, opp_1, opp_2 (= opp_4) and opp_6 to 1e-13 of their
    largest entry, opp_3 and opp_5 to 1e-12.  The largest differences
    (up to 8e-13, prisms' quadrilateral faces) are the reference's: it
    interpolates each edge's correction polynomial in Jacobi polynomials of
    the edge length coordinate t in [0, 2 sqrt 2] (src/funcs.cpp:806-893), a
    badly conditioned basis.  test_triangle_lift_is_exact checks the
    library's lift against an independent quadrature to 1e-13, where the
    reference's misses by 8e-13;
  * metrics (JGinv, detJ, tdA, normals): bit for bit;
  * wiring: the same interface points, with the same left and right sides,
    and the same boundary points.

The GPU test runs three RK45 steps of each fixture mesh through the
per-operator entry points with the library's own set-up and compares the
state with the reference's."""
import json
import os
import sys

import numpy as np
import pytest

from golden_util import load, rel

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_mixed as MM  # noqa: E402
from hifiles_b200 import mixed as X  # noqa: E402

CASES = ["mixed_pritet_p3", "mixed_pritet_p2", "mixed_hexpri_p3", "mixed_channel_p2", "mixed_channel_p3",
         "mixed_triquad_p3", "mixed_triquad_p2"]
# Gambit hex node g sits in the reference's hex slot k = G2I.index(g)
# (src/geometry.cpp:1860-1866)
G2I = [0, 4, 1, 5, 2, 6, 3, 7]


def fixture_mesh(meta):
    """(xv, cells, period, bfaces, opts) of a fixture's mesh in the library's
    terms, from the same generator and seed the fixture writer used."""
    if meta["kind"] == "triquad":
        lo, hi = (0.0, 0.0), (2 * np.pi, 2 * np.pi)
        xv, eles = MM.mixed_cells_2d(meta["n"], lo, hi, meta["jitter"], seed=12345)
        cells = [({3: X.TRI, 2: X.QUAD}[gt], list(vs)) for gt, vs, _ in eles]
        opts = X.ElementOpts(upts_type_tri=meta["tri_upts"], fpts_type_tri=meta["tri_fpts"],
                             vcjh_scheme_tri=meta["vcjh_tri"], upts_type_quad=0, vcjh_scheme_quad=1)
        return xv, cells, [hi[0] - lo[0], hi[1] - lo[1]], [], opts
    lo, hi = (0.0,) * 3, (2 * np.pi,) * 3
    xv, eles = MM.mixed_cells(meta["kind"], meta["n"], lo, hi, meta["jitter"], seed=12345)
    sbc = meta.get("side_bc", [0] * 6)
    cells, bfaces = [], []
    for ci, (gt, vs, bf) in enumerate(eles):
        t = {6: X.TET, 5: X.PRISM, 4: X.HEX}[gt]
        if t == X.HEX:
            vs = [vs[G2I[k]] for k in range(8)]
        cells.append((t, list(vs)))
        for side, code in bf:
            if sbc[side]:
                table = MM.PRI_GAMBIT if t == X.PRISM else MM.TET_GAMBIT
                bfaces.append((ci, [f for f, c in table.items() if c == code][0], sbc[side]))
    period = [hi[d] - lo[d] if sbc[2 * d] == 0 else 0.0 for d in range(3)]
    opts = X.ElementOpts(upts_type_tet=meta["tet_upts"], fpts_type_tet=0, vcjh_scheme_tet=2, upts_type_pri_tri=0,
                         upts_type_pri_1d=0, vcjh_scheme_tri=1, vcjh_scheme_pri_1d=1, upts_type_hexa=0,
                         vcjh_scheme_hexa=1)
    return xv, cells, period, bfaces, opts


def _maxrel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("case", CASES)
def test_element_operators_match_the_reference(case):
    meta, a = load(case)
    *_, opts = fixture_mesh(meta)
    for t in meta["types"]:
        et = t["ele_type"]
        T = "t%d_" % et
        ops = X.element_operators(et, meta["order"], opts)
        assert ops["opp_0"].shape == a[T + "opp_0"].shape
        assert _maxrel(ops["opp_0"], a[T + "opp_0"]) <= 1e-13
        assert _maxrel(ops["opp_6"], a[T + "opp_6"]) <= 1e-13
        assert _maxrel(ops["opp_3"], a[T + "opp_3"]) <= 1e-12, et
        for w, tol in ((1, 1e-13), (2, 1e-13), (4, 1e-13), (5, 1e-12)):
            for d in range(meta.get("dims", 3)):
                assert _maxrel(ops["opp_%d" % w][d], a[T + "opp_%d_%d" % (w, d)]) <= tol, (et, w, d)


@pytest.mark.parametrize("tag", ["triquad_p1", "triquad_p4", "triquad_p5", "pritet_p1", "pritet_p4", "pritet_p5",
                                 "triquad_p4_s2", "pritet_p4_s3", "pritet_p5_s4"])
def test_element_operators_match_the_reference_at_other_orders(tag):
    """Orders 1, 4 and 5 with the DG correction, and the SD-like, HU-like
    and c_+ schemes at orders 4 and 5, against the reference's own operators,
    metrics and interface wiring (tests/golden/ops_<tag>.npz, make_mixed.py
    --operators).  At order 5 the
    triangle lift (triangles and the prisms' triangular faces) follows the
    reference's 5-point edge rule."""
    z = np.load(os.path.join(HERE, "golden", "ops_%s.npz" % tag))
    meta = json.loads(str(z["meta"]))
    order = meta["order"]
    if meta["kind"] == "triquad":
        opts = X.ElementOpts(upts_type_tri=meta["tri_upts"], fpts_type_tri=meta["tri_fpts"],
                             vcjh_scheme_tri=meta["vcjh_tri"])
        types, D = (X.TRI, X.QUAD), 2
    else:
        opts = X.ElementOpts(upts_type_tet=meta["tet_upts"], vcjh_scheme_tet=meta["vcjh_tet"],
                             vcjh_scheme_tri=meta["vcjh_tri"], vcjh_scheme_pri_1d=1)
        types, D = (X.TET, X.PRISM), 3
    # the metrics of the library's own set-up of the same mesh
    xv, cells, period, bfaces, _ = fixture_mesh(dict(meta, vcjh_tri=meta["vcjh_tri"]))
    M = X.MixedMesh(order, xv, cells, period, bfaces, opts)
    assert sorted(M.types) == sorted(types)
    for et, m in M.types.items():
        for k in ("JGinv_upts", "detjac_upts", "tdA_fpts", "norm_fpts"):
            assert m[k].shape == z["t%d_%s" % (et, k)].shape
            assert rel(m[k], z["t%d_%s" % (et, k)]) <= 1e-15, (et, k)
    # and its interface wiring, left and right sides included
    ref = [z["int_inters_%d" % i] for i in meta["inters"]]
    assert [w.shape for w in M.int_inters] == [w.shape for w in ref]
    for w, r in zip(M.int_inters, ref):
        left_right = lambda x: {tuple(x[:3, q, i]): tuple(x[3:, q, i])  # noqa: E731
                                for i in range(x.shape[2]) for q in range(x.shape[1])}
        assert left_right(w) == left_right(r)
    for et in types:
        T = "t%d_" % et
        ops = X.element_operators(et, order, opts)
        assert ops["opp_0"].shape == z[T + "opp_0"].shape
        assert _maxrel(ops["opp_0"], z[T + "opp_0"]) <= 1e-13
        assert _maxrel(ops["opp_6"], z[T + "opp_6"]) <= 1e-13
        assert _maxrel(ops["opp_3"], z[T + "opp_3"]) <= 1e-12, et
        for w, tol in ((1, 1e-13), (2, 1e-13), (4, 1e-13), (5, 1e-12)):
            for d in range(D):
                assert _maxrel(ops["opp_%d" % w][d], z[T + "opp_%d_%d" % (w, d)]) <= tol, (et, w, d)


def test_triangle_lift_is_exact():
    """The DG lift of a unit jump at edge point m, in the orthonormal basis,
    has the coefficients int_edge phi_i l_m ds; checked with an independent
    20-point Gauss rule and scipy's Jacobi polynomials (prism P = 3, the
    triangle correction of its quadrilateral faces)."""
    from scipy.special import eval_jacobi, gamma
    P, n1, nt = 3, 4, 10
    meta, a = load("mixed_pritet_p3")
    opts = fixture_mesh(meta)[-1]
    ops = X.element_operators(X.PRISM, P, opts)
    tri = ops["loc_upts"][:2, :nt].T
    x1d = ops["loc_upts"][2, ::nt]

    def jac(x, al, be, n):
        g0 = 2 ** (al + be + 1) / (2 * n + al + be + 1) * gamma(n + al + 1) * gamma(n + be + 1) / \
            gamma(n + al + be + 1) / gamma(n + 1)
        return eval_jacobi(n, al, be, x) / np.sqrt(g0)

    def dub2(r, s, i, j):
        aa = np.where(s == 1, -1.0, 2 * (1 + r) / np.where(s == 1, 1.0, 1 - s) - 1)
        return np.sqrt(2) * jac(aa, 0, 0, i) * jac(s, 2 * i + 1, 0, j) * (1 - s) ** i

    modes = [(k - j, j) for k in range(P + 1) for j in range(k + 1)]
    Vi = np.linalg.inv(np.array([[dub2(tri[q, 0], tri[q, 1], *md) for md in modes] for q in range(nt)]))
    gx, gw = np.polynomial.legendre.leggauss(20)

    def lag(x, m):
        v = np.ones_like(x)
        for k in range(n1):
            if k != m:
                v = v * (x - x1d[k]) / (x1d[m] - x1d[k])
        return v

    err = {"library": 0.0, "reference": 0.0}
    for e in range(3):
        half = np.sqrt(2) if e == 1 else 1.0
        r, s = [(gx, -np.ones(20)), (-gx, gx), (-np.ones(20), -gx)][e]
        for m in range(n1):
            exact = np.array([half * np.sum(gw * dub2(r, s, *md) * lag(gx, m)) for md in modes])
            col = 2 * nt + e * n1 * n1 + m
            for name, M in (("library", ops["opp_3"]), ("reference", a["t3_opp_3"])):
                err[name] = max(err[name], _maxrel(Vi @ M[:nt, col], exact))
    print(err)
    assert err["library"] < 1e-13
    assert err["reference"] > err["library"]


@pytest.mark.parametrize("case", CASES)
def test_metrics_and_wiring_match_the_reference(case):
    meta, a = load(case)
    xv, cells, period, bfaces, opts = fixture_mesh(meta)
    M = X.MixedMesh(meta["order"], xv, cells, period, bfaces, opts)
    assert sorted(M.types) == sorted(t["ele_type"] for t in meta["types"])
    for t, m in M.types.items():
        T = "t%d_" % t
        for k in ("JGinv_upts", "detjac_upts", "tdA_fpts", "norm_fpts"):
            assert m[k].shape == a[T + k].shape
            assert rel(m[k], a[T + k]) <= 1e-15, (t, k)
    ref = [a["int_inters_%d" % it["index"]] for it in meta["inters"]]
    assert [w.shape for w in M.int_inters] == [w.shape for w in ref]
    for w, r in zip(M.int_inters, ref):
        left_right = lambda x: {tuple(x[:3, q, i]): tuple(x[3:, q, i])  # noqa: E731
                                for i in range(x.shape[2]) for q in range(x.shape[1])}
        assert left_right(w) == left_right(r)
    refb = [a["bdy_inters_%d" % it["index"]] for it in meta.get("bdy_inters", [])]
    points = lambda ws: {tuple(x) for w in ws for x in np.asarray(w).reshape(4, -1, order="F").T}  # noqa: E731
    assert points(M.bdy_inters) == points(refb)


def test_channel_mesh_is_a_conforming_walled_channel():
    """A small channel of the bench's kind: every cell positive, every
    interior face matched, walls only on the prisms' outer triangles."""
    n = (6, 5, 4)
    xv, cells, period, bfaces = X.channel_mesh(n, jitter=0.15, seed=3)
    ntet = 6 * n[0] * (n[1] - 2) * n[2]
    npri = 2 * n[0] * 2 * n[2]
    assert sum(1 for t, _ in cells if t == X.TET) == ntet
    assert sum(1 for t, _ in cells if t == X.PRISM) == npri
    assert len(bfaces) == npri
    M = X.MixedMesh(2, xv, cells, period, bfaces, X.ElementOpts(vcjh_scheme_tet=2, vcjh_scheme_tri=1,
                                                               vcjh_scheme_pri_1d=1))
    assert all((m["detjac_upts"] > 0).all() for m in M.types.values())
    seen = {t: np.zeros((m["n_fpts"], m["n_eles"]), dtype=int) for t, m in M.types.items()}
    for w in M.int_inters:
        x = w.reshape(6, -1, order="F")
        for s in (0, 3):
            np.add.at(seen[X.TET], (x[s + 2][x[s] == X.TET], x[s + 1][x[s] == X.TET]), 1)
            np.add.at(seen[X.PRISM], (x[s + 2][x[s] == X.PRISM], x[s + 1][x[s] == X.PRISM]), 1)
    for w in M.bdy_inters:
        x = w.reshape(4, -1, order="F")
        assert set(x[0]) == {X.PRISM} and set(x[3]) == {11, 12}
        np.add.at(seen[X.PRISM], (x[2], x[1]), 1)
    assert all((s == 1).all() for s in seen.values())
    assert M.n_dofs == 10 * ntet + 18 * npri


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_own_setup_advances_like_the_reference(case):
    """Three RK45 steps of the fixture mesh through the per-operator entry
    points, with operators, metrics and wiring from the library's set-up:
    the state ends where the reference's ends."""
    pytest.importorskip("torch")
    from hifiles_b200 import seam
    meta, a = load(case)
    xv, cells, period, bfaces, opts = fixture_mesh(meta)
    M = X.MixedMesh(meta["order"], xv, cells, period, bfaces, opts)
    states = {t: a["t%d_disu_upts_init" % t] for t in M.types}
    types, ints, bdys = M.operator_inputs(states)
    mesh = seam.MixedOperatorMesh(types, ints, meta["physics"], bdys, meta["bdy"], meta["R_ref"])
    mesh.advance(meta["steps"], meta["dt"])
    for t in M.types:
        got = mesh.get_state(t)
        assert rel(got, a["t%d_final_disu_upts0" % t]) <= 1e-12, (case, t)


def test_mixed_setup_rejects_bad_input():
    """Unmatched faces, inverted cells, unknown types and boundary codes are
    reported through fr_status, never by exiting."""
    import hifiles_b200 as H
    xv, cells, period, bfaces = X.channel_mesh((3, 3, 2), jitter=0.0, seed=1)
    opts = X.ElementOpts(vcjh_scheme_tet=2, vcjh_scheme_tri=1, vcjh_scheme_pri_1d=1)
    # walls removed: the prisms' outer faces are left unmatched
    with pytest.raises(H.FrError, match="unmatched"):
        X.MixedMesh(2, xv, cells, period, [], opts)
    # an inverted tet
    bad = list(cells)
    i = next(i for i, (t, _) in enumerate(bad) if t == X.TET)
    t, vs = bad[i]
    bad[i] = (t, [vs[0], vs[2], vs[1], vs[3]])
    with pytest.raises(H.FrError, match="Jacobian"):
        X.MixedMesh(2, xv, bad, period, bfaces, opts)
    # unknown boundary type
    with pytest.raises(H.FrError):
        X.MixedMesh(2, xv, cells, period, [(bfaces[0][0], bfaces[0][1], 9)] + list(bfaces[1:]), opts)
    # orders outside the simplex tables, schemes without constants
    with pytest.raises(H.FrError):
        X.element_operators(X.TET, 6)
    with pytest.raises(H.FrError):
        X.element_operators(X.TRI, 5, X.ElementOpts(vcjh_scheme_tri=2))
    # mixing 2-D and 3-D cells
    with pytest.raises(ValueError):
        X.MixedMesh(2, xv, [(X.TRI, [0, 1, 2, 3])], period, [], opts)


@pytest.mark.parametrize("ele_type,P", [(X.TRI, 1), (X.TRI, 4), (X.QUAD, 2), (X.TET, 1), (X.TET, 4), (X.PRISM, 1),
                                        (X.PRISM, 5), (X.HEX, 2)])
def test_element_operators_are_consistent(ele_type, P):
    """Properties every FR element's operators have: the nodal basis is a
    partition of unity (opp_0 rows sum to 1), derivatives of a constant vanish
    (opp_2 rows sum to 0), and opp_1 / opp_5 are opp_0 / opp_3 times the
    reference normals."""
    ops = X.element_operators(ele_type, P, X.ElementOpts(vcjh_scheme_tet=1, vcjh_scheme_tri=1,
                                                          vcjh_scheme_pri_1d=1))
    D = ops["loc_upts"].shape[0]
    assert np.allclose(ops["opp_0"].sum(axis=1), 1.0, atol=1e-12)
    for d in range(D):
        assert np.allclose(ops["opp_2"][d].sum(axis=1), 0.0, atol=1e-11)
        assert np.allclose(ops["opp_1"][d], ops["opp_0"] * ops["tnorm_fpts"][d][:, None], atol=0, rtol=0)
        assert np.allclose(ops["opp_5"][d], ops["opp_3"] * ops["tnorm_fpts"][d][None, :], atol=0, rtol=0)
    # the nodal basis at the solution points is the identity
    nu = ops["opp_0"].shape[1]
    assert ops["opp_2"][0].shape == (nu, nu)
