"""Restart files of triangles, tets and prisms (fr_restart_write /
fr_restart_read_points, host only) against the files the reference itself
wrote for the mixed fixtures (write_restart, src/output.cpp:1057-1107, with
write_restart_info of src/eles_tris.cpp:546-563, src/eles_tets.cpp:782-800,
src/eles_pris.cpp:700-726), and reading at another order through the nodal
basis on the file's points (eles::set_opp_r, src/eles.cpp:4135-4153).

The element ids of each block are taken from the reference's file; values
cross the file as 15 significant digits, so states are compared at 1e-14
normwise relative; files are compared byte for byte."""
import json
import os

import numpy as np
import pytest

import hifiles_b200 as H
import oracle as O
from golden_util import GOLDEN, rel
from hifiles_b200 import mixed as X

NAMES = {0: "TRIS", 1: "QUADS", 2: "TETS", 3: "PRIS", 4: "HEXAS"}


def fixture(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    meta = json.loads(str(z["meta"]))
    if meta["kind"] == "triquad":
        opts = X.ElementOpts(upts_type_tri=meta["tri_upts"], fpts_type_tri=meta["tri_fpts"])
    else:
        opts = X.ElementOpts(upts_type_tet=meta["tet_upts"], vcjh_scheme_tet=2, vcjh_scheme_tri=1,
                             vcjh_scheme_pri_1d=1)
    return meta, z, opts


def file_ids(path, ele_type):
    """The ele2global array of one block of a restart file."""
    lines = open(path).read().split("\n")
    i = lines.index(NAMES[ele_type])
    j = lines.index("ele2global_ele array", i)
    return np.array([int(v) for v in lines[j + 1].split()], dtype=np.int32)


def blocks(meta, z, opts, path):
    out = []
    for t in meta["types"]:
        et, P = t["ele_type"], meta["order"]
        b = dict(ele_type=et, order=P, disu_upts=z["t%d_final_disu_upts0" % t["index"]],
                 ele2global=file_ids(path, et))
        if et in (1, 4):
            b["loc_1d"] = O.points_1d(P)
        else:
            b["loc_pts"] = X.element_operators(et, P, opts)["loc_upts"].T
        out.append(b)
    return out


CASES = ["mixed_triquad_p2", "mixed_pritet_p2", "mixed_hexpri_p3"]


@pytest.mark.parametrize("name", CASES)
def test_writer_reproduces_reference_mixed_file_byte_for_byte(name, tmp_path):
    meta, z, opts = fixture(name)
    path = os.path.join(GOLDEN, "rest_%s.dat" % name)
    out = tmp_path / "Rest.dat"
    bl = blocks(meta, z, opts, path)
    H.restart_write(out, meta["steps"] * meta["dt"], bl[::-1])      # any block order: types go in code order
    assert out.read_bytes() == open(path, "rb").read()


@pytest.mark.parametrize("name", CASES)
def test_reader_on_reference_mixed_file_gives_reference_state(name):
    meta, z, opts = fixture(name)
    path = os.path.join(GOLDEN, "rest_%s.dat" % name)
    for b in blocks(meta, z, opts, path):
        et = b["ele_type"]
        pts = b.get("loc_pts")
        if pts is None:                                # quads, hexes: tensor points, x fastest
            n1, D = meta["order"] + 1, 2 if et == 1 else 3
            x = O.points_1d(meta["order"])
            pts = np.array([[x[(j // n1 ** d) % n1] for d in range(D)] for j in range(n1 ** D)])
        u, t = H.restart_read_points(path, et, pts, b["disu_upts"].shape[1], b["disu_upts"].shape[2],
                                     ele2global=b["ele2global"])
        assert abs(t - meta["steps"] * meta["dt"]) < 1e-12
        assert rel(u, b["disu_upts"]) <= 1e-14


def _block(et, order, pts, u):
    b = dict(ele_type=et, order=order, disu_upts=u)
    if et in (1, 4):
        b["loc_1d"] = pts[:order + 1, 0]
    else:
        b["loc_pts"] = pts
    return b


@pytest.mark.parametrize("et", [0, 1, 2, 3, 4])
def test_another_order_carries_polynomials_exactly(et, tmp_path):
    """A field of degree <= 2 written at order 2 and read at order 3 equals
    the field at the order-3 points, and reading those back at order 2
    returns what was written."""
    opts = X.ElementOpts(upts_type_tet=1, vcjh_scheme_tet=2, vcjh_scheme_tri=1, vcjh_scheme_pri_1d=1)
    p2 = X.element_operators(et, 2, opts)["loc_upts"].T.copy()
    p3 = X.element_operators(et, 3, opts)["loc_upts"].T.copy()
    rng = np.random.default_rng(7)
    ne, F = 5, 4
    c = rng.normal(size=(ne, F, 10))

    def field(p):
        x, y = p[:, 0], p[:, 1]
        zz = p[:, 2] if p.shape[1] == 3 else 0.0 * x
        mon = np.stack([np.ones_like(x), x, y, zz, x * x, x * y, y * y, x * zz, y * zz, zz * zz])
        return np.einsum("efm,mj->jef", c, mon)

    u2 = np.asfortranarray(field(p2))
    f1 = tmp_path / "Rest2.dat"
    H.restart_write(f1, 1.5, [_block(et, 2, p2, u2)])
    u3, t = H.restart_read_points(f1, et, p3, ne, F)
    assert t == 1.5
    assert rel(u3, field(p3)) <= 1e-13
    f2 = tmp_path / "Rest3.dat"
    H.restart_write(f2, 1.5, [_block(et, 3, p3, u3)])
    u2b, _ = H.restart_read_points(f2, et, p2, ne, F)
    assert rel(u2b, u2) <= 1e-13


def test_mixed_reader_and_writer_errors(tmp_path):
    path = os.path.join(GOLDEN, "rest_mixed_triquad_p2.dat")
    meta, z, opts = fixture("mixed_triquad_p2")
    p2 = X.element_operators(0, 2, opts)["loc_upts"].T
    ids = file_ids(path, 0)
    with pytest.raises(H.FrError):
        H.restart_read_points(path, 2, np.zeros((10, 3)), 4, 4)        # no TETS block
    with pytest.raises(H.FrError):
        H.restart_read_points(path, 0, p2, 17, 4)                      # ids 0..16: not all in the file
    with pytest.raises(ValueError):
        H.restart_read_points(path, 0, p2.T, 16, 4, ele2global=ids)    # points must be (n_upts, dims)
    with pytest.raises(H.FrError, match="4 fields per point, not 5"):
        H.restart_read_points(path, 0, p2, 16, 5, ele2global=ids)      # a 2-D file has 4 fields
    u = np.zeros((6, 2, 4), order="F")
    with pytest.raises(H.FrError):                                    # triangles need their points
        H.restart_write(tmp_path / "a.dat", 0.0, [dict(ele_type=0, order=2, disu_upts=u)])
    with pytest.raises(H.FrError):                                    # one block per type
        H.restart_write(tmp_path / "a.dat", 0.0, [dict(ele_type=0, order=2, loc_pts=p2, disu_upts=u)] * 2)
    with pytest.raises(H.FrError):                                    # 6 points are order 2
        H.restart_write(tmp_path / "a.dat", 0.0, [dict(ele_type=0, order=3, loc_pts=p2, disu_upts=u)])
    # global ids select the elements: reversed ids give the reversed state
    want = z["t0_final_disu_upts0"]
    u, _ = H.restart_read_points(path, 0, p2, 16, 4, ele2global=ids[::-1].copy())
    assert rel(u, want[:, ::-1, :]) <= 1e-14


@pytest.mark.parametrize("name", CASES)
def test_mixed_mesh_writes_the_reference_file(name, tmp_path):
    """The library's own set-up of the fixture mesh (cell order = the
    reference's element ids) writes the reference's file from the
    reference's final state."""
    from test_mixed_setup import fixture_mesh
    meta, z, _ = fixture(name)
    xv, cells, period, bfaces, opts = fixture_mesh(meta)
    M = X.MixedMesh(meta["order"], xv, cells, period, bfaces, opts)
    out = tmp_path / "Rest.dat"
    M.write_restart(out, meta["steps"] * meta["dt"], {t: z["t%d_final_disu_upts0" % t] for t in M.types})
    assert out.read_bytes() == open(os.path.join(GOLDEN, "rest_%s.dat" % name), "rb").read()
    u, t = M.read_restart(out)
    assert abs(t - meta["steps"] * meta["dt"]) < 1e-15
    for et in M.types:
        assert rel(u[et], z["t%d_final_disu_upts0" % et]) <= 1e-14


@pytest.mark.parametrize("name", CASES)
def test_mixed_mesh_reads_a_file_of_another_order(name, tmp_path):
    """A quadratic field of the physical coordinates, written from the
    order-2 mesh, read by the order-3 mesh of the same cells: every element
    type's map is at most bilinear, so the field lies in both spaces and
    arrives exactly at the order-3 points."""
    from test_mixed_setup import fixture_mesh
    meta, _, _ = fixture(name)
    xv, cells, period, bfaces, opts = fixture_mesh(meta)
    M2 = X.MixedMesh(2, xv, cells, period, bfaces, opts)
    M3 = X.MixedMesh(3, xv, cells, period, bfaces, opts)
    D = M2.dims
    rng = np.random.default_rng(3)
    c = rng.normal(size=(D + 2, 1 + D + D * D))

    def field(pos):                                    # pos (n_upts, n_eles, D)
        mon = [np.ones(pos.shape[:2])] + [pos[..., d] for d in range(D)] + \
              [pos[..., d] * pos[..., e] for d in range(D) for e in range(D)]
        return np.asfortranarray(np.stack([sum(ck * m for ck, m in zip(c[k], mon)) for k in range(D + 2)], axis=-1))

    out = tmp_path / "Rest.dat"
    M2.write_restart(out, 0.25, {t: field(m["pos_upts"]) for t, m in M2.types.items()})
    u, t = M3.read_restart(out)
    assert t == 0.25
    for et, m in M3.types.items():
        assert rel(u[et], field(m["pos_upts"])) <= 1e-12, et


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_fused_run_continues_from_a_restart_file(name, tmp_path):
    """The fused stage, restarted from the reference's restart file (state
    after the fixture's steps) and from this library's own file of the same
    run, continues like the uninterrupted run: 15 digits through the file
    keep the next two steps within 1e-12 (normwise relative)."""
    pytest.importorskip("torch")
    from hifiles_b200 import seam
    from test_mixed_setup import fixture_mesh
    meta, z, _ = fixture(name)
    xv, cells, period, bfaces, opts = fixture_mesh(meta)
    M = X.MixedMesh(meta["order"], xv, cells, period, bfaces, opts)

    def fused(states):
        types, ints, bdys = M.operator_inputs(states)
        return seam.FusedMixedMesh(types, ints, meta["physics"], bdys, meta["bdy"], meta["R_ref"])

    m1 = fused({t: z["t%d_disu_upts_init" % t] for t in M.types})
    m1.advance(meta["steps"], meta["dt"])
    ours = tmp_path / "Rest.dat"
    M.write_restart(ours, meta["steps"] * meta["dt"], {t: m1.get_state(t) for t in M.types})
    m1.advance(2, meta["dt"])
    for path in (os.path.join(GOLDEN, "rest_%s.dat" % name), ours):
        u, t = M.read_restart(path)
        assert abs(t - meta["steps"] * meta["dt"]) < 1e-15
        m2 = fused(u)
        m2.advance(2, meta["dt"])
        for et in M.types:
            assert rel(m2.get_state(et), m1.get_state(et)) <= 1e-12, (path, et)


@pytest.mark.parametrize("name,order", [("mixed_triquad_p2", 3), ("mixed_pritet_p2", 3), ("mixed_hexpri_p3", 2)])
def test_order_change_matches_the_reference_reading_its_own_file(name, order):
    """The reference set up at another order on a fixture's mesh, restarted
    from its own restart file (rest_read_<kind>_p<a>_to_p<b>.npz, made by
    make_mixed.py --restart-read), against MixedMesh.read_restart of the same
    file at that order: every element type through the nodal bases on the
    file's points, up (2 -> 3) and down (3 -> 2)."""
    from test_mixed_setup import fixture_mesh
    meta, _, _ = fixture(name)
    want = np.load(os.path.join(GOLDEN, "rest_read_%s_p%d_to_p%d.npz" % (meta["kind"], meta["order"], order)))
    xv, cells, period, bfaces, opts = fixture_mesh(meta)
    M = X.MixedMesh(order, xv, cells, period, bfaces, opts)
    u, t = M.read_restart(os.path.join(GOLDEN, "rest_%s.dat" % name))
    assert abs(t - float(want["time"])) < 1e-15
    assert sorted(u) == sorted(int(k[1]) for k in want.files if k.endswith("_u_ref"))
    for et in u:
        assert rel(u[et], want["t%d_u_ref" % et]) <= 1e-14, (et, rel(u[et], want["t%d_u_ref" % et]))


@pytest.mark.parametrize("et,order", [(0, 2), (0, 4), (1, 3), (2, 2), (2, 3), (3, 2), (3, 4), (4, 3)])
def test_file_basis_equals_the_element_basis(et, order, tmp_path):
    """Reading a file onto an element's flux points applies the nodal basis
    built from the file's points; at the element's own solution points that
    is the element's opp_0 (the extrapolation the reference builds in
    set_opp_0, src/eles.cpp:3620-3676)."""
    opts = X.ElementOpts(upts_type_tet=1, vcjh_scheme_tet=1, vcjh_scheme_tri=1, vcjh_scheme_pri_1d=1)
    ops = X.element_operators(et, order, opts)
    pts = ops["loc_upts"].T.copy()
    rng = np.random.default_rng(11)
    ne, F = 3, 4 if et in (0, 1) else 5
    u = np.asfortranarray(rng.normal(size=(pts.shape[0], ne, F)))
    path = tmp_path / "Rest.dat"
    H.restart_write(path, 0.0, [_block(et, order, pts, u)])
    got, _ = H.restart_read_points(path, et, ops["tloc_fpts"].T, ne, F)
    u15 = H.restart_read_points(path, et, pts, ne, F)[0]           # the values as the file holds them
    want = np.einsum("qj,jef->qef", ops["opp_0"], u15)
    assert rel(got, want) <= 1e-13, rel(got, want)
