"""The .vtu writers (fr_vtu_write, fr_vtu_write_mixed, host only): the file
parses as VTK XML, its base64 arrays decode to the state's density,
velocity and pressure at the solution points (quads, hexes) or the plot
lattice (triangles, tets, prisms), and the sub-cells are well formed."""
import base64
import struct
import xml.etree.ElementTree as ET

import numpy as np
import pytest

import hifiles_b200 as H
import oracle as O


def _arrays(path):
    root = ET.parse(path).getroot()
    out = {}
    piece = root.find("UnstructuredGrid/Piece")
    for da in root.iter("DataArray"):
        raw = base64.b64decode(da.text.strip())
        nb = struct.unpack("<I", raw[:4])[0]
        dt = {"Float32": np.float32, "Int32": np.int32, "UInt8": np.uint8}[da.get("type")]
        out[da.get("Name") or "Points"] = np.frombuffer(raw[4:4 + nb], dtype=dt)
    return out, int(piece.get("NumberOfPoints")), int(piece.get("NumberOfCells"))


@pytest.mark.parametrize("dims,P,n", [(3, 3, (2, 3, 2)), (2, 2, (4, 3))])
def test_vtu_round_trip(dims, P, n, tmp_path):
    m = O.Mesh.box(dims, P, n, [0.0] * dims, [2 * np.pi] * dims, jitter=0.1, seed=1)
    pos = m.geometry()["pos_upts"]
    u = O.ic_tgv(pos) if dims == 3 else O.ic_vortex(pos)
    path = tmp_path / "s.vtu"
    H.vtu_write(path, dims, P, pos, u)
    a, npts, ncells = _arrays(path)
    F = dims + 2
    q = u.reshape(-1, F, order="F")
    assert npts == q.shape[0] and ncells == m.n_eles * P ** dims
    assert np.allclose(a["Density"], q[:, 0], rtol=1e-6)
    vel = a["Velocity"].reshape(-1, 3)
    assert np.allclose(vel[:, :dims], q[:, 1:1 + dims] / q[:, :1], rtol=1e-5, atol=1e-6)
    p = 0.4 * (q[:, -1] - 0.5 * (q[:, 1:1 + dims] ** 2).sum(axis=1) / q[:, 0])
    assert np.allclose(a["Pressure"], p, rtol=1e-5)
    assert np.allclose(a["Points"].reshape(-1, 3)[:, :dims], pos.reshape(-1, dims, order="F"), atol=1e-5)
    nv = 4 if dims == 2 else 8
    assert a["connectivity"].size == ncells * nv and a["offsets"][-1] == ncells * nv
    assert a["connectivity"].min() == 0 and a["connectivity"].max() == npts - 1
    assert set(a["types"].tolist()) == {9 if dims == 2 else 12}


def _cells(a):
    conn, offs, types = a["connectivity"], a["offsets"], a["types"]
    start = np.concatenate([[0], offs[:-1]])
    return [(int(t), conn[s:e]) for t, s, e in zip(types, start, offs)]


def _tet_vol(x):
    return np.dot(np.cross(x[1] - x[0], x[2] - x[0]), x[3] - x[0]) / 6.0


@pytest.mark.parametrize("name", ["mixed_triquad_p2", "mixed_pritet_p2", "mixed_hexpri_p3"])
def test_mixed_vtu(name, tmp_path):
    """fr_vtu_write_mixed on a mixed fixture mesh set up by the library: a
    field linear in the coordinates arrives exactly at every plot point (the
    positions and the state go through the same nodal interpolation), the
    sub-cells of every type are counted and oriented as VTK wants them, and
    the sub-tetrahedra fill each tet."""
    from hifiles_b200 import mixed as X
    from test_mixed_setup import fixture_mesh
    import json
    import os
    from golden_util import GOLDEN
    meta = json.loads(str(np.load(os.path.join(GOLDEN, name + ".npz"))["meta"]))
    xv, cells, period, bfaces, opts = fixture_mesh(meta)
    P = meta["order"]
    M = X.MixedMesh(P, xv, cells, period, bfaces, opts)
    D = M.dims
    cf = np.array([0.05, -0.03, 0.02][:D])

    def state(pos):
        rho = 1.0 + pos @ cf
        u = np.zeros(pos.shape[:2] + (D + 2,))
        u[..., 0] = rho
        u[..., 1] = 0.3 * rho
        u[..., -1] = 180.0 + pos[..., 0]
        return np.asfortranarray(u)

    path = tmp_path / "m.vtu"
    M.write_vtu(path, {t: state(m["pos_upts"]) for t, m in M.types.items()})
    a, npts, ncells = _arrays(path)
    xyz = a["Points"].reshape(-1, 3).astype(np.float64)
    assert np.allclose(a["Density"], 1.0 + xyz[:, :D] @ cf, rtol=0, atol=2e-6)
    assert np.allclose(a["Energy"], 180.0 + xyz[:, 0], rtol=2e-7, atol=0)
    assert np.allclose(a["Velocity"].reshape(-1, 3)[:, 0], 0.3, rtol=1e-6)
    per = {0: (5, P * P), 1: (9, P * P), 2: (10, P ** 3), 3: (13, P ** 3), 4: (12, P ** 3)}
    want = sorted(sum([[per[t][0]] * (per[t][1] * m["n_eles"]) for t, m in M.types.items()], []))
    cl = _cells(a)
    assert sorted(t for t, _ in cl) == want and ncells == len(want)
    assert a["connectivity"].min() == 0 and a["connectivity"].max() == npts - 1
    tet_vol = 0.0
    for t, v in cl:
        x = xyz[v]
        if t == 10:
            vol = _tet_vol(x)
            assert vol > 0
            tet_vol += vol
        elif t == 13:                        # base normal points away from the top triangle
            n = np.cross(x[1] - x[0], x[2] - x[0])
            assert np.dot(n, x[3:].mean(axis=0) - x[:3].mean(axis=0)) < 0
        elif t == 5:                         # counter-clockwise in the plane
            e1, e2 = x[1, :2] - x[0, :2], x[2, :2] - x[0, :2]
            assert e1[0] * e2[1] - e1[1] * e2[0] > 0
    if 2 in M.types:
        want_vol = sum(abs(X._tet_volume(xv, vs)) / 6.0 for ty, vs in cells if ty == X.TET)
        assert abs(tet_vol - want_vol) <= 1e-5 * want_vol


def test_tensor_vtu_unchanged_through_the_mixed_writer(tmp_path):
    """fr_vtu_write (one quad or hex block) and fr_vtu_write_mixed with that
    block write the same file."""
    m = O.Mesh.box(3, 2, (2, 2, 2), [0.0] * 3, [2 * np.pi] * 3, jitter=0.1, seed=1)
    pos = m.geometry()["pos_upts"]
    u = O.ic_tgv(pos)
    H.vtu_write(tmp_path / "a.vtu", 3, 2, pos, u)
    H.vtu_write_mixed(tmp_path / "b.vtu", 2, [dict(ele_type=4, pos_upts=pos, disu_upts=u)])
    assert (tmp_path / "a.vtu").read_bytes() == (tmp_path / "b.vtu").read_bytes()
