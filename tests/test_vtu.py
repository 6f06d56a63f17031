"""The .vtu writer (fr_vtu_write, host only): the file parses as VTK XML,
its base64 arrays decode to the state's density, velocity and pressure at
the solution points, and the sub-cells are well formed."""
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
