"""Restart files in the reference's format (fr_restart_write / fr_restart_read,
host only), against files the reference itself wrote (write_restart,
src/output.cpp:1057-1107) and against the reference reading a file this
library wrote at another order (read_restart + eles::set_opp_r,
src/solver.cpp:390-445, src/eles.cpp:4135-4153).

Values cross the file as 15 significant digits, so states are compared at
1e-14 normwise relative; files are compared byte for byte."""
import os

import numpy as np
import pytest

import hifiles_b200 as H
import oracle as O
from golden_util import GOLDEN, load, rel

CASES = [("quad_vortex_p3_n6", 1, 3), ("hex_tgv_p2_n3_jit", 4, 2)]


@pytest.mark.parametrize("case,etype,order", CASES)
def test_reader_on_reference_file_gives_reference_state(case, etype, order):
    meta, a = load(case)
    u, t = H.restart_read(os.path.join(GOLDEN, "rest_%s.dat" % case), etype, order, a["uN"].shape[1],
                          a["uN"].shape[2])
    assert abs(t - meta["steps"] * meta["dt"]) < 1e-12
    assert rel(u, a["uN"]) <= 1e-14


@pytest.mark.parametrize("case,etype,order", CASES)
def test_writer_reproduces_reference_file_byte_for_byte(case, etype, order, tmp_path):
    _, a = load(case)
    path = os.path.join(GOLDEN, "rest_%s.dat" % case)
    u, t = H.restart_read(path, etype, order, a["uN"].shape[1], a["uN"].shape[2])
    out = tmp_path / "Rest.dat"
    H.restart_write(out, t, [dict(ele_type=etype, order=order, loc_1d=O.points_1d(order), disu_upts=u)])
    assert out.read_bytes() == open(path, "rb").read()


def test_reference_reading_our_file_at_another_order_matches_our_reader(tmp_path):
    z = np.load(os.path.join(GOLDEN, "rest_read_p2_to_p3.npz"))
    u2, want = np.asfortranarray(z["u_p2"]), z["u_p3_ref"]
    out = tmp_path / "Rest.dat"
    H.restart_write(out, float(z["time"]), [dict(ele_type=4, order=2, loc_1d=O.points_1d(2), disu_upts=u2)])
    u3, t = H.restart_read(out, 4, 3, u2.shape[1], u2.shape[2])
    assert abs(t - float(z["time"])) < 1e-15
    assert rel(u3, want) <= 1e-14
    # and the same order reads back what was written (to 15 digits)
    u2b, _ = H.restart_read(out, 4, 2, u2.shape[1], u2.shape[2])
    assert rel(u2b, u2) <= 1e-14


def test_reader_errors(tmp_path):
    path = os.path.join(GOLDEN, "rest_quad_vortex_p3_n6.dat")
    with pytest.raises(H.FrError):
        H.restart_read(path, 4, 3, 36, 5)                      # no HEXAS block
    with pytest.raises(H.FrError):
        H.restart_read(path, 1, 3, 37, 4)                      # element 36 missing
    with pytest.raises(H.FrError):
        H.restart_read(tmp_path / "absent.dat", 1, 3, 36, 4)
    # global ids select the elements: reversed ids give the reversed state
    _, a = load("quad_vortex_p3_n6")
    ids = np.arange(36)[::-1].copy()
    u, _ = H.restart_read(path, 1, 3, 36, 4, ele2global=ids)
    assert rel(u, a["uN"][:, ::-1, :]) <= 1e-14
