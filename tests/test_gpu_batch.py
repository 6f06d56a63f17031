"""Batches of independent meshes (fr_batch_*): instances of different sizes,
orders, element types and equations advanced together, each group merged
into one mesh and a whole step of all groups replayed as one CUDA graph.
Every instance must end bit for bit where a solver of its own ends: the
per-element arithmetic and the interface pairs are the same."""
import numpy as np
import pytest

import hifiles_b200 as H
import oracle as O

pytestmark = pytest.mark.gpu

NS = dict(viscous=True, gamma=1.4, prandtl=0.71, mu_inf=1.0 / 1600.0, tau=1.0, pen_fact=0.5)
EU = dict(viscous=False, gamma=1.4)
TGV = dict(lo=(0, 0, 0), hi=(2 * np.pi,) * 3)
INSTANCES = [
    dict(dims=3, order=3, n=(3, 3, 3), **TGV, **NS),
    dict(dims=3, order=3, n=(4, 3, 2), jitter=0.1, seed=4, **TGV, **NS),
    dict(dims=3, order=2, n=(2, 2, 2), **TGV, **NS),
    dict(dims=2, order=3, n=(4, 5), lo=(-5, -5), hi=(5, 5), **EU),
    dict(dims=3, order=3, n=(2, 3, 2), **TGV, **NS),
    dict(dims=3, order=2, n=(3, 2, 2), side_bc=(0, 0, 12, 12, 0, 0), **TGV, **NS),   # adiabatic walls
]


def _state(inst, s):
    pos = s.geometry()["pos_upts"]
    return np.asfortranarray(O.ic_tgv(pos) if inst["dims"] == 3 else O.ic_vortex(pos))


@pytest.mark.parametrize("tune", [False, True])
def test_batch_instances_equal_their_own_solvers(tune):
    b = H.Batch(INSTANCES)
    assert b.n_groups == 3          # hex P3 NS x3, hex P2 NS x2 (periodic and walled), quad P3 Euler
    refs = []
    for i, inst in enumerate(INSTANCES):
        kw = dict(inst)
        s = H.Solver.box(kw.pop("dims"), kw.pop("order"), kw.pop("n"), kw.pop("lo"), kw.pop("hi"), **kw)
        u0 = _state(inst, s)
        s.set_state(u0)
        b.set_state(i, u0)
        s.advance(3, 1e-3)
        refs.append(s.get_state())
    if tune:
        b.autotune(2)
    l0 = b.launch_count()
    b.advance(3, 1e-3)
    # hex P3 NS: gradient + fused interface/update; hex P2 NS: gradient, interface, update (runs of an odd
    # number of points); quad P3 Euler: the fused interface/update kernel alone
    assert b.launch_count() - l0 == 3 * 5 * (2 + 3 + 1)
    for i in range(len(INSTANCES)):
        assert np.array_equal(b.get_state(i), refs[i]), i


def test_batch_errors():
    with pytest.raises(H.FrError):
        H.Batch([dict(dims=3, order=5, n=(2, 2, 2), **TGV, **NS)])
    b = H.Batch(INSTANCES[:1])
    with pytest.raises(ValueError):
        b.set_state(0, np.zeros((3, 3, 3)))
    bad = np.full(b.shapes[0], np.nan, order="F")
    with pytest.raises(H.FrError):
        b.set_state(0, bad)


# hexahedral Navier-Stokes groups of orders 2, 3 and 4 (periodic and walled):
# the merged launches run each stage kernel once for all three groups
MERGEABLE = [
    dict(dims=3, order=2, n=(3, 2, 2), jitter=0.1, seed=5, **TGV, **NS),
    dict(dims=3, order=3, n=(3, 3, 2), **TGV, **NS),
    dict(dims=3, order=3, n=(2, 2, 2), side_bc=(0, 0, 12, 12, 0, 0), **TGV, **NS),
    dict(dims=3, order=4, n=(2, 2, 3), **TGV, **NS),
    dict(dims=3, order=2, n=(2, 3, 2), side_bc=(0, 0, 12, 12, 0, 0), **TGV, **NS),
]


@pytest.mark.parametrize("precision,minb", [(0, 4), (0, 3), (0, 1), (1, 4)])
def test_merged_launches_equal_per_group_launches(precision, minb):
    insts = [dict(inst, precision=precision) for inst in MERGEABLE]
    grouped, merged = H.Batch(insts), H.Batch(insts)
    for b in (grouped, merged):
        for i, inst in enumerate(insts):
            kw = dict(inst)
            s = H.Solver.box(kw.pop("dims"), kw.pop("order"), kw.pop("n"), kw.pop("lo"), kw.pop("hi"), **kw)
            b.set_state(i, _state(inst, s))
            s.close()
    merged.set_merged(True, minb)
    assert merged.merged == minb and grouped.merged == 0
    l0 = merged.launch_count()
    grouped.advance(3, 1e-3)
    merged.advance(3, 1e-3)
    # gradient, interface flux (orders 2 and 4), update: three launches per stage for all groups
    assert merged.launch_count() - l0 == 3 * 5 * 3
    for i in range(len(insts)):
        u = grouped.get_state(i)
        assert np.isfinite(u).all(), i
        assert np.array_equal(merged.get_state(i), u), i


def test_merged_launches_refuse_other_batches():
    b = H.Batch(INSTANCES)
    with pytest.raises(H.FrError):
        b.set_merged(True)
    b.autotune(1)
    assert b.merged == 0

