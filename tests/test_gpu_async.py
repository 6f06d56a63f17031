"""Asynchronous state upload and advance (fr_solver_set_state_async,
fr_solver_advance_async): the pipelined pattern gives the same states, bit for
bit, as set_state + advance, and one state is staged at a time."""
import numpy as np
import pytest
import torch

import hifiles_b200 as H

pytestmark = pytest.mark.gpu

GAMMA, MACH, RE, PR = 1.4, 0.1, 1600.0, 0.71


def _tgv(pos, amp=1.0):
    x, y, z = pos[..., 0], pos[..., 1], pos[..., 2]
    p = 1.0 / (GAMMA * MACH * MACH) + (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0) / 16.0
    u = amp * np.sin(x) * np.cos(y) * np.cos(z)
    v = -amp * np.cos(x) * np.sin(y) * np.cos(z)
    return np.asfortranarray(np.stack([np.ones_like(x), u, v, np.zeros_like(x),
                                       p / (GAMMA - 1.0) + 0.5 * (u * u + v * v)], axis=-1))


def _pinned_like(a):
    t = torch.empty(a.size, dtype=torch.float64, pin_memory=True)
    h = t.numpy().reshape(a.shape, order="F")
    h[...] = a
    return t, h


def test_async_upload_and_advance_match_the_synchronous_path():
    L = 2 * np.pi
    s = H.Solver.box(3, 3, (4, 4, 4), (0, 0, 0), (L, L, L), viscous=True, vcjh_scheme=1, gamma=GAMMA, prandtl=PR,
                     mu_inf=1.0 / RE, tau=1.0, pen_fact=0.5)
    pos = s.geometry()["pos_upts"]
    states = [_tgv(pos, a) for a in (1.0, 0.8, 1.2)]
    ref = []
    for u in states:
        s.set_state(u)
        s.advance(1, 1e-3)
        ref.append(s.get_state())
    keep = [_pinned_like(u) for u in states]
    norms_t = torch.zeros((len(states), s.n_fields), dtype=torch.float64, pin_memory=True)
    norms = norms_t.numpy()
    out = []
    for i, (_, h) in enumerate(keep):
        s.set_state_async(h)
        s.advance_async(1, 1e-3, norms[i])
        s.sync()
        out.append(s.get_state())
    for a, b in zip(out, ref):
        assert np.array_equal(a, b)
    assert np.isfinite(norms).all() and (norms > 0).all()
    # pipelined: the next upload is queued while the step before runs
    for _, h in keep:
        s.set_state_async(h)
        s.advance_async(1, 1e-3)
    s.sync()
    assert np.array_equal(s.get_state(), ref[-1])
    # one staged state at a time; a bad density is refused before anything is copied
    s.set_state_async(keep[0][1])
    with pytest.raises(H.FrError) as ei:
        s.set_state_async(keep[1][1])
    assert ei.value.status == 1
    s.advance(1, 1e-3)
    assert np.array_equal(s.get_state(), ref[0])
    bad = np.array(states[0], order="F")
    bad[3, 5, 0] = -1.0
    _, hb = _pinned_like(bad)
    with pytest.raises(H.FrError) as ei:
        s.set_state_async(hb)
    assert ei.value.status == 3
    with pytest.raises(ValueError):
        s.set_state_async(np.ascontiguousarray(states[0]))
