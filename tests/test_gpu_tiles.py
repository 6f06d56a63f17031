"""Every compiled tile variant of the gradient and update kernels -- elements
and threads per block, register budget, and persistent blocks that prefetch
their next element block -- gives the same state, bit for bit.

The mesh (12^3 hexes, P = 3) has more element blocks than the B200 keeps
resident at once, so the persistent variants run several blocks each and
their prefetch path is exercised."""
import numpy as np
import pytest

import hifiles_b200 as H

pytestmark = pytest.mark.gpu

GAMMA, MACH, RE, PR = 1.4, 0.1, 1600.0, 0.71


def _tgv(pos):
    x, y, z = pos[..., 0], pos[..., 1], pos[..., 2]
    p = 1.0 / (GAMMA * MACH * MACH) + (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0) / 16.0
    u = np.sin(x) * np.cos(y) * np.cos(z)
    v = -np.cos(x) * np.sin(y) * np.cos(z)
    return np.asfortranarray(np.stack([np.ones_like(x), u, v, np.zeros_like(x),
                                       p / (GAMMA - 1.0) + 0.5 * (u * u + v * v)], axis=-1))


@pytest.mark.parametrize("precision", [0, 1])
def test_every_tile_variant_gives_identical_states(precision):
    L = 2 * np.pi
    s = H.Solver.box(3, 3, (12, 12, 12), (0, 0, 0), (L, L, L), viscous=True, vcjh_scheme=1, gamma=GAMMA,
                     prandtl=PR, mu_inf=1.0 / RE, rt_inf=1.0, c_sth=1.0, fix_vis=1.0, tau=1.0, pen_fact=0.5,
                     precision=precision)
    u0 = _tgv(s.geometry()["pos_upts"])
    ng, nu = s.tile_count()
    assert any(s.tile_info(0, g)[3] for g in range(ng)), "no persistent gradient variant compiled"
    ref = None
    runs = [(g, 0) for g in range(ng)] + [(0, u) for u in range(1, nu)]
    for g, u in runs:
        s.set_state(u0)
        s.select_tiles(g, u)
        s.advance(2, 1e-3)
        st = s.get_state()
        if ref is None:
            ref = st
            assert np.isfinite(ref).all()
        else:
            assert np.array_equal(st, ref), ("gradient", s.tile_info(0, g), "update", s.tile_info(1, u))
    with pytest.raises(H.FrError):
        s.select_tiles(ng, 0)


@pytest.mark.parametrize("case", ["hex_channel_p2", "hex_channel_char_p3"])
def test_every_tile_variant_matches_the_reference_on_walled_meshes(case):
    """The reference's walled channels (isothermal, adiabatic, slip and
    characteristic boundaries): every tile variant ends where the reference
    ends, so the boundary branches hold for every block shape."""
    from golden_util import load, rel
    meta, a = load(case)
    s = H.Solver.box(meta["dims"], meta["order"], meta["n"], meta["lo"], meta["hi"], jitter=meta["jitter"],
                     seed=meta["seed"], viscous=bool(meta["viscous"]), vcjh_scheme=meta["vcjh"],
                     side_bc=meta.get("side_bc"), **meta["physics"])
    ng, nu = s.tile_count()
    bad = []
    for g, u in [(g, 0) for g in range(ng)] + [(0, u) for u in range(1, nu)]:
        s.set_state(a["u0"])
        s.select_tiles(g, u)
        s.advance(meta["steps"], meta["dt"])
        r = rel(s.get_state(), a["uN"])
        if not r <= 1e-12:
            bad.append((s.tile_info(0, g), s.tile_info(1, u), r))
    assert not bad, bad
