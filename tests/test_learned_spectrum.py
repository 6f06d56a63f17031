"""The energy spectrum of the learned-closure experiment (learned_sgs.energy_spectrum)
on a single Fourier mode: the velocity interpolated from the solution points of
each element to a uniform grid and transformed gives E(k) = 1/4 at |k| = 2 for
u = (sin 2x, 0, 0), and nothing elsewhere.  Host-only (the element geometry comes
from the library's host set-up)."""
import numpy as np

import hifiles_b200 as H
from hifiles_b200 import learned_sgs as L


class _BoxGeometry:
    def __init__(self, n, P):
        xv, c2v = H.box_mesh(3, (n, n, n), (0, 0, 0), (2 * np.pi,) * 3)
        self.g = H.mesh_geometry(3, xv, c2v, [2 * np.pi] * 3, P)
        self.n_upts = (P + 1) ** 3

    def geometry(self):
        return self.g


def test_single_mode_spectrum():
    n, P = 6, 3
    s = _BoxGeometry(n, P)
    x = s.g["pos_upts"]
    q = np.zeros(x.shape[:2] + (5,))
    q[..., 0] = 1.0
    q[..., 1] = np.sin(2 * x[..., 0])
    spec = L.energy_spectrum(s, q, n)
    assert len(spec) == n * (P + 1) // 2
    assert abs(spec[1] - 0.25) < 1e-3, spec[:4]
    assert np.abs(np.delete(spec, 1)).max() < 1e-3 * spec[1]
