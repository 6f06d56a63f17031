"""The numpy restatement of the learned closure (oracle/mlp.py), which checks
the CUDA training and inference kernels: its analytic gradient against
central finite differences, and the closure switched off (c ~ 2e-9) in the C
oracle leaves the viscous residual unchanged."""
import numpy as np

import mlp as M
import oracle as O
from golden_util import rel


def _data(n, seed):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, M.NIN))
    Y = rng.uniform(0.0, 0.3, n)
    return X, Y


def test_mlp_gradient_matches_finite_differences():
    w = M.init_params(3, xmean=np.full(6, 0.1, dtype=np.float32), xscale=np.full(6, 0.9, dtype=np.float32))
    w = w.astype(np.float64)
    w[M.B3] = 0.2
    X, Y = _data(40, 1)
    _, g = M.loss_grad(w, X, Y)
    rng = np.random.default_rng(0)
    for p in list(rng.choice(M.NTRAIN, 60, replace=False)) + [M.B3, M.W3, M.B1, M.W1 + 5]:
        h = 1e-6
        wp, wm = w.copy(), w.copy()
        wp[p] += h
        wm[p] -= h
        fd = (M.loss_grad(wp, X, Y)[0] - M.loss_grad(wm, X, Y)[0]) / (2 * h)
        assert abs(fd - g[p]) <= 1e-6 * max(1.0, abs(g[p])) + 1e-9, (p, fd, g[p])


def test_forward_is_softplus_of_the_network():
    w = M.init_params(5)
    X, _ = _data(10, 2)
    c = M.forward(w, X)
    assert np.all(c > 0)
    w2 = w.copy()
    w2[M.W3:M.B3] = 0.0
    w2[M.B3] = 0.0
    assert np.allclose(M.forward(w2, X), np.log(2.0))


def test_oracle_closure_switched_off_leaves_residual():
    kw = dict(gamma=1.4, prandtl=0.71, mu_inf=1e-3, tau=1.0, pen_fact=0.5)
    m = O.Mesh.box(3, 2, (2, 2, 2), (0, 0, 0), (2 * np.pi,) * 3, jitter=0.1, seed=4)
    u = O.ic_tgv(m.geometry()["pos_upts"])
    w = np.zeros(M.NPARAM, dtype=np.float32)
    w[M.B3] = -20.0
    w[M.XS:] = 1.0
    off = m.residual(O.physics(viscous=1, les=1, sgs_model=5, mlp=w, **kw), u)
    plain = m.residual(O.physics(viscous=1, **kw), u)
    assert rel(off, plain) < 1e-6
    w[M.B3] = 0.0
    on = m.residual(O.physics(viscous=1, les=1, sgs_model=5, mlp=w, **kw), u)
    assert rel(on, plain) > 1e-4
