"""Restatement of the learned SGS closure in numpy (forward pass, loss and its
gradient, the closure's inputs), the checker for the CUDA training and
inference kernels.

TEST INFRASTRUCTURE ONLY.  The product never imports this module.

The closure has no counterpart in the reference (whose eddy-viscosity models
are Smagorinsky and WALE, src/eles.cpp:2456-2778).  Model: c = softplus(w3 .
tanh(W2 tanh(W1 x_n + b1) + b2) + b3), x_n = (x - xmean) * xscale, and
mu_t = rho Delta^2 |S| c.  Parameter vector (float32):
W1[64][6], b1[64], W2[64][64], b2[64], w3[64], b3, xmean[6], xscale[6].
"""
import numpy as np

NIN, NH = 6, 64
W1, B1 = 0, 384
W2, B2 = 448, 4544
W3, B3 = 4608, 4672
NTRAIN = 4673
XM, XS = 4673, 4679
NPARAM = 4685


def unpack(w):
    w = np.asarray(w, dtype=np.float64)
    return (w[W1:B1].reshape(NH, NIN), w[B1:W2], w[W2:B2].reshape(NH, NH), w[B2:W3], w[W3:B3], w[B3],
            w[XM:XS], w[XS:NPARAM])


def init_params(seed, xmean=None, xscale=None):
    """Glorot-uniform weights, zero biases, b3 = -3 (c ~ 0.05 at the start)."""
    rng = np.random.default_rng(seed)
    w = np.zeros(NPARAM, dtype=np.float32)
    a1 = np.sqrt(6.0 / (NIN + NH))
    a2 = np.sqrt(6.0 / (NH + NH))
    a3 = np.sqrt(6.0 / (NH + 1))
    w[W1:B1] = rng.uniform(-a1, a1, NH * NIN)
    w[W2:B2] = rng.uniform(-a2, a2, NH * NH)
    w[W3:B3] = rng.uniform(-a3, a3, NH)
    w[B3] = -3.0
    w[XM:XS] = 0.0 if xmean is None else xmean
    w[XS:NPARAM] = 1.0 if xscale is None else xscale
    return w


def _softplus(o):
    return np.where(o > 20.0, o, np.log1p(np.exp(np.minimum(o, 20.0))))


def forward(w, X):
    """c for every row of X (float64 arithmetic)."""
    w1, b1, w2, b2, w3, b3, xm, xs = unpack(w)
    xn = (np.asarray(X, dtype=np.float64) - xm) * xs
    h1 = np.tanh(xn @ w1.T + b1)
    h2 = np.tanh(h1 @ w2.T + b2)
    return _softplus(h2 @ w3 + b3)


def loss_grad(w, X, Y, sw=None):
    """(loss, gradient over the 4673 trained parameters) of mean sw (c - y)^2."""
    w1, b1, w2, b2, w3, b3, xm, xs = unpack(w)
    X = np.asarray(X, dtype=np.float64)
    Y = np.asarray(Y, dtype=np.float64)
    n = X.shape[0]
    xn = (X - xm) * xs
    h1 = np.tanh(xn @ w1.T + b1)
    h2 = np.tanh(h1 @ w2.T + b2)
    o = h2 @ w3 + b3
    r = _softplus(o) - Y
    sw = np.ones(n) if sw is None else np.asarray(sw, dtype=np.float64)
    do = 2.0 * sw * r / (1.0 + np.exp(-o)) / n
    g = np.zeros(NTRAIN)
    g[W3:B3] = do @ h2
    g[B3] = do.sum()
    da2 = do[:, None] * w3[None, :] * (1.0 - h2 * h2)
    g[W2:B2] = (da2.T @ h1).ravel()
    g[B2:W3] = da2.sum(axis=0)
    da1 = (da2 @ w2) * (1.0 - h1 * h1)
    g[W1:B1] = (da1.T @ xn).ravel()
    g[B1:W2] = da1.sum(axis=0)
    return float((sw * r * r).mean()), g


def inputs(q, g, detjac, order, filter_ratio):
    """Closure inputs x (n, 6) and (Delta, |S|, S) at n points from the state
    q (n, F) and its physical gradient g (n, F, D), D = F - 2."""
    q = np.asarray(q, dtype=np.float64)
    g = np.asarray(g, dtype=np.float64)
    n, F = q.shape
    D = F - 2
    rho = q[:, 0]
    u = q[:, 1:1 + D] / rho[:, None]
    A = (g[:, 1:1 + D, :] - u[:, :, None] * g[:, 0:1, :]) / rho[:, None, None]     # A[n, i, j] = d u_i / d x_j
    tr = np.trace(A, axis1=1, axis2=2)
    S = 0.5 * (A + A.transpose(0, 2, 1)) - np.eye(D)[None] * (tr / 3.0)[:, None, None]
    W = 0.5 * (A - A.transpose(0, 2, 1))
    a2 = (A * A).sum(axis=(1, 2)) + 1e-30
    S2, W2 = S @ S, W @ W
    tr_ = lambda M: np.trace(M, axis1=1, axis2=2)
    trS2, trW2 = tr_(S @ S), tr_(W @ W)
    x = np.stack([trS2 / a2, trW2 / a2, tr_(S2 @ S) / a2 ** 1.5, tr_(S @ W2) / a2 ** 1.5, tr_(S2 @ W2) / a2 ** 2],
                 axis=1)
    vol = np.asarray(detjac, dtype=np.float64) * (8.0 if D == 3 else 4.0)
    delta = filter_ratio * vol ** (1.0 / D) / (order + 1.0)
    x = np.concatenate([x, np.log(delta)[:, None]], axis=1)
    return x, delta, np.sqrt(2.0 * trS2), S
