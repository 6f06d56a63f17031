"""The learned SGS closure on the GPU: the hand-written CUDA forward, loss
gradient and Adam kernels against the numpy restatement (oracle/mlp.py),
the closure's inputs evaluated by the solver against the same restatement,
the LES residual with the closure against the C oracle, and a short training
run.

Tolerances: the network runs in FP32, so kernel outputs are compared at
1e-5 (forward, inputs) and 1e-4 (gradients, summed over 10^4 samples in
FP32) relative; the solver residual with the closure at 1e-7 relative (the
FP32 network differs from the oracle's by ~1 ulp of c, which moves the SGS
flux, about 1 % of the residual, by ~1e-7 of itself)."""
import numpy as np
import pytest

import hifiles_b200 as H
import mlp as M
import oracle as O
from golden_util import load, rel

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

KW = dict(gamma=1.4, prandtl=0.71, mu_inf=1e-3, tau=1.0, pen_fact=0.5)


def _params(seed):
    rng = np.random.default_rng(seed)
    w = M.init_params(seed, xmean=rng.normal(0, 0.2, 6).astype(np.float32),
                      xscale=rng.uniform(0.5, 2.0, 6).astype(np.float32))
    w[M.B3] = 0.3
    return w


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _data(n, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((n, 6)).astype(np.float32), rng.uniform(0.0, 0.5, n).astype(np.float32)


def test_forward_kernel_matches_numpy():
    w = _params(1)
    X, _ = _data(5000, 2)
    out = torch.empty(5000, dtype=torch.float32, device="cuda")
    dw, dx = _dev(w), _dev(X)          # held: a freed temporary's memory would be reused
    H.mlp_forward(dw.data_ptr(), dx.data_ptr(), 5000, out.data_ptr())
    torch.cuda.synchronize()
    assert rel(out.cpu().numpy(), M.forward(w, X)) < 1e-5


def test_loss_gradient_kernel_matches_numpy_and_is_deterministic():
    w = _params(3)
    X, Y = _data(10000, 4)
    n = len(Y)
    dw, dx, dy = _dev(w), _dev(X), _dev(Y)
    grads = []
    for _ in range(2):
        g = torch.empty(H.mlp_n_trained(), dtype=torch.float32, device="cuda")
        loss = torch.empty(1, dtype=torch.float32, device="cuda")
        ns = H.mlp_scratch_floats(n)
        scratch = torch.empty(ns, dtype=torch.float32, device="cuda")
        H.mlp_loss_grad(dw.data_ptr(), dx.data_ptr(), dy.data_ptr(), n, g.data_ptr(), loss.data_ptr(),
                        scratch.data_ptr(), ns)
        torch.cuda.synchronize()
        grads.append(g.cpu().numpy())
    l_ref, g_ref = M.loss_grad(w, X, Y)
    assert abs(loss.item() - l_ref) <= 1e-5 * l_ref
    assert rel(grads[0], g_ref) < 1e-4
    for a, b in ((M.W1, M.B1), (M.W2, M.B2), (M.W3, M.B3)):
        assert rel(grads[0][a:b], g_ref[a:b]) < 1e-4
    assert np.array_equal(grads[0], grads[1])
    # per-sample weights
    sw = np.random.default_rng(8).uniform(0.0, 3.0, n).astype(np.float32)
    dsw = _dev(sw)
    H.mlp_loss_grad(dw.data_ptr(), dx.data_ptr(), dy.data_ptr(), n, g.data_ptr(), loss.data_ptr(),
                    scratch.data_ptr(), ns, d_sw=dsw.data_ptr())
    torch.cuda.synchronize()
    l_ref, g_ref = M.loss_grad(w, X, Y, sw)
    assert abs(loss.item() - l_ref) <= 1e-5 * l_ref
    assert rel(g.cpu().numpy(), g_ref) < 1e-4


def test_adam_kernel_matches_numpy():
    rng = np.random.default_rng(5)
    w = _params(6)
    g = rng.standard_normal(M.NTRAIN).astype(np.float32)
    m = rng.standard_normal(M.NTRAIN).astype(np.float32) * 0.1
    v = rng.uniform(0, 0.1, M.NTRAIN).astype(np.float32)
    dw, dg, dm, dv = _dev(w), _dev(g), _dev(m), _dev(v)
    H.mlp_adam(dw.data_ptr(), dg.data_ptr(), dm.data_ptr(), dv.data_ptr(), 3, 1e-3)
    torch.cuda.synchronize()
    m1 = 0.9 * m + 0.1 * g
    v1 = 0.999 * v + 0.001 * g * g
    w1 = w[:M.NTRAIN] - 1e-3 * (m1 / (1 - 0.9 ** 3)) / (np.sqrt(v1 / (1 - 0.999 ** 3)) + 1e-8)
    assert rel(dw.cpu().numpy()[:M.NTRAIN], w1) < 1e-6
    assert np.array_equal(dw.cpu().numpy()[M.NTRAIN:], w[M.NTRAIN:])


def test_solver_gradient_matches_reference_stage_array():
    meta, a = load("hex_tgv_p3_n3")
    ph = meta["physics"]
    s = H.Solver.box(3, 3, meta["n"], meta["lo"], meta["hi"], jitter=meta["jitter"], seed=meta["seed"],
                     viscous=True, vcjh_scheme=meta["vcjh"], **ph)
    s.set_state(a["u0"])
    assert rel(s.gradient(), a["grad_disu_upts0"]) <= 1e-12


@pytest.mark.parametrize("dims,P", [(3, 3), (3, 2), (2, 3)])
def test_closure_inputs_match_numpy(dims, P):
    lo, hi = [0.0] * dims, [2 * np.pi] * dims
    n = (3, 2, 3)[:dims]
    s = H.Solver.box(dims, P, n, lo, hi, jitter=0.1, seed=2, viscous=True, les=1, sgs_model=5, filter_ratio=1.5, **KW)
    m = O.Mesh.box(dims, P, n, lo, hi, jitter=0.1, seed=2)
    g = m.geometry()
    u = O.ic_tgv(g["pos_upts"]) if dims == 3 else O.ic_vortex(g["pos_upts"] * (10 / (2 * np.pi)) - 5)
    u = np.asfortranarray(u + 0.02 * np.random.default_rng(1).standard_normal(u.shape) * (np.arange(u.shape[2]) > 0))
    s.set_state(u)
    x = s.sgs_features()
    grad = s.gradient()
    F = dims + 2
    q = u.reshape(-1, F, order="F")
    gg = grad.reshape(-1, F, dims, order="F")
    xr, _, _, _ = M.inputs(q, gg, g["detjac_upts"].reshape(-1, order="F"), P, 1.5)
    assert rel(x, xr) < 1e-5


@pytest.mark.parametrize("dims,P,n", [(3, 3, (3, 2, 3)), (3, 2, (2, 3, 2)), (2, 3, (4, 3))])
def test_les_residual_with_learned_closure_matches_oracle(dims, P, n):
    lo, hi = [0.0] * dims, [2 * np.pi] * dims
    w = _params(9)
    w[M.XM:M.XS] = 0.0
    w[M.XS:] = 1.0
    w[M.B3] = -1.0
    s = H.Solver.box(dims, P, n, lo, hi, jitter=0.1, seed=7, viscous=True, les=1, sgs_model=5, **KW)
    s.set_sgs_mlp(w)
    m = O.Mesh.box(dims, P, n, lo, hi, jitter=0.1, seed=7)
    pos = m.geometry()["pos_upts"]
    u = O.ic_tgv(pos) if dims == 3 else O.ic_vortex(pos * (10 / (2 * np.pi)) - 5)
    u = np.asfortranarray(u + 0.05 * np.random.default_rng(3).standard_normal(u.shape) * (np.arange(u.shape[2]) > 0))
    s.set_state(u)
    want = m.residual(O.physics(viscous=1, les=1, sgs_model=5, mlp=w, **KW), u)
    plain = m.residual(O.physics(viscous=1, **KW), u)
    assert rel(plain, want) > 1e-4                  # the closure matters at this bar
    assert rel(s.residual(), want) <= 1e-7


def test_training_reduces_the_loss():
    """200 Adam steps on a smooth synthetic target cut the loss tenfold."""
    rng = np.random.default_rng(11)
    X = rng.standard_normal((20000, 6)).astype(np.float32)
    Y = (0.1 + 0.05 * np.tanh(X[:, 0] - 0.5 * X[:, 1]) + 0.02 * X[:, 5] ** 2).astype(np.float32)
    w = M.init_params(12)
    n = len(Y)
    dw, dx, dy = _dev(w), _dev(X), _dev(Y)
    g = torch.zeros(M.NTRAIN, dtype=torch.float32, device="cuda")
    mm, vv = torch.zeros_like(g), torch.zeros_like(g)
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    ns = H.mlp_scratch_floats(n)
    scratch = torch.empty(ns, dtype=torch.float32, device="cuda")
    hist = []
    for step in range(1, 201):
        H.mlp_loss_grad(dw.data_ptr(), dx.data_ptr(), dy.data_ptr(), n, g.data_ptr(), loss.data_ptr(),
                        scratch.data_ptr(), ns)
        H.mlp_adam(dw.data_ptr(), g.data_ptr(), mm.data_ptr(), vv.data_ptr(), step, 3e-3)
        if step in (1, 200):
            torch.cuda.synchronize()
            hist.append(loss.item())
    assert hist[1] < 0.1 * hist[0], hist
