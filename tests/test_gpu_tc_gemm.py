"""The tensor-core form of the per-operator path: the operator product in
BF16 with a 3-term split (tcgen05, FP32 accumulation) against FP64, and a
whole RK45 step through the per-operator entry points against the fused
solver."""
import ctypes as C

import numpy as np
import pytest
import torch

import hifiles_b200 as H
from hifiles_b200 import seam

pytestmark = pytest.mark.gpu

VP = C.c_void_p
GAMMA, MACH, RE, PR = 1.4, 0.1, 1600.0, 0.71


def _lib():
    L = seam._bind(H.lib())
    return L


def _dev(a):
    return torch.from_numpy(np.asfortranarray(a).ravel(order="F").copy()).cuda()


def _host(t, shape):
    torch.cuda.synchronize()
    return t.cpu().numpy().reshape(shape, order="F")


def _product(L, A, B, mode):
    m, k = A.shape
    n = B.shape[1]
    dA, dB = _dev(A), _dev(B)
    dC = torch.zeros(m * n, dtype=torch.float64, device="cuda")
    assert L.fr_op_set_gemm_precision(mode) == 0
    try:
        st = L.fr_op_extrapolate_solution(m, k, 1, n, dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), None)
        assert st == 0, H.lib().fr_last_error().decode()
        assert L.fr_op_check(None) == 0, H.lib().fr_last_error().decode()
    finally:
        L.fr_op_set_gemm_precision(0)
    return _host(dC, (m, n))


@pytest.mark.parametrize("m,k,n", [(96, 64, 5 * 1000 + 3), (64, 96, 777), (128, 128, 64 * 40), (16, 16, 100),
                                   (1, 1, 5), (64, 64, 64), (96, 64, 5 * 32 ** 3), (150, 125, 5 * 200 + 7),
                                   (125, 150, 333), (256, 128, 96)])
def test_bf16x3_product_against_fp64(m, k, n):
    rng = np.random.default_rng(7 + m + k)
    A = rng.standard_normal((m, k))
    B = rng.standard_normal((k, n))
    ref = A @ B
    L = _lib()
    c64 = _product(L, A, B, 0)
    assert np.abs(c64 - ref).max() <= 1e-12 * np.abs(ref).max() * max(1, k)
    c3 = _product(L, A, B, 1)
    err = np.linalg.norm(c3 - ref) / np.linalg.norm(ref)
    if k == 1:
        # a one-entry column is all column shift: the product is the FP64 one
        assert err < 1e-15, err
        return
    # x0 + x1 keeps ~16 bits of each operand: a few 1e-6 relative
    assert 1e-9 < err < 3e-5, err
    if (m <= 128 and k <= 192) or k <= 128:
        c6 = _product(L, A, B, 2)
        err6 = np.linalg.norm(c6 - ref) / np.linalg.norm(ref)
        # x0 + x1 + x2 keeps ~24 bits; the FP32 accumulation over the 6 k
        # products (about 1e-6 relative on random data, more for long k) is
        # then the limit
        assert err6 < 3e-6 and err6 < err / 2, (err6, err)


def test_split_carries_only_the_variation_of_each_column():
    """Columns with a large common level (the TGV energy is ~178 at Mach 0.1
    against variations of order 1): the BF16 parts carry B minus each
    column's first entry, so the error scales with the variation, not the level."""
    rng = np.random.default_rng(11)
    m, k, n = 96, 64, 500
    A = rng.standard_normal((m, k)) / k
    V = rng.standard_normal((k, n))
    L = _lib()
    ref0 = A @ V
    e_var = np.linalg.norm(_product(L, A, V, 1) - ref0)
    B = V + 178.0
    e_lvl = np.linalg.norm(_product(L, A, B, 1) - A @ B)
    # the level adds only its FP64 row-sum term: the error stays that of the variation
    assert e_lvl < 2.0 * e_var, (e_lvl, e_var)


def test_bf16x3_accumulates_into_c():
    """beta = 1 (div += opp_3 (norm_tconf - norm_tdisf)) in the tensor-core form."""
    rng = np.random.default_rng(3)
    nu, nf, F, E = 64, 96, 5, 300
    A = rng.standard_normal((nu, nf))
    ntd, ntc, div = (rng.standard_normal((nf, F * E)), rng.standard_normal((nf, F * E)),
                     rng.standard_normal((nu, F * E)))
    ref = div + A @ (ntc - ntd)
    L = _lib()
    dA, d_ntd, d_ntc, d_div = _dev(A), _dev(ntd), _dev(ntc), _dev(div)
    assert L.fr_op_set_gemm_precision(1) == 0
    try:
        assert L.fr_op_calculate_corrected_divergence(nu, nf, F, E, dA.data_ptr(), d_ntd.data_ptr(), d_ntc.data_ptr(),
                                                      d_div.data_ptr(), None) == 0
        assert L.fr_op_check(None) == 0
    finally:
        L.fr_op_set_gemm_precision(0)
    out = _host(d_div, (nu, F * E))
    assert np.linalg.norm(out - ref) / np.linalg.norm(ref) < 3e-5


def test_split_products_reject_operators_beyond_shared_memory():
    L = _lib()
    big = torch.zeros(300 * 300, dtype=torch.float64, device="cuda")
    col = torch.zeros(300 * 10, dtype=torch.float64, device="cuda")
    out = torch.zeros(300 * 10, dtype=torch.float64, device="cuda")
    for mode, (m, k) in ((1, (300, 64)), (1, (200, 200)), (2, (150, 140)), (2, (64, 200))):
        assert L.fr_op_set_gemm_precision(mode) == 0
        try:
            st = L.fr_op_extrapolate_solution(m, k, 1, 10, big.data_ptr(), col.data_ptr(), out.data_ptr(), None)
        finally:
            L.fr_op_set_gemm_precision(0)
        assert st == 5, (mode, m, k)
    assert L.fr_op_set_gemm_precision(4) == 1


def _tgv(pos):
    x, y, z = pos[..., 0], pos[..., 1], pos[..., 2]
    p = 1.0 / (GAMMA * MACH * MACH) + (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0) / 16.0
    u = np.sin(x) * np.cos(y) * np.cos(z)
    v = -np.cos(x) * np.sin(y) * np.cos(z)
    return np.asfortranarray(np.stack([np.ones_like(x), u, v, np.zeros_like(x),
                                       p / (GAMMA - 1.0) + 0.5 * (u * u + v * v)], axis=-1))


def test_operator_path_step_matches_fused_solver_and_bf16x3_error_is_small():
    L2 = 2 * np.pi
    phys = dict(gamma=GAMMA, prandtl=PR, mu_inf=1.0 / RE, rt_inf=1.0, c_sth=1.0, fix_vis=1.0, tau=1.0, pen_fact=0.5)
    s = H.Solver.box(3, 3, (4, 4, 4), (0, 0, 0), (L2, L2, L2), viscous=True, vcjh_scheme=1, **phys)
    u0 = _tgv(s.geometry()["pos_upts"])
    s.set_state(u0)
    s.advance(2, 1e-3)
    fused = s.get_state()
    op = seam.OperatorStage(s, phys, 3, vcjh_scheme=1)
    op.set_state(u0)
    op.advance(2, 1e-3)
    u64 = op.get_state()
    assert np.linalg.norm(u64 - fused) / np.linalg.norm(fused) < 1e-13
    op.set_state(u0)
    op.advance(2, 1e-3, gemm_precision=1)
    u3 = op.get_state()
    err = np.linalg.norm(u3 - u64) / np.linalg.norm(u64)
    # ~16-bit operands: the state (energy ~178 at p0 = 1/(gamma M^2)) carries
    # a few 1e-6 relative error into every product of a stage
    assert 1e-12 < err < 1e-5, err
    op.set_state(u0)
    op.advance(2, 1e-3, gemm_precision=2)
    err6 = np.linalg.norm(op.get_state() - u64) / np.linalg.norm(u64)
    assert err6 < 1e-7 and err6 < err / 10, (err6, err)


@pytest.mark.parametrize("m,k,n", [(96, 64, 5 * 1000 + 3), (64, 64, 64 * 37 + 5), (150, 125, 5 * 200 + 7),
                                   (96, 64, 5 * 32 ** 3)])
@pytest.mark.parametrize("mode", [1, 2])
def test_pipelined_b_tiles_give_identical_products(m, k, n, mode):
    """The next column tile loaded into registers during the current tile's
    MMAs (fr_op_set_gemm_pipelining) changes no value of the product."""
    rng = np.random.default_rng(11 + m + k + n)
    A = rng.standard_normal((m, k))
    B = rng.standard_normal((k, n)) + 3.0
    L = _lib()
    L.fr_op_set_gemm_pipelining.argtypes = [C.c_int]
    try:
        assert L.fr_op_set_gemm_pipelining(0) == 0
        plain = _product(L, A, B, mode)
        assert L.fr_op_set_gemm_pipelining(1) == 0
        piped = _product(L, A, B, mode)
    finally:
        L.fr_op_set_gemm_pipelining(1)
    assert np.isfinite(piped).all()
    assert np.array_equal(plain, piped)


@pytest.mark.parametrize("m,k,n", [(96, 64, 5 * 1000 + 3), (64, 96, 777), (40, 20, 5 * 8 + 3), (20, 40, 64),
                                   (10, 24, 129), (1, 1, 5), (68, 40, 333), (250, 150, 70), (20, 20, 100),
                                   (64, 64, 5 * 4096)])
def test_fp64_tensor_core_product_matches_cuda_cores(m, k, n):
    """Precision mode 0 (FP64 tensor cores) against mode 3 (FP64 CUDA cores)
    and numpy: single products (extrapolate_solution), products fanned out
    over the dimensions (calculate_gradient) and summed over them
    (extrapolate_totalFlux); the two FP64 forms agree bit for bit."""
    rng = np.random.default_rng(11 + m + k)
    A = rng.standard_normal((m, k))
    B = rng.standard_normal((k, n))
    ref = A @ B
    L = _lib()
    c0, c3 = _product(L, A, B, 0), _product(L, A, B, 3)
    assert np.abs(c0 - ref).max() <= 1e-13 * np.abs(ref).max() * max(1, k) ** 0.5
    # the tensor-core product accumulates each k-step of 4 as successive
    # fused multiply-adds in k order, like the CUDA-core chain: same bits
    assert np.array_equal(c0, c3)
    D, F = 3, 1
    As = [rng.standard_normal((m, k)) for _ in range(D)]
    Bs = [rng.standard_normal((k, n)) for _ in range(D)]
    dA = [_dev(a) for a in As]
    tab = (VP * D)(*[a.data_ptr() for a in dA])
    out = {}
    for mode in (0, 3):
        assert L.fr_op_set_gemm_precision(mode) == 0
        try:
            # fan: G_d = A_d B (calculate_gradient: n_upts = m = k square only)
            dB = _dev(Bs[0])
            dS = _dev(np.concatenate([b.ravel(order="F") for b in Bs]))
            dC = torch.zeros(m * n, dtype=torch.float64, device="cuda")
            st = L.fr_op_extrapolate_totalFlux(m, k, D, F, n, C.cast(tab, VP), dS.data_ptr(), dC.data_ptr(), None)
            assert st == 0, H.lib().fr_last_error().decode()
            out[mode] = _host(dC, (m, n))
            if m == k:
                dG = torch.zeros(m * n * D, dtype=torch.float64, device="cuda")
                st = L.fr_op_calculate_gradient(m, D, F, n, C.cast(tab, VP), dB.data_ptr(), dG.data_ptr(), None)
                assert st == 0, H.lib().fr_last_error().decode()
                out[(mode, "fan")] = _host(dG, (m, n, D))
            assert L.fr_op_check(None) == 0
        finally:
            L.fr_op_set_gemm_precision(0)
    want = sum(a @ b for a, b in zip(As, Bs))
    scale = np.abs(want).max() * (D * k) ** 0.5
    assert np.abs(out[0] - want).max() <= 1e-13 * scale
    assert np.array_equal(out[0], out[3])
    if m == k:
        for d in range(D):
            assert np.abs(out[(0, "fan")][..., d] - As[d] @ Bs[0]).max() <= 1e-13 * np.abs(ref).max() * k ** 0.5


@pytest.mark.parametrize("nu,nf,E", [(20, 40, 300), (64, 96, 200), (40, 68, 77)])
def test_fp64_tensor_core_products_that_add_to_their_output(nu, nf, E):
    """The products that accumulate into existing data (beta = 1):
    calculate_corrected_divergence (div += opp_3 (ntc - ntd)) and
    correct_gradient (grad_d += opp_5[d] delta, then the JGinv/detJ
    transform) give the same bits on the FP64 tensor cores (mode 0) as on the
    CUDA cores (mode 3), and match numpy."""
    rng = np.random.default_rng(nu + nf + E)
    F, D = 5, 3
    opp3 = rng.standard_normal((nu, nf))
    opp5 = [rng.standard_normal((nu, nf)) for _ in range(D)]
    ntd, ntc = rng.standard_normal((nf, E, F)), rng.standard_normal((nf, E, F))
    div0 = rng.standard_normal((nu, E, F))
    delta = rng.standard_normal((nf, E, F))
    grad0 = rng.standard_normal((nu, E, F, D))
    JG = rng.standard_normal((D, D, nu, E))
    dj = 1.0 + rng.random((nu, E))
    L = _lib()
    d5 = [_dev(a) for a in opp5]
    tab = (VP * D)(*[a.data_ptr() for a in d5])
    out = {}
    for mode in (0, 3):
        assert L.fr_op_set_gemm_precision(mode) == 0
        try:
            dA, dntd, dntc, ddiv = _dev(opp3), _dev(ntd), _dev(ntc), _dev(div0)
            st = L.fr_op_calculate_corrected_divergence(nu, nf, F, E, dA.data_ptr(), dntd.data_ptr(), dntc.data_ptr(),
                                                        ddiv.data_ptr(), None)
            assert st == 0, H.lib().fr_last_error().decode()
            dd, dg, dJ, ddj = _dev(delta), _dev(grad0), _dev(JG), _dev(dj)
            st = L.fr_op_correct_gradient(nu, nf, D, F, E, C.cast(tab, VP), dd.data_ptr(), dJ.data_ptr(),
                                          ddj.data_ptr(), dg.data_ptr(), None)
            assert st == 0, H.lib().fr_last_error().decode()
            assert L.fr_op_check(None) == 0
            out[mode] = (_host(ddiv, (nu, E, F)), _host(dg, (nu, E, F, D)))
        finally:
            L.fr_op_set_gemm_precision(0)
    assert np.array_equal(out[0][0], out[3][0]) and np.array_equal(out[0][1], out[3][1])
    want = div0 + np.einsum("uf,fek->uek", opp3, ntc - ntd)
    assert np.abs(out[0][0] - want).max() <= 1e-13 * np.abs(want).max() * nf ** 0.5
