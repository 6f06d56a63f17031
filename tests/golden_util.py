"""Loading of the committed golden fixtures (tests/golden/*.npz, made by
tests/golden/make_golden.py from runs of the reference itself)."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# eddy-viscosity LES cases (WALE and Smagorinsky SGS flux)
LES_CASES = ["hex_wale_p3_n3_jit", "hex_smag_p2_n3", "quad_wale_p3_n6_jit"]
# Roe common flux (2-D)
ROE_CASES = ["quad_vortex_roe_p3_n6_jit", "quad_ns_roe_p2_n5"]
# boundary conditions (every Euler/Navier-Stokes boundary type of the reference)
BC_CASES = ["quad_bc_euler_p3", "quad_bc_euler2_p2", "quad_bc_roe_p3", "quad_ns_bc_p3", "hex_channel_p2",
            "hex_channel_char_p3"]
CASES = ["quad_vortex_p3_n6", "quad_vortex_p2_n5_jit", "quad_vortex_p3_n20", "hex_tgv_p3_n3",
         "hex_tgv_p2_n3_jit", "hex_tgv_p4_n2", "hex_euler_p3_n3", "quad_vortex_p1_n8_jit", "quad_vortex_p5_n4",
         "hex_tgv_p1_n4_jit"] + LES_CASES + ROE_CASES


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    meta = json.loads(str(z["meta"]))
    arrs = {k: np.asfortranarray(z[k]) for k in z.files if k != "meta"}
    return meta, arrs


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


# integral quantities on the reference's volume cubature (iq_*.npz from make_golden.py --integrals)
IQ_CASES = ["iq_hex_tgv_p3_n3_jit", "iq_hex_tgv_p2_n3_jit_cub5", "iq_quad_vortex_p3_n6_jit_cub4"]


def integral_quantities_numpy(u, grad, opp, weight, detjac, dims, gamma):
    """numpy restatement of eles::CalcIntegralQuantities (src/eles.cpp:6503-6641):
    state and gradient interpolated to the cubature points with opp (nc, nu),
    the five quantities, weights x detJ at the cubature points.  Returns the
    five integrals and the integrals of their absolute values (the scale
    against which a cancelling sum such as the pressure dilatation is compared)."""
    F = dims + 2
    uc = np.einsum("jk,kem->jem", opp, u)                     # (nc, E, F)
    gc = np.einsum("jk,kemn->jemn", opp, grad)                # (nc, E, F, D)
    irho = 1.0 / uc[..., 0]
    A = irho[..., None, None] * (gc[..., 1:1 + dims, :] - uc[..., 1:1 + dims, None] * irho[..., None, None] *
                                 gc[..., 0:1, :])          # A[a][b] = d u_a / d x_b
    tke = (0.5 * uc[..., 1:F - 1] * uc[..., 1:F - 1]).sum(axis=-1)
    ke = irho * tke
    wz = A[..., 1, 0] - A[..., 0, 1]
    vort = wz * wz
    if dims == 3:
        vort = vort + (A[..., 2, 1] - A[..., 1, 2]) ** 2 + (A[..., 0, 2] - A[..., 2, 0]) ** 2
    vort = vort * 0.5 / irho
    p = (gamma - 1.0) * (uc[..., F - 1] - irho * tke)
    pd = p * np.trace(A, axis1=-2, axis2=-1)
    S = 0.5 * (A + np.swapaxes(A, -1, -2))
    sc = (S * S).sum(axis=(-2, -1))
    Sd = S - np.eye(dims) * (np.trace(S, axis1=-2, axis2=-1) / 3.0)[..., None, None]
    dsc = (Sd * Sd).sum(axis=(-2, -1))
    wj = weight[:, None] * detjac                             # (nc, E)
    vals = [float((x * wj).sum()) for x in (ke, vort, pd, sc, dsc)]
    mags = [float((np.abs(x) * wj).sum()) for x in (ke, vort, pd, sc, dsc)]
    return vals, mags


def _lagrange_matrix(xs, xq):
    n = len(xs)
    M = np.ones((len(xq), n))
    for m in range(n):
        for i in range(n):
            if i != m:
                M[:, m] *= (xq - xs[i]) / (xs[m] - xs[i])
    return M


def over_integrated_density_error(u, pos, P, h, t):
    """L2 error of the density of a 2-D vortex state u (nu, E, 4) on a uniform
    quad mesh of spacing h: the solution and the positions interpolated to the
    (P + 3)-point Gauss rule of each element, the exact vortex (initial field
    shifted by (t, 0)) evaluated there, weights times the constant Jacobian."""
    import oracle as O
    x1 = O.points_1d(P)
    xq, wq = np.polynomial.legendre.leggauss(P + 3)
    M1 = _lagrange_matrix(x1, xq)
    M = np.kron(M1, M1)                       # point i + nq j <- a + n1 b
    W = np.kron(wq, wq)
    rq = M @ u[:, :, 0]
    pq = np.stack([M @ pos[:, :, d] for d in range(2)], axis=-1)
    ex = O.ic_vortex(pq, t=t)[..., 0]
    return float(np.sqrt((W[:, None] * (h / 2) ** 2 * (rq - ex) ** 2).sum()))
