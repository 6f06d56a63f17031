"""Training and evaluation of the learned SGS closure (sgs_model 5) on
decaying homogeneous isotropic turbulence, with this solver producing its own
training data.

Pipeline (every heavy step runs on the GPU):
  1. initial field: random-phase (seeded) solenoidal velocity on the periodic
     box [0, 2 pi]^3 with spectrum E(k) ~ k^4 exp(-2 (k/k0)^2), k0 = 4,
     scaled to u_rms = 1; rho = 1, p = 1/(gamma M^2) (Mach 0.1);
  2. a fine hex mesh (nf^3, order P) advanced without a model;
  3. snapshots projected onto the coarse mesh (nc^3, same P, nf = r nc): the
     L2 projection of the fine piecewise polynomials onto each coarse
     element's polynomial space (exact Gauss quadrature on the r^3 nested
     fine elements) is the filter; SGS stress
     tau_ij = bar(rho u_i u_j) - bar(rho u_i) bar(rho u_j) / bar(rho);
  4. target: the SGS dissipation eps* = -tau^d : S (S the deviatoric strain
     of the filtered field), which the closure's form gives as
     c * s with s = rho Delta^2 |S|^3; the closure is fitted to
     c* = eps* / s with sample weights s^2, i.e. least squares on the
     dissipation itself; inputs from the solver (fr_solver_sgs_features), so
     training and use see the same numbers;
  5. training with the library's CUDA kernels (fr_mlp_loss_grad, fr_mlp_adam);
  6. evaluation: a priori on a held-out snapshot (SGS dissipation
     tau^d : S predicted by the closure, by WALE and by no model), and a
     posteriori (coarse LES from the filtered initial field with no model,
     WALE and the closure, resolved kinetic energy against the filtered fine
     solution).
"""
import math

import numpy as np

from . import Solver, mlp_adam, mlp_loss_grad, mlp_n_params, mlp_n_trained, mlp_scratch_floats

GAMMA = 1.4
IN, H = 6, 64


def _torch():
    import torch
    return torch


# ------------------------------------------------------------------ initial field

def hit_velocity(pos, seed, k0=4.0, kmax=12, urms=1.0):
    """Solenoidal random-phase velocity at points pos (..., 3); E(k) ~ k^4
    exp(-2 (k/k0)^2) over integer wavevectors |k| <= kmax, scaled so that
    the mean of |u|^2 / 3 over the points is urms^2."""
    torch = _torch()
    rng = np.random.default_rng(seed)
    r = np.arange(-kmax, kmax + 1)
    K = np.stack(np.meshgrid(r, r, r, indexing="ij"), axis=-1).reshape(-1, 3)
    kk = np.linalg.norm(K, axis=1)
    # half space: one of each +-k pair (the real part supplies the conjugate)
    half = (K[:, 0] > 0) | ((K[:, 0] == 0) & (K[:, 1] > 0)) | ((K[:, 0] == 0) & (K[:, 1] == 0) & (K[:, 2] > 0))
    K, kk = K[half & (kk <= kmax)], kk[half & (kk <= kmax)]
    E = kk ** 4 * np.exp(-2.0 * (kk / k0) ** 2)
    amp = np.sqrt(E / (4.0 * np.pi * kk ** 2))
    a = rng.standard_normal((len(K), 3)) + 1j * rng.standard_normal((len(K), 3))
    khat = K / kk[:, None]
    a -= (a * khat).sum(axis=1, keepdims=True) * khat          # solenoidal: a . k = 0
    a *= (amp / np.sqrt((np.abs(a) ** 2).sum(axis=1)))[:, None]
    dev = "cuda"
    Kt = torch.tensor(K, dtype=torch.float64, device=dev)
    ar = torch.tensor(a.real, dtype=torch.float64, device=dev)
    ai = torch.tensor(a.imag, dtype=torch.float64, device=dev)
    P = pos.reshape(-1, 3)
    out = np.empty_like(P)
    for s in range(0, len(P), 1 << 15):
        x = torch.tensor(P[s:s + (1 << 15)], dtype=torch.float64, device=dev)
        ph = x @ Kt.T
        u = torch.cos(ph) @ ar - torch.sin(ph) @ ai
        out[s:s + (1 << 15)] = (2.0 * u).cpu().numpy()
    out *= urms / math.sqrt((out ** 2).sum(axis=1).mean() / 3.0)
    return out.reshape(pos.shape)


def hit_state(pos, seed, mach=0.1, **kw):
    u = hit_velocity(pos, seed, **kw)
    p0 = 1.0 / (GAMMA * mach * mach)
    rho = np.ones(pos.shape[:-1])
    E = p0 / (GAMMA - 1.0) + 0.5 * rho * (u ** 2).sum(axis=-1)
    return np.asfortranarray(np.concatenate([rho[..., None], rho[..., None] * u, E[..., None]], axis=-1))


# ------------------------------------------------------------------ projection filter

def _gauss(P):
    return np.polynomial.legendre.leggauss(P + 1)


def _lagrange(nodes, x):
    """L[a, i] = l_a(x_i) for the Lagrange basis on nodes."""
    L = np.ones((len(nodes), len(x)))
    for a in range(len(nodes)):
        for b in range(len(nodes)):
            if b != a:
                L[a] *= (x - nodes[b]) / (nodes[a] - nodes[b])
    return L


def projection_matrix(P, r):
    """Pi (P+1, r(P+1)): nodal values at the coarse Gauss points of the L2
    projection onto one coarse interval of a function given by its values at
    the Gauss points of r equal sub-intervals (exact for piecewise degree P)."""
    xg, wg = _gauss(P)
    xs = np.concatenate([-1.0 + (2 * j + 1 + xg) / r for j in range(r)])
    ws = np.concatenate([wg / r for _ in range(r)])
    return _lagrange(xg, xs) * ws[None, :] / wg[:, None]


def _grid(s, n):
    """Element grid index (i, j, k) of every element of a box solver, from its
    solution points, and a check of the tensor point order (x fastest)."""
    g = s.geometry()["pos_upts"]                       # (nu, E, 3)
    c = g.mean(axis=0)
    h = 2 * np.pi / n
    ijk = np.floor(c / h).astype(np.int64)
    N1 = round(s.n_upts ** (1 / 3))
    x = g[:, 0, :].reshape(N1, N1, N1, 3, order="F")   # [a, b, c]
    assert np.all(np.diff(x[:, 0, 0, 0]) > 0) and np.all(np.diff(x[0, :, 0, 1]) > 0)
    return ijk, N1


def filter_fields(fields, fine, coarse, nf, nc):
    """Project fine-mesh point fields (nu_f, E_f, m) onto the coarse mesh ->
    (nu_c, E_c, m)."""
    torch = _torch()
    r = nf // nc
    ijk_f, N1 = _grid(fine, nf)
    ijk_c, _ = _grid(coarse, nc)
    m = fields.shape[2]
    Pm = torch.tensor(projection_matrix(N1 - 1, r), dtype=torch.float64, device="cuda")
    # fine values on a global grid [I, J, K, a, b, c]
    order = np.argsort((ijk_f[:, 0] + nf * (ijk_f[:, 1] + nf * ijk_f[:, 2])))
    out = np.empty((N1 ** 3, nc ** 3, m))
    corder = np.argsort((ijk_c[:, 0] + nc * (ijk_c[:, 1] + nc * ijk_c[:, 2])))
    for q in range(m):
        v = torch.tensor(np.ascontiguousarray(fields[:, order, q].T), dtype=torch.float64, device="cuda")
        v = v.reshape(nc, r, nc, r, nc, r, N1, N1, N1)           # [Kc, rk, Jc, rj, Ic, ri, c, b, a]
        v = v.permute(4, 2, 0, 5, 8, 3, 7, 1, 6).reshape(nc, nc, nc, r * N1, r * N1, r * N1)
        w = torch.einsum("ax,by,cz,IJKxyz->IJKabc", Pm, Pm, Pm, v)  # [Ic, Jc, Kc, a, b, c]
        w = w.permute(2, 1, 0, 5, 4, 3).reshape(nc ** 3, N1 ** 3)   # element k-major, point c-major
        out[:, corder, q] = w.cpu().numpy().T
    return out


# ------------------------------------------------------------------ targets and reference models

def _strain(q, g):
    """Deviatoric strain S (n, 3, 3) and |S| from state q (n, 5) and gradient g (n, 5, 3)."""
    rho = q[:, 0]
    u = q[:, 1:4] / rho[:, None]
    A = (g[:, 1:4, :] - u[:, :, None] * g[:, 0:1, :]) / rho[:, None, None]
    tr = np.trace(A, axis1=1, axis2=2)
    S = 0.5 * (A + A.transpose(0, 2, 1)) - np.eye(3)[None] * (tr / 3.0)[:, None, None]
    return S, A, np.sqrt(2.0 * (S * S).sum(axis=(1, 2)))


def _delta(detj, P, filter_ratio):
    return filter_ratio * np.cbrt(8.0 * detj) / (P + 1.0)


def sgs_targets(coarse, q, tau, P, filter_ratio=1.0):
    """(inputs X, target c* = eps* / s, dissipation scale s, |S|, Delta, S) at
    the coarse points for a filtered state q (nu, E, 5) set into `coarse` and
    the SGS stress tau (n, 3, 3)."""
    coarse.set_state(q)
    X = coarse.sgs_features()
    g = coarse.gradient().reshape(-1, 5, 3, order="F")
    qq = q.reshape(-1, 5, order="F")
    S, _, smag = _strain(qq, g)
    trt = np.trace(tau, axis1=1, axis2=2)
    taud = tau - np.eye(3)[None] * (trt / 3.0)[:, None, None]
    eps = -(taud * S).sum(axis=(1, 2))
    detj = coarse.geometry()["detjac_upts"].reshape(-1, order="F")
    delta = _delta(detj, P, filter_ratio)
    s = qq[:, 0] * delta ** 2 * smag ** 3
    return X, eps / (s + 1e-30), s, smag, delta, S


def wale_coefficient(q, g, delta, smag):
    """c of the WALE eddy viscosity (Cw = 0.5) in the closure's form."""
    S, A, _ = _strain(q, g)
    A2 = A @ A
    Sq = 0.5 * (A2 + A2.transpose(0, 2, 1)) - np.eye(3)[None] * (np.trace(A2, axis1=1, axis2=2) / 3.0)[:, None, None]
    num = (Sq * Sq).sum(axis=(1, 2))
    den = (S * S).sum(axis=(1, 2))
    mu = q[:, 0] * 0.25 * delta ** 2 * num ** 1.5 / (den ** 2.5 + num ** 1.25 + 1e-12)
    return mu / (q[:, 0] * delta ** 2 * smag + 1e-30)


# ------------------------------------------------------------------ training

def train(X, Y, W=None, epochs=60, batch=65536, lr=2e-3, seed=0, cmax=2.0):
    """Fit the closure to targets Y (clipped to [-cmax, cmax]) with sample
    weights W (normalised to mean 1 and capped at 50) using the library's CUDA
    kernels; returns the parameter vector (float32) and the mean loss of each
    epoch."""
    torch = _torch()
    rng = np.random.default_rng(seed)
    X = np.asarray(X, dtype=np.float32)
    Y = np.clip(np.asarray(Y, dtype=np.float32), -cmax, cmax)
    if W is None:
        W = np.ones(len(Y))
    W = np.asarray(W, dtype=np.float64)
    W = np.minimum(W / W.mean(), 50.0).astype(np.float32)
    xm = X.mean(axis=0)
    xs = 1.0 / (X.std(axis=0) + 1e-6)
    npar, ntr = mlp_n_params(), mlp_n_trained()
    w = np.zeros(npar, dtype=np.float32)
    a1, a2, a3 = math.sqrt(6.0 / (IN + H)), math.sqrt(6.0 / (2 * H)), math.sqrt(6.0 / (H + 1))
    w[0:H * IN] = rng.uniform(-a1, a1, H * IN)
    w[H * IN + H:H * IN + H + H * H] = rng.uniform(-a2, a2, H * H)
    o3 = H * IN + H + H * H + H
    w[o3:o3 + H] = rng.uniform(-a3, a3, H)
    ymean = float((W * Y).sum() / W.sum())
    w[ntr - 1] = math.log(math.expm1(max(ymean, 1e-4)))         # start at the mean coefficient
    w[ntr:ntr + IN] = xm
    w[ntr + IN:] = xs
    dev = "cuda"
    dw = torch.tensor(w, device=dev)
    dX = torch.tensor(X, device=dev)
    dY = torch.tensor(Y, device=dev)
    dW = torch.tensor(W, device=dev)
    g = torch.zeros(ntr, dtype=torch.float32, device=dev)
    m, v = torch.zeros_like(g), torch.zeros_like(g)
    loss = torch.zeros(1, dtype=torch.float32, device=dev)
    nb = min(batch, len(Y))
    ns = mlp_scratch_floats(nb)
    scratch = torch.empty(ns, dtype=torch.float32, device=dev)
    hist, step = [], 0
    n = len(Y)
    for ep in range(epochs):
        perm = torch.tensor(rng.permutation(n), device=dev)
        tot = 0.0
        for s in range(0, n - nb + 1, nb):
            idx = perm[s:s + nb]
            bx, by, bw = dX[idx].contiguous(), dY[idx].contiguous(), dW[idx].contiguous()
            mlp_loss_grad(dw.data_ptr(), bx.data_ptr(), by.data_ptr(), nb, g.data_ptr(), loss.data_ptr(),
                          scratch.data_ptr(), ns, d_sw=bw.data_ptr())
            step += 1
            mlp_adam(dw.data_ptr(), g.data_ptr(), m.data_ptr(), v.data_ptr(), step, lr)
            tot += float(loss.item())
        hist.append(tot / max(1, n // nb))
    return dw.cpu().numpy(), hist


def predict(w, X):
    """c of the closure for inputs X on the GPU (fr_mlp_forward)."""
    torch = _torch()
    from . import mlp_forward
    dw = torch.tensor(np.asarray(w, dtype=np.float32), device="cuda")
    dX = torch.tensor(np.asarray(X, dtype=np.float32), device="cuda")
    out = torch.empty(len(X), dtype=torch.float32, device="cuda")
    mlp_forward(dw.data_ptr(), dX.data_ptr(), len(X), out.data_ptr())
    return out.cpu().numpy().astype(np.float64)


# ------------------------------------------------------------------ experiment

def _filtered_snapshot(fine, coarse, nf, nc):
    u = fine.get_state()
    rho = u[:, :, 0]
    vel = u[:, :, 1:4] / rho[..., None]
    prod = [u[:, :, 1 + i] * vel[..., j] for i in range(3) for j in range(i, 3)]
    f = filter_fields(np.concatenate([u, np.stack(prod, axis=-1)], axis=-1), fine, coarse, nf, nc)
    q = np.asfortranarray(f[:, :, :5])
    qq = q.reshape(-1, 5, order="F")
    rr = f[:, :, 5:].reshape(-1, 6, order="F")
    tau = np.empty((len(qq), 3, 3))
    it = 0
    for i in range(3):
        for j in range(i, 3):
            tau[:, i, j] = tau[:, j, i] = rr[:, it] - qq[:, 1 + i] * qq[:, 1 + j] / qq[:, 0]
            it += 1
    return q, tau


def run_experiment(nf=24, nc=6, P=3, mu=2e-3, dt=1e-3, t_snaps=(0.25, 0.5), t_eval=0.75, seed=1, epochs=60,
                   filter_ratio=1.0, log=print):
    """Whole pipeline; returns a dict of a-priori and a-posteriori figures."""
    box = dict(lo=(0.0, 0.0, 0.0), hi=(2 * np.pi,) * 3)
    kw = dict(viscous=True, gamma=GAMMA, prandtl=0.71, mu_inf=mu, tau=1.0, pen_fact=0.5)
    fine = Solver.box(3, P, (nf,) * 3, box["lo"], box["hi"], **kw)
    coarse = Solver.box(3, P, (nc,) * 3, box["lo"], box["hi"], les=1, sgs_model=5, filter_ratio=filter_ratio, **kw)
    fine.set_state(hit_state(fine.geometry()["pos_upts"], seed))
    q0, _ = _filtered_snapshot(fine, coarse, nf, nc)
    ke_f = {0.0: _ke(coarse, q0)}
    data, t = [], 0.0
    for ts in list(t_snaps) + [t_eval]:
        ns = int(round((ts - t) / dt))
        fine.advance(ns, dt)
        t = ts
        q, tau = _filtered_snapshot(fine, coarse, nf, nc)
        ke_f[ts] = _ke(coarse, q)
        data.append((ts, q, tau))
        log("fine t=%.3f filtered KE %.6f" % (ts, ke_f[ts]))
    Xs, Ys, Ws = [], [], []
    for ts, q, tau in data[:-1]:
        X, c, s, smag, delta, S = sgs_targets(coarse, q, tau, P, filter_ratio)
        Xs.append(X)
        Ys.append(c)
        Ws.append(s * s)
    X, Y, W = np.concatenate(Xs), np.concatenate(Ys), np.concatenate(Ws)
    w, hist = train(X, Y, W, epochs=epochs, seed=seed)
    log("training loss %.4e -> %.4e over %d epochs, %d samples" % (hist[0], hist[-1], len(hist), len(Y)))
    # a priori on the held-out snapshot: SGS dissipation tau^d:S against the models'
    ts, q, tau = data[-1]
    X, c, scale, smag, delta, S = sgs_targets(coarse, q, tau, P, filter_ratio)
    qq = q.reshape(-1, 5, order="F")
    g = coarse.gradient().reshape(-1, 5, 3, order="F")
    eps_true = c * scale                                          # SGS dissipation (>0 forward scatter)
    c_mlp = predict(w, X)
    c_wale = wale_coefficient(qq, g, delta, smag)
    apriori = {}
    for name, cm in (("none", np.zeros_like(c)), ("wale", c_wale), ("learned", c_mlp)):
        e = cm * scale
        apriori[name] = {"mean_dissipation": float(e.mean()),
                         "rel_l2_error": float(np.linalg.norm(e - eps_true) / np.linalg.norm(eps_true)),
                         "corr": float(np.corrcoef(e, eps_true)[0, 1]) if name != "none" else 0.0}
    apriori["true_mean_dissipation"] = float(eps_true.mean())
    # a posteriori: coarse LES from the filtered initial field
    post = {}
    spec_f = energy_spectrum(coarse, data[-1][1], nc)
    kmax = nc * (P + 1) // 3                      # the well-resolved wavenumbers of the coarse mesh
    tk = sorted(float(k) for k in ke_f)
    diss_f = -np.diff([ke_f[k] for k in tk]) / np.diff(tk)
    for name in ("none", "wale", "learned"):
        kw2 = dict(kw)
        if name == "wale":
            les = dict(les=1, sgs_model=1, filter_ratio=filter_ratio)
        elif name == "learned":
            les = dict(les=1, sgs_model=5, filter_ratio=filter_ratio)
        else:
            les = {}
        s = Solver.box(3, P, (nc,) * 3, box["lo"], box["hi"], **les, **kw2)
        if name == "learned":
            s.set_sgs_mlp(w)
        s.set_state(q0)
        kes, t = {}, 0.0
        for ts in list(t_snaps) + [t_eval]:
            s.advance(int(round((ts - t) / dt)), dt)
            t = ts
            kes[ts] = s.kinetic_energy()
        err = [abs(kes[ts] - ke_f[ts]) / ke_f[ts] for ts in kes]
        spec = energy_spectrum(s, s.get_state(), nc)
        kes0 = {**kes, 0.0: ke_f[0.0]}
        diss = -np.diff([kes0[k] for k in tk]) / np.diff(tk)
        post[name] = {"ke": {str(k): v for k, v in kes.items()}, "mean_rel_ke_error": float(np.mean(err)),
                      "spectrum_t_eval": spec.tolist(), "spectrum_log_error": spectrum_error(spec, spec_f, kmax),
                      "dissipation_rate": diss.tolist(),
                      "dissipation_rel_error": float(np.linalg.norm(diss - diss_f) / np.linalg.norm(diss_f))}
        s.close()
    return {"config": {"fine": nf, "coarse": nc, "order": P, "mu": mu, "dt": dt, "t_snaps": list(t_snaps),
                       "t_eval": t_eval, "seed": seed, "samples": int(len(Y))},
            "loss_history": [float(h) for h in hist], "filtered_fine_ke": {str(k): v for k, v in ke_f.items()},
            "filtered_fine_spectrum_t_eval": spec_f.tolist(), "filtered_fine_dissipation_rate": diss_f.tolist(),
            "spectrum_kmax": int(kmax),
            "a_priori": apriori, "a_posteriori": post, "params": w}


def energy_spectrum(solver, q, n):
    """Shell-averaged kinetic-energy spectrum E(k), k = 1 .. n(P+1)/2, of the
    velocity of a state q (nu, E, 5) on the periodic box of n^3 elements:
    the velocity is interpolated to the (P+1)^3 uniform cell centres of every
    element, Fourier transformed on the n(P+1) grid, and E(k) sums
    |u_hat|^2 / 2 over the wavenumbers with |k| in [k - 1/2, k + 1/2)."""
    ijk, N1 = _grid(solver, n)
    xg, _ = _gauss(N1 - 1)
    xu = -1.0 + (2 * np.arange(N1) + 1) / N1
    Lm = _lagrange(xg, xu)                              # [a, a'] = l_a(x_a')
    M = n * N1
    vel = q[:, :, 1:4] / q[:, :, :1]                    # (nu, E, 3)
    grid = np.zeros((3, M, M, M))
    v = vel.reshape(N1, N1, N1, -1, 3, order="F")       # [a, b, c, e, comp]
    w = np.einsum("aA,bB,cC,abcem->ABCem", Lm, Lm, Lm, v)
    for e in range(vel.shape[1]):
        i, j, k = ijk[e]
        grid[:, k * N1:(k + 1) * N1, j * N1:(j + 1) * N1, i * N1:(i + 1) * N1] = \
            w[:, :, :, e, :].transpose(3, 2, 1, 0)      # [comp, z, y, x]
    uh = np.fft.fftn(grid, axes=(1, 2, 3)) / M ** 3
    e3 = 0.5 * (np.abs(uh) ** 2).sum(axis=0)
    kk = np.fft.fftfreq(M, 1.0 / M)
    kz, ky, kx = np.meshgrid(kk, kk, kk, indexing="ij")
    kmag = np.sqrt(kx ** 2 + ky ** 2 + kz ** 2)
    shells = np.rint(kmag).astype(np.int64)
    spec = np.bincount(shells.ravel(), weights=e3.ravel(), minlength=M)
    return spec[1:M // 2 + 1]


def spectrum_error(spec, ref, kmax):
    """Relative L2 distance of log E(k) from the reference's over k = 1 .. kmax."""
    a, b = np.log(spec[:kmax]), np.log(ref[:kmax])
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _ke(coarse, q):
    coarse.set_state(q)
    return coarse.kinetic_energy()


if __name__ == "__main__":
    import argparse
    import json
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--fine", type=int, default=96)
    ap.add_argument("--coarse", type=int, default=24)
    ap.add_argument("--order", type=int, default=3)
    ap.add_argument("--mu", type=float, default=5e-4)
    ap.add_argument("--dt", type=float, default=2.5e-4)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    r = run_experiment(a.fine, a.coarse, a.order, a.mu, a.dt, epochs=a.epochs)
    w = r.pop("params")
    print(json.dumps(r, indent=1))
    if a.out:
        with open(a.out, "w") as f:
            json.dump(r, f, indent=1)
        np.save(a.out + ".params.npy", w)
