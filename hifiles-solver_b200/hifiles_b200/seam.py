"""The reference's residual as a sequence of per-operator calls.

`OperatorStage` runs CalcResidual (src/solver.cpp:65-225) and
eles::AdvanceSolution (src/eles.cpp:1091-1188) for one element type through
the fr_op_* entry points of include/fr_b200.h: the dense operators
opp_0 .. opp_6 applied to all elements (the reference's cublasDgemm calls),
the pointwise flux kernels, and the interface kernels over tables of
pointers (int_inters' disu_fpts_l / _r ... pointer arrays).  The operator
products run in FP64 (0) or as BF16 split products on the tensor cores,
BF16x3 (1) or BF16x6 (2) (`fr_op_set_gemm_precision`); `gemm_precision`
selects it per call.

The dense operators are built from the library's 1-D factors (`fr_line_operators`):
for Gauss solution points every row of opp_0 .. opp_6 has one non-zero 1-D
factor per line, so the Kronecker construction below reproduces the
reference's matrices (eles::set_opp_0 .. set_opp_6, src/eles.cpp:3620-4052)
entry for entry.
"""
import ctypes as C

import numpy as np

from . import _check, lib, line_operators

_VP = C.c_void_p


class PhysDesc(C.Structure):
    """fr_phys_desc of include/fr_b200.h."""
    _fields_ = [(n, C.c_double) for n in ("gamma", "prandtl", "mu_inf", "rt_inf", "c_sth", "fix_vis", "tau",
                                          "pen_fact")]


def _face_lines(dims, P):
    """Per flux point: (fixed coordinates, axis, plus) of the line of solution
    points through it, in the reference's flux-point order (quads
    src/eles_quads.cpp:259-300, hexes src/eles_hexas.cpp:262-324)."""
    n = P + 1
    nfpf = n ** (dims - 1)
    out = []
    for f in range(2 * dims * nfpf):
        fc, r = divmod(f, nfpf)
        if dims == 2:
            j = r
            out.append({0: ((j, None), 1, 0), 1: ((None, j), 0, 1), 2: ((P - j, None), 1, 1),
                        3: ((None, P - j), 0, 0)}[fc])
        else:
            j, k = divmod(r, n)
            out.append({0: ((P - k, j, None), 2, 0), 1: ((k, None, j), 1, 0), 2: ((None, k, j), 0, 1),
                        3: ((P - k, None, j), 1, 1), 4: ((None, P - k, j), 0, 0), 5: ((k, j, None), 2, 1)}[fc])
    return out


def dense_operators(dims, P, upts_type=0, vcjh_scheme=1, eta=0.0):
    """opp_0 (nf x nu), opp_1[d] (nf x nu), opp_2[d] = opp_4[d] (nu x nu),
    opp_3 (nu x nf), opp_5[d] (nu x nf), opp_6 = opp_0, column-major float64."""
    L = line_operators(P, upts_type, vcjh_scheme, eta)
    n = P + 1
    nu = n ** dims
    lines = _face_lines(dims, P)
    nf = len(lines)

    def abc(u):
        return (u % n, (u // n) % n, u // (n * n)) if dims == 3 else (u % n, u // n, 0)

    o0 = np.zeros((nf, nu))
    o3 = np.zeros((nu, nf))
    nrm = np.zeros((nf, dims))            # reference-element unit normal of each flux point
    for f, (fixed, ax, plus) in enumerate(lines):
        nrm[f, ax] = 1.0 if plus else -1.0
        for u in range(nu):
            c = abc(u)
            if all(fixed[d] is None or fixed[d] == c[d] for d in range(dims)):
                o0[f, u] = (L["Lp"] if plus else L["Lm"])[c[ax]]
                o3[u, f] = L["gR"][c[ax]] if plus else -L["gL"][c[ax]]
    o2 = []
    for d in range(dims):
        Dm = np.zeros((nu, nu))
        for k in range(nu):
            ck = abc(k)
            for u in range(nu):
                cu = abc(u)
                if all(cu[e] == ck[e] for e in range(dims) if e != d):
                    Dm[k, u] = L["D"][ck[d], cu[d]]
        o2.append(Dm)
    o1 = [o0 * nrm[:, d][:, None] for d in range(dims)]
    o5 = [o3 * nrm[:, d][None, :] for d in range(dims)]
    F = lambda a: np.asfortranarray(a)  # noqa: E731
    return dict(opp_0=F(o0), opp_1=[F(a) for a in o1], opp_2=[F(a) for a in o2], opp_3=F(o3),
                opp_4=[F(a) for a in o2], opp_5=[F(a) for a in o5], opp_6=F(o0))


def ellpack(a, zero_tol=1e-12):
    """(data, indices, nnz_per_row) of a dense operator in the ELL layout of
    array_to_ellpack (src/funcs.cpp:961-1011): entries with |a| >= 1e-12, in
    increasing column order, slot s of row i at i + m s; padding slots hold 0
    at column 0."""
    a = np.asarray(a, dtype=np.float64)
    m = a.shape[0]
    keep = np.abs(a) >= zero_tol
    nnz = int(keep.sum(axis=1).max()) if m else 0
    data = np.zeros(nnz * m)
    idx = np.zeros(nnz * m, dtype=np.int32)
    for i in range(m):
        cols = np.nonzero(keep[i])[0]
        data[i + m * np.arange(len(cols))] = a[i, cols]
        idx[i + m * np.arange(len(cols))] = cols
    return data, idx, nnz


def _bind(L):
    i, vp = C.c_int, _VP
    sig = {
        "fr_op_extrapolate_solution": [i, i, i, i, vp, vp, vp, vp],
        "fr_op_evaluate_invFlux": [i, i, i, i, vp, vp, vp, vp, vp],
        "fr_op_calculate_gradient": [i, i, i, i, vp, vp, vp, vp],
        "fr_op_correct_gradient": [i, i, i, i, i, vp, vp, vp, vp, vp, vp],
        "fr_op_extrapolate_corrected_gradient": [i, i, i, i, i, vp, vp, vp, vp],
        "fr_op_evaluate_viscFlux": [i, i, i, i, vp, vp, vp, vp, vp, vp],
        "fr_op_extrapolate_totalFlux": [i, i, i, i, i, vp, vp, vp, vp],
        "fr_op_calculate_divergence": [i, i, i, i, vp, vp, vp, vp],
        "fr_op_calculate_corrected_divergence": [i, i, i, i, vp, vp, vp, vp, vp],
        "fr_op_int_inters_common_invFlux": [i, i, i, i] + [vp] * 9 + [vp, i, i, vp],
        "fr_op_int_inters_common_viscFlux": [i, i, i, i] + [vp] * 9 + [vp, vp],
        "fr_op_advance_rk45": [i, i, i, i, C.c_double, C.c_double, vp, vp, vp, vp, vp, vp],
        "fr_op_spmv_ell": [i, i, i, i, vp, vp, i, vp, vp, i, i, i, vp],
        "fr_op_set_gemm_precision": [i],
        "fr_op_check": [vp],
    }
    for name, args in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = C.c_int
    L.fr_op_gemm_precision.restype = C.c_int
    return L


class OperatorStage:
    """One element type of a periodic mesh, advanced through the per-operator
    entry points.  `solver` (a hifiles_b200.Solver of the same scheme) supplies
    the metrics and the interface wiring; the state lives here as a torch
    tensor of layout (n_upts, n_eles, n_fields)."""

    def __init__(self, solver, physics, order, vcjh_scheme=1, eta=0.0, upts_type=0, viscous=True):
        import torch
        self.torch = torch
        self.L = _bind(lib())
        s = solver
        self.E, self.nu, self.nf, self.F, self.D = s.n_eles, s.n_upts, s.n_fpts, s.n_fields, s.dims
        self.visc = bool(viscous)
        E, nu, nf, F, D = self.E, self.nu, self.nf, self.F, self.D
        dev = "cuda:%d" % s.device
        z = lambda n: torch.zeros(n, dtype=torch.float64, device=dev)  # noqa: E731
        t = lambda a: torch.from_numpy(np.asfortranarray(a).ravel(order="F")).to(dev)  # noqa: E731
        ops = dense_operators(D, order, upts_type, vcjh_scheme, eta)
        self._ops = {k: (t(v) if not isinstance(v, list) else [t(a) for a in v]) for k, v in ops.items()}
        self._tabs = {k: (C.c_void_p * D)(*[a.data_ptr() for a in self._ops[k]])
                      for k in ("opp_1", "opp_2", "opp_4", "opp_5")}
        g = s.geometry()
        self.JG, self.dj, self.tdA, self.nrm = (t(g[k]) for k in ("JGinv_upts", "detjac_upts", "tdA_fpts",
                                                                   "norm_fpts"))
        self.u, self.reg, self.div = z(nu * E * F), z(nu * E * F), z(nu * E * F)
        self.ufp, self.ntc, self.ntd, self.ddu = z(nf * E * F), z(nf * E * F), z(nf * E * F), z(nf * E * F)
        self.tf, self.gup, self.gfp = z(nu * E * F * D), z(nu * E * F * D), z(nf * E * F * D)
        il, ir = s.interfaces()
        il, ir = il.astype(np.int64), ir.astype(np.int64)
        self.ni = len(il)
        fk = np.arange(F)[None, :] * (nf * E)
        gk = (np.arange(F)[:, None] + F * np.arange(D)[None, :]).ravel(order="F")[None, :] * (nf * E)

        def table(base, offsets):
            a = base.data_ptr() + 8 * np.asarray(offsets, dtype=np.int64).ravel(order="F")
            return torch.from_numpy(a.astype(np.int64)).to(dev)

        self._pt = dict(ul=table(self.ufp, il[:, None] + fk), ur=table(self.ufp, ir[:, None] + fk),
                        tl=table(self.ntc, il[:, None] + fk), tr=table(self.ntc, ir[:, None] + fk),
                        dl=table(self.ddu, il[:, None] + fk), dr=table(self.ddu, ir[:, None] + fk),
                        al=table(self.tdA, il), ar=table(self.tdA, ir),
                        n=table(self.nrm, il[:, None] + np.arange(D)[None, :] * (nf * E)),
                        gl=table(self.gfp, il[:, None] + gk), gr=table(self.gfp, ir[:, None] + gk))
        self.ph = PhysDesc(**physics)
        self.stream = torch.cuda.current_stream(dev)

    # -- state
    def set_state(self, u):
        self.u.copy_(self.torch.from_numpy(np.asfortranarray(u).ravel(order="F")))

    def get_state(self):
        self.torch.cuda.synchronize()
        return self.u.cpu().numpy().reshape((self.nu, self.E, self.F), order="F")

    def _ok(self, st):
        if st != 0:
            raise RuntimeError(lib().fr_last_error().decode())

    def residual(self, gemm_precision=0):
        """div_tconf_upts of the current state (CalcResidual)."""
        L, P = self.L, (lambda a: a.data_ptr())
        E, nu, nf, F, D = self.E, self.nu, self.nf, self.F, self.D
        sp = C.c_void_p(self.stream.cuda_stream)
        ph = C.byref(self.ph)
        pt = {k: P(v) for k, v in self._pt.items()}
        self._ok(L.fr_op_set_gemm_precision(int(gemm_precision)))
        try:
            self._ok(L.fr_op_extrapolate_solution(nf, nu, F, E, P(self._ops["opp_0"]), P(self.u), P(self.ufp), sp))
            if self.visc:
                self._ok(L.fr_op_calculate_gradient(nu, D, F, E, C.cast(self._tabs["opp_4"], _VP), P(self.u),
                                                    P(self.gup), sp))
            self._ok(L.fr_op_evaluate_invFlux(nu, D, F, E, P(self.u), P(self.JG), P(self.tf), ph, sp))
            self._ok(L.fr_op_int_inters_common_invFlux(1, D, F, self.ni, pt["ul"], pt["ur"], pt["tl"], pt["tr"],
                                                       pt["al"], pt["ar"], pt["n"], pt["dl"], pt["dr"], ph, 0,
                                                       int(self.visc), sp))
            if self.visc:
                self._ok(L.fr_op_correct_gradient(nu, nf, D, F, E, C.cast(self._tabs["opp_5"], _VP), P(self.ddu),
                                                  P(self.JG), P(self.dj), P(self.gup), sp))
                self._ok(L.fr_op_extrapolate_corrected_gradient(nf, nu, D, F, E, P(self._ops["opp_6"]),
                                                                P(self.gup), P(self.gfp), sp))
                self._ok(L.fr_op_evaluate_viscFlux(nu, D, F, E, P(self.u), P(self.gup), P(self.JG), P(self.tf),
                                                   ph, sp))
            self._ok(L.fr_op_extrapolate_totalFlux(nf, nu, D, F, E, C.cast(self._tabs["opp_1"], _VP), P(self.tf),
                                                   P(self.ntd), sp))
            self._ok(L.fr_op_calculate_divergence(nu, D, F, E, C.cast(self._tabs["opp_2"], _VP), P(self.tf),
                                                  P(self.div), sp))
            if self.visc:
                self._ok(L.fr_op_int_inters_common_viscFlux(1, D, F, self.ni, pt["ul"], pt["ur"], pt["gl"],
                                                            pt["gr"], pt["tl"], pt["tr"], pt["al"], pt["ar"],
                                                            pt["n"], ph, sp))
            self._ok(L.fr_op_calculate_corrected_divergence(nu, nf, F, E, P(self._ops["opp_3"]), P(self.ntd),
                                                            P(self.ntc), P(self.div), sp))
        finally:
            L.fr_op_set_gemm_precision(0)
        return self.div

    def advance(self, n_steps, dt, gemm_precision=0):
        """n_steps RK45 steps (5 stages each) through the operator seam."""
        L, P = self.L, (lambda a: a.data_ptr())
        sp = C.c_void_p(self.stream.cuda_stream)
        for _ in range(n_steps):
            for k in range(5):
                self.residual(gemm_precision)
                self._ok(L.fr_op_advance_rk45(self.nu, self.F, self.E, k, float(dt), 0.0, P(self.u), P(self.reg),
                                              P(self.div), P(self.dj), None, sp))
        self._ok(L.fr_op_check(sp))


def _bind_bdy(L):
    i, vp = C.c_int, _VP
    L.fr_op_bdy_inters_common_invFlux.argtypes = [i, i, i, i] + [vp] * 7 + [vp, C.c_double, i, i, vp]
    L.fr_op_bdy_inters_common_viscFlux.argtypes = [i, i, i, i] + [vp] * 7 + [vp, C.c_double, vp]
    L.fr_op_bdy_inters_common_invFlux.restype = C.c_int
    L.fr_op_bdy_inters_common_viscFlux.restype = C.c_int
    return L


class MixedOperatorMesh:
    """A mesh of several element types (tets, prisms, hexes, ...) advanced
    through the per-operator entry points, in the order of CalcResidual
    (src/solver.cpp:65-225): every element type for each element step, every
    interface type for each interface step.

    `types` maps the caller's element-type index to a dict with that type's
    dense operators as the caller's classes build them (opp_0, opp_3, opp_6;
    lists of n_dims matrices opp_1, opp_2, opp_4, opp_5), its metrics
    (JGinv_upts, detjac_upts, tdA_fpts, norm_fpts) and its state u
    (n_upts, n_eles, n_fields).  `int_inters` lists int32 arrays
    (6, n_fpts_per_inter, n_inters) of (type, element, flux point) of the left
    and right side of every interface point (int_inters' pointer tables,
    src/int_inters.cpp:95-178, as indices); `bdy_inters` lists
    (4, n_fpts_per_inter, n_inters) arrays of the owning side's triple and the
    boundary type (bdy_inters, src/bdy_inters.cpp:111-203), whose boundary
    values `bdy` (14, bdy_inters::set_bdy_params order) and gas constant
    `R_ref` apply.  Navier-Stokes in 2-D (tris, quads) or 3-D; the state
    lives on the device."""

    def __init__(self, types, int_inters, physics, bdy_inters=(), bdy=None, R_ref=1.0, device=0):
        import torch
        self.torch = torch
        self.L = _bind_bdy(_bind(lib()))
        dev = "cuda:%d" % device
        self.dev = dev
        D = int(np.asarray(next(iter(types.values()))["JGinv_upts"]).shape[0])
        F = D + 2
        self.D, self.F = D, F
        t = lambda a: torch.from_numpy(np.asfortranarray(a, dtype=np.float64).ravel(order="F").copy()).to(dev)  # noqa
        z = lambda n: torch.zeros(n, dtype=torch.float64, device=dev)  # noqa: E731
        self.S = {}
        for i, ty in types.items():
            nu, E, _ = ty["u"].shape
            nf = ty["opp_0"].shape[0]
            s = dict(nu=nu, nf=nf, E=E)
            for k in ("opp_0", "opp_3", "opp_6"):
                s[k] = t(ty[k])
            for k in ("opp_1", "opp_2", "opp_4", "opp_5"):
                s[k] = [t(a) for a in ty[k]]
                s[k + "_tab"] = (C.c_void_p * D)(*[a.data_ptr() for a in s[k]])
            s["JG"], s["dj"], s["tdA"], s["nrm"] = (t(ty[k]) for k in ("JGinv_upts", "detjac_upts", "tdA_fpts",
                                                                         "norm_fpts"))
            s["u"], s["reg"], s["div"] = t(ty["u"]), z(nu * E * F), z(nu * E * F)
            s["ufp"], s["ntc"], s["ntd"], s["ddu"] = z(nf * E * F), z(nf * E * F), z(nf * E * F), z(nf * E * F)
            s["tf"], s["gup"], s["gfp"] = z(nu * E * F * D), z(nu * E * F * D), z(nf * E * F * D)
            self.S[i] = s

        def table(w, side, arr, comps):
            tt, e, f = (np.asarray(w[side + q]).reshape(-1, order="F").astype(np.int64) for q in range(3))
            rows = np.zeros((tt.size, comps), dtype=np.int64)
            for i, s in self.S.items():
                m = tt == i
                if m.any():
                    slot = f[m] + s["nf"] * e[m]
                    rows[m] = s[arr].data_ptr() + 8 * (slot[:, None] + s["nf"] * s["E"] * np.arange(comps)[None, :])
            return torch.from_numpy(np.asfortranarray(rows).ravel(order="F").copy()).to(dev)

        self.inters = []
        for w in int_inters:
            tb = dict(nfpi=int(w.shape[1]), ni=int(w.shape[2]))
            for side, sx in ((0, "l"), (3, "r")):
                tb["u" + sx], tb["t" + sx] = table(w, side, "ufp", F), table(w, side, "ntc", F)
                tb["d" + sx], tb["g" + sx] = table(w, side, "ddu", F), table(w, side, "gfp", F * D)
                tb["a" + sx] = table(w, side, "tdA", 1)
            tb["n"] = table(w, 0, "nrm", D)
            self.inters.append(tb)
        self.bdys = []
        for w in bdy_inters:
            tb = dict(nfpi=int(w.shape[1]), ni=int(w.shape[2]))
            tb["ul"], tb["tl"], tb["dl"] = table(w, 0, "ufp", F), table(w, 0, "ntc", F), table(w, 0, "ddu", F)
            tb["gl"], tb["al"], tb["n"] = table(w, 0, "gfp", F * D), table(w, 0, "tdA", 1), table(w, 0, "nrm", D)
            tb["type"] = torch.from_numpy(np.ascontiguousarray(np.asarray(w)[3, 0, :]).astype(np.int32)).to(dev)
            self.bdys.append(tb)
        self.bdy = torch.tensor(list(bdy) if bdy is not None else [0.0] * 14, dtype=torch.float64, device=dev)
        self.R_ref = float(R_ref)
        self.ph = PhysDesc(**physics)
        self.stream = torch.cuda.current_stream(dev)

    @property
    def dofs(self):
        """Solution DOFs (points x fields) over all element types."""
        return sum(s["nu"] * s["E"] * self.F for s in self.S.values())

    def get_state(self, i):
        self.torch.cuda.synchronize()
        s = self.S[i]
        return s["u"].cpu().numpy().reshape((s["nu"], s["E"], self.F), order="F")

    def _ok(self, st):
        if st != 0:
            raise RuntimeError(lib().fr_last_error().decode())

    def residual(self, gemm_precision=0):
        """div_tconf_upts of every element type (CalcResidual)."""
        L, P, ok, D, F = self.L, (lambda a: a.data_ptr()), self._ok, self.D, self.F
        sp = C.c_void_p(self.stream.cuda_stream)
        ph = C.byref(self.ph)
        cast = lambda tab: C.cast(tab, _VP)  # noqa: E731
        ok(L.fr_op_set_gemm_precision(int(gemm_precision)))
        try:
            for s in self.S.values():
                nu, nf, E = s["nu"], s["nf"], s["E"]
                ok(L.fr_op_extrapolate_solution(nf, nu, F, E, P(s["opp_0"]), P(s["u"]), P(s["ufp"]), sp))
                ok(L.fr_op_calculate_gradient(nu, D, F, E, cast(s["opp_4_tab"]), P(s["u"]), P(s["gup"]), sp))
                ok(L.fr_op_evaluate_invFlux(nu, D, F, E, P(s["u"]), P(s["JG"]), P(s["tf"]), ph, sp))
            for tb in self.inters:
                ok(L.fr_op_int_inters_common_invFlux(tb["nfpi"], D, F, tb["ni"], P(tb["ul"]), P(tb["ur"]),
                                                     P(tb["tl"]), P(tb["tr"]), P(tb["al"]), P(tb["ar"]), P(tb["n"]),
                                                     P(tb["dl"]), P(tb["dr"]), ph, 0, 1, sp))
            for tb in self.bdys:
                ok(L.fr_op_bdy_inters_common_invFlux(tb["nfpi"], D, F, tb["ni"], P(tb["ul"]), P(tb["tl"]),
                                                     P(tb["al"]), P(tb["n"]), P(tb["type"]), P(self.bdy),
                                                     P(tb["dl"]), ph, self.R_ref, 0, 1, sp))
            for s in self.S.values():
                nu, nf, E = s["nu"], s["nf"], s["E"]
                ok(L.fr_op_correct_gradient(nu, nf, D, F, E, cast(s["opp_5_tab"]), P(s["ddu"]), P(s["JG"]),
                                            P(s["dj"]), P(s["gup"]), sp))
                ok(L.fr_op_extrapolate_corrected_gradient(nf, nu, D, F, E, P(s["opp_6"]), P(s["gup"]), P(s["gfp"]),
                                                          sp))
                ok(L.fr_op_evaluate_viscFlux(nu, D, F, E, P(s["u"]), P(s["gup"]), P(s["JG"]), P(s["tf"]), ph, sp))
                ok(L.fr_op_extrapolate_totalFlux(nf, nu, D, F, E, cast(s["opp_1_tab"]), P(s["tf"]), P(s["ntd"]), sp))
                ok(L.fr_op_calculate_divergence(nu, D, F, E, cast(s["opp_2_tab"]), P(s["tf"]), P(s["div"]), sp))
            for tb in self.inters:
                ok(L.fr_op_int_inters_common_viscFlux(tb["nfpi"], D, F, tb["ni"], P(tb["ul"]), P(tb["ur"]),
                                                      P(tb["gl"]), P(tb["gr"]), P(tb["tl"]), P(tb["tr"]),
                                                      P(tb["al"]), P(tb["ar"]), P(tb["n"]), ph, sp))
            for tb in self.bdys:
                ok(L.fr_op_bdy_inters_common_viscFlux(tb["nfpi"], D, F, tb["ni"], P(tb["ul"]), P(tb["gl"]),
                                                      P(tb["tl"]), P(tb["al"]), P(tb["n"]), P(tb["type"]),
                                                      P(self.bdy), ph, self.R_ref, sp))
            for s in self.S.values():
                ok(L.fr_op_calculate_corrected_divergence(s["nu"], s["nf"], F, s["E"], P(s["opp_3"]), P(s["ntd"]),
                                                          P(s["ntc"]), P(s["div"]), sp))
        finally:
            L.fr_op_set_gemm_precision(0)

    def advance(self, n_steps, dt, gemm_precision=0):
        """n_steps RK45 steps (5 stages each), eles::AdvanceSolution per type."""
        L, P = self.L, (lambda a: a.data_ptr())
        sp = C.c_void_p(self.stream.cuda_stream)
        for _ in range(n_steps):
            for k in range(5):
                self.residual(gemm_precision)
                for s in self.S.values():
                    self._ok(L.fr_op_advance_rk45(s["nu"], self.F, s["E"], k, float(dt), 0.0, P(s["u"]),
                                                  P(s["reg"]), P(s["div"]), P(s["dj"]), None, sp))
        self._ok(L.fr_op_check(sp))


class _MixedStageType(C.Structure):
    _fields_ = [("n_upts", C.c_int), ("n_fpts", C.c_int), ("n_eles", C.c_longlong), ("opp_0", _VP),
                ("opp_1", _VP * 3), ("opp_2", _VP * 3), ("opp_3", _VP), ("opp_4", _VP * 3), ("opp_5", _VP * 3),
                ("opp_6", _VP), ("JGinv_upts", _VP), ("detjac_upts", _VP), ("tdA_fpts", _VP), ("norm_fpts", _VP),
                ("disu_upts", _VP), ("div_tconf_upts", _VP)]


def _bind_stage(L):
    i, vp, ll = C.c_int, _VP, C.c_longlong
    L.fr_mixed_stage_create.argtypes = [i, i, vp, i, vp, vp, vp, i, vp, vp, vp, vp, C.c_double, vp, i, i, vp]
    L.fr_mixed_stage_destroy.argtypes = [vp]
    L.fr_mixed_stage_residual.argtypes = [vp, vp]
    L.fr_mixed_stage_advance.argtypes = [vp, i, C.c_double, vp]
    L.fr_mixed_stage_info.argtypes = [vp, C.POINTER(ll), C.POINTER(ll), C.POINTER(i)]
    L.fr_mixed_stage_set_launch.argtypes = [vp, i, i, i]
    L.fr_mixed_stage_get_launch.argtypes = [vp, i, C.POINTER(i), C.POINTER(i)]
    L.fr_mixed_stage_autotune.argtypes = [vp, vp]
    L.fr_mixed_stage_set_concurrent.argtypes = [vp, i]
    L.fr_mixed_stage_advance_norms.argtypes = [vp, i, C.c_double, vp, vp]
    for f in ("fr_mixed_stage_create", "fr_mixed_stage_destroy", "fr_mixed_stage_residual", "fr_mixed_stage_advance",
              "fr_mixed_stage_info", "fr_mixed_stage_set_launch", "fr_mixed_stage_get_launch",
              "fr_mixed_stage_autotune", "fr_mixed_stage_set_concurrent", "fr_mixed_stage_advance_norms"):
        getattr(L, f).restype = C.c_int
    return L


class FusedMixedMesh:
    """The mesh of `MixedOperatorMesh` (same arguments) advanced by the fused
    stage of include/fr_b200.h (`fr_mixed_stage_*`): per element type and RK
    stage one gradient kernel and one interface/update kernel, operator
    products on the FP64 tensor cores.  Navier-Stokes (viscous) or Euler
    (Rusanov, or Roe in 2-D: riemann 2) in 2-D (triangles, quads) or 3-D
    (tets, prisms, hexes), orders 1 to 4 (hexes 1 to 3).  The
    state of type i is `S[i]["u"]` (n_upts, n_eles, n_fields) on the device,
    advanced in place; `residual()` writes `S[i]["div"]`."""

    def __init__(self, types, int_inters, physics, bdy_inters=(), bdy=None, R_ref=1.0, device=0, viscous=True,
                 riemann=0):
        import torch
        self.torch = torch
        self.L = _bind_stage(lib())
        dev = "cuda:%d" % device
        self.dev = dev
        keys = list(types.keys())
        pos = {k: j for j, k in enumerate(keys)}
        D = int(np.asarray(types[keys[0]]["JGinv_upts"]).shape[0])
        self.D, self.F = D, D + 2
        keep = []  # host arrays the C call reads

        def host(a):
            a = np.asfortranarray(a, dtype=np.float64)
            keep.append(a)
            return a.ctypes.data

        descs = (_MixedStageType * len(keys))()
        self.S = {}
        for j, k in enumerate(keys):
            ty = types[k]
            nu, E, _ = ty["u"].shape
            nf = ty["opp_0"].shape[0]
            s = dict(nu=nu, nf=nf, E=E)
            s["u"] = torch.from_numpy(np.asfortranarray(ty["u"], dtype=np.float64).ravel(order="F").copy()).to(dev)
            s["div"] = torch.zeros(nu * E * self.F, dtype=torch.float64, device=dev)
            self.S[k] = s
            d = descs[j]
            d.n_upts, d.n_fpts, d.n_eles = nu, nf, E
            d.opp_0, d.opp_3 = host(ty["opp_0"]), host(ty["opp_3"])
            d.opp_6 = host(ty["opp_6"]) if ty.get("opp_6") is not None else None
            for name in ("opp_1", "opp_2", "opp_4", "opp_5"):
                if ty.get(name) is None:
                    continue  # Euler: no gradient operators
                arr = getattr(d, name)
                for q in range(D):
                    arr[q] = host(ty[name][q])
            d.JGinv_upts, d.detjac_upts = host(ty["JGinv_upts"]), host(ty["detjac_upts"])
            d.tdA_fpts, d.norm_fpts = host(ty["tdA_fpts"]), host(ty["norm_fpts"])
            d.disu_upts, d.div_tconf_upts = s["u"].data_ptr(), s["div"].data_ptr()

        def tables(ws, type_rows):
            ptrs, nfpi, ni = [], [], []
            for w in ws:
                w = np.array(w, dtype=np.int32, order="F", copy=True)
                for r in type_rows:
                    t = w[r].copy()
                    w[r] = -1
                    for k, j in pos.items():
                        w[r][t == k] = j
                keep.append(w)
                ptrs.append(w.ctypes.data)
                nfpi.append(w.shape[1])
                ni.append(w.shape[2])
            n = len(ws)
            return (n, (_VP * max(n, 1))(*ptrs), (C.c_int * max(n, 1))(*nfpi), (C.c_longlong * max(n, 1))(*ni))

        ni_, ip, inf, inn = tables(int_inters, (0, 3))
        nb_, bp, bnf, bnn = tables(bdy_inters, (0,))
        bdy_arr = (C.c_double * 14)(*(list(bdy) if bdy is not None else [0.0] * 14))
        self.ph = PhysDesc(**physics)
        h = _VP()
        _check(self.L.fr_mixed_stage_create(D, len(keys), descs, ni_, ip, inf, inn, nb_, bp, bnf, bnn, bdy_arr,
                                            float(R_ref), C.byref(self.ph), int(bool(viscous)), int(riemann),
                                            C.byref(h)))
        self.h = h
        self._pos = pos
        self.stream = torch.cuda.current_stream(dev)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.fr_mixed_stage_destroy(self.h)
            self.h = None

    @property
    def dofs(self):
        """Solution DOFs (points x fields) over all element types."""
        return sum(s["nu"] * s["E"] * self.F for s in self.S.values())

    @property
    def launches_per_stage(self):
        n = C.c_int()
        _check(self.L.fr_mixed_stage_info(self.h, None, None, C.byref(n)))
        return n.value

    def get_state(self, i):
        self.torch.cuda.synchronize()
        s = self.S[i]
        return s["u"].cpu().numpy().reshape((s["nu"], s["E"], self.F), order="F")

    def set_state(self, i, u):
        s = self.S[i]
        s["u"].copy_(self.torch.from_numpy(np.asfortranarray(u, dtype=np.float64).ravel(order="F")))

    def launch(self, i):
        """(gradient, update) launch shapes of element type i."""
        g, u = C.c_int(), C.c_int()
        _check(self.L.fr_mixed_stage_get_launch(self.h, self._pos[i], C.byref(g), C.byref(u)))
        return g.value, u.value

    def set_launch(self, i, grad_shape, update_shape):
        _check(self.L.fr_mixed_stage_set_launch(self.h, self._pos[i], int(grad_shape), int(update_shape)))

    def set_concurrent(self, on):
        """Element types on side streams (True, default) or all on one stream."""
        _check(self.L.fr_mixed_stage_set_concurrent(self.h, int(bool(on))))

    def autotune(self):
        """Time every launch shape on the current state, keep the fastest."""
        _check(self.L.fr_mixed_stage_autotune(self.h, _VP(self.stream.cuda_stream)))
        return {i: self.launch(i) for i in self.S}

    def residual(self):
        """div_tconf_upts of every element type (one CalcResidual) into S[i]["div"]."""
        _check(self.L.fr_mixed_stage_residual(self.h, _VP(self.stream.cuda_stream)))

    def advance(self, n_steps, dt, norms=False):
        """n_steps RK45 steps (5 stages each); with norms, returns the L1
        residual norms of the last step (CalcNormResidual, res_norm_type 1)."""
        if not norms:
            _check(self.L.fr_mixed_stage_advance(self.h, int(n_steps), float(dt), _VP(self.stream.cuda_stream)))
            return None
        out = np.zeros(self.F)
        _check(self.L.fr_mixed_stage_advance_norms(self.h, int(n_steps), float(dt), out.ctypes.data,
                                                   _VP(self.stream.cuda_stream)))
        return out


def tile_mixed_mesh(types, int_inters, bdy_inters, copies):
    """`copies` independent copies of a mixed mesh (element axis tiled, every
    copy's interfaces wired to its own elements), for throughput runs on a
    mesh whose operators and metrics come from one small set-up."""
    out = {}
    for i, ty in types.items():
        E = ty["u"].shape[1]
        o = {k: ty[k] for k in ("opp_0", "opp_1", "opp_2", "opp_3", "opp_4", "opp_5", "opp_6")}
        o["JGinv_upts"] = np.tile(ty["JGinv_upts"], (1, 1, 1, copies))
        o["detjac_upts"] = np.tile(ty["detjac_upts"], (1, copies))
        o["tdA_fpts"] = np.tile(ty["tdA_fpts"], (1, copies))
        o["norm_fpts"] = np.tile(ty["norm_fpts"], (1, copies, 1))
        o["u"] = np.tile(ty["u"], (1, copies, 1))
        o["_E"] = E
        out[i] = o

    def shift(w, sides):
        w = np.asarray(w)
        parts = []
        for c in range(copies):
            x = w.copy()
            for s in sides:
                for i, o in out.items():
                    m = x[s] == i
                    x[s + 1][m] += c * o["_E"]
            parts.append(x)
        return np.concatenate(parts, axis=2)

    ints = [shift(w, (0, 3)) for w in int_inters]
    bdys = [shift(w, (0,)) for w in bdy_inters]
    for o in out.values():
        del o["_E"]
    return out, ints, bdys


def mixed_mesh_inputs(meta, arrays, state_key="disu_upts_init"):
    """(types, int_inters, bdy_inters) for MixedOperatorMesh from arrays named
    as the reference's objects dump them: per element type with ele_type et,
    t<et>_opp_0, t<et>_opp_<w>_<d>, t<et>_JGinv_upts ... t<et>_<state_key>;
    int_inters_<k> / bdy_inters_<k> wiring; `meta` lists the element types
    ({"index", "ele_type"}), interface and boundary types ({"index"})."""
    types = {}
    dims = int(meta.get("dims", 3))
    for t in meta["types"]:
        X = "t%d_" % t["ele_type"]
        ty = {k: arrays.get(X + k) for k in ("opp_0", "opp_3", "opp_6", "JGinv_upts", "detjac_upts", "tdA_fpts",
                                             "norm_fpts")}
        for w in (1, 2, 4, 5):  # an Euler run's objects have no opp_4 / opp_5 / opp_6
            ops = [arrays.get(X + "opp_%d_%d" % (w, d)) for d in range(dims)]
            ty["opp_%d" % w] = None if any(o is None for o in ops) else ops
        ty["u"] = arrays[X + state_key]
        types[t["index"]] = ty
    ints = [arrays["int_inters_%d" % it["index"]] for it in meta["inters"]]
    bdys = [arrays["bdy_inters_%d" % it["index"]] for it in meta.get("bdy_inters", [])]
    return types, ints, bdys
