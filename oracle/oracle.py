"""ctypes binding of oracle/liboracle.so (the CPU restatement in fr_oracle.c).

TEST INFRASTRUCTURE ONLY.  The product never imports this module; tests/, the
smoke check and bench.py's CPU-baseline leg use it as the checker.

Arrays use the reference's array<T> layouts (first index fastest), exposed to
numpy as Fortran-ordered arrays: u[upt, ele, field], grad[upt, ele, field, dim].
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")


def build():
    """Compile liboracle.so (and nothing from the reference)."""
    subprocess.run(["make", "-s", "-C", HERE, os.path.join(HERE, "liboracle.so")], check=True)


def _lib():
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(os.path.join(HERE, "fr_oracle.c")):
        build()
    lib = C.CDLL(LIB)
    P = C.c_void_p
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int)
    lib.or_box_new_bc.restype = P
    lib.or_box_new_bc.argtypes = [C.c_int, C.c_int, ip, dp, dp, C.c_double, C.c_ulonglong, ip, C.c_int, C.c_int,
                                  C.c_double]
    lib.or_n_boundary.restype = C.c_int
    lib.or_n_boundary.argtypes = [P]
    lib.or_get_boundary.argtypes = [P, ip, ip]
    lib.or_box_new.restype = P
    lib.or_box_new.argtypes = [C.c_int, C.c_int, ip, dp, dp, C.c_double, C.c_ulonglong, C.c_int, C.c_int, C.c_double]
    lib.or_mesh_new.restype = P
    lib.or_mesh_new.argtypes = [C.c_int, C.c_int, C.c_int, dp, C.c_int, ip, dp, C.c_int, C.c_int, C.c_double]
    lib.or_mesh_free.argtypes = [P]
    lib.or_sizes.argtypes = [P, ip]
    lib.or_get_geometry.argtypes = [P, dp, dp, dp, dp, dp, dp]
    lib.or_get_interfaces.argtypes = [P, ip, ip]
    lib.or_set_geometry.argtypes = [P, dp, dp, dp, dp]
    lib.or_set_interfaces.argtypes = [P, C.c_int, ip, ip]
    lib.or_get_operator.argtypes = [P, C.c_int, C.c_int, dp, ip]
    lib.or_residual.argtypes = [P, C.c_void_p, dp, dp, dp]
    lib.or_stage_offsets.argtypes = [P, C.POINTER(C.c_longlong)]
    lib.or_rk45.argtypes = [P, C.c_void_p, dp, dp, C.c_double, C.c_int, dp]
    lib.or_kinetic_energy.restype = C.c_double
    lib.or_kinetic_energy.argtypes = [P, dp]
    lib.or_points_1d.argtypes = [C.c_int, C.c_int, dp]
    return lib


_L = None


def lib():
    global _L
    if _L is None:
        _L = _lib()
    return _L


class Physics(C.Structure):
    _fields_ = [("viscous", C.c_int), ("gamma", C.c_double), ("prandtl", C.c_double),
                ("mu_inf", C.c_double), ("rt_inf", C.c_double), ("c_sth", C.c_double),
                ("fix_vis", C.c_double), ("tau", C.c_double), ("pen_fact", C.c_double),
                ("les", C.c_int), ("sgs_model", C.c_int), ("filter_ratio", C.c_double),
                ("mlp", C.POINTER(C.c_float)), ("riemann", C.c_int), ("bdy", C.c_double * 14),
                ("R_ref", C.c_double)]


def physics(viscous=0, gamma=1.4, prandtl=0.72, mu_inf=0.0, rt_inf=1.0, c_sth=1.0, fix_vis=1.0,
            tau=1.0, pen_fact=0.5, les=0, sgs_model=1, filter_ratio=1.0, mlp=None, riemann=0, bdy=None, R_ref=1.0):
    """mlp: float32 parameter vector of the learned closure (sgs_model 5); the
    returned structure keeps a reference to it."""
    ptr = None
    if mlp is not None:
        mlp = np.ascontiguousarray(mlp, dtype=np.float32)
        ptr = mlp.ctypes.data_as(C.POINTER(C.c_float))
    ph = Physics(int(viscous), gamma, prandtl, mu_inf, rt_inf, c_sth, fix_vis, tau, pen_fact, int(les),
                 int(sgs_model), float(filter_ratio), ptr, int(riemann),
                 (C.c_double * 14)(*(list(bdy) if bdy is not None else [0.0] * 14)), float(R_ref))
    ph._keep = mlp
    return ph


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def points_1d(order, upts_type=0):
    out = np.zeros(order + 1)
    lib().or_points_1d(order, upts_type, _dp(out))
    return out


class Mesh:
    """One element type (quads in 2-D or hexes in 3-D) on a conforming periodic mesh."""

    def __init__(self, handle):
        if not handle:
            raise RuntimeError("oracle mesh construction failed")
        self.h = handle
        s = (C.c_int * 6)()
        lib().or_sizes(self.h, s)
        self.n_eles, self.n_upts, self.n_fpts, self.n_fields, self.dims, self.n_int = list(s)

    @classmethod
    def box(cls, dims, order, n, lo, hi, jitter=0.0, seed=0, upts_type=0, vcjh_scheme=1, eta=0.0, side_bc=None):
        """side_bc: boundary type of the sides x-, x+, y-, y+(, z-, z+); 0 = periodic."""
        n = np.ascontiguousarray(list(n) + [1] * (3 - len(n)), dtype=np.int32)
        lo = np.ascontiguousarray(list(lo) + [0.0] * (3 - len(lo)), dtype=np.float64)
        hi = np.ascontiguousarray(list(hi) + [0.0] * (3 - len(hi)), dtype=np.float64)
        if side_bc is not None:
            sb = np.ascontiguousarray(side_bc, dtype=np.int32)
            return cls(lib().or_box_new_bc(dims, order, _ip(n), _dp(lo), _dp(hi), float(jitter), int(seed), _ip(sb),
                                           upts_type, vcjh_scheme, float(eta)))
        return cls(lib().or_box_new(dims, order, _ip(n), _dp(lo), _dp(hi), float(jitter), int(seed),
                                    upts_type, vcjh_scheme, float(eta)))

    def boundary(self):
        """(flat flux-point index, boundary type) of every boundary flux point."""
        nb = lib().or_n_boundary(self.h)
        i = np.zeros(nb, dtype=np.int32)
        t = np.zeros(nb, dtype=np.int32)
        if nb:
            lib().or_get_boundary(self.h, _ip(i), _ip(t))
        return i, t

    @classmethod
    def from_vertices(cls, dims, order, xv, c2v, shift, upts_type=0, vcjh_scheme=1, eta=0.0):
        xv = np.ascontiguousarray(xv, dtype=np.float64)
        c2v = np.ascontiguousarray(c2v, dtype=np.int32)
        shift = np.ascontiguousarray(list(shift) + [0.0] * (3 - len(shift)), dtype=np.float64)
        return cls(lib().or_mesh_new(dims, order, xv.shape[0], _dp(xv), c2v.shape[0], _ip(c2v), _dp(shift),
                                     upts_type, vcjh_scheme, float(eta)))

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_mesh_free(self.h)
            self.h = None

    def _f(self, *shape):
        return np.zeros(shape, dtype=np.float64, order="F")

    def geometry(self):
        E, nu, nf, D = self.n_eles, self.n_upts, self.n_fpts, self.dims
        g = dict(pos_upts=self._f(nu, E, D), detjac_upts=self._f(nu, E), JGinv_upts=self._f(D, D, nu, E),
                 tdA_fpts=self._f(nf, E), norm_fpts=self._f(nf, E, D), pos_fpts=self._f(nf, E, D))
        lib().or_get_geometry(self.h, *[_dp(g[k]) for k in
                                        ("pos_upts", "detjac_upts", "JGinv_upts", "tdA_fpts", "norm_fpts", "pos_fpts")])
        return g

    def interfaces(self):
        l = np.zeros(self.n_int, dtype=np.int32)
        r = np.zeros(self.n_int, dtype=np.int32)
        lib().or_get_interfaces(self.h, _ip(l), _ip(r))
        return l, r

    def set_geometry(self, detjac_upts, JGinv_upts, tdA_fpts, norm_fpts):
        a = [np.asfortranarray(x, dtype=np.float64) for x in (detjac_upts, JGinv_upts, tdA_fpts, norm_fpts)]
        lib().or_set_geometry(self.h, *[_dp(x) for x in a])

    def set_interfaces(self, left, right):
        l = np.ascontiguousarray(left, dtype=np.int32)
        r = np.ascontiguousarray(right, dtype=np.int32)
        lib().or_set_interfaces(self.h, len(l), _ip(l), _ip(r))
        self.n_int = len(l)

    def operator(self, which, dim=0):
        shape = (C.c_int * 2)()
        lib().or_get_operator(self.h, which, dim, None, shape)
        out = np.zeros((shape[0], shape[1]), dtype=np.float64, order="F")
        lib().or_get_operator(self.h, which, dim, _dp(out), shape)
        return out

    def state_shape(self):
        return (self.n_upts, self.n_eles, self.n_fields)

    def residual(self, ph, u, stages=False):
        """div_tconf_upts of one CalcResidual; optionally the intermediate arrays."""
        u = np.asfortranarray(u, dtype=np.float64)
        div = np.zeros(self.state_shape(), order="F")
        st = None
        if stages:
            off = (C.c_longlong * 10)()
            lib().or_stage_offsets(self.h, off)
            st = np.zeros(off[9], dtype=np.float64)
            lib().or_residual(self.h, C.byref(ph), _dp(u), _dp(div), _dp(st))
            E, nu, nf, F, D = self.n_eles, self.n_upts, self.n_fpts, self.n_fields, self.dims
            shapes = [(nf, E, F), (nu, E, F, D), (nf, E, F, D), (nu, E, F, D), (nf, E, F), (nf, E, F), (nf, E, F),
                      (nu, E, F, D), (nf, E, F, D)]
            names = ["disu_fpts", "grad_disu_upts", "grad_disu_fpts", "tdisf_upts", "norm_tdisf_fpts",
                     "norm_tconf_fpts", "delta_disu_fpts", "sgsf_upts", "sgsf_fpts"]
            st = {n: st[off[i]:off[i + 1]].reshape(s, order="F") for i, (n, s) in enumerate(zip(names, shapes))}
            return div, st
        lib().or_residual(self.h, C.byref(ph), _dp(u), _dp(div), None)
        return div

    def rk45(self, ph, u, dt, n_steps, reg=None, norms=True):
        """Advance n_steps RK45 steps in place on a Fortran copy; returns (u, reg, norms)."""
        u = np.array(u, dtype=np.float64, order="F", copy=True)
        reg = np.zeros_like(u, order="F") if reg is None else np.array(reg, dtype=np.float64, order="F", copy=True)
        nrm = np.zeros((self.n_fields, n_steps), order="F") if norms else None
        lib().or_rk45(self.h, C.byref(ph), _dp(u), _dp(reg), float(dt), int(n_steps),
                      _dp(nrm) if norms else None)
        return u, reg, nrm

    def kinetic_energy(self, u):
        u = np.asfortranarray(u, dtype=np.float64)
        return lib().or_kinetic_energy(self.h, _dp(u))


# ---------------------------------------------------------------- initial states

def ic_vortex(pos, gamma=1.4, beta=5.0, t=0.0):
    """Isentropic vortex of strength beta in a free stream rho=1, u=1, v=0, p=1,
    advected along x (the vortex profile of the reference's src/funcs.cpp:1646-1657)."""
    x = pos[..., 0] - t
    y = pos[..., 1]
    f = 1.0 - (x * x + y * y)
    rho = (1.0 - beta * beta * (gamma - 1.0) / (8.0 * gamma * np.pi * np.pi) * np.exp(f)) ** (1.0 / (gamma - 1.0))
    vx = 1.0 - beta * y / (2.0 * np.pi) * np.exp(f / 2.0)
    vy = beta * x / (2.0 * np.pi) * np.exp(f / 2.0)
    p = rho ** gamma
    return np.stack([rho, rho * vx, rho * vy, p / (gamma - 1.0) + 0.5 * rho * (vx * vx + vy * vy)], axis=-1)


def ic_tgv(pos, gamma=1.4, p0=None, mach=0.1):
    """Taylor-Green vortex, rho0 = U0 = 1, background pressure p0 (default 1/(gamma M^2))."""
    if p0 is None:
        p0 = 1.0 / (gamma * mach * mach)
    x, y, z = pos[..., 0], pos[..., 1], pos[..., 2]
    p = p0 + 1.0 / 16.0 * (np.cos(2.0 * x) + np.cos(2.0 * y)) * (np.cos(2.0 * z) + 2.0)
    u = np.sin(x) * np.cos(y) * np.cos(z)
    v = -np.cos(x) * np.sin(y) * np.cos(z)
    rho = np.ones_like(x)
    return np.stack([rho, u, v, np.zeros_like(x), p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)], axis=-1)


def tgv_kat_physics():
    """Non-dimensional constants of the reference's TGV regression input
    (testcases/navier-stokes/Taylor_Green_vortex/input_TGV_SD_hex), computed as
    input::setup_params does (src/input.cpp:400-440) for fix_vis = 1."""
    gamma, R, T, mu_gas, Re, M, L = 1.4, 286.9, 300.0, 1.827e-05, 1600.0, 0.08, 1.0
    uvw = M * np.sqrt(gamma * R * T)
    rho_ref = (mu_gas * Re) / (uvw * L)
    mu_ref = rho_ref * uvw * L
    return physics(viscous=1, gamma=gamma, prandtl=0.72, mu_inf=mu_gas / mu_ref,
                   rt_inf=291.15 * R / (uvw * uvw), c_sth=120.0 / 291.15, fix_vis=1.0, tau=1.0, pen_fact=0.5)
