"""Python mirror of the HiFiLES per-element-type FR path over the C ABI of
include/fr_b200.h (libfrb200.so, built in-tree by hifiles-solver_b200/build.py).

The names follow the reference: a Solver holds one element type on a periodic
conforming mesh and exposes CalcResidual (`residual`), one RK45 stage of
eles::AdvanceSolution (`rk_stage`), the time loop (`advance`) and the
diagnostics (`norms`, `kinetic_energy`).  Arrays are numpy arrays in the
reference's array<T> layouts (Fortran order): state[upt, ele, field].

There is no CPU fallback: constructing a Solver without the CUDA library or
without a GPU raises.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(HERE, "libfrb200.so")

FR_OK = 0
STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "non-finite residual", 4: "device wait timed out",
          5: "unsupported configuration", 6: "mesh wiring failed"}


class FrError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s (%d): %s" % (STATUS.get(status, "?"), status, msg))
        self.status = status


class MeshDesc(C.Structure):
    _fields_ = [("dims", C.c_int), ("n_verts", C.c_int), ("xv", C.POINTER(C.c_double)), ("n_eles", C.c_int),
                ("c2v", C.POINTER(C.c_int)), ("shift", C.c_double * 3), ("bctype", C.POINTER(C.c_int))]


class SchemeDesc(C.Structure):
    _fields_ = [("order", C.c_int), ("upts_type", C.c_int), ("vcjh_scheme", C.c_int), ("eta", C.c_double),
                ("viscous", C.c_int), ("riemann", C.c_int), ("precision", C.c_int), ("gamma", C.c_double),
                ("prandtl", C.c_double), ("mu_inf", C.c_double), ("rt_inf", C.c_double), ("c_sth", C.c_double),
                ("fix_vis", C.c_double), ("tau", C.c_double), ("pen_fact", C.c_double), ("les", C.c_int),
                ("sgs_model", C.c_int), ("filter_ratio", C.c_double), ("bdy", C.c_double * 14), ("R_ref", C.c_double)]


# local face of each box side (x-, x+, y-, y+, z-, z+) in the reference's numbering
_QUAD_SIDE_FACE = (3, 1, 0, 2)
_HEX_SIDE_FACE = (4, 2, 1, 3, 0, 5)


def box_bctype(dims, n, side_bc):
    """(n_eles, 2*dims) boundary type per local face of a box mesh whose sides
    x-, x+, y-, y+(, z-, z+) carry the types side_bc (0 = periodic)."""
    nx, ny = int(n[0]), int(n[1])
    nz = int(n[2]) if dims == 3 else 1
    bct = np.zeros((nx * ny * nz, 2 * dims), dtype=np.int32)
    ijk = np.indices((nz, ny, nx)).reshape(3, -1)[::-1]          # i, j, k with i fastest
    nn = (nx, ny, nz)
    side_face = _QUAD_SIDE_FACE if dims == 2 else _HEX_SIDE_FACE
    for d in range(dims):
        for sd in range(2):
            b = int(side_bc[2 * d + sd])
            if b:
                sel = ijk[d] == (0 if sd == 0 else nn[d] - 1)
                bct[sel, side_face[2 * d + sd]] = b
    return bct


_LIB = None


def lib():
    """Load libfrb200.so; raises if it has not been built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise ImportError("libfrb200.so is missing: run `python hifiles-solver_b200/build.py`")
    L = C.CDLL(LIB_PATH)
    vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)
    sigs = {
        "fr_status_string": (C.c_char_p, [C.c_int]),
        "fr_last_error": (C.c_char_p, []),
        "fr_solver_create": (C.c_int, [C.POINTER(MeshDesc), C.POINTER(SchemeDesc), C.c_int, C.POINTER(vp)]),
        "fr_solver_destroy": (C.c_int, [vp]),
        "fr_solver_sizes": (C.c_int, [vp, ip]),
        "fr_solver_get_geometry": (C.c_int, [vp, dp, dp, dp, dp, dp]),
        "fr_solver_get_interfaces": (C.c_int, [vp, ip, ip]),
        "fr_solver_set_geometry": (C.c_int, [vp, dp, dp, dp, dp]),
        "fr_solver_set_state": (C.c_int, [vp, dp, vp]),
        "fr_solver_set_state_async": (C.c_int, [vp, dp]),
        "fr_solver_get_state": (C.c_int, [vp, dp, vp]),
        "fr_solver_state_ptrs": (C.c_int, [vp, C.POINTER(vp), C.POINTER(vp)]),
        "fr_solver_state_updated": (C.c_int, [vp, vp]),
        "fr_solver_residual": (C.c_int, [vp, dp, vp]),
        "fr_solver_rk_stage": (C.c_int, [vp, C.c_int, C.c_double, vp]),
        "fr_solver_advance": (C.c_int, [vp, C.c_int, C.c_double, dp, vp]),
        "fr_solver_advance_async": (C.c_int, [vp, C.c_int, C.c_double, dp, vp]),
        "fr_solver_kinetic_energy": (C.c_int, [vp, dp, vp]),
        "fr_solver_set_volume_cubature": (C.c_int, [vp, C.c_int, dp, dp]),
        "fr_volume_cubature": (C.c_int, [C.c_int, C.c_int, dp, dp]),
        "fr_solver_launch_count": (C.c_longlong, [vp]),
        "fr_solver_stream": (vp, [vp]),
        "fr_solver_sync": (C.c_int, [vp]),
        "fr_solver_profile_stage": (C.c_int, [vp, C.c_int, C.c_double, dp]),
        "fr_solver_autotune": (C.c_int, [vp, C.c_int, ip]),
        "fr_solver_tile_count": (C.c_int, [vp, ip]),
        "fr_solver_tile_info": (C.c_int, [vp, C.c_int, C.c_int, ip]),
        "fr_solver_select_tiles": (C.c_int, [vp, C.c_int, C.c_int]),
        "fr_mesh_geometry": (C.c_int, [C.POINTER(MeshDesc), C.POINTER(SchemeDesc), ip, dp, dp, dp, dp, dp, ip, ip]),
        "fr_line_operators": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double, dp]),
        "fr_solver_gradient": (C.c_int, [vp, dp, vp]),
        "fr_solver_integral_quantities": (C.c_int, [vp, dp, vp]),
        "fr_vtu_write": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, dp, dp, C.c_double]),
        "fr_solver_write_vtu": (C.c_int, [vp, C.c_char_p]),
        "fr_batch_create": (C.c_int, [vp, vp, C.c_int, C.c_int, C.POINTER(vp)]),
        "fr_batch_destroy": (C.c_int, [vp]),
        "fr_batch_n_groups": (C.c_int, [vp]),
        "fr_batch_group": (C.c_int, [vp, C.c_int, C.POINTER(vp)]),
        "fr_batch_instance": (C.c_int, [vp, C.c_int, ip]),
        "fr_batch_set_state": (C.c_int, [vp, C.c_int, dp]),
        "fr_batch_get_state": (C.c_int, [vp, C.c_int, dp]),
        "fr_batch_autotune": (C.c_int, [vp, C.c_int]),
        "fr_batch_set_merged": (C.c_int, [vp, C.c_int, C.c_int]),
        "fr_batch_merged": (C.c_int, [vp]),
        "fr_batch_advance": (C.c_int, [vp, C.c_int, C.c_double, vp]),
        "fr_batch_launch_count": (C.c_longlong, [vp]),
        "fr_batch_stream": (vp, [vp]),
        "fr_restart_write": (C.c_int, [C.c_char_p, C.c_double, vp, C.c_int]),
        "fr_restart_read": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, vp, dp, dp]),
        "fr_restart_read_points": (C.c_int, [C.c_char_p, C.c_int, C.c_int, dp, C.c_int, C.c_int, vp, dp, dp]),
        "fr_vtu_write_mixed": (C.c_int, [C.c_char_p, C.c_int, vp, C.c_int, C.c_double]),
        "fr_solver_write_restart": (C.c_int, [vp, C.c_char_p, C.c_double]),
        "fr_solver_read_restart": (C.c_int, [vp, C.c_char_p, dp]),
        "fr_solver_sgs_features": (C.c_int, [vp, C.POINTER(C.c_float), vp]),
        "fr_solver_set_sgs_mlp": (C.c_int, [vp, C.POINTER(C.c_float)]),
        "fr_mlp_n_params": (C.c_int, []),
        "fr_mlp_n_trained": (C.c_int, []),
        "fr_mlp_scratch_floats": (C.c_longlong, [C.c_longlong]),
        "fr_mlp_forward": (C.c_int, [vp, vp, C.c_longlong, vp, vp]),
        "fr_mlp_loss_grad": (C.c_int, [vp, vp, vp, vp, C.c_longlong, vp, vp, vp, C.c_longlong, vp]),
        "fr_mlp_adam": (C.c_int, [vp, vp, vp, vp, C.c_int, C.c_float, vp]),
    }
    for name, (res, args) in sigs.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _LIB = L
    return L


def _check(st):
    if st != FR_OK:
        raise FrError(st, lib().fr_last_error().decode())


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def box_mesh(dims, n, lo, hi, jitter=0.0, seed=0):
    """Vertices and tensor-ordered element->vertex map of a structured box,
    interior vertices moved by a seeded uniform jitter of +-jitter*h (64-bit
    LCG, so a seed names one mesh on every machine)."""
    nx, ny = int(n[0]), int(n[1])
    nz = int(n[2]) if dims == 3 else 1
    vx, vy, vz = nx + 1, ny + 1, (nz + 1 if dims == 3 else 1)
    nn = [nx, ny, nz]
    idx = np.indices((vz, vy, vx)).reshape(3, -1)      # k, j, i with i fastest
    ijk = [idx[2], idx[1], idx[0]]
    nv = vx * vy * vz
    mask = (1 << 64) - 1
    A, B = 6364136223846793005, 1442695040888963407
    rnd = np.zeros((nv, dims))
    s = (int(seed) * A + B) & mask
    for v in range(nv if jitter > 0 else 0):
        for d in range(dims):
            s = (s * A + B) & mask
            rnd[v, d] = ((s >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0
    xv = np.empty((nv, dims))
    interior = np.ones(nv, dtype=bool)
    for d in range(dims):
        interior &= (ijk[d] > 0) & (ijk[d] < nn[d])
    for d in range(dims):
        h = (hi[d] - lo[d]) / nn[d]
        x = lo[d] + (hi[d] - lo[d]) * ijk[d] / nn[d]
        if jitter > 0:
            x = np.where(interior, x + jitter * h * rnd[:, d], x)
        xv[:, d] = x
    ex, ey, ez = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    ex, ey, ez = ex.transpose(2, 1, 0).ravel(), ey.transpose(2, 1, 0).ravel(), ez.transpose(2, 1, 0).ravel()
    cols = []
    for c in range(2 if dims == 3 else 1):
        for b in range(2):
            for a in range(2):
                cols.append((ex + a) + vx * ((ey + b) + vy * (ez + c)))
    c2v = np.stack(cols, axis=1).astype(np.int32)
    return xv, c2v


def _bdy(bdy):
    return (C.c_double * 14)(*(list(bdy) if bdy is not None else [0.0] * 14))


def _descs(dims, xv, c2v, shift, order, viscous=False, gamma=1.4, prandtl=0.72, mu_inf=0.0, rt_inf=1.0,
           c_sth=1.0, fix_vis=1.0, tau=1.0, pen_fact=0.5, vcjh_scheme=1, eta=0.0, upts_type=0, precision=0,
           les=0, sgs_model=1, filter_ratio=1.0, riemann=0, bctype=None, bdy=None, R_ref=1.0):
    xv = np.ascontiguousarray(xv, dtype=np.float64)
    c2v = np.ascontiguousarray(c2v, dtype=np.int32)
    bct = None if bctype is None else np.ascontiguousarray(bctype, dtype=np.int32)
    md = MeshDesc(int(dims), xv.shape[0], _dp(xv), c2v.shape[0], c2v.ctypes.data_as(C.POINTER(C.c_int)),
                  (C.c_double * 3)(*(list(shift) + [0.0] * (3 - len(shift)))),
                  None if bct is None else bct.ctypes.data_as(C.POINTER(C.c_int)))
    sd = SchemeDesc(int(order), int(upts_type), int(vcjh_scheme), float(eta), int(bool(viscous)), int(riemann),
                    int(precision),
                    gamma, prandtl, mu_inf, rt_inf, c_sth, fix_vis, tau, pen_fact, int(les), int(sgs_model),
                    float(filter_ratio), _bdy(bdy), float(R_ref))
    return md, sd, (xv, c2v, bct)


def mesh_geometry(dims, xv, c2v, shift, order, **kw):
    """Host-only: metrics and interface wiring as the solver builds them."""
    md, sd, keep = _descs(dims, xv, c2v, shift, order, **kw)
    sz = (C.c_int * 6)()
    _check(lib().fr_mesh_geometry(C.byref(md), C.byref(sd), sz, None, None, None, None, None, None, None))
    E, nu, nf, F, D, ni = list(sz)
    g = dict(pos_upts=np.zeros((nu, E, D), order="F"), detjac_upts=np.zeros((nu, E), order="F"),
             JGinv_upts=np.zeros((D, D, nu, E), order="F"), tdA_fpts=np.zeros((nf, E), order="F"),
             norm_fpts=np.zeros((nf, E, D), order="F"), left=np.zeros(ni, dtype=np.int32),
             right=np.zeros(ni, dtype=np.int32))
    ipp = C.POINTER(C.c_int)
    _check(lib().fr_mesh_geometry(C.byref(md), C.byref(sd), sz, *[_dp(g[k]) for k in
                                  ("pos_upts", "detjac_upts", "JGinv_upts", "tdA_fpts", "norm_fpts")],
                                  g["left"].ctypes.data_as(ipp), g["right"].ctypes.data_as(ipp)))
    return g


def line_operators(order, upts_type=0, vcjh_scheme=1, eta=0.0):
    """The 1-D operator factors (see fr_line_operators in include/fr_b200.h)."""
    n = order + 1
    out = np.zeros(n * n + 6 * n + 1)
    _check(lib().fr_line_operators(int(order), int(upts_type), int(vcjh_scheme), float(eta), _dp(out)))
    o = iter(np.split(out, np.cumsum([n, n, n, n * n, n, n, n])))
    loc, Lm, Lp, D, gL, gR, w, eta = [next(o) for _ in range(8)]
    return dict(loc=loc, Lm=Lm, Lp=Lp, D=D.reshape(n, n), gL=gL, gR=gR, w=w, eta=float(eta[0]))


def volume_cubature(dims, rule):
    """The tensor Gauss-Legendre volume cubature of `rule` points per direction
    in the reference's point order, full double precision: (loc (dims, n),
    weights (n))."""
    n = lib().fr_volume_cubature(int(dims), int(rule), None, None)
    if n <= 0:
        raise ValueError("cubature rule must be 1..12")
    loc = np.zeros((dims, n), order="F")
    w = np.zeros(n)
    lib().fr_volume_cubature(int(dims), int(rule), _dp(loc), _dp(w))
    return loc, w


def read_reference_cubature(path, dims, rule):
    """A rule of the reference's cubature tables (data/cubature_quad.dat or
    data/cubature_hexa.dat: a line "rule=N", then "locs(x)", "locs(y)"
    [, "locs(z)"] and "weights", each followed by one value per line), for a
    caller that has the reference's data directory: (loc (dims, n), weights)."""
    n = rule ** dims
    lines = [ln.strip() for ln in open(path)]
    i = lines.index("rule=%d" % rule)
    cols = []
    for _ in range(dims + 1):
        i += 1                          # the section title
        cols.append([float(lines[i + 1 + q].split()[0]) for q in range(n)])
        i += n
    return np.asfortranarray(np.array(cols[:dims])), np.array(cols[dims])


class Solver:
    """One element type (quads or hexes) on a periodic conforming mesh, resident on one GPU."""

    def __init__(self, dims, xv, c2v, shift, order, viscous=False, gamma=1.4, prandtl=0.72, mu_inf=0.0,
                 rt_inf=1.0, c_sth=1.0, fix_vis=1.0, tau=1.0, pen_fact=0.5, vcjh_scheme=1, eta=0.0, upts_type=0,
                 precision=0, device=0, les=0, sgs_model=1, filter_ratio=1.0, riemann=0, bctype=None, bdy=None,
                 R_ref=1.0):
        L = lib()
        self._xv = np.ascontiguousarray(xv, dtype=np.float64)
        self._c2v = np.ascontiguousarray(c2v, dtype=np.int32)
        self._bct = None if bctype is None else np.ascontiguousarray(bctype, dtype=np.int32)
        md = MeshDesc(int(dims), self._xv.shape[0], _dp(self._xv), self._c2v.shape[0],
                      self._c2v.ctypes.data_as(C.POINTER(C.c_int)),
                      (C.c_double * 3)(*(list(shift) + [0.0] * (3 - len(shift)))),
                      None if self._bct is None else self._bct.ctypes.data_as(C.POINTER(C.c_int)))
        sd = SchemeDesc(int(order), int(upts_type), int(vcjh_scheme), float(eta), int(bool(viscous)), int(riemann),
                        int(precision), gamma, prandtl, mu_inf, rt_inf, c_sth, fix_vis, tau, pen_fact, int(les),
                        int(sgs_model), float(filter_ratio), _bdy(bdy), float(R_ref))
        h = C.c_void_p()
        self.h = None
        _check(L.fr_solver_create(C.byref(md), C.byref(sd), int(device), C.byref(h)))
        self.h = h
        sz = (C.c_int * 6)()
        _check(L.fr_solver_sizes(self.h, sz))
        self.n_eles, self.n_upts, self.n_fpts, self.n_fields, self.dims, self.n_int = list(sz)
        self.viscous = bool(viscous)
        self.order = int(order)
        self.precision = precision
        self.device = int(device)

    @classmethod
    def box(cls, dims, order, n, lo, hi, jitter=0.0, seed=0, side_bc=None, **kw):
        """Structured box; side_bc: boundary types of the sides x-, x+, y-, y+(,
        z-, z+), 0 = periodic (the default for every side)."""
        xv, c2v = box_mesh(dims, n, lo, hi, jitter, seed)
        shift = [hi[d] - lo[d] for d in range(dims)]
        if side_bc is not None:
            shift = [0.0 if (side_bc[2 * d] or side_bc[2 * d + 1]) else shift[d] for d in range(dims)]
            kw["bctype"] = box_bctype(dims, n, side_bc)
        return cls(dims, xv, c2v, shift, order, **kw)

    def close(self):
        if self.h is not None:
            lib().fr_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def state_shape(self):
        return (self.n_upts, self.n_eles, self.n_fields)

    def geometry(self):
        E, nu, nf, D = self.n_eles, self.n_upts, self.n_fpts, self.dims
        g = dict(pos_upts=np.zeros((nu, E, D), order="F"), detjac_upts=np.zeros((nu, E), order="F"),
                 JGinv_upts=np.zeros((D, D, nu, E), order="F"), tdA_fpts=np.zeros((nf, E), order="F"),
                 norm_fpts=np.zeros((nf, E, D), order="F"))
        _check(lib().fr_solver_get_geometry(self.h, *[_dp(g[k]) for k in
                                                      ("pos_upts", "detjac_upts", "JGinv_upts", "tdA_fpts",
                                                       "norm_fpts")]))
        return g

    def interfaces(self):
        l = np.zeros(self.n_int, dtype=np.int32)
        r = np.zeros(self.n_int, dtype=np.int32)
        _check(lib().fr_solver_get_interfaces(self.h, l.ctypes.data_as(C.POINTER(C.c_int)),
                                              r.ctypes.data_as(C.POINTER(C.c_int))))
        return l, r

    def set_geometry(self, detjac_upts, JGinv_upts, tdA_fpts, norm_fpts):
        a = [np.asfortranarray(x, dtype=np.float64) for x in (detjac_upts, JGinv_upts, tdA_fpts, norm_fpts)]
        _check(lib().fr_solver_set_geometry(self.h, *[_dp(x) for x in a]))

    def set_state(self, u, stream=None):
        u = np.asfortranarray(u, dtype=np.float64)
        if u.shape != self.state_shape:
            raise ValueError("state shape %s != %s" % (u.shape, self.state_shape))
        _check(lib().fr_solver_set_state(self.h, _dp(u), stream))

    def set_state_async(self, u):
        """Stage a state for the next advance (fr_solver_set_state_async): u must
        be a Fortran-ordered float64 array, ideally in pinned memory, left
        unchanged until that advance has run."""
        if not (isinstance(u, np.ndarray) and u.dtype == np.float64 and u.flags.f_contiguous):
            raise ValueError("set_state_async needs a Fortran-ordered float64 array")
        if u.shape != self.state_shape:
            raise ValueError("state shape %s != %s" % (u.shape, self.state_shape))
        _check(lib().fr_solver_set_state_async(self.h, _dp(u)))
        self._staged_host = u

    def advance_async(self, n_steps, dt, norms_out=None, stream=None):
        """advance without waiting; norms_out (float64, n_fields, pinned memory
        for an asynchronous copy) holds the L1 norms once the stream is synced."""
        _check(lib().fr_solver_advance_async(self.h, int(n_steps), float(dt),
                                             _dp(norms_out) if norms_out is not None else None, stream))

    def get_state(self, stream=None):
        u = np.zeros(self.state_shape, order="F")
        _check(lib().fr_solver_get_state(self.h, _dp(u), stream))
        return u

    def state_ptrs(self):
        u, r = C.c_void_p(), C.c_void_p()
        _check(lib().fr_solver_state_ptrs(self.h, C.byref(u), C.byref(r)))
        return u.value, r.value

    def state_updated(self, stream=None):
        _check(lib().fr_solver_state_updated(self.h, stream))

    def residual(self, stream=None):
        """div_tconf_upts(0) of one CalcResidual on the current state."""
        d = np.zeros(self.state_shape, order="F")
        _check(lib().fr_solver_residual(self.h, _dp(d), stream))
        return d

    def rk_stage(self, stage, dt, stream=None):
        _check(lib().fr_solver_rk_stage(self.h, int(stage), float(dt), stream))

    def advance(self, n_steps, dt, norms=False, stream=None):
        """n_steps RK45 steps; returns the L1 residual norms of the last stage if norms."""
        out = np.zeros(self.n_fields) if norms else None
        _check(lib().fr_solver_advance(self.h, int(n_steps), float(dt), _dp(out) if norms else None, stream))
        return out

    def write_restart(self, path, time=0.0):
        """The state as a restart file in the reference's format."""
        _check(lib().fr_solver_write_restart(self.h, str(path).encode(), float(time)))

    def read_restart(self, path):
        """Sets the state from a restart file (any order of the same element
        type); returns the file's time."""
        t = C.c_double()
        _check(lib().fr_solver_read_restart(self.h, str(path).encode(), C.byref(t)))
        return t.value

    def write_vtu(self, path):
        """The current state as a .vtu file (solution points, sub-cells per element)."""
        _check(lib().fr_solver_write_vtu(self.h, str(path).encode()))

    def integral_quantities(self, stream=None):
        """kinetic energy, enstrophy, pressure dilatation, strain colon product,
        deviatoric strain colon product of the current state (viscous solvers)."""
        out = np.zeros(5)
        _check(lib().fr_solver_integral_quantities(self.h, _dp(out), stream))
        return dict(zip(("kineticenergy", "vorticity", "pressuredilatation", "straincolonproduct",
                         "devstraincolonproduct"), out.tolist()))

    def gradient(self, stream=None):
        """Corrected physical gradient grad_disu_upts (n_upts, n_eles, n_fields, n_dims)."""
        g = np.zeros((self.n_upts, self.n_eles, self.n_fields, self.dims), order="F")
        _check(lib().fr_solver_gradient(self.h, _dp(g), stream))
        return g

    def sgs_features(self, stream=None):
        """Inputs of the learned closure at every solution point, (n_upts * n_eles, 6) float32."""
        x = np.zeros((self.n_upts * self.n_eles, 6), dtype=np.float32)
        _check(lib().fr_solver_sgs_features(self.h, x.ctypes.data_as(C.POINTER(C.c_float)), stream))
        return x

    def set_sgs_mlp(self, w):
        """Parameters of the learned closure (solvers made with les=1, sgs_model=5)."""
        w = np.ascontiguousarray(w, dtype=np.float32)
        if w.size != mlp_n_params():
            raise ValueError("expected %d parameters" % mlp_n_params())
        _check(lib().fr_solver_set_sgs_mlp(self.h, w.ctypes.data_as(C.POINTER(C.c_float))))

    def set_volume_cubature(self, loc, weights):
        """Volume cubature of the integral diagnostics: loc (dims, n) points in
        [-1, 1]^dims, weights (n) -- e.g. a rule of the reference's own
        data/cubature_*.dat tables (read_reference_cubature)."""
        loc = np.asfortranarray(loc, dtype=np.float64)
        w = np.ascontiguousarray(weights, dtype=np.float64)
        if loc.shape != (self.dims, w.size):
            raise ValueError("loc must be (dims, n) with n = len(weights)")
        _check(lib().fr_solver_set_volume_cubature(self.h, int(w.size), _dp(loc), _dp(w)))

    def kinetic_energy(self, stream=None):
        v = C.c_double()
        _check(lib().fr_solver_kinetic_energy(self.h, C.byref(v), stream))
        return v.value

    def launch_count(self):
        return int(lib().fr_solver_launch_count(self.h))

    def stream(self):
        return lib().fr_solver_stream(self.h)

    def sync(self):
        _check(lib().fr_solver_sync(self.h))

    def autotune(self, reps=5):
        """Pick the fastest compiled tile variants; returns (grad EPB, grad NT, update EPB, update NT)."""
        out = (C.c_int * 4)()
        _check(lib().fr_solver_autotune(self.h, int(reps), out))
        return tuple(out)

    def tile_count(self):
        """(gradient variants, update variants) compiled for this solver's shape."""
        out = (C.c_int * 2)()
        _check(lib().fr_solver_tile_count(self.h, out))
        return tuple(out)

    def tile_info(self, kind, i):
        """(elements, threads, CTAs per SM, persistent) of gradient (kind 0) or update (kind 1) variant i."""
        out = (C.c_int * 4)()
        _check(lib().fr_solver_tile_info(self.h, int(kind), int(i), out))
        return tuple(out)

    def select_tiles(self, g, u):
        """Use gradient variant g and update variant u (as the autotuner would)."""
        _check(lib().fr_solver_select_tiles(self.h, int(g), int(u)))

    def profile_stage(self, reps, dt):
        """Mean CUDA-event ms of the (gradient, interface-flux, update) kernels over reps stages."""
        out = np.zeros(3)
        _check(lib().fr_solver_profile_stage(self.h, int(reps), float(dt), _dp(out)))
        return tuple(out)


# ---------------------------------------------------------------- learned closure kernels
# Device arrays are passed as integer addresses (e.g. torch's data_ptr()).

def mlp_n_params():
    return int(lib().fr_mlp_n_params())


def mlp_n_trained():
    return int(lib().fr_mlp_n_trained())


def mlp_scratch_floats(n):
    return int(lib().fr_mlp_scratch_floats(int(n)))


def mlp_forward(d_w, d_x, n, d_out, stream=None):
    _check(lib().fr_mlp_forward(d_w, d_x, int(n), d_out, stream))


def mlp_loss_grad(d_w, d_x, d_y, n, d_grad, d_loss, d_scratch, scratch_floats, d_sw=None, stream=None):
    _check(lib().fr_mlp_loss_grad(d_w, d_x, d_y, d_sw, int(n), d_grad, d_loss, d_scratch, int(scratch_floats),
                                  stream))


def mlp_adam(d_w, d_grad, d_m, d_v, step, lr, stream=None):
    _check(lib().fr_mlp_adam(d_w, d_grad, d_m, d_v, int(step), float(lr), stream))


# ---------------------------------------------------------------- restart files (host only)

class RestartBlock(C.Structure):
    _fields_ = [("ele_type", C.c_int), ("order", C.c_int), ("n_upts", C.c_int), ("n_eles", C.c_int),
                ("n_fields", C.c_int), ("loc_1d", C.POINTER(C.c_double)), ("ele2global", C.POINTER(C.c_int)),
                ("disu_upts", C.POINTER(C.c_double)), ("loc_pts", C.POINTER(C.c_double))]


def _points(loc_pts, ele_type):
    """Solution points as a C-ordered (n_upts, dims) array (element_operators' loc_upts is (dims, n_upts):
    pass its transpose)."""
    pts = np.ascontiguousarray(loc_pts, dtype=np.float64)
    if pts.ndim != 2 or pts.shape[1] != (2 if ele_type in (0, 1) else 3):
        raise ValueError("loc_pts must be (n_upts, dims)")
    return pts


def restart_write(path, time, blocks):
    """blocks: list of dicts(ele_type, order, disu_upts (n_upts, n_eles, F), ele2global=None) with loc_1d
    (quads, hexes: the 1-D points) or loc_pts (triangles, tets, prisms: the (n_upts, dims) solution points
    of element_operators)."""
    keep, arr = [], (RestartBlock * len(blocks))()
    for i, b in enumerate(blocks):
        u = np.asfortranarray(b["disu_upts"], dtype=np.float64)
        loc = None if b.get("loc_1d") is None else np.ascontiguousarray(b["loc_1d"], dtype=np.float64)
        pts = None if b.get("loc_pts") is None else _points(b["loc_pts"], b["ele_type"])
        g = None if b.get("ele2global") is None else np.ascontiguousarray(b["ele2global"], dtype=np.int32)
        keep += [u, loc, pts, g]
        arr[i] = RestartBlock(int(b["ele_type"]), int(b["order"]), u.shape[0], u.shape[1], u.shape[2],
                              None if loc is None else _dp(loc),
                              None if g is None else g.ctypes.data_as(C.POINTER(C.c_int)), _dp(u),
                              None if pts is None else _dp(pts))
    _check(lib().fr_restart_write(str(path).encode(), float(time), arr, len(blocks)))


def restart_read(path, ele_type, order, n_eles, n_fields, upts_type=0, ele2global=None):
    """(disu_upts (n_upts, n_eles, F), time) of the quad or hex block."""
    dims = 2 if ele_type == 1 else 3
    u = np.zeros(((order + 1) ** dims, n_eles, n_fields), order="F")
    g = None if ele2global is None else np.ascontiguousarray(ele2global, dtype=np.int32)
    t = C.c_double()
    _check(lib().fr_restart_read(str(path).encode(), int(ele_type), int(order), int(upts_type), int(n_eles),
                                 int(n_fields), None if g is None else g.ctypes.data, _dp(u), C.byref(t)))
    return u, t.value


def restart_read_points(path, ele_type, loc_pts, n_eles, n_fields, ele2global=None):
    """(disu_upts (n_upts, n_eles, F), time) of one element type's block carried to the solution points
    loc_pts ((n_upts, dims), as element_operators gives them)."""
    pts = _points(loc_pts, ele_type)
    u = np.zeros((pts.shape[0], n_eles, n_fields), order="F")
    g = None if ele2global is None else np.ascontiguousarray(ele2global, dtype=np.int32)
    t = C.c_double()
    _check(lib().fr_restart_read_points(str(path).encode(), int(ele_type), pts.shape[0], _dp(pts), int(n_eles),
                                        int(n_fields), None if g is None else g.ctypes.data, _dp(u), C.byref(t)))
    return u, t.value


# ---------------------------------------------------------------- batches

class Batch:
    """Independent meshes advanced together: instances with the same dims and
    scheme are merged into one group (one launch per stage kernel), and a
    step of all groups is one CUDA graph.  instances: list of dicts with the
    Solver.box arguments (dims, order, n, lo, hi, jitter, seed, side_bc and
    the scheme keywords)."""

    def __init__(self, instances, device=0):
        L = lib()
        n = len(instances)
        mds, sds = (MeshDesc * n)(), (SchemeDesc * n)()
        self._keep = []
        for i, inst in enumerate(instances):
            kw = dict(inst)
            dims, order, nn, lo, hi = kw.pop("dims"), kw.pop("order"), kw.pop("n"), kw.pop("lo"), kw.pop("hi")
            xv, c2v = box_mesh(dims, nn, lo, hi, kw.pop("jitter", 0.0), kw.pop("seed", 0))
            shift = [hi[d] - lo[d] for d in range(dims)]
            side_bc = kw.pop("side_bc", None)
            if side_bc is not None:
                shift = [0.0 if (side_bc[2 * d] or side_bc[2 * d + 1]) else shift[d] for d in range(dims)]
                kw["bctype"] = box_bctype(dims, nn, side_bc)
            md, sd, keep = _descs(dims, xv, c2v, shift, order, **kw)
            mds[i], sds[i] = md, sd
            self._keep.append(keep)
        h = C.c_void_p()
        self.h = None
        _check(L.fr_batch_create(mds, sds, n, int(device), C.byref(h)))
        self.h = h
        self.n = n
        self.shapes = []
        for i in range(n):
            o = (C.c_int * 4)()
            _check(L.fr_batch_instance(self.h, i, o))
            inst = instances[i]
            self.shapes.append((o[3], o[2], inst["dims"] + 2))
        self.n_groups = int(L.fr_batch_n_groups(self.h))

    def close(self):
        if self.h is not None:
            lib().fr_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, i, u):
        u = np.asfortranarray(u, dtype=np.float64)
        if u.shape != self.shapes[i]:
            raise ValueError("state of instance %d must have shape %s" % (i, self.shapes[i]))
        _check(lib().fr_batch_set_state(self.h, int(i), _dp(u)))

    def get_state(self, i):
        u = np.zeros(self.shapes[i], order="F")
        _check(lib().fr_batch_get_state(self.h, int(i), _dp(u)))
        return u

    def autotune(self, reps=3):
        """Tiles per group, then per-group launches against merged launches (fr_batch_autotune)."""
        _check(lib().fr_batch_autotune(self.h, int(reps)))

    def set_merged(self, on, minb=4):
        """One launch per stage kernel for all groups (hex NS groups of orders 2-4; fr_batch_set_merged)."""
        _check(lib().fr_batch_set_merged(self.h, int(bool(on)), int(minb)))

    @property
    def merged(self):
        """Register cap (CTAs per SM) of the merged launches in use, 0 when the groups launch one by one."""
        return int(lib().fr_batch_merged(self.h))

    def advance(self, n_steps, dt, stream=None):
        _check(lib().fr_batch_advance(self.h, int(n_steps), float(dt), stream))

    def launch_count(self):
        return int(lib().fr_batch_launch_count(self.h))

    def stream(self):
        return lib().fr_batch_stream(self.h)

    def dof(self):
        """Degrees of freedom of the whole batch (sum of n_upts * n_eles * n_fields)."""
        return int(sum(a * b * c for a, b, c in self.shapes))


class VtuBlock(C.Structure):
    _fields_ = [("ele_type", C.c_int), ("n_eles", C.c_int), ("loc_pts", C.POINTER(C.c_double)),
                ("pos_upts", C.POINTER(C.c_double)), ("disu_upts", C.POINTER(C.c_double))]


def vtu_write_mixed(path, order, blocks, gamma=1.4):
    """Host-only .vtu writer of a mixed mesh (see fr_vtu_write_mixed): blocks is a list of dicts(ele_type,
    pos_upts (n_upts, n_eles, dims), disu_upts (n_upts, n_eles, dims + 2), loc_pts (triangles, tets,
    prisms: the (n_upts, dims) solution points))."""
    keep, arr = [], (VtuBlock * len(blocks))()
    for i, b in enumerate(blocks):
        pos = np.asfortranarray(b["pos_upts"], dtype=np.float64)
        u = np.asfortranarray(b["disu_upts"], dtype=np.float64)
        pts = None if b.get("loc_pts") is None else _points(b["loc_pts"], b["ele_type"])
        keep += [pos, u, pts]
        arr[i] = VtuBlock(int(b["ele_type"]), u.shape[1], None if pts is None else _dp(pts), _dp(pos), _dp(u))
    _check(lib().fr_vtu_write_mixed(str(path).encode(), int(order), arr, len(blocks), float(gamma)))


def vtu_write(path, dims, order, pos_upts, disu_upts, gamma=1.4):
    """Host-only .vtu writer (see fr_vtu_write)."""
    pos = np.asfortranarray(pos_upts, dtype=np.float64)
    u = np.asfortranarray(disu_upts, dtype=np.float64)
    _check(lib().fr_vtu_write(str(path).encode(), int(dims), int(order), u.shape[1], _dp(pos), _dp(u), float(gamma)))
