"""Meshes of triangles and quadrilaterals (2-D) or tetrahedra, prisms and
hexahedra (3-D) for the per-operator path: the library's host set-up
(include/fr_b200.h, fr_element_* and fr_mixed_*) and the jittered channel
mesh (prism wall layers, tetrahedral core).

`MixedMesh(...).operator_inputs(states)` gives the (types, int_inters,
bdy_inters) triple that `seam.MixedOperatorMesh` advances, the same arrays the
reference's eles_tris / eles_quads / eles_tets / eles_pris / eles_hexas and
int_inters / bdy_inters objects hold after their set-up
(src/eles_tris.cpp:66-648, src/eles_tets.cpp:68-1415,
src/eles_pris.cpp:51-1194, src/eles.cpp:3620-4800, src/int_inters.cpp:95-178,
src/bdy_inters.cpp:111-203).
"""
import ctypes as C
import itertools

import numpy as np

from . import _check, box_mesh, lib, restart_read_points, restart_write, vtu_write_mixed

TRI, QUAD, TET, PRISM, HEX = 0, 1, 2, 3, 4
_NODES = {TRI: 3, QUAD: 4, TET: 4, PRISM: 6, HEX: 8}
_DIMS = {TRI: 2, QUAD: 2, TET: 3, PRISM: 3, HEX: 3}


class ElementOpts(C.Structure):
    """fr_element_opts: point types and VCJH schemes per element type (the
    reference's input keys of the same names)."""
    _fields_ = [("upts_type_tet", C.c_int), ("fpts_type_tet", C.c_int), ("vcjh_scheme_tet", C.c_int),
                ("c_tet", C.c_double), ("upts_type_pri_tri", C.c_int), ("upts_type_pri_1d", C.c_int),
                ("vcjh_scheme_tri", C.c_int), ("c_tri", C.c_double), ("vcjh_scheme_pri_1d", C.c_int),
                ("eta_pri", C.c_double), ("upts_type_hexa", C.c_int), ("vcjh_scheme_hexa", C.c_int),
                ("eta_hexa", C.c_double), ("upts_type_tri", C.c_int), ("fpts_type_tri", C.c_int),
                ("upts_type_quad", C.c_int), ("vcjh_scheme_quad", C.c_int), ("eta_quad", C.c_double)]

    def __init__(self, **kw):
        d = dict(upts_type_tet=0, fpts_type_tet=0, vcjh_scheme_tet=0, c_tet=0.0, upts_type_pri_tri=0,
                 upts_type_pri_1d=0, vcjh_scheme_tri=0, c_tri=0.0, vcjh_scheme_pri_1d=0, eta_pri=0.0,
                 upts_type_hexa=0, vcjh_scheme_hexa=1, eta_hexa=0.0, upts_type_tri=0, fpts_type_tri=0,
                 upts_type_quad=0, vcjh_scheme_quad=1, eta_quad=0.0)
        unknown = set(kw) - set(d)
        if unknown:
            raise TypeError("unknown options: %s" % sorted(unknown))
        d.update(kw)
        super().__init__(**d)


_BOUND = None


def _lib():
    global _BOUND
    if _BOUND is not None:
        return _BOUND
    L = lib()
    vp, dp, ip, lp = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_longlong)
    i, ll = C.c_int, C.c_longlong
    sigs = {
        "fr_element_sizes": [i, i, ip, ip, ip, ip],
        "fr_element_operators": [i, i, C.POINTER(ElementOpts), dp, dp, dp, dp, dp, dp, dp, dp],
        "fr_mixed_create": [i, i, C.POINTER(ElementOpts), ll, dp, ll, ip, ip, dp, ll, lp, ip, ip, C.POINTER(vp)],
        "fr_mixed_destroy": [vp],
        "fr_mixed_info": [vp, ip, ip, lp, ip, ip],
        "fr_mixed_metrics": [vp, i, dp, dp, dp, dp, dp, lp],
        "fr_mixed_inters": [vp, i, ip, lp, ip],
        "fr_mixed_bdy_inters": [vp, i, ip, lp, ip],
    }
    for name, args in sigs.items():
        f = getattr(L, name)
        f.restype = C.c_int
        f.argtypes = args
    _BOUND = L
    return L


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def element_sizes(ele_type, order):
    """(n_upts, n_fpts, n_fpts per face) of one element type."""
    L = _lib()
    nu, nf, nfc = C.c_int(), C.c_int(), C.c_int()
    per = (C.c_int * 6)()
    _check(L.fr_element_sizes(ele_type, order, C.byref(nu), C.byref(nf), C.byref(nfc), per))
    return nu.value, nf.value, list(per)[:nfc.value]


def element_operators(ele_type, order, opts=None):
    """Point sets and dense operators of one element type, as the
    reference's set_opp_0 .. set_opp_6 build them: opp_0, opp_3, opp_6
    matrices, opp_1, opp_2, opp_4, opp_5 lists of D (column-major)."""
    L = _lib()
    nu, nf, _ = element_sizes(ele_type, order)
    D = _DIMS[ele_type]
    A = lambda *s: np.zeros(s, order="F")  # noqa: E731
    lu, tf, tn = A(D, nu), A(D, nf), A(D, nf)
    o0, o1, o2, o3, o5 = A(nf, nu), A(nf, nu, D), A(nu, nu, D), A(nu, nf), A(nu, nf, D)
    o = opts if opts is not None else ElementOpts()
    _check(L.fr_element_operators(ele_type, order, C.byref(o), _dp(lu), _dp(tf), _dp(tn), _dp(o0), _dp(o1),
                                  _dp(o2), _dp(o3), _dp(o5)))
    split = lambda a: [np.asfortranarray(a[..., d]) for d in range(D)]  # noqa: E731
    return dict(loc_upts=lu, tloc_fpts=tf, tnorm_fpts=tn, opp_0=o0, opp_1=split(o1), opp_2=split(o2), opp_3=o3,
                opp_4=split(o2), opp_5=split(o5), opp_6=o0.copy(order="F"))


class MixedMesh:
    """A conforming mesh of one order, triangles and quads (xv (n_verts, 2))
    or tets, prisms and hexes (xv (n_verts, 3)), set up on the host by the
    library: per element type its operators and metrics, the interface tables
    (edges in 2-D; triangular faces, then quadrilateral, in 3-D) and the
    boundary tables.

    cells is a list of (ele_type, vertex ids) in the reference's vertex orders
    (quads in tensor order a + 2 b, hexes a + 2 b + 4 c); period (dims,)
    periodic lengths (0: not periodic); bfaces a list of (cell, local face,
    boundary type)."""

    def __init__(self, order, xv, cells, period=None, bfaces=(), opts=None):
        L = _lib()
        self.order = int(order)
        self.opts = opts if opts is not None else ElementOpts()
        xv = np.ascontiguousarray(xv, dtype=np.float64)
        self.dims = D = xv.shape[1]
        n = len(cells)
        ct = np.array([c[0] for c in cells], dtype=np.int32)
        cv = np.full((n, 8), -1, dtype=np.int32)
        for k, (t, vs) in enumerate(cells):
            if t not in _NODES or len(vs) != _NODES[t]:
                raise ValueError("cell %d: type %r with %d vertices" % (k, t, len(vs)))
            cv[k, :len(vs)] = vs
        per = np.zeros(D) if period is None else np.ascontiguousarray(period, dtype=np.float64)
        bf = np.array([b[0] for b in bfaces], dtype=np.int64)
        bfc = np.array([b[1] for b in bfaces], dtype=np.int32)
        bft = np.array([b[2] for b in bfaces], dtype=np.int32)
        h = C.c_void_p()
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))  # noqa: E731
        _check(L.fr_mixed_create(D, self.order, C.byref(self.opts), xv.shape[0], _dp(xv), n, ip(ct), ip(cv), _dp(per),
                                 len(bf), bf.ctypes.data_as(C.POINTER(C.c_longlong)), ip(bfc), ip(bft), C.byref(h)))
        self._h = h
        try:
            nt, ni, nb = C.c_int(), C.c_int(), C.c_int()
            et = (C.c_int * 3)()
            ne = (C.c_longlong * 3)()
            _check(L.fr_mixed_info(h, C.byref(nt), et, ne, C.byref(ni), C.byref(nb)))
            self.types = {}
            for s in range(nt.value):
                t = et[s]
                nu, nf, _ = element_sizes(t, self.order)
                E = ne[s]
                A = lambda *shape: np.zeros(shape, order="F")  # noqa: E731
                m = dict(JGinv_upts=A(D, D, nu, E), detjac_upts=A(nu, E), tdA_fpts=A(nf, E), norm_fpts=A(nf, E, D),
                         pos_upts=A(nu, E, D), cell=np.zeros(E, dtype=np.int64))
                _check(L.fr_mixed_metrics(h, s, _dp(m["JGinv_upts"]), _dp(m["detjac_upts"]), _dp(m["tdA_fpts"]),
                                          _dp(m["norm_fpts"]), _dp(m["pos_upts"]),
                                          m["cell"].ctypes.data_as(C.POINTER(C.c_longlong))))
                m.update(element_operators(t, self.order, self.opts))
                m["n_upts"], m["n_fpts"], m["n_eles"] = nu, nf, E
                self.types[t] = m
            self.int_inters = [self._table(L.fr_mixed_inters, g, 6) for g in range(ni.value)]
            self.bdy_inters = [self._table(L.fr_mixed_bdy_inters, g, 4) for g in range(nb.value)]
        finally:
            L.fr_mixed_destroy(h)
            self._h = None

    def _table(self, fn, g, rows):
        npi, ni = C.c_int(), C.c_longlong()
        _check(fn(self._h, g, C.byref(npi), C.byref(ni), None))
        t = np.zeros((rows, npi.value, ni.value), dtype=np.int32, order="F")
        _check(fn(self._h, g, None, None, t.ctypes.data_as(C.POINTER(C.c_int))))
        return t

    @property
    def n_dofs(self):
        """Solution points over all element types."""
        return sum(m["n_upts"] * m["n_eles"] for m in self.types.values())

    def operator_inputs(self, states):
        """(types, int_inters, bdy_inters) for seam.MixedOperatorMesh; states
        maps each element type to its state (n_upts, n_eles, 5)."""
        keys = ("opp_0", "opp_1", "opp_2", "opp_3", "opp_4", "opp_5", "opp_6", "JGinv_upts", "detjac_upts",
                "tdA_fpts", "norm_fpts")
        types = {t: dict({k: m[k] for k in keys}, u=np.asfortranarray(states[t])) for t, m in self.types.items()}
        return types, list(self.int_inters), list(self.bdy_inters)

    def write_restart(self, path, time, states):
        """states (element type -> (n_upts, n_eles, F)) as a restart file in
        the reference's format (write_restart, src/output.cpp:1057-1107); the
        element ids are the cells' indices, the reference's ele2global."""
        blocks = []
        for t, m in sorted(self.types.items()):
            b = dict(ele_type=t, order=self.order, disu_upts=states[t], ele2global=m["cell"].astype(np.int32))
            if t in (QUAD, HEX):
                b["loc_1d"] = m["loc_upts"][0, :self.order + 1]
            else:
                b["loc_pts"] = m["loc_upts"].T
            blocks.append(b)
        restart_write(path, time, blocks)

    def write_vtu(self, path, states, gamma=1.4):
        """states (element type -> (n_upts, n_eles, dims + 2)) as one .vtu
        file (fr_vtu_write_mixed): the role of the reference's Paraview
        output (src/output.cpp:580-1055)."""
        vtu_write_mixed(path, self.order, [dict(ele_type=t, pos_upts=m["pos_upts"], disu_upts=states[t],
                                                loc_pts=None if t in (QUAD, HEX) else m["loc_upts"].T)
                                           for t, m in sorted(self.types.items())], gamma)

    def read_restart(self, path, n_fields=None):
        """({element type: state (n_upts, n_eles, F)}, time) from a restart
        file of any order, each block carried to this mesh's solution points
        (read_restart, src/solver.cpp:390-445); F defaults to dims + 2."""
        F = self.dims + 2 if n_fields is None else int(n_fields)
        out, time = {}, None
        for t, m in sorted(self.types.items()):
            out[t], time = restart_read_points(path, t, m["loc_upts"].T, m["n_eles"], F,
                                               ele2global=m["cell"].astype(np.int32))
        return out, time


def _tet_volume(xv, t):
    a, b, c, d = (xv[v] for v in t)
    return float(np.dot(np.cross(b - a, c - a), d - a))


# the prisms' local faces: 0 = nodes (0, 2, 1) at the bottom of the
# extrusion, 1 = nodes (3, 4, 5) at the top (src/geometry.cpp:3240-3290)
PRISM_BOTTOM, PRISM_TOP = 0, 1


def channel_mesh(n=(40, 20, 20), lo=(0.0, 0.0, 0.0), hi=(2 * np.pi, 2.0, np.pi), jitter=0.15, seed=2024,
                 wall_bc=(11, 12)):
    """Jittered channel of nx x ny x nz cells: the first and the last layer
    of cells in y are prisms (each x-z square split along its (0,0)-(1,1)
    diagonal into two triangles, extruded in y), the core is six tets per cell
    (Kuhn split along the main diagonal, whose y-faces carry the same
    diagonal), interior vertices move by a seeded uniform jitter of up to
    +-jitter cell sizes; periodic in x and z, walls at y = lo and y = hi with
    the reference boundary types wall_bc (default: isothermal and adiabatic
    fixed walls).  A conforming mesh cannot hold hexes next to tets (the
    reference has no pyramid), so the channel has none.

    Returns (xv (n_verts, 3), cells [(ele_type, vertex ids)], period (3,),
    bfaces [(cell, local face, boundary type)])."""
    nx, ny, nz = (int(v) for v in n)
    xv, _ = box_mesh(3, (nx, ny, nz), lo, hi, jitter=jitter, seed=seed)
    vx, vy = nx + 1, ny + 1

    def vid(i, j, k):
        return i + vx * (j + vy * k)

    cells, bfaces = [], []
    paths = []
    for perm in itertools.permutations(range(3)):
        p = [0, 0, 0]
        path = [tuple(p)]
        for ax in perm:
            p[ax] = 1
            path.append(tuple(p))
        paths.append(path)
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                def c(a, b, cc):
                    return vid(i + a, j + b, k + cc)
                if j in (0, ny - 1):
                    for tri in (((0, 0), (1, 1), (1, 0)), ((0, 0), (0, 1), (1, 1))):
                        bot = [c(a, 0, cc) for a, cc in tri]
                        top = [c(a, 1, cc) for a, cc in tri]
                        if j == 0:
                            bfaces.append((len(cells), PRISM_BOTTOM, wall_bc[0]))
                        if j == ny - 1:
                            bfaces.append((len(cells), PRISM_TOP, wall_bc[1]))
                        cells.append((PRISM, bot + top))
                else:
                    for path in paths:
                        t = [c(*q) for q in path]
                        if _tet_volume(xv, t) < 0:
                            t = [t[0], t[2], t[1], t[3]]
                        cells.append((TET, t))
    period = np.array([hi[0] - lo[0], 0.0, hi[2] - lo[2]])
    return xv, cells, period, bfaces
