#!/usr/bin/env python3
"""Golden fixtures of mixed-element meshes (tets, prisms, hexes), made by
running the reference itself.

TEST INFRASTRUCTURE ONLY.  Runs where the reference sources are available and
oracle/_ref/ref_harness is built (`make -C oracle REF=<reference checkout> ref`).  For every case it

  1. writes a jittered periodic box of mixed elements as a Gambit neutral file
     (element reader src/geometry.cpp:1706-1880: linear tets = Gambit type 6,
     linear prisms = type 5, hexes = type 4; face numbers of the boundary
     reader src/geometry.cpp:1236-1290),
  2. runs the unmodified reference objects through ref_harness, which dumps
     every element type's operators opp_0..opp_6 (eles_tets / eles_pris /
     eles_hexas set-up), metrics, the interface wiring of every interface type
     (triangular and quadrilateral faces), the intermediate arrays of one
     CalcResidual and the state after N RK45 steps,
  3. stores a compact .npz per case.

The per-operator entry points take exactly these operators and tables, as the
reference's own per-type methods would pass them; tests/test_gpu_mixed.py runs
the stage through them and compares with the reference's arrays.

Meshes (a conforming mix of the three types needs pyramids, which the
reference has no element for, so hexes and tets never share a face):
  * "pritet": prism layers at the bottom and top of y (each x-z cell square
    split along its (0,0)-(1,1) diagonal into two triangles, extruded in y)
    and a core of six tets per cell (Kuhn split along the main diagonal, whose
    y-faces carry the same diagonal), periodic in x, y and z;
  * "hexpri": hexes for the first half of the x cells and y-extruded prisms
    for the second half (hex and prism meet on quadrilateral faces), periodic.
Interior vertices move by a seeded jitter of up to `jitter` cell sizes.

With --restart-only it reruns mixed_triquad_p2, mixed_pritet_p2 and
mixed_hexpri_p3 with the
harness's --write-restart and keeps the reference's own restart files
(write_restart, src/output.cpp:1057-1107) verbatim as rest_<name>.dat.  With --restart-read it runs the reference at order 3 on
the meshes of mixed_triquad_p2 and mixed_pritet_p2, restarted from those
order-2 files, and keeps its states (rest_read_<kind>_p2_to_p3.npz).

Usage:  python tests/golden/make_mixed.py --ref <reference checkout>   (or HIFILES_REF=<dir>)
"""
import argparse
import itertools
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, HERE)
import make_golden as G  # noqa: E402

# reference local faces (src/geometry.cpp:3075-3290) and the Gambit face
# number the boundary reader maps to each (inverse of src/geometry.cpp:1255-1282)
TET_FACES = [(1, 2, 3), (0, 3, 2), (0, 1, 3), (0, 2, 1)]
TET_GAMBIT = {0: 3, 1: 4, 2: 2, 3: 1}
PRI_FACES = [(0, 2, 1), (3, 4, 5), (0, 1, 4, 3), (1, 2, 5, 4), (2, 0, 3, 5)]
PRI_GAMBIT = {0: 4, 1: 5, 2: 1, 3: 2, 4: 3}
# hex: Gambit node g = ag + 2 bg + 4 cg is tensor node (a, b, c) = (cg, ag, bg)
HEX_ORDER = [((g >> 2) & 1) + 2 * (g & 1) + 4 * ((g >> 1) & 1) for g in range(8)]


def _vol(xv, t):
    a, b, c, d = (xv[v] for v in t)
    return float(np.dot(np.cross(b - a, c - a), d - a))


def mixed_cells(kind, n, lo, hi, jitter, seed):
    """Vertices and elements [(gambit_type, vertex ids), ...] of a mixed box,
    plus per element its boundary faces [(side, gambit_face)]."""
    xv, c2v = G.box_vertices(3, n, lo, hi, jitter, seed=seed)
    nx, ny, nz = n
    vx, vy = nx + 1, ny + 1

    def vid(i, j, k):
        return i + vx * (j + vy * k)

    def ijk(v):
        return v % vx, (v // vx) % vy, v // (vx * vy)

    eles = []
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                c = lambda a, b, cc: vid(i + a, j + b, k + cc)  # noqa: E731
                if kind == "pritet":
                    use = "pri" if j in (0, ny - 1) else "tet"
                else:
                    use = "hex" if i < nx // 2 else "pri"
                if use == "hex":
                    e = c2v[i + nx * (j + ny * k)]
                    eles.append((4, [int(e[HEX_ORDER[g]]) for g in range(8)]))
                elif use == "pri":
                    # triangles in (x, z): (00, 11, 10) and (00, 01, 11); node 0->1
                    # x node 0->2 along +y gives a positive volume
                    for tri in (((0, 0), (1, 1), (1, 0)), ((0, 0), (0, 1), (1, 1))):
                        bot = [c(a, 0, cc) for a, cc in tri]
                        top = [c(a, 1, cc) for a, cc in tri]
                        eles.append((5, bot + top))
                else:
                    for perm in itertools.permutations(range(3)):
                        p = [0, 0, 0]
                        path = [tuple(p)]
                        for ax in perm:
                            p[ax] = 1
                            path.append(tuple(p))
                        t = [c(*q) for q in (path[0], path[1], path[2], path[3])]
                        if _vol(xv, t) < 0:
                            t = [t[0], t[2], t[1], t[3]]
                        eles.append((6, t))
    # orientation and boundary faces
    out = []
    for gt, vs in eles:
        if gt == 6:
            assert _vol(xv, vs) > 0
            faces = [(f, TET_GAMBIT[f], [vs[q] for q in TET_FACES[f]]) for f in range(4)]
        elif gt == 5:
            assert _vol(xv, [vs[0], vs[1], vs[2], vs[3]]) > 0
            faces = [(f, PRI_GAMBIT[f], [vs[q] for q in PRI_FACES[f]]) for f in range(5)]
        else:
            faces = None
        bf = []
        if faces is None:
            I = [ijk(v) for v in vs]
            for side, code in ((0, 5), (1, 6), (2, 4), (3, 2), (4, 1), (5, 3)):
                ax, hi_side = side // 2, side % 2
                lim = n[ax] if hi_side else 0
                if sum(1 for q in I if q[ax] == lim) == 4:
                    bf.append((side, code))
        else:
            for f, code, fv in faces:
                I = [ijk(v) for v in fv]
                for side in range(6):
                    ax, hi_side = side // 2, side % 2
                    lim = n[ax] if hi_side else 0
                    if all(q[ax] == lim for q in I):
                        bf.append((side, code))
        out.append((gt, vs, bf))
    return xv, out


# 2-D: reference local edges (src/geometry.cpp:3078-3120): triangles
# (0,1), (1,2), (2,0); quads in tensor slots (0,1), (1,3), (3,2), (2,0); the
# boundary reader maps Gambit face k to edge k - 1 for both (:1240-1241)
TRI_EDGES = [(0, 1), (1, 2), (2, 0)]
QUAD_EDGES = [(0, 1), (1, 3), (3, 2), (2, 0)]


def mixed_cells_2d(n, lo, hi, jitter, seed):
    """Jittered periodic 2-D box: quads for the first half of the x cells,
    each other cell split along its (0,0)-(1,1) diagonal into two
    counter-clockwise triangles.  Elements [(gambit_type, vertex ids in the
    reference's order, boundary edges [(side, gambit face)])]."""
    xv, c2v = G.box_vertices(2, n, lo, hi, jitter, seed=seed)
    nx, ny = n
    vx = nx + 1

    def ij(v):
        return v % vx, v // vx

    out = []
    for j in range(ny):
        for i in range(nx):
            c = lambda a, b: (i + a) + vx * (j + b)  # noqa: E731
            if i < nx // 2:
                eles = [(2, [c(0, 0), c(1, 0), c(0, 1), c(1, 1)], QUAD_EDGES)]
            else:
                eles = [(3, [c(0, 0), c(1, 0), c(1, 1)], TRI_EDGES), (3, [c(0, 0), c(1, 1), c(0, 1)], TRI_EDGES)]
            for gt, vs, edges in eles:
                bf = []
                for k, (a, b) in enumerate(edges):
                    I = [ij(vs[a]), ij(vs[b])]
                    for side in range(4):
                        ax, hi_side = side // 2, side % 2
                        lim = n[ax] if hi_side else 0
                        if all(q[ax] == lim for q in I):
                            bf.append((side, k + 1))
                out.append((gt, vs, bf))
    return xv, out


def write_mixed_gambit(path, xv, eles, side_bc=None):
    side_bc = list(side_bc) if side_bc is not None else [0] * 6
    names = ["Cyclic" if b == 0 else G.BC_NAMES[b] for b in side_bc]
    groups = sorted(set(names), key=names.index)
    ne = len(eles)
    lines = ["        CONTROL INFO 2.3.16", "** GAMBIT NEUTRAL FILE", "mixed", "PROGRAM:  fixture", "",
             "     NUMNP     NELEM     NGRPS    NBSETS     NDFCD     NDFVL",
             "%10d%10d%10d%10d%10d%10d" % (xv.shape[0], ne, 1, len(groups), xv.shape[1], xv.shape[1]),
             "ENDOFSECTION", "   NODAL COORDINATES 2.3.16"]
    for v in range(xv.shape[0]):
        lines.append("%10d " % (v + 1) + " ".join("%.17e" % c for c in xv[v]))
    lines += ["ENDOFSECTION", "      ELEMENTS/CELLS 2.3.16"]
    for e, (gt, vs, _) in enumerate(eles):
        nodes = [v + 1 for v in vs]
        if gt == 2:     # quad: Gambit's counter-clockwise order from tensor slots (0, 1, 3, 2)
            nodes = [nodes[0], nodes[1], nodes[3], nodes[2]]
        lines.append("%8d %2d %2d " % (e + 1, gt, len(nodes)) + " ".join("%8d" % x for x in nodes[:7]))
        if len(nodes) > 7:
            lines.append("               " + " ".join("%8d" % x for x in nodes[7:]))
    lines += ["ENDOFSECTION", "       ELEMENT GROUP 2.3.16",
              "GROUP:          1 ELEMENTS: %10d MATERIAL:          2 NFLAGS:          1" % ne,
              "                           fluid", "       0"]
    ids = [str(e + 1) for e in range(ne)]
    for i in range(0, ne, 10):
        lines.append(" ".join("%7s" % x for x in ids[i:i + 10]))
    bnd = {g: [] for g in groups}
    for e, (gt, _, bf) in enumerate(eles):
        for side, code in bf:
            bnd[names[side]].append((e + 1, gt, code))
    for g in groups:
        lines += ["ENDOFSECTION", " BOUNDARY CONDITIONS 2.3.16"]
        lines.append("%32s%8d%8d%8d%8d" % (g, 1, len(bnd[g]), 0, 6))
        for b in bnd[g]:
            lines.append("%10d%5d%5d" % b)
    lines.append("ENDOFSECTION")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


CASES = [
    # tet_upts: upts_type_tet (0 interior quadrature points, 1 alpha-optimised nodes)
    dict(name="mixed_pritet_p3", kind="pritet", order=3, n=(2, 3, 2), jitter=0.1, steps=3, dt=1e-3, tet_upts=0),
    dict(name="mixed_pritet_p2", kind="pritet", order=2, n=(2, 4, 2), jitter=0.15, steps=3, dt=1e-3, tet_upts=1),
    dict(name="mixed_hexpri_p3", kind="hexpri", order=3, n=(4, 2, 2), jitter=0.1, steps=3, dt=1e-3, tet_upts=0),
    # channel: isothermal wall at y = 0, adiabatic wall at y = 2 pi, on the
    # prisms' triangular faces; periodic in x and z
    dict(name="mixed_channel_p2", kind="pritet", order=2, n=(3, 4, 2), jitter=0.15, steps=3, dt=1e-3, tet_upts=0,
         side_bc=(0, 0, 11, 12, 0, 0), ic="channel_mach01"),
    dict(name="mixed_channel_p3", kind="pritet", order=3, n=(2, 3, 2), jitter=0.1, steps=2, dt=1e-3, tet_upts=1,
         side_bc=(0, 0, 11, 12, 0, 0), ic="channel_mach01"),
]

# 2-D triangle / quadrilateral meshes (conforming in 2-D), Navier-Stokes,
# periodic: the SD-like triangle filter on interior points, and the c+ member
# on alpha-optimised points.  Edge points are Gauss points in both: the
# reference's reader asks for the key " fpts_type_tri" with a leading space
# (src/input.cpp:283), which no input line can match, so its triangles always
# keep the default fpts_type_tri 0.
CASES_2D = [
    dict(name="mixed_triquad_p3", kind="triquad", order=3, n=(4, 3), jitter=0.1, steps=3, dt=1e-3, tri_upts=0,
         tri_fpts=0, vcjh_tri=2),
    dict(name="mixed_triquad_p2", kind="triquad", order=2, n=(4, 4), jitter=0.15, steps=3, dt=1e-3, tri_upts=1,
         tri_fpts=0, vcjh_tri=4),
]


def keep_restart(d, c):
    """The reference's own restart file of a run, kept verbatim as a fixture."""
    src = os.path.join(d, "Rest_%09d_p%04d.dat" % (c["steps"], 0))
    with open(src) as fi, open(os.path.join(HERE, "rest_" + c["name"] + ".dat"), "w") as fo:
        fo.write(fi.read())


def run_case_2d(ref, c, work, restart=False):
    d = os.path.join(work, c["name"])
    os.makedirs(d, exist_ok=True)
    lo, hi = (0.0, 0.0), (2 * np.pi, 2 * np.pi)
    xv, eles = mixed_cells_2d(c["n"], lo, hi, c["jitter"], seed=12345)
    write_mixed_gambit(os.path.join(d, "mesh.neu"), xv, eles, [0, 0, 0, 0])
    vals = input_values_2d(c, lo, hi)
    G.write_input(os.path.join(d, "input"), os.path.join(ref, G.TGV_INPUT), vals)
    out = os.path.join(d, "out")
    os.makedirs(out, exist_ok=True)
    env = dict(os.environ, HIFILES_HOME=os.path.join(REPO, "oracle", "_ref"))
    args = [G.HARNESS, "input", out, "--ic", "channel_mach01", "--steps", str(c["steps"]), "--stages"]
    if restart:
        args += ["--write-restart", str(c["steps"])]
    r = subprocess.run(args, cwd=d, env=env, capture_output=True, text=True)
    if r.returncode != 0:
        print(r.stdout[-3000:], r.stderr[-3000:])
        raise RuntimeError("harness failed for " + c["name"])
    if restart:
        keep_restart(d, c)
    arr, par = G.load_npy_dir(out)
    return arr, par, eles


def input_values_2d(c, lo, hi):
    """The reference's input keys of a 2-D triangle/quad case."""
    return {
        "equation": 0, "viscous": 1, "riemann_solve_type": 0, "vis_riemann_solve_type": 0, "ic_form": 7,
        "order": c["order"], "dt_type": 0, "dt": c["dt"], "n_steps": c["steps"], "adv_type": 3, "tau": 1.0,
        "pen_fact": 0.5, "mesh_file": "mesh.neu", "dx_cyclic": "%.17g" % (hi[0] - lo[0]),
        "dy_cyclic": "%.17g" % (hi[1] - lo[1]), "dz_cyclic": 0.0, "monitor_res_freq": 100000,
        "plot_freq": 100000, "restart_dump_freq": 100000,
        "upts_type_quad": 0, "vcjh_scheme_quad": 1, "upts_type_tri": c["tri_upts"], "fpts_type_tri": c["tri_fpts"],
        "vcjh_scheme_tri": c["vcjh_tri"],
        "prandtl": 0.71, "Mach_free_stream": 0.1, "Re_free_stream": 1600.0, "gamma": 1.4, "fix_vis": 1,
        "res_norm_type": 1,
    }


# arrays kept per element type (prefix t<ele_type>_ in the harness output)
SETUP = ["opp_0", "opp_3", "opp_6", "detjac_upts", "JGinv_upts", "tdA_fpts", "norm_fpts", "disu_upts_init"]
# s03 / s04 arrays are the final flux and common flux of inviscid runs only
INVISCID_ONLY = ("s03_tdisf_upts", "s04_norm_tconf_fpts")
STAGES = ["s01_disu_fpts", "s03_tdisf_upts", "s04_norm_tconf_fpts", "s04_delta_disu_fpts", "s05_grad_disu_upts", "s06_grad_disu_fpts", "s07_tdisf_upts",
          "s08_norm_tdisf_fpts", "s09_div_tconf_upts", "s10_norm_tconf_fpts", "s11_div_tconf_upts",
          "s12_disu_upts0", "final_disu_upts0"]


def run_case(ref, c, work, restart=False):
    d = os.path.join(work, c["name"])
    os.makedirs(d, exist_ok=True)
    lo, hi = (0.0, 0.0, 0.0), (2 * np.pi,) * 3
    xv, eles = mixed_cells(c["kind"], c["n"], lo, hi, c["jitter"], seed=12345)
    write_mixed_gambit(os.path.join(d, "mesh.neu"), xv, eles, c.get("side_bc"))
    vals = input_values_3d(c, [hi[i] - lo[i] for i in range(3)])
    G.write_input(os.path.join(d, "input"), os.path.join(ref, G.TGV_INPUT), vals)
    out = os.path.join(d, "out")
    os.makedirs(out, exist_ok=True)
    env = dict(os.environ, HIFILES_HOME=os.path.join(REPO, "oracle", "_ref"))
    args = [G.HARNESS, "input", out, "--ic", c.get("ic", "tgv_mach01"), "--steps", str(c["steps"]), "--stages"]
    if restart:
        args += ["--write-restart", str(c["steps"])]
    r = subprocess.run(args, cwd=d, env=env, capture_output=True, text=True)
    if r.returncode != 0:
        print(r.stdout[-3000:], r.stderr[-3000:])
        raise RuntimeError("harness failed for " + c["name"])
    if restart:
        keep_restart(d, c)
    arr, par = G.load_npy_dir(out)
    types = []
    for line in open(os.path.join(out, "params.txt")):
        p = line.split()
        if p[0] == "type" and int(p[5]) > 0:
            types.append(dict(index=int(p[1]), ele_type=int(p[3]), n_eles=int(p[5]), n_upts=int(p[7]),
                              n_fpts=int(p[9])))
    return arr, par, types, eles


def input_values_3d(c, L):
    """The reference's input keys of a 3-D mixed case (periodic lengths L)."""
    vals = {
        "equation": 0, "viscous": 1, "riemann_solve_type": 0, "vis_riemann_solve_type": 0, "ic_form": 7,
        "order": c["order"], "dt_type": 0, "dt": c["dt"], "n_steps": c["steps"], "adv_type": 3, "tau": 1.0,
        "pen_fact": 0.5, "mesh_file": "mesh.neu", "dx_cyclic": "%.17g" % L[0], "dy_cyclic": "%.17g" % L[1],
        "dz_cyclic": "%.17g" % L[2], "monitor_res_freq": 100000, "plot_freq": 100000, "restart_dump_freq": 100000,
        "upts_type_hexa": 0, "vcjh_scheme_hexa": 1, "upts_type_tet": c["tet_upts"], "fpts_type_tet": 0, "vcjh_scheme_tet": 2,
        "upts_type_pri_tri": 0, "upts_type_pri_1d": 0, "vcjh_scheme_pri_1d": 1, "vcjh_scheme_tri": 1,
        "prandtl": 0.71, "Mach_free_stream": 0.1, "Re_free_stream": 1600.0, "gamma": 1.4, "fix_vis": 1,
        "res_norm_type": 1,
    }
    if c.get("side_bc"):
        # free stream along x, wall temperature = free-stream temperature
        vals.update({"nx_free_stream": 1.0, "ny_free_stream": 0.0, "nz_free_stream": 0.0, "Mach_wall": 0.0,
                     "nx_wall": 1.0, "ny_wall": 0.0, "nz_wall": 0.0, "rho_bound": 1.0, "u_bound": 1.0,
                     "v_bound": 0.0, "w_bound": 0.0, "p_bound": 1.0, "T_wall": 300.0, "T_free_stream": 300.0})
    return vals


def restart_read_fixture(ref, work):
    """The reference reading its own restart files of mixed_triquad_p2 and
    mixed_pritet_p2 (order 2, read at order 3) and of mixed_hexpri_p3 (order
    3, read at order 2) on the same meshes: read_restart with each type's
    read_restart_info and eles::set_opp_r (src/solver.cpp:390-445,
    src/eles_tris.cpp:511-543, src/eles_tets.cpp:749-780,
    src/eles_pris.cpp:655-698, src/eles.cpp:4135-4153) -> every type's
    disu_upts(0) at the new order, kept as rest_read_<kind>_p<a>_to_p<b>.npz."""
    import shutil
    for name, new_order in (("mixed_triquad_p2", 3), ("mixed_pritet_p2", 3), ("mixed_hexpri_p3", 2)):
        two_d = name == "mixed_triquad_p2"
        c0 = [c for c in (CASES_2D if two_d else CASES) if c["name"] == name][0]
        c = dict(c0, order=new_order)
        d = os.path.join(work, "restart_read_" + c["kind"])
        os.makedirs(d, exist_ok=True)
        shutil.copy(os.path.join(HERE, "rest_%s.dat" % name), os.path.join(d, "Rest_%09d_p%04d.dat" % (c["steps"], 0)))
        if two_d:
            lo, hi = (0.0, 0.0), (2 * np.pi, 2 * np.pi)
            xv, eles = mixed_cells_2d(c["n"], lo, hi, c["jitter"], seed=12345)
            write_mixed_gambit(os.path.join(d, "mesh.neu"), xv, eles, [0, 0, 0, 0])
            vals = input_values_2d(c, lo, hi)
            kinds = (0, 1)
        else:
            lo, hi = (0.0, 0.0, 0.0), (2 * np.pi,) * 3
            xv, eles = mixed_cells(c["kind"], c["n"], lo, hi, c["jitter"], seed=12345)
            write_mixed_gambit(os.path.join(d, "mesh.neu"), xv, eles, None)
            vals = input_values_3d(c, [hi[i] - lo[i] for i in range(3)])
            kinds = (2, 3) if c["kind"] == "pritet" else (3, 4)
        vals.update({"restart_flag": 1, "restart_iter": c["steps"], "n_restart_files": 1})
        G.write_input(os.path.join(d, "input"), os.path.join(ref, G.TGV_INPUT), vals)
        out = os.path.join(d, "out")
        os.makedirs(out, exist_ok=True)
        env = dict(os.environ, HIFILES_HOME=os.path.join(REPO, "oracle", "_ref"))
        r = subprocess.run([G.HARNESS, "input", out, "--steps", "0"], cwd=d, env=env, capture_output=True, text=True)
        if r.returncode != 0:
            print(r.stdout[-3000:], r.stderr[-3000:])
            raise RuntimeError("harness failed reading a restart file")
        arr, _ = G.load_npy_dir(out)
        keep = {"t%d_u_ref" % t: np.asfortranarray(arr["t%d_disu_upts_init" % t]) for t in kinds}
        np.savez_compressed(os.path.join(HERE, "rest_read_%s_p%d_to_p%d.npz" % (c["kind"], c0["order"], new_order)),
                            time=c["steps"] * c["dt"], **keep)
        print("restart read fixture", c["kind"], {k: v.shape for k, v in keep.items()})


def operator_fixture(ref, work):
    """The reference's element operators opp_0 .. opp_6 (per-type set-up of
    eles_tris / eles_tets / eles_pris, src/eles.cpp:3620-4052) at the orders
    and correction schemes the mixed fixtures do not cover, on small meshes
    of the fixtures' kinds, kept as ops_<kind>_p<order>.npz (DG, vcjh scheme
    1) or ops_<kind>_p<order>_s<scheme>.npz.  Tets take the scheme, and so do
    triangles and the prisms' triangles where the reference defines it
    (orders 2-4; src/funcs.cpp:586-635)."""
    for kind, order, scheme in (("triquad", 1, 1), ("triquad", 4, 1), ("triquad", 5, 1), ("pritet", 1, 1),
                                ("pritet", 4, 1), ("pritet", 5, 1), ("triquad", 4, 2), ("pritet", 4, 3),
                                ("pritet", 5, 4)):
        two_d = kind == "triquad"
        tri_scheme = scheme if order <= 4 else 1
        base = [c for c in (CASES_2D if two_d else CASES) if c["name"] == "mixed_%s_p2" % kind][0]
        c = dict(base, order=order, steps=1, vcjh_tri=tri_scheme)
        tag = "ops_%s_p%d" % (kind, order) + ("" if scheme == 1 else "_s%d" % scheme)
        d = os.path.join(work, tag)
        os.makedirs(d, exist_ok=True)
        if two_d:
            lo, hi = (0.0, 0.0), (2 * np.pi, 2 * np.pi)
            xv, eles = mixed_cells_2d(c["n"], lo, hi, c["jitter"], seed=12345)
            write_mixed_gambit(os.path.join(d, "mesh.neu"), xv, eles, [0, 0, 0, 0])
            vals = input_values_2d(c, lo, hi)
            ic, kinds = "channel_mach01", (0, 1)
        else:
            lo, hi = (0.0, 0.0, 0.0), (2 * np.pi,) * 3
            xv, eles = mixed_cells(c["kind"], c["n"], lo, hi, c["jitter"], seed=12345)
            write_mixed_gambit(os.path.join(d, "mesh.neu"), xv, eles, None)
            vals = input_values_3d(c, [hi[i] - lo[i] for i in range(3)])
            vals["vcjh_scheme_tet"] = scheme
            vals["vcjh_scheme_tri"] = tri_scheme
            ic, kinds = "tgv_mach01", (2, 3)
        G.write_input(os.path.join(d, "input"), os.path.join(ref, G.TGV_INPUT), vals)
        out = os.path.join(d, "out")
        os.makedirs(out, exist_ok=True)
        env = dict(os.environ, HIFILES_HOME=os.path.join(REPO, "oracle", "_ref"))
        r = subprocess.run([G.HARNESS, "input", out, "--ic", ic, "--steps", "0"], cwd=d, env=env,
                           capture_output=True, text=True)
        if r.returncode != 0:
            print(r.stdout[-3000:], r.stderr[-3000:])
            raise RuntimeError("harness failed for operators of %s P%d" % (kind, order))
        arr, _ = G.load_npy_dir(out)
        metrics = ("detjac_upts", "JGinv_upts", "tdA_fpts", "norm_fpts")
        keep = {k: np.asfortranarray(v) for k, v in arr.items()
                if (k[:3] in ("t%d_" % kinds[0], "t%d_" % kinds[1]) and (k[3:].startswith("opp_") or k[3:] in metrics))
                or k.startswith("int_inters_")}
        inters = sorted(int(k[len("int_inters_"):]) for k in keep if k.startswith("int_inters_"))
        meta = dict(kind=kind, order=order, n=list(c["n"]), jitter=c["jitter"], tri_upts=c.get("tri_upts"),
                    tri_fpts=c.get("tri_fpts"), tet_upts=c.get("tet_upts"), vcjh_tet=scheme, vcjh_tri=tri_scheme,
                    inters=inters)
        np.savez_compressed(os.path.join(HERE, tag + ".npz"), meta=json.dumps(meta), **keep)
        print("operators", tag, len(keep))


# 2-D quadrilateral boxes with boundaries on every side (side order x-, x+,
# y-, y+), run through make_golden's writer and input; they exercise the
# boundary entry points in 2-D and every boundary type but the moving walls'
# 3-D forms
SEAM_2D = [
    dict(name="seam_quad_bc_euler_p3", dims=2, order=3, n=(5, 4), lo=(-5, -5), hi=(5, 5), viscous=0,
         ic="vortex_u1v0", vcjh=1, jitter=0.1, steps=3, dt=1e-3, stages=True, side_bc=(15, 4, 7, 16)),
    dict(name="seam_quad_bc_euler2_p2", dims=2, order=2, n=(4, 5), lo=(-5, -5), hi=(5, 5), viscous=0,
         ic="vortex_u1v0", vcjh=2, jitter=0.1, steps=3, dt=1e-3, stages=True, side_bc=(1, 2, 5, 6)),
    dict(name="seam_quad_ns_bc_p3", dims=2, order=3, n=(5, 4), lo=(0, 0), hi=(2 * np.pi, 2 * np.pi), viscous=1,
         ic="channel_mach01", vcjh=1, jitter=0.1, steps=3, dt=1e-3, stages=True, side_bc=(3, 4, 13, 14)),
    # Roe common flux (riemann_solve_type 2, 2-D only in the reference)
    dict(name="seam_quad_roe_bc_p3", dims=2, order=3, n=(4, 4), lo=(-5, -5), hi=(5, 5), viscous=0,
         ic="vortex_u1v0", vcjh=1, jitter=0.1, steps=3, dt=1e-3, stages=True, side_bc=(15, 4, 7, 16), riemann=2),
    dict(name="seam_quad_roe_p3_jit", dims=2, order=3, n=(6, 6), lo=(-5, -5), hi=(5, 5), viscous=0,
         ic="vortex_u1v0", vcjh=1, jitter=0.15, steps=3, dt=1e-3, stages=True, side_bc=(0, 0, 0, 0), riemann=2),
]


def pack(out_dir, arr, par, meta):
    """Fixture arrays of one harness run (every element, interface and boundary type)."""
    types = []
    for line in open(os.path.join(out_dir, "params.txt")):
        p = line.split()
        if p[0] == "type" and int(p[5]) > 0:
            types.append(dict(index=int(p[1]), ele_type=int(p[3]), n_eles=int(p[5]), n_upts=int(p[7]),
                              n_fpts=int(p[9])))
    D = int(par["n_dims"])
    fx = {}
    for t in types:
        T = "t%d_" % t["ele_type"]
        for k in SETUP:
            if T + k in arr:
                fx[T + k] = arr[T + k]
        for w in (1, 2, 4, 5):
            for dd in range(D):
                if T + "opp_%d_%d" % (w, dd) in arr:
                    fx[T + "opp_%d_%d" % (w, dd)] = arr[T + "opp_%d_%d" % (w, dd)]
        for k in STAGES:
            if T + k in arr and not (meta["viscous"] and k in INVISCID_ONLY):
                fx[T + k] = arr[T + k]
    inters, bdys = [], []
    for it in range(8):
        for key, lst in (("int_inters_%d" % it, inters), ("bdy_inters_%d" % it, bdys)):
            if key in arr:
                fx[key] = arr[key]
                lst.append(dict(index=it, n_fpts=int(arr[key].shape[1]), n_inters=int(arr[key].shape[2])))
    fx["res_norms"] = arr["res_norms"]
    meta = dict(meta)
    meta.update(types=types, inters=inters, bdy_inters=bdys, dims=D,
                physics={k: par[k] for k in ("gamma", "prandtl", "mu_inf", "rt_inf", "c_sth", "fix_vis", "tau",
                                             "pen_fact")},
                bdy=[par.get("bdy%d" % i, 0.0) for i in range(14)], R_ref=par.get("R_ref", 1.0))
    return fx, meta


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("HIFILES_REF"), required="HIFILES_REF" not in os.environ,
                    help="the reference checkout (or set HIFILES_REF)")
    ap.add_argument("--work", default=None)
    ap.add_argument("--only-2d", action="store_true", help="write the 2-D triangle/quad fixtures only")
    ap.add_argument("--restart-only", action="store_true",
                    help="write only the reference's restart files of mixed_triquad_p2 and mixed_pritet_p2")
    ap.add_argument("--operators", action="store_true",
                    help="write only the reference's element operators at orders 1, 4 and 5 and other schemes")
    ap.add_argument("--restart-read", action="store_true",
                    help="write only the fixtures of the reference reading the order-2 restart files at order 3")
    a = ap.parse_args()
    if not os.path.exists(G.HARNESS):
        subprocess.run(["make", "-C", os.path.join(REPO, "oracle"), "REF=" + a.ref, "ref"], check=True)
    work = a.work or tempfile.mkdtemp(prefix="fr_mixed_")
    if a.operators:
        operator_fixture(a.ref, work)
        return
    if a.restart_read:
        restart_read_fixture(a.ref, work)
        return
    if a.restart_only:
        run_case_2d(a.ref, [c for c in CASES_2D if c["name"] == "mixed_triquad_p2"][0], work, restart=True)
        for name in ("mixed_pritet_p2", "mixed_hexpri_p3"):
            run_case(a.ref, [c for c in CASES if c["name"] == name][0], work, restart=True)
        return
    for c in CASES_2D:
        arr, par, eles = run_case_2d(a.ref, c, work)
        meta = {k: (list(v) if isinstance(v, tuple) else v) for k, v in c.items()}
        meta["viscous"] = 1
        fx, meta = pack(os.path.join(work, c["name"], "out"), arr, par, meta)
        meta["element_counts"] = {str(gt): sum(1 for e in eles if e[0] == gt) for gt in (2, 3)}
        np.savez_compressed(os.path.join(HERE, c["name"] + ".npz"), meta=json.dumps(meta),
                            **{k: np.asfortranarray(v) for k, v in fx.items()})
        print(c["name"], json.dumps({"types": meta["types"], "inters": meta["inters"]}))
    if a.only_2d:
        return
    for c in SEAM_2D:
        arr, par = G.run_case(a.ref, c, work)
        meta = {k: (list(v) if isinstance(v, tuple) else v) for k, v in c.items()}
        fx, meta = pack(os.path.join(work, c["name"], "out"), arr, par, meta)
        np.savez_compressed(os.path.join(HERE, c["name"] + ".npz"), meta=json.dumps(meta),
                            **{k: np.asfortranarray(v) for k, v in fx.items()})
        print(c["name"], json.dumps({"types": meta["types"], "bdy_inters": meta["bdy_inters"]}))
    for c in CASES:
        arr, par, types, eles = run_case(a.ref, c, work)
        fx = {}
        for t in types:
            T = "t%d_" % t["ele_type"]
            for k in SETUP:
                fx[T + k] = arr[T + k]
            for w in (1, 2, 4, 5):
                for dd in range(3):
                    fx[T + "opp_%d_%d" % (w, dd)] = arr[T + "opp_%d_%d" % (w, dd)]
            for k in STAGES:
                if k not in INVISCID_ONLY:
                    fx[T + k] = arr[T + k]
        inters = []
        for it in range(8):
            key = "int_inters_%d" % it
            if key in arr:
                fx[key] = arr[key]
                inters.append(dict(index=it, n_fpts=int(arr[key].shape[1]), n_inters=int(arr[key].shape[2])))
        bdys = []
        for it in range(8):
            key = "bdy_inters_%d" % it
            if key in arr:
                fx[key] = arr[key]
                bdys.append(dict(index=it, n_fpts=int(arr[key].shape[1]), n_inters=int(arr[key].shape[2])))
        fx["res_norms"] = arr["res_norms"]
        meta = dict(c)
        meta["n"] = list(c["n"])
        meta["types"] = types
        meta["inters"] = inters
        meta["bdy_inters"] = bdys
        meta["bdy"] = [par.get("bdy%d" % i, 0.0) for i in range(14)]
        meta["R_ref"] = par.get("R_ref", 1.0)
        if c.get("side_bc"):
            meta["side_bc"] = list(c["side_bc"])
        meta["physics"] = {k: par[k] for k in ("gamma", "prandtl", "mu_inf", "rt_inf", "c_sth", "fix_vis", "tau",
                                                 "pen_fact")}
        meta["element_counts"] = {str(gt): sum(1 for e in eles if e[0] == gt) for gt in (4, 5, 6)}
        np.savez_compressed(os.path.join(HERE, c["name"] + ".npz"), meta=json.dumps(meta),
                            **{k: np.asfortranarray(v) for k, v in fx.items()})
        print(c["name"], json.dumps({"types": types, "inters": inters}))


if __name__ == "__main__":
    main()
