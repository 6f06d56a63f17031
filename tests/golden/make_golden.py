#!/usr/bin/env python3
"""Generate the golden fixtures in tests/golden/ by running the reference itself.

Runs only where the reference sources are available (it reads them under
--ref or HIFILES_REF) and where oracle/_ref/ref_harness has been built
(`make -C oracle REF=<reference checkout> ref`).  For every case it

  1. writes a periodic box mesh (Gambit neutral format, the reader of
     src/geometry.cpp:1706-1880 and 1122-1307) and an input file derived from
     the reference's own TGV regression input,
  2. runs oracle/_ref/ref_harness (the unmodified reference objects) which
     dumps the reference's operators, metrics, interface wiring, the
     intermediate arrays of one CalcResidual, and the state + L1 residual norms
     after N RK45 steps,
  3. checks that the reference's element / point ordering equals the one the
     box generator defines (so the arrays below need no permutation),
  4. pins the C restatement (oracle/fr_oracle.c) against those dumps and
     records the maximum normwise relative difference,
  5. stores a compact .npz fixture.

The regression known-answer values of the reference's TGV test
(testcases/regression_tests.py:300-310) are recorded in kat.json together
with the value this script reproduces with the oracle.

Usage:  python tests/golden/make_golden.py --ref <reference checkout>   (or HIFILES_REF=<dir>)
"""
import argparse
import json
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, os.path.join(REPO, "oracle"))
import oracle as O  # noqa: E402

HARNESS = os.path.join(REPO, "oracle", "_ref", "ref_harness")
TGV_INPUT = "testcases/navier-stokes/Taylor_Green_vortex/input_TGV_SD_hex"


# ----------------------------------------------------------------- mesh writer

def box_vertices(dims, n, lo, hi, jitter=0.0, seed=0):
    """Same vertex set and element->vertex map (tensor order) as or_box_new."""
    m = O.Mesh.box(dims, 1, n, lo, hi, jitter=jitter, seed=seed)
    del m
    # Rebuild in Python with the identical LCG so both agree bit-for-bit.
    nx, ny = n[0], n[1]
    nz = n[2] if dims == 3 else 1
    vx, vy, vz = nx + 1, ny + 1, (nz + 1 if dims == 3 else 1)
    mask = (1 << 64) - 1
    s = (seed * 6364136223846793005 + 1442695040888963407) & mask
    xv = np.zeros((vx * vy * vz, dims))
    nn = [nx, ny, nz]
    for k in range(vz):
        for j in range(vy):
            for i in range(vx):
                v = i + vx * (j + vy * k)
                ijk = [i, j, k]
                interior = all(0 < ijk[d] < nn[d] for d in range(dims))
                for d in range(dims):
                    h = (hi[d] - lo[d]) / nn[d]
                    x = lo[d] + (hi[d] - lo[d]) * ijk[d] / nn[d]
                    s = (s * 6364136223846793005 + 1442695040888963407) & mask
                    r = ((s >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0
                    if interior and jitter > 0:
                        x += jitter * h * r
                    xv[v, d] = x
    nsp = 1 << dims
    c2v = np.zeros((nx * ny * nz, nsp), dtype=np.int64)
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                e = i + nx * (j + ny * k)
                for c in range(2 if dims == 3 else 1):
                    for b in range(2):
                        for a in range(2):
                            c2v[e, a + 2 * b + 4 * c] = (i + a) + vx * ((j + b) + vy * (k + c))
    return xv, c2v


BC_NAMES = {1: "sub_in_simp", 2: "sub_out_simp", 3: "sub_in_char", 4: "sub_out_char", 5: "sup_in", 6: "sup_out",
            7: "slip_wall", 11: "isotherm_fix", 12: "adiabat_fix", 13: "isotherm_move", 14: "adiabat_move",
            15: "char", 16: "slip_wall_dual"}


def write_gambit(path, dims, xv, c2v, n, side_bc=None):
    """Gambit neutral file.  Node order is chosen so that the reference's local
    axes (xi, eta, zeta) equal physical (x, y, z): the hex reader stores Gambit
    nodes 0..7 in c2v slots (0,2,4,6,1,3,5,7) (src/geometry.cpp:1840-1843) and
    the quad reader stores them in slots (0,1,3,2) (src/geometry.cpp:1800-1803)."""
    ne = c2v.shape[0]
    side_bc = list(side_bc) if side_bc is not None else [0] * (2 * dims)
    names = ["Cyclic" if b == 0 else BC_NAMES[b] for b in side_bc]
    groups = sorted(set(names), key=names.index)
    lines = ["        CONTROL INFO 2.3.16", "** GAMBIT NEUTRAL FILE", "box", "PROGRAM:  fixture", "",
             "     NUMNP     NELEM     NGRPS    NBSETS     NDFCD     NDFVL",
             "%10d%10d%10d%10d%10d%10d" % (xv.shape[0], ne, 1, len(groups), dims, dims),
             "ENDOFSECTION", "   NODAL COORDINATES 2.3.16"]
    for v in range(xv.shape[0]):
        lines.append("%10d " % (v + 1) + " ".join("%.17e" % c for c in xv[v]))
    lines += ["ENDOFSECTION", "      ELEMENTS/CELLS 2.3.16"]
    if dims == 3:
        # Gambit node g = ag + 2 bg + 4 cg  <->  tensor node a + 2b + 4c with a=cg, b=ag, c=bg
        order = [((g >> 2) & 1) + 2 * (g & 1) + 4 * ((g >> 1) & 1) for g in range(8)]
        for e in range(ne):
            nodes = [c2v[e, order[g]] + 1 for g in range(8)]
            lines.append("%8d %2d %2d " % (e + 1, 4, 8) + " ".join("%8d" % x for x in nodes[:7]))
            lines.append("               %8d" % nodes[7])
    else:
        for e in range(ne):
            nodes = [c2v[e, 0] + 1, c2v[e, 1] + 1, c2v[e, 3] + 1, c2v[e, 2] + 1]
            lines.append("%8d %2d %2d " % (e + 1, 2, 4) + " ".join("%8d" % x for x in nodes))
    lines += ["ENDOFSECTION", "       ELEMENT GROUP 2.3.16",
              "GROUP:          1 ELEMENTS: %10d MATERIAL:          2 NFLAGS:          1" % ne,
              "                           fluid", "       0"]
    ids = [str(e + 1) for e in range(ne)]
    for i in range(0, ne, 10):
        lines.append(" ".join("%7s" % x for x in ids[i:i + 10]))
    bnd = {g: [] for g in groups}
    nx, ny = n[0], n[1]
    nz = n[2] if dims == 3 else 1
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                e = i + nx * (j + ny * k) + 1
                if dims == 3:   # Gambit hex faces: x- 5, x+ 6, y- 4, y+ 2, z- 1, z+ 3
                    if i == 0: bnd[names[0]].append((e, 4, 5))
                    if i == nx - 1: bnd[names[1]].append((e, 4, 6))
                    if j == 0: bnd[names[2]].append((e, 4, 4))
                    if j == ny - 1: bnd[names[3]].append((e, 4, 2))
                    if k == 0: bnd[names[4]].append((e, 4, 1))
                    if k == nz - 1: bnd[names[5]].append((e, 4, 3))
                else:           # Gambit quad faces: y- 1, x+ 2, y+ 3, x- 4
                    if j == 0: bnd[names[2]].append((e, 2, 1))
                    if i == nx - 1: bnd[names[1]].append((e, 2, 2))
                    if j == ny - 1: bnd[names[3]].append((e, 2, 3))
                    if i == 0: bnd[names[0]].append((e, 2, 4))
    for gi, g in enumerate(groups):
        lines += ["ENDOFSECTION", " BOUNDARY CONDITIONS 2.3.16"]
        lines.append("%32s%8d%8d%8d%8d" % (g, 1, len(bnd[g]), 0, 6))
        for b in bnd[g]:
            lines.append("%10d%5d%5d" % b)
    lines.append("ENDOFSECTION")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_input(path, template, values):
    txt = open(template).read()
    for k, v in values.items():
        pat = re.compile(r"^(\s*%s\s+)\S+" % re.escape(k), re.M)
        if pat.search(txt):
            txt = pat.sub(lambda mm: mm.group(1) + str(v), txt, count=1)
        else:
            txt += "\n%s %s\n" % (k, v)
    with open(path, "w") as f:
        f.write(txt)


def load_npy_dir(d):
    out = {}
    for fn in os.listdir(d):
        if fn.endswith(".npy"):
            out[fn[:-4]] = np.load(os.path.join(d, fn))
    params = {}
    for line in open(os.path.join(d, "params.txt")):
        p = line.split()
        if p[0] != "type":
            params[p[0]] = float(p[1])
    return out, params


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


# ------------------------------------------------------------------------ cases

CASES = [
    # name, dims, order, n, lo, hi, viscous, ic, vcjh, jitter, steps, dt, stages
    dict(name="quad_vortex_p3_n6", dims=2, order=3, n=(6, 6), lo=(-5, -5), hi=(5, 5), viscous=0,
         ic="vortex_u1v0", vcjh=1, jitter=0.0, steps=20, dt=1e-3, stages=True, restart_out=True),
    dict(name="quad_vortex_p2_n5_jit", dims=2, order=2, n=(5, 5), lo=(-5, -5), hi=(5, 5), viscous=0,
         ic="vortex_u1v0", vcjh=2, jitter=0.15, steps=10, dt=1e-3, stages=True),
    dict(name="quad_vortex_p3_n20", dims=2, order=3, n=(20, 20), lo=(-5, -5), hi=(5, 5), viscous=0,
         ic="vortex_u1v0", vcjh=1, jitter=0.0, steps=1000, dt=1e-3, stages=False),
    dict(name="hex_tgv_p3_n3", dims=3, order=3, n=(3, 3, 3), lo=(0, 0, 0), hi=(2 * np.pi,) * 3, viscous=1,
         ic="tgv_mach01", vcjh=1, jitter=0.0, steps=5, dt=1e-3, stages=True),
    dict(name="hex_tgv_p2_n3_jit", dims=3, order=2, n=(3, 3, 3), lo=(0, 0, 0), hi=(2 * np.pi,) * 3, viscous=1,
         ic="tgv_mach01", vcjh=2, jitter=0.1, steps=5, dt=1e-3, stages=True, restart_out=True),
    dict(name="hex_tgv_p4_n2", dims=3, order=4, n=(2, 2, 2), lo=(0, 0, 0), hi=(2 * np.pi,) * 3, viscous=1,
         ic="tgv_mach01", vcjh=1, jitter=0.0, steps=3, dt=1e-3, stages=False),
    dict(name="hex_euler_p3_n3", dims=3, order=3, n=(3, 3, 3), lo=(0, 0, 0), hi=(2 * np.pi,) * 3, viscous=0,
         ic="tgv_mach01", vcjh=1, jitter=0.0, steps=3, dt=1e-3, stages=True),
    # the ends of the built order range
    dict(name="quad_vortex_p1_n8_jit", dims=2, order=1, n=(8, 8), lo=(-5, -5), hi=(5, 5), viscous=0,
         ic="vortex_u1v0", vcjh=1, jitter=0.1, steps=10, dt=1e-3, stages=True),
    dict(name="quad_vortex_p5_n4", dims=2, order=5, n=(4, 4), lo=(-5, -5), hi=(5, 5), viscous=0,
         ic="vortex_u1v0", vcjh=2, jitter=0.0, steps=10, dt=1e-3, stages=True),
    dict(name="hex_tgv_p1_n4_jit", dims=3, order=1, n=(4, 4, 4), lo=(0, 0, 0), hi=(2 * np.pi,) * 3, viscous=1,
         ic="tgv_mach01", vcjh=2, jitter=0.1, steps=5, dt=1e-3, stages=True),
    # eddy-viscosity LES (input keys LES 1, SGS_model 1 = WALE / 0 = Smagorinsky)
    dict(name="hex_wale_p3_n3_jit", dims=3, order=3, n=(3, 3, 3), lo=(0, 0, 0), hi=(2 * np.pi,) * 3, viscous=1,
         ic="tgv_mach01", vcjh=1, jitter=0.1, steps=5, dt=1e-3, stages=True, les=1, sgs=1, filter_ratio=1.0),
    dict(name="hex_smag_p2_n3", dims=3, order=2, n=(3, 3, 3), lo=(0, 0, 0), hi=(2 * np.pi,) * 3, viscous=1,
         ic="tgv_mach01", vcjh=2, jitter=0.0, steps=3, dt=1e-3, stages=True, les=1, sgs=0, filter_ratio=2.0),
    dict(name="quad_wale_p3_n6_jit", dims=2, order=3, n=(6, 6), lo=(-5, -5), hi=(5, 5), viscous=1,
         ic="vortex_u1v0", vcjh=1, jitter=0.15, steps=5, dt=1e-3, stages=True, les=1, sgs=1, filter_ratio=1.0),
    # Roe common flux (riemann_solve_type 2; 2-D only in the reference)
    dict(name="quad_vortex_roe_p3_n6_jit", dims=2, order=3, n=(6, 6), lo=(-5, -5), hi=(5, 5), viscous=0,
         ic="vortex_u1v0", vcjh=1, jitter=0.15, steps=10, dt=1e-3, stages=True, riemann=2),
    dict(name="quad_ns_roe_p2_n5", dims=2, order=2, n=(5, 5), lo=(-5, -5), hi=(5, 5), viscous=1,
         ic="vortex_u1v0", vcjh=2, jitter=0.0, steps=5, dt=1e-3, stages=True, riemann=2),
    # boundary conditions (side types x-, x+, y-, y+, z-, z+; 0 = periodic)
    dict(name="quad_bc_euler_p3", dims=2, order=3, n=(5, 4), lo=(-5, -5), hi=(5, 5), viscous=0,
         ic="vortex_u1v0", vcjh=1, jitter=0.1, steps=10, dt=1e-3, stages=True, side_bc=(15, 4, 7, 16)),
    dict(name="quad_bc_euler2_p2", dims=2, order=2, n=(4, 5), lo=(-5, -5), hi=(5, 5), viscous=0,
         ic="vortex_u1v0", vcjh=2, jitter=0.1, steps=10, dt=1e-3, stages=True, side_bc=(1, 2, 5, 6)),
    dict(name="quad_bc_roe_p3", dims=2, order=3, n=(4, 4), lo=(-5, -5), hi=(5, 5), viscous=0,
         ic="vortex_u1v0", vcjh=1, jitter=0.1, steps=10, dt=1e-3, stages=True, side_bc=(15, 4, 7, 16), riemann=2),
    dict(name="quad_ns_bc_p3", dims=2, order=3, n=(5, 4), lo=(0, 0), hi=(2 * np.pi, 2 * np.pi), viscous=1,
         ic="channel_mach01", vcjh=1, jitter=0.1, steps=5, dt=1e-3, stages=True, side_bc=(3, 4, 13, 14)),
    dict(name="hex_channel_p2", dims=3, order=2, n=(4, 3, 3), lo=(0, 0, 0), hi=(2 * np.pi,) * 3, viscous=1,
         ic="channel_mach01", vcjh=1, jitter=0.1, steps=5, dt=1e-3, stages=True, side_bc=(0, 0, 11, 12, 0, 0)),
    dict(name="hex_channel_char_p3", dims=3, order=3, n=(3, 2, 2), lo=(0, 0, 0), hi=(2 * np.pi,) * 3, viscous=1,
         ic="channel_mach01", vcjh=1, jitter=0.0, steps=3, dt=1e-3, stages=True, side_bc=(15, 15, 11, 7, 0, 0)),
]


def run_case(ref, c, work):
    d = os.path.join(work, c["name"])
    os.makedirs(d, exist_ok=True)
    xv, c2v = box_vertices(c["dims"], c["n"], c["lo"], c["hi"], c["jitter"], seed=12345)
    write_gambit(os.path.join(d, "mesh.neu"), c["dims"], xv, c2v, c["n"], c.get("side_bc"))
    L = [c["hi"][i] - c["lo"][i] for i in range(c["dims"])]
    # the cyclic lengths stay the box lengths in every direction, walls too:
    # with a zero length check_cyclic (src/geometry.cpp:3634-3664) matches a
    # periodic face with itself and flips the orientation of the real pairs
    vals = {
        "equation": 0, "viscous": c["viscous"], "riemann_solve_type": 0, "vis_riemann_solve_type": 0,
        "ic_form": 7 if c["ic"].startswith("tgv") else 1, "order": c["order"], "dt_type": 0, "dt": c["dt"],
        "n_steps": max(c["steps"], 1), "adv_type": 3, "tau": 1.0, "pen_fact": 0.5,
        "mesh_file": "mesh.neu", "dx_cyclic": "%.17g" % L[0], "dy_cyclic": "%.17g" % L[1],
        "dz_cyclic": "%.17g" % (L[2] if c["dims"] == 3 else 0.0),
        "monitor_res_freq": 100000, "plot_freq": 100000, "restart_dump_freq": 100000,
        "upts_type_quad": 0, "vcjh_scheme_quad": c["vcjh"], "upts_type_hexa": 0, "vcjh_scheme_hexa": c["vcjh"],
        "prandtl": 0.71, "Mach_free_stream": 0.1, "Re_free_stream": 1600.0, "gamma": 1.4, "fix_vis": 1,
        "res_norm_type": 1,
    }
    vals["riemann_solve_type"] = c.get("riemann", 0)
    if c.get("side_bc"):
        # free stream along x; inviscid runs take the boundary state as given
        vals.update({"nx_free_stream": 1.0, "ny_free_stream": 0.0, "nz_free_stream": 0.0, "Mach_wall": 0.05,
                     "nx_wall": 1.0, "ny_wall": 0.0, "nz_wall": 0.0, "rho_bound": 1.0, "u_bound": 1.0,
                     "v_bound": 0.0, "w_bound": 0.0, "p_bound": 1.0, "T_wall": 300.0, "T_free_stream": 300.0})
    if c.get("les"):
        vals.update({"LES": 1, "filter_type": 0, "filter_ratio": "%.17g" % c["filter_ratio"],
                     "SGS_model": c["sgs"], "wall_model": 0, "wall_layer_thickness": 0.0})
    write_input(os.path.join(d, "input"), os.path.join(ref, TGV_INPUT), vals)
    out = os.path.join(d, "out")
    os.makedirs(out, exist_ok=True)
    args = [HARNESS, "input", out, "--ic", c["ic"], "--steps", str(c["steps"])]
    if c["stages"]:
        args.append("--stages")
    if c.get("restart_out"):
        args += ["--write-restart", str(c["steps"])]
    env = dict(os.environ, HIFILES_HOME=os.path.join(REPO, "oracle", "_ref"))
    r = subprocess.run(args, cwd=d, env=env, capture_output=True, text=True)
    if r.returncode != 0:
        print(r.stdout[-2000:], r.stderr[-2000:])
        raise RuntimeError("harness failed for " + c["name"])
    if c.get("restart_out"):
        # the reference's own restart file, kept verbatim as a fixture
        src = os.path.join(d, "Rest_%09d_p%04d.dat" % (c["steps"], 0))
        with open(src) as fi, open(os.path.join(HERE, "rest_" + c["name"] + ".dat"), "w") as fo:
            fo.write(fi.read())
    return load_npy_dir(out)


def restart_read_fixture(ref, work):
    """The reference reading a restart file written by this library's writer
    (fr_restart_write) at another order: the TGV P=2 jittered case's final
    state, written as order 2, read by the reference set up at order 3
    (read_restart + eles::set_opp_r interpolation) -> its disu_upts(0)."""
    sys.path.insert(0, os.path.join(REPO, "hifiles-solver_b200"))
    import hifiles_b200 as H
    meta, fx = None, np.load(os.path.join(HERE, "hex_tgv_p2_n3_jit.npz"))
    meta = json.loads(str(fx["meta"]))
    u2 = np.asfortranarray(fx["uN"])
    d = os.path.join(work, "restart_read")
    os.makedirs(d, exist_ok=True)
    H.restart_write(os.path.join(d, "Rest_%09d_p%04d.dat" % (7, 0)), 0.005,
                    [dict(ele_type=4, order=2, loc_1d=O.points_1d(2), disu_upts=u2)])
    xv, c2v = box_vertices(3, meta["n"], meta["lo"], meta["hi"], meta["jitter"], seed=12345)
    write_gambit(os.path.join(d, "mesh.neu"), 3, xv, c2v, meta["n"])
    L = [meta["hi"][i] - meta["lo"][i] for i in range(3)]
    vals = {"equation": 0, "viscous": 1, "order": 3, "dt_type": 0, "dt": 1e-3, "n_steps": 1, "adv_type": 3,
            "mesh_file": "mesh.neu", "dx_cyclic": "%.17g" % L[0], "dy_cyclic": "%.17g" % L[1],
            "dz_cyclic": "%.17g" % L[2], "monitor_res_freq": 100000, "plot_freq": 100000,
            "restart_dump_freq": 100000, "upts_type_hexa": 0, "vcjh_scheme_hexa": 2, "prandtl": 0.71,
            "Mach_free_stream": 0.1, "Re_free_stream": 1600.0, "gamma": 1.4, "fix_vis": 1, "ic_form": 7,
            "restart_flag": 1, "restart_iter": 7, "n_restart_files": 1}
    write_input(os.path.join(d, "input"), os.path.join(ref, TGV_INPUT), vals)
    out = os.path.join(d, "out")
    os.makedirs(out, exist_ok=True)
    env = dict(os.environ, HIFILES_HOME=os.path.join(REPO, "oracle", "_ref"))
    r = subprocess.run([HARNESS, "input", out, "--steps", "0"], cwd=d, env=env, capture_output=True, text=True)
    if r.returncode != 0:
        print(r.stdout[-2000:], r.stderr[-2000:])
        raise RuntimeError("harness failed reading a restart file")
    arr, _ = load_npy_dir(out)
    np.savez_compressed(os.path.join(HERE, "rest_read_p2_to_p3.npz"), u_p2=u2,
                        u_p3_ref=np.asfortranarray(arr["t4_disu_upts_init"]), time=0.005)
    print("restart read fixture: reference P3 state from our P2 file, shape", arr["t4_disu_upts_init"].shape)


# integral quantities on the reference's volume cubature (volume_cub_order)
IQ_CASES = [
    dict(name="iq_hex_tgv_p3_n3_jit", dims=3, order=3, n=(3, 3, 3), lo=(0, 0, 0), hi=(2 * np.pi,) * 3, viscous=1,
         ic="tgv_mach01", vcjh=1, jitter=0.1, cub=3),
    dict(name="iq_hex_tgv_p2_n3_jit_cub5", dims=3, order=2, n=(3, 2, 3), lo=(0, 0, 0), hi=(2 * np.pi,) * 3,
         viscous=1, ic="tgv_mach01", vcjh=2, jitter=0.1, cub=5),
    dict(name="iq_quad_vortex_p3_n6_jit_cub4", dims=2, order=3, n=(6, 5), lo=(-5, -5), hi=(5, 5), viscous=1,
         ic="vortex_u1v0", vcjh=1, jitter=0.15, cub=4),
]
IQ_NAMES = "5 kineticenergy vorticity pressuredilatation straincolonproduct devstraincolonproduct"


def integral_fixtures(ref, work):
    """The reference's own integral quantities (eles::CalcIntegralQuantities on
    its volume cubature) of a state after one residual evaluation, with the
    cubature points, weights, interpolation operator and Jacobians it used."""
    env = dict(os.environ, HIFILES_HOME=os.path.join(REPO, "oracle", "_ref"))
    for c in IQ_CASES:
        d = os.path.join(work, c["name"])
        os.makedirs(d, exist_ok=True)
        xv, c2v = box_vertices(c["dims"], c["n"], c["lo"], c["hi"], c["jitter"], seed=12345)
        write_gambit(os.path.join(d, "mesh.neu"), c["dims"], xv, c2v, c["n"])
        L = [c["hi"][i] - c["lo"][i] for i in range(c["dims"])]
        vals = {"equation": 0, "viscous": c["viscous"], "ic_form": 7 if c["ic"].startswith("tgv") else 1,
                "order": c["order"], "dt_type": 0, "dt": 1e-3, "n_steps": 1, "adv_type": 3, "tau": 1.0,
                "pen_fact": 0.5, "mesh_file": "mesh.neu", "dx_cyclic": "%.17g" % L[0], "dy_cyclic": "%.17g" % L[1],
                "dz_cyclic": "%.17g" % (L[2] if c["dims"] == 3 else 0.0), "monitor_res_freq": 100000,
                "plot_freq": 100000, "restart_dump_freq": 100000, "upts_type_quad": 0,
                "vcjh_scheme_quad": c["vcjh"], "upts_type_hexa": 0, "vcjh_scheme_hexa": c["vcjh"], "prandtl": 0.71,
                "Mach_free_stream": 0.1, "Re_free_stream": 1600.0, "gamma": 1.4, "fix_vis": 1, "res_norm_type": 1,
                "volume_cub_order": c["cub"], "integral_quantities": IQ_NAMES}
        write_input(os.path.join(d, "input"), os.path.join(ref, TGV_INPUT), vals)
        out = os.path.join(d, "out")
        os.makedirs(out, exist_ok=True)
        r = subprocess.run([HARNESS, "input", out, "--ic", c["ic"], "--integrals"], cwd=d, env=env,
                           capture_output=True, text=True)
        if r.returncode != 0:
            print(r.stdout[-2000:], r.stderr[-2000:])
            raise RuntimeError("harness failed for " + c["name"])
        arr, par = load_npy_dir(out)
        T = "t%d_" % (1 if c["dims"] == 2 else 4)
        meta = {k: (list(v) if isinstance(v, tuple) else v) for k, v in c.items()}
        meta["physics"] = {k: par[k] for k in ("gamma", "prandtl", "mu_inf", "rt_inf", "c_sth", "fix_vis", "tau",
                                                 "pen_fact")}
        meta["quantities"] = IQ_NAMES.split()[1:]
        meta["seed"] = 12345
        fx = dict(u0=arr[T + "disu_upts_iq"], grad=arr[T + "grad_disu_upts_iq"], iq=arr["integral_quantities"],
                  loc=arr[T + "loc_volume_cubpts"], weight=arr[T + "weight_volume_cubpts"],
                  opp=arr[T + "opp_volume_cubpts"], detjac=arr[T + "vol_detjac_vol_cubpts"])
        np.savez_compressed(os.path.join(HERE, c["name"] + ".npz"), meta=json.dumps(meta),
                            **{k: np.asfortranarray(v) for k, v in fx.items()})
        print(c["name"], "integral quantities", arr["integral_quantities"])


# the BASELINE vortex (periodic [-5, 5]^2, quads, c_dg, Rusanov, RK45, dt 1e-3)
# advanced to t = 1 by the reference at P = 2 on three meshes: its own
# convergence rate, against which the CUDA path's rate and states are checked
ORDER_CASES = [dict(name="order_vortex_p2_n%d" % n, dims=2, order=2, n=(n, n), lo=(-5, -5), hi=(5, 5), viscous=0,
                    ic="vortex_u1v0", vcjh=1, jitter=0.0, steps=1000, dt=1e-3, stages=False) for n in (10, 20, 40)]


def order_fixtures(ref, work):
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(len(ORDER_CASES)) as ex:
        res = list(ex.map(lambda c: run_case(ref, c, work), ORDER_CASES))
    for c, (arr, par) in zip(ORDER_CASES, res):
        meta = {k: (list(v) if isinstance(v, tuple) else v) for k, v in c.items()}
        meta["physics"] = {k: par[k] for k in ("gamma", "prandtl", "mu_inf", "rt_inf", "c_sth", "fix_vis", "tau",
                                                 "pen_fact")}
        meta["seed"] = 12345
        np.savez_compressed(os.path.join(HERE, c["name"] + ".npz"), meta=json.dumps(meta),
                            u0=np.asfortranarray(arr["t1_disu_upts_init"]),
                            uN=np.asfortranarray(arr["t1_final_disu_upts0"]),
                            pos=np.asfortranarray(arr["t1_pos_upts"]))
        print(c["name"], "done")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("HIFILES_REF"), required="HIFILES_REF" not in os.environ,
                    help="the reference checkout (or set HIFILES_REF)")
    ap.add_argument("--work", default=None)
    ap.add_argument("--integrals", action="store_true", help="only the integral-quantity fixtures (iq_*.npz)")
    ap.add_argument("--order", action="store_true", help="only the reference convergence fixtures (order_*.npz)")
    a = ap.parse_args()
    if not os.path.exists(HARNESS):
        subprocess.run(["make", "-C", os.path.join(REPO, "oracle"), "REF=" + a.ref, "ref"], check=True)
    work = a.work or tempfile.mkdtemp(prefix="fr_golden_")
    if a.integrals:
        integral_fixtures(a.ref, work)
        return
    if a.order:
        order_fixtures(a.ref, work)
        return
    summary = {}
    for c in CASES:
        arr, par = run_case(a.ref, c, work)
        et = 1 if c["dims"] == 2 else 4
        T = "t%d_" % et
        m = O.Mesh.box(c["dims"], c["order"], c["n"], c["lo"], c["hi"], jitter=c["jitter"], seed=12345,
                       vcjh_scheme=c["vcjh"], side_bc=c.get("side_bc"))
        bdy = [par.get("bdy%d" % i, 0.0) for i in range(14)]
        g = m.geometry()
        # 3. ordering check: the reference's solution points sit where ours do
        dpos = np.abs(arr[T + "pos_upts"] - g["pos_upts"]).max()
        assert dpos < 1e-12, (c["name"], dpos)
        ph = O.physics(viscous=c["viscous"], gamma=par["gamma"], prandtl=par["prandtl"], mu_inf=par["mu_inf"],
                       rt_inf=par["rt_inf"], c_sth=par["c_sth"], fix_vis=par["fix_vis"], tau=par["tau"],
                       pen_fact=par["pen_fact"], les=c.get("les", 0), sgs_model=c.get("sgs", 1),
                       filter_ratio=c.get("filter_ratio", 1.0), riemann=c.get("riemann", 0), bdy=bdy,
                       R_ref=par.get("R_ref", 1.0))
        u0 = arr[T + "disu_upts_init"]
        pins = {}
        pins["metrics_detjac"] = rel(g["detjac_upts"], arr[T + "detjac_upts"])
        pins["metrics_JGinv"] = rel(g["JGinv_upts"], arr[T + "JGinv_upts"])
        pins["metrics_tdA"] = rel(g["tdA_fpts"], arr[T + "tdA_fpts"])
        pins["metrics_norm"] = rel(g["norm_fpts"], arr[T + "norm_fpts"])
        for w, dd in ((0, 0), (3, 0), (1, 0), (2, 0)):
            pins["opp_%d" % w] = rel(m.operator(w, dd), arr[T + "opp_%d" % w if w in (0, 3) else T + "opp_%d_%d" % (w, dd)])
        fx = dict(u0=u0)
        if c["stages"]:
            div, st = m.residual(ph, u0, stages=True)
            pins["residual"] = rel(div, arr[T + "s11_div_tconf_upts"])
            pins["disu_fpts"] = rel(st["disu_fpts"], arr[T + "s01_disu_fpts"])
            pins["norm_tdisf_fpts"] = rel(st["norm_tdisf_fpts"], arr[T + "s08_norm_tdisf_fpts"])
            ntc_key = T + ("s10_norm_tconf_fpts" if c["viscous"] else "s04_norm_tconf_fpts")
            pins["norm_tconf_fpts"] = rel(st["norm_tconf_fpts"], arr[ntc_key])
            pins["tdisf_upts"] = rel(st["tdisf_upts"], arr[T + ("s07_tdisf_upts" if c["viscous"] else "s03_tdisf_upts")])
            fx["div0"] = arr[T + "s11_div_tconf_upts"]
            fx["disu_fpts0"] = arr[T + "s01_disu_fpts"]
            fx["norm_tconf_fpts0"] = arr[ntc_key]
            fx["norm_tdisf_fpts0"] = arr[T + "s08_norm_tdisf_fpts"]
            fx["tdisf_upts0"] = arr[T + ("s07_tdisf_upts" if c["viscous"] else "s03_tdisf_upts")]
            if c["viscous"]:
                pins["grad_disu_upts"] = rel(st["grad_disu_upts"], arr[T + "s05_grad_disu_upts"])
                pins["grad_disu_fpts"] = rel(st["grad_disu_fpts"], arr[T + "s06_grad_disu_fpts"])
                pins["delta_disu_fpts"] = rel(st["delta_disu_fpts"], arr[T + "s04_delta_disu_fpts"])
                fx["grad_disu_upts0"] = arr[T + "s05_grad_disu_upts"]
                fx["grad_disu_fpts0"] = arr[T + "s06_grad_disu_fpts"]
                fx["delta_disu_fpts0"] = arr[T + "s04_delta_disu_fpts"]
            if c.get("les"):
                pins["sgsf_upts"] = rel(st["sgsf_upts"], arr[T + "s07_sgsf_upts"])
                pins["sgsf_fpts"] = rel(st["sgsf_fpts"], arr[T + "s07_sgsf_fpts"])
                fx["sgsf_upts0"] = arr[T + "s07_sgsf_upts"]
        else:
            div = m.residual(ph, u0)
            fx["div0"] = div  # not dumped by the harness in this mode: the pinned oracle's value
        if c["steps"] > 0:
            uN, _, nrm = m.rk45(ph, u0, c["dt"], c["steps"])
            pins["state_after_steps"] = rel(uN, arr[T + "final_disu_upts0"])
            pins["res_norms"] = rel(nrm, arr["res_norms"])
            fx["uN"] = arr[T + "final_disu_upts0"]
            fx["norms"] = arr["res_norms"]
        meta = {k: (list(v) if isinstance(v, tuple) else v) for k, v in c.items()}
        meta["physics"] = {k: par[k] for k in ("gamma", "prandtl", "mu_inf", "rt_inf", "c_sth", "fix_vis", "tau",
                                                 "pen_fact")}
        meta["physics"].update(les=c.get("les", 0), sgs_model=c.get("sgs", 1), filter_ratio=c.get("filter_ratio", 1.0),
                               riemann=c.get("riemann", 0))
        if c.get("side_bc"):
            meta["physics"].update(bdy=bdy, R_ref=par.get("R_ref", 1.0))
        meta["pins"] = pins
        meta["seed"] = 12345
        np.savez_compressed(os.path.join(HERE, c["name"] + ".npz"), meta=json.dumps(meta),
                            **{k: np.asfortranarray(v) for k, v in fx.items()})
        summary[c["name"]] = pins
        print(c["name"], json.dumps({k: "%.2e" % v for k, v in pins.items()}))

    # the regression known-answer test of the reference, re-evaluated by the oracle
    ph = O.tgv_kat_physics()
    m = O.Mesh.box(3, 3, (15, 15, 15), (0, 0, 0), (2 * np.pi,) * 3, vcjh_scheme=2)
    u0 = O.ic_tgv(m.geometry()["pos_upts"], p0=100.0)
    _, _, nrm = m.rk45(ph, u0, 1e-3, 25)
    kat = {
        "source": "testcases/regression_tests.py:300-310 (tgv.test_vals, tol 1e-5, iter 25)",
        "config": "15^3 periodic hex on [0,2pi]^3, P=3 Gauss points, SD correction (vcjh_scheme_hexa 2), "
                  "Rusanov + LDG (tau 1, pen_fact 0.5), RK45, dt 1e-3, Mach 0.08, Re 1600, Pr 0.72, "
                  "IC ic_form 7 (p0 = 100)",
        "test_iter": 25,
        "test_vals": [0.00013215, 0.05076817, 0.05076814, 0.06456282, 0.07476870],
        "tol": 1e-5,
        "oracle_vals": [float(x) for x in nrm[:, -1]],
        "oracle_all_iters": nrm.T.tolist(),
    }
    with open(os.path.join(HERE, "kat_tgv.json"), "w") as f:
        json.dump(kat, f, indent=1)
    # the reference's tabulated 1-D point sets (data/loc_1d_gauss_pts.dat,
    # data/loc_1d_gauss_lobatto_pts.dat), parsed as C literals
    tables = {}
    for key, fn in (("gauss", "loc_1d_gauss_pts.dat"), ("gauss_lobatto", "loc_1d_gauss_lobatto_pts.dat")):
        txt = open(os.path.join(a.ref, "data", fn)).read()
        tab = {}
        for blk in re.finditer(r"get_order==(\d+)\)\s*\{([^}]*)\}", txt):
            vals = re.findall(r"\(\d+\)\s*=\s*([-+0-9.eE]+)\s*;", blk.group(2))
            tab[blk.group(1)] = [float(v) for v in vals]
        tables[key] = tab
    with open(os.path.join(HERE, "points_1d.json"), "w") as f:
        json.dump(tables, f, indent=1)
    mism = [(k, p) for k, tab in tables.items() for p, v in tab.items()
            if O.points_1d(int(p), 0 if k == "gauss" else 1).tolist() != v]
    with open(os.path.join(HERE, "summary.json"), "w") as f:
        json.dump({"pins": summary, "kat_oracle": kat["oracle_vals"], "points_1d_mismatches": mism}, f, indent=1)
    print("kat", kat["oracle_vals"], "point-table mismatches", mism)
    restart_read_fixture(a.ref, work)


if __name__ == "__main__":
    main()
