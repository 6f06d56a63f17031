"""Input files for the reference executable built in oracle/_ref.

TEST INFRASTRUCTURE ONLY (the golden generator and bench.py's reference arm).
Writes, with no access to the reference's own source tree:
  * a periodic structured box as a Gambit neutral mesh, vertex for vertex the
    box of hifiles_b200.box_mesh / or_box_new (same seeded jitter), with node
    order chosen so the reference's local axes equal the physical axes;
  * a complete key/value input file for its reader (src/input.cpp:89-330).
"""
import numpy as np


def box_vertices(dims, n, lo, hi, jitter=0.0, seed=0):
    """Vertices (nv, dims) and tensor-ordered element->vertex map of the box."""
    nx, ny = n[0], n[1]
    nz = n[2] if dims == 3 else 1
    vx, vy, vz = nx + 1, ny + 1, (nz + 1 if dims == 3 else 1)
    mask = (1 << 64) - 1
    A, B = 6364136223846793005, 1442695040888963407
    s = (seed * A + B) & mask
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
                    s = (s * A + B) & mask
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


def write_gambit(path, dims, xv, c2v, n):
    """Gambit neutral file of a periodic box; every boundary face is listed in
    a "Cyclic" group.  The hex reader stores Gambit nodes 0..7 in shape slots
    (0,2,4,6,1,3,5,7) and the quad reader in (0,1,3,2)
    (src/geometry.cpp:1800-1843), so writing Gambit node g = ag + 2bg + 4cg as
    tensor node (a, b, c) = (cg, ag, bg) makes the reference's (xi, eta, zeta)
    the physical (x, y, z)."""
    ne = c2v.shape[0]
    out = ["        CONTROL INFO 2.3.16", "** GAMBIT NEUTRAL FILE", "box", "PROGRAM:  fixture", "",
           "     NUMNP     NELEM     NGRPS    NBSETS     NDFCD     NDFVL",
           "%10d%10d%10d%10d%10d%10d" % (xv.shape[0], ne, 1, 1, dims, dims),
           "ENDOFSECTION", "   NODAL COORDINATES 2.3.16"]
    for v in range(xv.shape[0]):
        out.append("%10d " % (v + 1) + " ".join("%.17e" % c for c in xv[v]))
    out += ["ENDOFSECTION", "      ELEMENTS/CELLS 2.3.16"]
    if dims == 3:
        order = [((g >> 2) & 1) + 2 * (g & 1) + 4 * ((g >> 1) & 1) for g in range(8)]
        for e in range(ne):
            nodes = [c2v[e, order[g]] + 1 for g in range(8)]
            out.append("%8d %2d %2d " % (e + 1, 4, 8) + " ".join("%8d" % x for x in nodes[:7]))
            out.append("               %8d" % nodes[7])
    else:
        for e in range(ne):
            nodes = [c2v[e, 0] + 1, c2v[e, 1] + 1, c2v[e, 3] + 1, c2v[e, 2] + 1]
            out.append("%8d %2d %2d " % (e + 1, 2, 4) + " ".join("%8d" % x for x in nodes))
    out += ["ENDOFSECTION", "       ELEMENT GROUP 2.3.16",
            "GROUP:          1 ELEMENTS: %10d MATERIAL:          2 NFLAGS:          1" % ne,
            "                           fluid", "       0"]
    ids = [str(e + 1) for e in range(ne)]
    for i in range(0, ne, 10):
        out.append(" ".join("%7s" % x for x in ids[i:i + 10]))
    out += ["ENDOFSECTION", " BOUNDARY CONDITIONS 2.3.16"]
    bnd = []
    nx, ny = n[0], n[1]
    nz = n[2] if dims == 3 else 1
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                e = i + nx * (j + ny * k) + 1
                if dims == 3:   # Gambit hex faces: x- 5, x+ 6, y- 4, y+ 2, z- 1, z+ 3
                    for cond, fc in ((i == 0, 5), (i == nx - 1, 6), (j == 0, 4), (j == ny - 1, 2),
                                     (k == 0, 1), (k == nz - 1, 3)):
                        if cond:
                            bnd.append((e, 4, fc))
                else:           # Gambit quad faces: y- 1, x+ 2, y+ 3, x- 4
                    for cond, fc in ((j == 0, 1), (i == nx - 1, 2), (j == ny - 1, 3), (i == 0, 4)):
                        if cond:
                            bnd.append((e, 2, fc))
    out.append("%32s%8d%8d%8d%8d" % ("Cyclic", 1, len(bnd), 0, 6))
    for b in bnd:
        out.append("%10d%5d%5d" % b)
    out.append("ENDOFSECTION")
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


def write_input(path, **over):
    """A complete input file for the reference's reader.  Defaults describe a
    viscous periodic case with Rusanov + LDG, RK45 and fixed viscosity."""
    v = dict(equation=0, viscous=1, riemann_solve_type=0, vis_riemann_solve_type=0, ic_form=1, test_case=0,
             order=3, dt_type=0, dt=1e-3, CFL=0.1, n_steps=1, adv_type=3, tau=1.0, pen_fact=0.5, restart_flag=0,
             mesh_file="mesh.neu", dx_cyclic=0.0, dy_cyclic=0.0, dz_cyclic=0.0, p_res=2, write_type=0,
             inters_cub_order=3, volume_cub_order=3, monitor_res_freq=100000, plot_freq=100000,
             data_file_name="run", restart_dump_freq=100000, res_norm_type=1, error_norm_type=1, res_norm_field=0,
             upts_type_tri=0, fpts_type_tri=0, vcjh_scheme_tri=0, c_tri=0.0, sparse_tri=0,
             upts_type_quad=0, vcjh_scheme_quad=1, eta_quad=0.0, sparse_quad=0,
             upts_type_hexa=0, vcjh_scheme_hexa=1, eta_hexa=0.0, sparse_hexa=0,
             upts_type_tet=1, fpts_type_tet=0, vcjh_scheme_tet=0, eta_tet=0.0, sparse_tet=0,
             upts_type_pri_tri=0, upts_type_pri_1d=0, vcjh_scheme_pri_1d=0, eta_pri=0.0, sparse_pri=0,
             gamma=1.4, prandtl=0.71, S_gas=120.0, T_gas=291.15, R_gas=286.9, mu_gas=1.827e-05, fix_vis=1,
             Mach_free_stream=0.1, nx_free_stream=0.0, ny_free_stream=0.0, nz_free_stream=0.0,
             Re_free_stream=1600.0, L_free_stream=1.0, T_free_stream=300.0, T_wall=300.0, rho_bound=1.0,
             u_bound=1.0, v_bound=0.0, w_bound=0.0, p_bound=1.0)
    v.update(over)
    with open(path, "w") as f:
        for k, x in v.items():
            f.write("%s %s\n" % (k, ("%.17g" % x) if isinstance(x, float) else x))
