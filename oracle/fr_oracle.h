/* fr_oracle.h -- CPU restatement of the HiFiLES flux-reconstruction residual
 * and low-storage RK45 stage for quadrilateral and hexahedral elements.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker that the CUDA path is
 * compared against; it is never linked into, loaded by, or called from the
 * product library.  Only tests/, the smoke check and the CPU-baseline leg of
 * bench.py may load it.
 *
 * Array layouts follow the reference's array<T> (first index fastest,
 * include/array.h:287-309):
 *   u, div          (n_upts, n_eles, n_fields)
 *   *_fpts          (n_fpts, n_eles, n_fields)
 *   grad_*          (n_pts,  n_eles, n_fields, n_dims)
 *   detjac_upts     (n_upts, n_eles)
 *   JGinv_upts      (n_dims, n_dims, n_upts, n_eles)
 *   tdA_fpts        (n_fpts, n_eles)
 *   norm_fpts       (n_fpts, n_eles, n_dims)
 */
#ifndef FR_ORACLE_H
#define FR_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_mesh or_mesh;

typedef struct {
  int viscous;           /* 0 Euler, 1 Navier-Stokes                       */
  double gamma, prandtl; /* gas constants                                  */
  double mu_inf, rt_inf, c_sth, fix_vis; /* viscosity law (flux.cpp:326-330) */
  double tau, pen_fact;  /* LDG penalties (inters.cpp:550-678)             */
  int les;               /* 0 none, 1 eddy-viscosity LES (input key LES)   */
  int sgs_model;         /* 0 Smagorinsky, 1 WALE (input key SGS_model)    */
  double filter_ratio;   /* input key filter_ratio                         */
  const float* mlp;      /* sgs_model 5: parameters of the learned closure
                            (no reference counterpart; layout in mlp.py)    */
  int riemann;           /* riemann_solve_type: 0 Rusanov, 2 Roe (2-D only) */
  double bdy[14];        /* boundary parameters in bdy_inters::set_bdy_params
                            order (src/bdy_inters.cpp:78-110): rho_bound,
                            v_bound[3], p_bound, v_wall[3], T_wall,
                            p_total_bound, T_total_bound, n_free_stream[3]   */
  double R_ref;          /* gas constant in reference units                 */
} or_physics;

/* Generic conforming mesh of one element type (4-node quads or 8-node hexes,
 * vertices listed in tensor order: node m = a + 2 b (+ 4 c) sits at reference
 * coordinates (a, b, c) in {-1, +1}).  Periodic directions are matched with the
 * translation vectors shift[d] (0 = not periodic).  Faces that find no partner
 * are an error (no boundary conditions in this oracle).
 * upts_type: 0 Gauss, 1 Gauss-Lobatto.  vcjh_scheme: 0 user eta, 1 DG, 2 SD,
 * 3 Hu, 4 c_+.  Returns NULL on error (message on stderr). */
or_mesh* or_mesh_new(int dims, int order, int n_verts, const double* xv /* (n_verts, dims) row-major */,
                     int n_eles, const int* c2v /* (n_eles, 2^dims) row-major */,
                     const double* shift /* dims */, int upts_type, int vcjh_scheme, double eta);

/* Structured box [lo, hi] with n[d] elements per direction, periodic in every
 * direction; interior vertices optionally moved by a seeded uniform jitter of
 * +-jitter*h (a 64-bit LCG, so the same seed gives the same mesh everywhere). */
or_mesh* or_box_new(int dims, int order, const int* n, const double* lo, const double* hi,
                    double jitter, unsigned long long seed, int upts_type, int vcjh_scheme, double eta);

/* Variants with boundaries.  bctype (n_eles, 2*dims): reference boundary
 * type of each local face (src/geometry.cpp:121-148: 1 sub_in_simp,
 * 2 sub_out_simp, 3 sub_in_char, 4 sub_out_char, 5 sup_in, 6 sup_out,
 * 7 slip_wall, 11 isotherm_fix, 12 adiabat_fix, 13 isotherm_move,
 * 14 adiabat_move, 15 char, 16 slip_wall_dual), 0 = matched with another
 * face.  side_bc (2*dims): type of the box sides x-, x+, y-, y+, z-, z+;
 * 0 = periodic pair. */
or_mesh* or_mesh_new_bc(int dims, int order, int n_verts, const double* xv, int n_eles, const int* c2v,
                        const double* shift, const int* bctype, int upts_type, int vcjh_scheme, double eta);
or_mesh* or_box_new_bc(int dims, int order, const int* n, const double* lo, const double* hi, double jitter,
                       unsigned long long seed, const int* side_bc, int upts_type, int vcjh_scheme, double eta);
/* Number of boundary flux points; their flat indices (fpt + n_fpts*ele) and types. */
int or_n_boundary(const or_mesh* m);
void or_get_boundary(const or_mesh* m, int* fpt_idx, int* type);

void or_mesh_free(or_mesh* m);

/* n_eles, n_upts, n_fpts, n_fields(for Euler/NS), n_dims, n_interface_fpts */
void or_sizes(const or_mesh* m, int* out6);

/* Copies of the set-up arrays (layouts above).  pos arrays: (n_pts, n_eles, dims). */
void or_get_geometry(const or_mesh* m, double* pos_upts, double* detjac_upts, double* JGinv_upts,
                     double* tdA_fpts, double* norm_fpts, double* pos_fpts);
/* Interface wiring: for interface flux point i, left_idx[i] = fpt + n_fpts*ele of
 * the left side, right_idx[i] likewise. */
void or_get_interfaces(const or_mesh* m, int* left_idx, int* right_idx);
/* Replace metrics / wiring by externally supplied arrays (same layouts). */
void or_set_geometry(or_mesh* m, const double* detjac_upts, const double* JGinv_upts,
                     const double* tdA_fpts, const double* norm_fpts);
void or_set_interfaces(or_mesh* m, int n_int_fpts, const int* left_idx, const int* right_idx);

/* Dense operator matrices exactly as the reference builds them
 * (which: 0..6 = opp_0..opp_6, dim selects the component of opp_1/2/4/5).
 * Column-major, (rows, cols) returned through shape. */
int or_get_operator(const or_mesh* m, int which, int dim, double* out, int* shape2);

/* With les != 0 the stage arrays gain sgsf_upts (n_upts, n_eles, F, D) and
 * sgsf_fpts (n_fpts, n_eles, F, D) at offsets 7 and 8 (or_stage_offsets
 * then returns 10 offsets). */

/* One evaluation of CalcResidual (src/solver.cpp:65-225):
 * div_tconf_upts = full FR residual (before division by detjac).
 * stages (optional, may be NULL): receives intermediate arrays in this order
 *   disu_fpts, grad_disu_upts(corrected, physical), grad_disu_fpts,
 *   tdisf_upts(total), norm_tdisf_fpts, norm_tconf_fpts(total common flux),
 *   delta_disu_fpts
 * each at the offsets returned by or_stage_offsets. */
void or_residual(or_mesh* m, const or_physics* ph, const double* u, double* div, double* stages);
void or_stage_offsets(const or_mesh* m, long long* off10);

/* n_steps low-storage RK45 steps (src/eles.cpp:1091-1188), in place on u
 * (stage register reg must hold zeros on the first call).  If norms != NULL it
 * receives the L1 residual norm per field after every step (src/output.cpp:
 * 1452-1523 with res_norm_type 1: mean |div/detjac| over all points). */
void or_rk45(or_mesh* m, const or_physics* ph, double* u, double* reg, double dt, int n_steps,
             double* norms /* (n_fields, n_steps) */);

/* Sum over elements of sum_pts w_pt * |J| * q, for q = 0.5 rho |v|^2 (the
 * kinetic energy) using the tensor-product Gauss weights of the solution points. */
double or_kinetic_energy(const or_mesh* m, const double* u);

/* 1-D solution-point locations for (order, upts_type), as tabulated by the
 * reference to 15 decimals (data/loc_1d_gauss_pts.dat, loc_1d_gauss_lobatto_pts.dat). */
void or_points_1d(int order, int upts_type, double* out);

#ifdef __cplusplus
}
#endif
#endif
