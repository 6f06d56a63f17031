/* fr_b200.h -- C ABI of the B200 (sm_100a) flux-reconstruction residual and
 * low-storage RK45 stage.  Drop-in for the GPU seam of HiFiLES's per-element
 * operator path (the `#ifdef _GPU` bodies of class eles / int_inters and the
 * wrappers of include/cuda_kernels.h in the reference).
 *
 * Conventions
 *  - Every entry point returns fr_status; nothing calls exit().  The reference
 *    reports errors through FatalError/exit (include/error.h:20-22,
 *    include/array.h:461-473); here the caller decides.
 *  - Array layouts are the reference's array<T> layouts (first index fastest,
 *    include/array.h:287-309): states (n_upts, n_eles, n_fields), flux-point
 *    arrays (n_fpts, n_eles, n_fields), gradients (n_pts, n_eles, n_fields,
 *    n_dims), JGinv (n_dims, n_dims, n_upts, n_eles).  Point orderings inside
 *    an element are the reference's (src/eles_hexas.cpp:240-324,
 *    src/eles_quads.cpp:237-300), so reference arrays can be passed unchanged.
 *  - `stream` is a cudaStream_t passed as void*; NULL selects the solver's own
 *    non-blocking stream.  Device pointers are caller-owned unless stated
 *    otherwise.
 *  - One GPU, one rank: there is no MPI interface path.
 */
#ifndef FR_B200_H
#define FR_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  FR_OK = 0,
  FR_ERR_ARG = 1,         /* bad size, pointer or option                      */
  FR_ERR_CUDA = 2,        /* a CUDA runtime call failed (fr_last_error says)  */
  FR_ERR_NONFINITE = 3,   /* NaN/Inf or non-positive density/pressure found   */
  FR_ERR_TIMEOUT = 4,     /* a bounded device-side wait gave up               */
  FR_ERR_UNSUPPORTED = 5, /* element type / order / option not built          */
  FR_ERR_MESH = 6         /* mesh cannot be wired (unmatched face, bad map)   */
} fr_status;

const char* fr_status_string(fr_status s);
/* Message of the last failing call on this host thread ("" if none). */
const char* fr_last_error(void);

/* ------------------------------------------------------------------------
 * Solver object: mesh wiring, metrics and operators built once on the host
 * (replaces GeoPreprocess' set_transforms / set_opp_* / int_inters::set_interior,
 * src/geometry.cpp:151-990, src/eles.cpp:3620-4847, src/int_inters.cpp:95-178),
 * state resident in HBM, fused stage kernels.
 * ---------------------------------------------------------------------- */

typedef struct fr_solver fr_solver;

typedef struct {
  int dims;              /* 2: 4-node quadrilaterals, 3: 8-node hexahedra      */
  int n_verts;
  const double* xv;      /* (n_verts, dims) row-major vertex coordinates       */
  int n_eles;
  const int* c2v;        /* (n_eles, 2^dims) row-major; vertex m = a + 2b + 4c
                            sits at reference corner (a, b, c) in {0,1}^dims    */
  double shift[3];       /* periodic translation per axis (dx/dy/dz_cyclic of
                            the reference input), 0 = not periodic             */
  const int* bctype;     /* (n_eles, 2*dims) boundary type of each local
                            face in the reference's face numbering (quads:
                            y- 0, x+ 1, y+ 2, x- 3; hexes: z- 0, y- 1, x+ 2,
                            y+ 3, x- 4, z+ 5), get_bc_number codes
                            (src/geometry.cpp:121-148): 1 sub_in_simp,
                            2 sub_out_simp, 3 sub_in_char, 4 sub_out_char,
                            5 sup_in, 6 sup_out, 7 slip_wall, 11 isotherm_fix,
                            12 adiabat_fix, 13 isotherm_move, 14 adiabat_move,
                            15 char, 16 slip_wall_dual; 0 = matched with
                            another face.  NULL: every face is matched.       */
} fr_mesh_desc;

typedef struct {
  int order;             /* polynomial order P (quads 1..5, hexes 1..4)        */
  int upts_type;         /* upts_type_quad/hexa: 0 Gauss (the only points the
                            solver object takes; 1, Gauss-Lobatto, returns
                            FR_ERR_UNSUPPORTED here and is accepted by
                            fr_line_operators)                                */
  int vcjh_scheme;       /* 0 VCJH with eta, 1 DG, 2 SD, 3 Hu, 4 c_+           */
  double eta;            /* used when vcjh_scheme == 0                         */
  int viscous;           /* 0 Euler, 1 Navier-Stokes                           */
  int riemann;           /* riemann_solve_type: 0 Rusanov; 2 Roe (2-D only, as
                            in the reference, src/inters.cpp:390-508)          */
  int precision;         /* 0 FP64 throughout; 1 FP32 traces/fluxes/operators
                            with FP64 state, RK register and reductions        */
  double gamma, prandtl, mu_inf, rt_inf, c_sth, fix_vis; /* gas + viscosity law */
  double tau, pen_fact;  /* LDG penalty parameters                             */
  int les;               /* 1 adds the eddy-viscosity SGS flux (input key LES;
                            viscous only; eles::calc_sgsf_upts,
                            src/eles.cpp:2456-2778); 0 none                    */
  int sgs_model;         /* with les: 0 Smagorinsky, 1 WALE (SGS_model), 5 the
                            learned closure below; the filter-based models
                            2-4 are not built                                 */
  double filter_ratio;   /* with les: filter width over the point spacing     */
  double bdy[14];        /* boundary values in bdy_inters::set_bdy_params
                            order (src/bdy_inters.cpp:78-110): rho_bound,
                            v_bound[3], p_bound, v_wall[3], T_wall,
                            p_total_bound, T_total_bound, n_free_stream[3]   */
  double R_ref;          /* gas constant in reference units (isothermal walls,
                            characteristic inflow)                            */
} fr_scheme_desc;

fr_status fr_solver_create(const fr_mesh_desc* mesh, const fr_scheme_desc* scheme, int device,
                           fr_solver** out);
fr_status fr_solver_destroy(fr_solver* s);

/* n_eles, n_upts_per_ele, n_fpts_per_ele, n_fields, n_dims, n_interface_fpts */
fr_status fr_solver_sizes(const fr_solver* s, int out6[6]);

/* Host copies of the set-up arrays (NULL entries are skipped). */
fr_status fr_solver_get_geometry(const fr_solver* s, double* pos_upts, double* detjac_upts,
                                 double* JGinv_upts, double* tdA_fpts, double* norm_fpts);
/* Left/right element flux point (fpt + n_fpts*ele) of every interface flux point. */
fr_status fr_solver_get_interfaces(const fr_solver* s, int* left_idx, int* right_idx);
/* Replace the metrics by caller-built arrays (e.g. the reference's own). */
fr_status fr_solver_set_geometry(fr_solver* s, const double* detjac_upts, const double* JGinv_upts,
                                 const double* tdA_fpts, const double* norm_fpts);

/* State transfer (disu_upts(0)), host memory, layout (n_upts, n_eles, n_fields).
 * set_state zeroes the RK register (disu_upts(1)), like InitSolution. */
fr_status fr_solver_set_state(fr_solver* s, const double* host_u, void* stream);

/* Asynchronous state upload for pipelined hosts: validates the densities
 * (as fr_solver_set_state), then copies host_u -- pinned host memory that
 * must stay unchanged until the copy is done -- into a device staging buffer
 * on the solver's copy stream, overlapping steps already queued.  The next
 * fr_solver_advance / fr_solver_advance_async takes it as the current state
 * (traces rebuilt in the same pass) in stream order; the RK register is not
 * cleared, since the first stage of the next step writes it without reading
 * it.  One state can be staged at a time (FR_ERR_ARG otherwise).  No
 * counterpart in the reference. */
fr_status fr_solver_set_state_async(fr_solver* s, const double* host_u);
fr_status fr_solver_get_state(fr_solver* s, double* host_u, void* stream);
/* Device pointers of the resident state and RK register (owned by the solver). */
fr_status fr_solver_state_ptrs(fr_solver* s, double** d_u, double** d_reg);
/* Re-derive the flux-point traces after the caller wrote the state in place. */
fr_status fr_solver_state_updated(fr_solver* s, void* stream);

/* One CalcResidual (src/solver.cpp:65-225): div_tconf_upts(0) to host memory
 * (layout (n_upts, n_eles, n_fields)); the state is not advanced. */
fr_status fr_solver_residual(fr_solver* s, double* host_div, void* stream);

/* RK45 stage `stage` (0..4) of eles::AdvanceSolution (src/eles.cpp:1091-1188)
 * preceded by its residual evaluation: the body of the reference's
 * HiFiLES.cpp:159-183 loop for one stage. */
fr_status fr_solver_rk_stage(fr_solver* s, int stage, double dt, void* stream);

/* n_steps full RK45 steps.  If norms_host != NULL it receives the L1 residual
 * norms per field of the last stage of the last step (CalcNormResidual,
 * src/output.cpp:1452-1523, res_norm_type 1).  Graph-replayed after the first
 * call with the same dt. */
fr_status fr_solver_advance(fr_solver* s, int n_steps, double dt, double* norms_host, void* stream);

/* fr_solver_advance without waiting: the norms (if requested) are copied to
 * norms_host asynchronously -- valid, and not yet checked for NaN/Inf, once
 * the stream is synchronised (fr_solver_sync). */
fr_status fr_solver_advance_async(fr_solver* s, int n_steps, double dt, double* norms_host, void* stream);

/* Volume integral of 0.5 rho |v|^2 on the solver's volume cubature (the
 * "kineticenergy" integral quantity of eles::CalcIntegralQuantities,
 * src/eles.cpp:6503-6641), FP64. */
fr_status fr_solver_kinetic_energy(fr_solver* s, double* out_host, void* stream);

/* The volume cubature of the integral diagnostics.  By default it is the
 * reference's default rule (volume_cub_order 3: the tensor Gauss-Legendre rule
 * of 3 points per direction) in full double precision; the reference's
 * data/cubature_{quad,hexa}.dat print these rules to 12-15 significant
 * digits.  fr_solver_set_volume_cubature takes any rule instead, e.g. the
 * reference's own table (bit for bit) or another volume_cub_order
 * (eles_quads / eles_hexas::set_volume_cubpts, src/eles_hexas.cpp:418-440):
 * loc (dims, n_cub) with the point index slowest, points in [-1, 1]^dims.
 * fr_volume_cubature writes the tensor Gauss-Legendre rule of `rule` points per
 * direction in the reference's point order (quads: first coordinate fastest;
 * hexes: first coordinate slowest), full double precision, and returns its point count (0: rule
 * outside 1..12); loc or weights may be null to query the count. */
fr_status fr_solver_set_volume_cubature(fr_solver* s, int n_cub, const double* loc, const double* weights);
int fr_volume_cubature(int dims, int rule, double* loc, double* weights);

/* Kernel launches issued by the solver since creation (for launch accounting). */
long long fr_solver_launch_count(const fr_solver* s);

/* The solver's own non-blocking stream (cudaStream_t), used whenever an entry
 * point is given stream == NULL; and a synchronisation of that stream. */
void* fr_solver_stream(fr_solver* s);
fr_status fr_solver_sync(fr_solver* s);

/* Autotuner: times every compiled tile variant (elements per CTA, threads per
 * CTA) of the gradient and update kernels on this solver's mesh, `reps`
 * launches each, keeps the fastest, and returns the choice as
 * {grad elements, grad threads, update elements, update threads}.  The state
 * is not changed.  Results do not depend on the tiles except for the
 * summation order of the residual norms. */
fr_status fr_solver_autotune(fr_solver* s, int reps, int out4[4]);

/* The compiled tile variants by index, as the autotuner walks them:
 * fr_solver_tile_count returns {gradient variants, update variants};
 * fr_solver_tile_info returns {elements, threads, CTAs per SM the registers
 * are sized for, persistent} of gradient variant i (kind 0) or update variant
 * i (kind 1); fr_solver_select_tiles makes variants g and u the ones used.
 * Results do not depend on the choice (except the summation order of the
 * residual norms). */
fr_status fr_solver_tile_count(const fr_solver* s, int out2[2]);
fr_status fr_solver_tile_info(const fr_solver* s, int kind, int i, int out4[4]);
fr_status fr_solver_select_tiles(fr_solver* s, int g, int u);

/* Runs `reps` RK stages one by one (advancing the state) and returns in ms3
 * the mean CUDA-event duration, on the solver's stream, of the three stage
 * kernels: gradient/flux (0 for inviscid runs), interface fluxes, and
 * correction + update.  For roofline accounting. */
fr_status fr_solver_profile_stage(fr_solver* s, int reps, double dt, double* ms3);

/* Corrected physical gradient of the current state, grad_disu_upts after
 * eles::correct_gradient (src/eles.cpp:1770-1968), to host memory in the
 * layout (n_upts, n_eles, n_fields, n_dims).  Viscous solvers only. */
fr_status fr_solver_gradient(fr_solver* s, double* host_grad, void* stream);

/* Integral diagnostics of the current state on the device, the quantities of
 * eles::CalcIntegralQuantities (src/eles.cpp:6503-6641): out5 = kinetic
 * energy, enstrophy (rho |curl u|^2 / 2, the reference's "vorticity"),
 * pressure dilatation, strain colon product, deviatoric strain colon
 * product.  As in the reference, the state and its corrected gradient are
 * interpolated to the volume cubature points (opp_volume_cubpts) and
 * integrated with the rule's weights times the Jacobian there.  Viscous
 * solvers only (the corrected gradient comes from the gradient kernel). */
fr_status fr_solver_integral_quantities(fr_solver* s, double out5[5], void* stream);

/* ------------------------------------------------------------------------
 * Batches of independent meshes (no reference counterpart: the reference
 * runs one mesh per process).  Instances with the same dims and scheme form a
 * group whose meshes are merged (each keeps its own periodic wiring), so a
 * group advances with one launch per stage kernel; fr_batch_advance runs a
 * whole RK45 step of every group as one CUDA graph.  All instances share dt.
 * ---------------------------------------------------------------------- */
typedef struct fr_batch fr_batch;
fr_status fr_batch_create(const fr_mesh_desc* meshes, const fr_scheme_desc* schemes, int n_instances, int device,
                          fr_batch** out);
fr_status fr_batch_destroy(fr_batch* b);
int fr_batch_n_groups(const fr_batch* b);
/* The solver object of group g (owned by the batch; for queries, autotuning,
 * kinetic energy of the whole group). */
fr_status fr_batch_group(fr_batch* b, int g, fr_solver** out);
/* group, first element in the group, n_eles, n_upts of instance i */
fr_status fr_batch_instance(const fr_batch* b, int i, int out4[4]);
/* State of one instance, host memory (n_upts, n_eles_i, n_fields); setting
 * it zeroes its RK register. */
fr_status fr_batch_set_state(fr_batch* b, int i, const double* host_u);
fr_status fr_batch_get_state(fr_batch* b, int i, double* host_u);
/* Picks every group's tiles (fr_solver_autotune), then times `reps` whole
 * steps run group by group against the merged launches below (registers
 * capped for 4 and for 3 CTAs per SM) from the same state, keeps the fastest
 * and restores the state. */
fr_status fr_batch_autotune(fr_batch* b, int reps);
/* Merged launches: each stage kernel (gradient, interface flux where an order
 * needs it, update) runs once for all groups, its grid the groups' element
 * blocks one after the other, each block running its group's order.  For
 * batches of hexahedral Navier-Stokes groups (Rusanov, no LES, one precision)
 * of orders 2, 3 and 4, at most one group per order; FR_ERR_UNSUPPORTED
 * otherwise.  on 0 returns to one launch per group and stage kernel; minb
 * (1, 3 or 4) caps the merged kernels' registers for that many CTAs per SM.
 * fr_batch_merged returns the cap in use, 0 when not merged. */
fr_status fr_batch_set_merged(fr_batch* b, int on, int minb);
int fr_batch_merged(const fr_batch* b);
fr_status fr_batch_advance(fr_batch* b, int n_steps, double dt, void* stream);
long long fr_batch_launch_count(const fr_batch* b);
void* fr_batch_stream(fr_batch* b);

/* ------------------------------------------------------------------------
 * Restart files in the reference's text format (write_restart,
 * src/output.cpp:1057-1107; read_restart, src/solver.cpp:390-445).  Host
 * memory only; no GPU is touched by fr_restart_*.
 * ---------------------------------------------------------------------- */
typedef struct {
  int ele_type;            /* reference codes: 0 triangles, 1 quads, 2 tets,
                              3 prisms, 4 hexes                                 */
  int order;               /* polynomial order of the block                    */
  int n_upts, n_eles, n_fields;
  const double* loc_1d;    /* quads, hexes: order + 1 solution-point locations
                              in 1-D                                          */
  const int* ele2global;   /* global element ids (NULL: 0 .. n_eles-1)         */
  const double* disu_upts; /* (n_upts, n_eles, n_fields)                       */
  const double* loc_pts;   /* triangles, tets, prisms: the solution points,
                              (n_upts, dims) point-major as
                              fr_element_operators gives them                  */
} fr_restart_block;

/* Writes a restart file exactly as the reference does (%.15g numbers,
 * each type's write_restart_info, src/eles_tris.cpp:546-563,
 * src/eles_tets.cpp:782-800, src/eles_pris.cpp:700-726,
 * src/eles_hexas.cpp:882-900, and eles::write_restart_data,
 * src/eles.cpp:697-722): element types in the order of their codes, at most
 * one block per type; blocks with no elements are left out. */
fr_status fr_restart_write(const char* path, double time, const fr_restart_block* blocks, int n_blocks);
/* Reads the quad (1) or hex (4) block into disu_upts (n_upts, n_eles,
 * n_fields) of a solver of the given order and point family, interpolating
 * from the file's order when it differs (eles::set_opp_r,
 * src/eles.cpp:4135-4153).  Elements are matched by global id; every
 * element must be present.  time_out may be NULL. */
fr_status fr_restart_read(const char* path, int ele_type, int order, int upts_type, int n_eles, int n_fields,
                          const int* ele2global, double* disu_upts, double* time_out);
/* The same for any element type (read_restart_info of src/eles_tris.cpp:511,
 * src/eles_tets.cpp:749, src/eles_pris.cpp:655): the file's block carried
 * to the solution points loc_pts ((n_upts, dims) point-major) through the
 * nodal basis on the file's points; points equal to the file's to 1e-13 take
 * the file's values as they are. */
fr_status fr_restart_read_points(const char* path, int ele_type, int n_upts, const double* loc_pts, int n_eles,
                                 int n_fields, const int* ele2global, double* disu_upts, double* time_out);
/* A solution as a VTK unstructured grid (.vtu, inline base64 binary), the
 * role of the reference's Paraview output (src/output.cpp:580-1055): points
 * are the solution points (pos_upts, (n_upts, n_eles, dims)), each element is
 * cut into order^dims sub-cells joining neighbouring points, point data
 * Density, Velocity, Pressure, Energy (float32).  Host memory only. */
fr_status fr_vtu_write(const char* path, int dims, int order, int n_eles, const double* pos_upts,
                       const double* disu_upts, double gamma);
/* The solver's current state as such a file (one device-to-host copy). */
fr_status fr_solver_write_vtu(fr_solver* s, const char* path);
/* One element type of a mixed mesh for fr_vtu_write_mixed. */
typedef struct {
  int ele_type;            /* 0 triangles, 1 quads, 2 tets, 3 prisms, 4 hexes   */
  int n_eles;
  const double* loc_pts;   /* triangles, tets, prisms: the solution points,
                              (n_upts, dims) point-major as
                              fr_element_operators gives them                  */
  const double* pos_upts;  /* (n_upts, n_eles, dims)                           */
  const double* disu_upts; /* (n_upts, n_eles, dims + 2)                       */
} fr_vtu_block;
/* A mixed mesh's solution as one .vtu file (all blocks of one dimension).
 * Quads and hexes as fr_vtu_write; triangles, tets and prisms interpolated
 * through their nodal basis to the equispaced lattice of order `order` (the
 * reference's plot points, eles::set_opp_p) and cut into order^dims
 * triangles, tetrahedra or wedges.  Host memory only. */
fr_status fr_vtu_write_mixed(const char* path, int order, const fr_vtu_block* blocks, int n_blocks, double gamma);

/* The solver's state to / from a restart file (global ids 0 .. n_eles-1). */
fr_status fr_solver_write_restart(fr_solver* s, const char* path, double time);
fr_status fr_solver_read_restart(fr_solver* s, const char* path, double* time_out);

/* ------------------------------------------------------------------------
 * Learned SGS closure (sgs_model 5).  No counterpart in the reference, whose
 * eddy-viscosity models are Smagorinsky and WALE (eles::calc_sgsf_upts,
 * src/eles.cpp:2456-2778); it uses the same flux with
 * mu_t = rho Delta^2 |S| c, where c >= 0 comes from a 6-64-64-1 perceptron
 * (tanh, tanh, softplus; FP32) of five invariants of the resolved velocity
 * gradient and log Delta.  Parameter vector: W1[64][6], b1[64], W2[64][64],
 * b2[64], w3[64], b3 (trained), then xmean[6], xscale[6] (input
 * normalisation (x - xmean) * xscale).
 * ---------------------------------------------------------------------- */
int fr_mlp_n_params(void);       /* 4685 floats in all */
int fr_mlp_n_trained(void);      /* 4673 trained ones (the leading part) */

/* Closure inputs at every solution point of the current state, host memory
 * (n_upts * n_eles, 6) floats, point index upt + n_upts * ele. */
fr_status fr_solver_sgs_features(fr_solver* s, float* host_x, void* stream);
/* Copies a parameter vector into a solver created with les = 1,
 * sgs_model = 5 (such a solver starts with the closure off, c ~ 2e-9). */
fr_status fr_solver_set_sgs_mlp(fr_solver* s, const float* host_w);

/* Training kernels on device arrays: x (n, 6), c* = y (n), sample weights
 * sw (n, or NULL for all ones), w, grad, m, v (fr_mlp_n_params() /
 * fr_mlp_n_trained() floats).  loss_grad gives the gradient of
 * (1/n) sum sw (c(x) - y)^2 over the trained parameters and the loss; it
 * needs fr_mlp_scratch_floats(n) floats of caller scratch and is
 * deterministic.  adam applies one Adam step (beta 0.9 / 0.999, eps 1e-8;
 * step counts from 1). */
long long fr_mlp_scratch_floats(long long n);
fr_status fr_mlp_forward(const float* d_w, const float* d_x, long long n, float* d_out, void* stream);
fr_status fr_mlp_loss_grad(const float* d_w, const float* d_x, const float* d_y, const float* d_sw, long long n,
                           float* d_grad, float* d_loss, float* d_scratch, long long scratch_floats, void* stream);
fr_status fr_mlp_adam(float* d_w, const float* d_grad, float* d_m, float* d_v, int step, float lr, void* stream);

/* ------------------------------------------------------------------------
 * Host-only set-up queries (no GPU is touched).
 * ---------------------------------------------------------------------- */

/* Wiring and metrics exactly as fr_solver_create builds them.  Call with NULL
 * arrays first to get the sizes (out6 as in fr_solver_sizes). */
fr_status fr_mesh_geometry(const fr_mesh_desc* mesh, const fr_scheme_desc* scheme, int out6[6],
                           double* pos_upts, double* detjac_upts, double* JGinv_upts, double* tdA_fpts,
                           double* norm_fpts, int* left_idx, int* right_idx);

/* The 1-D factors of the tensor-product operators for (order, upts_type,
 * vcjh_scheme, eta), packed as: loc[n], l_m(-1)[n], l_m(+1)[n], D[n][n]
 * (D[k][m] = l_m'(xi_k)), g_L'(xi_k)[n], g_R'(xi_k)[n], weights[n], eta;
 * n = order + 1, i.e. n*n + 6n + 1 doubles.  Every non-zero of the reference's
 * opp_0..opp_6 for quads / hexes (src/eles.cpp:3620-4052) is one of these. */
fr_status fr_line_operators(int order, int upts_type, int vcjh_scheme, double eta, double* out);

/* ------------------------------------------------------------------------
 * Per-operator entry points: the reference's GPU seam one method at a time,
 * on caller-owned device arrays in the reference's layouts.  Operators are
 * the caller's dense matrices (any element type, column-major, as built by
 * set_opp_0..6, src/eles.cpp:3620-4052); interface data come through device
 * tables of device pointers laid out like int_inters' arrays
 * (src/int_inters.cpp:95-178).  Each call enqueues on `stream` and returns;
 * nothing synchronises the device.
 * ---------------------------------------------------------------------- */

typedef struct {
  double gamma, prandtl, mu_inf, rt_inf, c_sth, fix_vis, tau, pen_fact;
} fr_phys_desc;

/* eles::extrapolate_solution, include/eles.h:109 (GPU body src/eles.cpp:1310-1314,
 * cublasDgemm on opp_0): disu_fpts = opp_0 * disu_upts. */
fr_status fr_op_extrapolate_solution(int n_fpts, int n_upts, int n_fields, int n_eles, const double* opp_0,
                                     const double* disu_upts, double* disu_fpts, void* stream);

/* eles::evaluate_invFlux, include/eles.h:115; replaces
 * evaluate_invFlux_gpu_kernel_wrapper, include/cuda_kernels.h:35 (static mesh). */
fr_status fr_op_evaluate_invFlux(int n_upts, int n_dims, int n_fields, int n_eles, const double* disu_upts,
                                 const double* JGinv_upts, double* tdisf_upts, const fr_phys_desc* phys,
                                 void* stream);

/* eles::calculate_gradient, include/eles.h:130 (cublasDgemm on opp_4[d]);
 * opp_4 is a host array of n_dims device pointers. */
fr_status fr_op_calculate_gradient(int n_upts, int n_dims, int n_fields, int n_eles, const double* const* opp_4,
                                   const double* disu_upts, double* grad_disu_upts, void* stream);

/* eles::correct_gradient, include/eles.h:133: grad += opp_5[d] * delta_disu_fpts,
 * then the transform of transform_grad_disu_upts_kernel_wrapper,
 * include/cuda_kernels.h:45. */
fr_status fr_op_correct_gradient(int n_upts, int n_fpts, int n_dims, int n_fields, int n_eles,
                                 const double* const* opp_5, const double* delta_disu_fpts, const double* JGinv_upts,
                                 const double* detjac_upts, double* grad_disu_upts, void* stream);

/* eles::extrapolate_corrected_gradient, include/eles.h:136 (cublasDgemm on opp_6 per dimension). */
fr_status fr_op_extrapolate_corrected_gradient(int n_fpts, int n_upts, int n_dims, int n_fields, int n_eles,
                                               const double* opp_6, const double* grad_disu_upts,
                                               double* grad_disu_fpts, void* stream);

/* eles::evaluate_viscFlux, include/eles.h:142; replaces
 * evaluate_viscFlux_gpu_kernel_wrapper, include/cuda_kernels.h:48 (no LES,
 * no wall model, no turbulence model): tdisf_upts += JGinv * F_visc. */
fr_status fr_op_evaluate_viscFlux(int n_upts, int n_dims, int n_fields, int n_eles, const double* disu_upts,
                                  const double* grad_disu_upts, const double* JGinv_upts, double* tdisf_upts,
                                  const fr_phys_desc* phys, void* stream);

/* eles::evaluate_viscFlux with LES (eddy-viscosity SGS models), include/eles.h:142,
 * src/eles.cpp:2321-2409 (the CPU path's form; its GPU wrapper
 * evaluate_viscFlux_gpu_kernel_wrapper, include/cuda_kernels.h:48, has the
 * same arguments plus sgsf_upts): tdisf_upts += JGinv (F_visc + F_sgs) and
 * sgsf_upts (n_upts, n_eles, n_fields, n_dims) = JGinv F_sgs.  sgs_model 0
 * Smagorinsky, 1 WALE (src/eles.cpp:2456-2778); the filter width uses detJ
 * and order as calc_sgsf_upts does. */
fr_status fr_op_evaluate_viscFlux_les(int n_upts, int n_dims, int n_fields, int n_eles, const double* disu_upts,
                                      const double* grad_disu_upts, const double* JGinv_upts,
                                      const double* detjac_upts, double* tdisf_upts, double* sgsf_upts,
                                      const fr_phys_desc* phys, int sgs_model, double filter_ratio, int order,
                                      void* stream);

/* eles::evaluate_sgsFlux, include/eles.h:124 (src/eles.cpp:3294-3368, cublasDgemm
 * on opp_0 per dimension): sgsf_fpts[.., d] = opp_0 * sgsf_upts[.., d]. */
fr_status fr_op_evaluate_sgsFlux(int n_fpts, int n_upts, int n_dims, int n_fields, int n_eles, const double* opp_0,
                                 const double* sgsf_upts, double* sgsf_fpts, void* stream);

/* int_inters::calculate_common_viscFlux with LES, include/int_inters.h:64
 * (src/int_inters.cpp:359-470): as fr_op_int_inters_common_viscFlux, each
 * side's SGS flux at the flux point (tables sgsf_fpts_l/_r shaped like
 * grad_disu_fpts_l/_r) added to its viscous flux before the LDG flux. */
fr_status fr_op_int_inters_common_viscFlux_les(int n_fpts_per_inter, int n_dims, int n_fields, int n_inters,
                                               double* const* disu_fpts_l, double* const* disu_fpts_r,
                                               double* const* grad_disu_fpts_l, double* const* grad_disu_fpts_r,
                                               double* const* norm_tconf_fpts_l, double* const* norm_tconf_fpts_r,
                                               double* const* tdA_fpts_l, double* const* tdA_fpts_r,
                                               double* const* norm_fpts, double* const* sgsf_fpts_l,
                                               double* const* sgsf_fpts_r, const fr_phys_desc* phys, void* stream);

/* eles::extrapolate_totalFlux, include/eles.h:121: norm_tdisf_fpts = sum_d opp_1[d] * tdisf_upts[d]. */
fr_status fr_op_extrapolate_totalFlux(int n_fpts, int n_upts, int n_dims, int n_fields, int n_eles,
                                      const double* const* opp_1, const double* tdisf_upts, double* norm_tdisf_fpts,
                                      void* stream);

/* eles::calculate_divergence, include/eles.h:118: div = sum_d opp_2[d] * tdisf_upts[d]. */
fr_status fr_op_calculate_divergence(int n_upts, int n_dims, int n_fields, int n_eles, const double* const* opp_2,
                                     const double* tdisf_upts, double* div_tconf_upts, void* stream);

/* eles::calculate_corrected_divergence, include/eles.h:127 (cublasDaxpy +
 * cublasDgemm on opp_3): norm_tconf -= norm_tdisf; div += opp_3 * norm_tconf. */
fr_status fr_op_calculate_corrected_divergence(int n_upts, int n_fpts, int n_fields, int n_eles, const double* opp_3,
                                               const double* norm_tdisf_fpts, double* norm_tconf_fpts,
                                               double* div_tconf_upts, void* stream);

/* int_inters::calculate_common_invFlux, include/int_inters.h:61; replaces
 * calculate_common_invFlux_gpu_kernel_wrapper, include/cuda_kernels.h:39
 * (static mesh): riemann_solve_type 0 Rusanov or 2 Roe (2-D, as the
 * reference); with viscous != 0 also the LDG common solution into
 * delta_disu_fpts_l/_r. */
fr_status fr_op_int_inters_common_invFlux(int n_fpts_per_inter, int n_dims, int n_fields, int n_inters,
                                          double* const* disu_fpts_l, double* const* disu_fpts_r,
                                          double* const* norm_tconf_fpts_l, double* const* norm_tconf_fpts_r,
                                          double* const* tdA_fpts_l, double* const* tdA_fpts_r,
                                          double* const* norm_fpts, double* const* delta_disu_fpts_l,
                                          double* const* delta_disu_fpts_r, const fr_phys_desc* phys,
                                          int riemann_solve_type, int viscous, void* stream);

/* int_inters::calculate_common_viscFlux, include/int_inters.h:64; replaces
 * calculate_common_viscFlux_gpu_kernel_wrapper, include/cuda_kernels.h:56
 * (LDG, no LES): norm_tconf_fpts_l/_r += +/- f_n * tdA. */
fr_status fr_op_int_inters_common_viscFlux(int n_fpts_per_inter, int n_dims, int n_fields, int n_inters,
                                           double* const* disu_fpts_l, double* const* disu_fpts_r,
                                           double* const* grad_disu_fpts_l, double* const* grad_disu_fpts_r,
                                           double* const* norm_tconf_fpts_l, double* const* norm_tconf_fpts_r,
                                           double* const* tdA_fpts_l, double* const* tdA_fpts_r,
                                           double* const* norm_fpts, const fr_phys_desc* phys, void* stream);

/* bdy_inters::evaluate_boundaryConditions_invFlux, include/bdy_inters.h:70;
 * replaces evaluate_boundaryConditions_invFlux_gpu_kernel_wrapper,
 * include/cuda_kernels.h:42 (static mesh, Euler/Navier-Stokes).  Tables as
 * bdy_inters keeps them (src/bdy_inters.cpp:111-203): (n_fpts_per_inter,
 * n_inters, n_fields) / (.., n_dims) device arrays of device pointers into the
 * owning elements' flux-point arrays; boundary_type (n_inters) and the 14
 * bdy_params of bdy_inters::set_bdy_params are device arrays.  Boundary types
 * 1-7 and 11-16 (get_bc_number, src/geometry.cpp:121-148); riemann_solve_type
 * 0 (central flux of own and ghost state) or 2 (Roe, 2-D).  Writes
 * norm_tconf_fpts_l = f_n tdA and, with viscous != 0, the LDG common solution
 * into delta_disu_fpts_l. */
fr_status fr_op_bdy_inters_common_invFlux(int n_fpts_per_inter, int n_dims, int n_fields, int n_inters,
                                          double* const* disu_fpts_l, double* const* norm_tconf_fpts_l,
                                          double* const* tdA_fpts_l, double* const* norm_fpts,
                                          const int* boundary_type, const double* bdy_params,
                                          double* const* delta_disu_fpts_l, const fr_phys_desc* phys, double R_ref,
                                          int riemann_solve_type, int viscous, void* stream);

/* bdy_inters::evaluate_boundaryConditions_viscFlux, include/bdy_inters.h:76;
 * replaces evaluate_boundaryConditions_viscFlux_gpu_kernel_wrapper,
 * include/cuda_kernels.h:59 (no LES, no turbulence model):
 * norm_tconf_fpts_l += (f_v + tau n (u_l - u_ghost)) . n tdA. */
fr_status fr_op_bdy_inters_common_viscFlux(int n_fpts_per_inter, int n_dims, int n_fields, int n_inters,
                                           double* const* disu_fpts_l, double* const* grad_disu_fpts_l,
                                           double* const* norm_tconf_fpts_l, double* const* tdA_fpts_l,
                                           double* const* norm_fpts, const int* boundary_type,
                                           const double* bdy_params, const fr_phys_desc* phys, double R_ref,
                                           void* stream);

/* The sparse operator product of the sparse_* options: replaces
 * bespoke_SPMV, include/cuda_kernels.h:81 (same arguments; cell_type and
 * order are accepted and unused).  The operator is m x n in the ELL layout of
 * array_to_ellpack (src/funcs.cpp:961-1011): nnz_per_row slots per row,
 * ell_data[i + m s] / ell_indices[i + m s]; b (n, n_eles, n_fields) and
 * c (m, n_eles, n_fields) in the state layouts; c = A b (add_flag 0) or
 * c += A b (add_flag 1).  m <= 256 and n <= ~850; entries whose column is
 * outside 0..n-1 are skipped. */
fr_status fr_op_spmv_ell(int m, int n, int n_fields, int n_eles, const double* ell_data, const int* ell_indices,
                         int nnz_per_row, const double* b, double* c, int cell_type, int order, int add_flag,
                         void* stream);

/* eles::AdvanceSolution(stage, adv_type 3), include/eles.h:157; replaces
 * RK45_update_kernel_wrapper, include/cuda_kernels.h:30 (fixed dt):
 * res = a_s res + dt (-div/detjac + const_src + src); u += b_s res.
 * src_upts may be NULL (zero source). */
fr_status fr_op_advance_rk45(int n_upts, int n_fields, int n_eles, int stage, double dt, double const_src,
                             double* disu_upts_0, double* disu_upts_1, const double* div_tconf_upts,
                             const double* detjac_upts, const double* src_upts, void* stream);

/* Precision of the operator products (opp_0 .. opp_6 applied to all
 * elements, the reference's cublasDgemm calls) of the fr_op_* entry points,
 * process-wide like the reference's run_input:
 *   0  FP64 (default; parity with the reference): operators of k >= 16
 *      columns on the FP64 tensor cores (mma.sync m8n8k4 f64), shorter ones
 *      and those whose 64-column operand tile exceeds shared memory on the
 *      CUDA cores; both forms accumulate each output as one chain of fused
 *      multiply-adds in k order, so they give the same bits,
 *   1  BF16x3: x = x0 + x1 + x2 in BF16, products x0y0 + x0y1 + x1y0 (about
 *      16 bits) on the tcgen05 tensor cores, FP32 accumulation, FP64 inputs
 *      and outputs; m x k operators with m <= 128 and k <= 288, or m <= 256
 *      and k <= 192 (hexes up to P = 4),
 *   2  BF16x6: the same plus x0y2 + x1y1 + x2y0 (about 24 bits); m <= 128
 *      and k <= 192, or m <= 256 and k <= 128 (hexes up to P = 4),
 *   3  FP64 on the CUDA cores;
 * larger operators return FR_ERR_UNSUPPORTED.
 * Pointwise kernels stay FP64.  fr_op_check synchronises the stream and
 * returns FR_ERR_TIMEOUT if a tensor-core product gave up waiting for its
 * MMAs since the last check. */
fr_status fr_op_set_gemm_precision(int mode);
int fr_op_gemm_precision(void);
/* Tensor-core BF16x3 products: on (default) loads each block's next column
 * tile into registers while the current tile's MMAs run (operators of up to
 * 64 columns with 64-column tiles, 128 with 32); off reads B at the split.
 * Both give identical results; the switch is for comparisons. */
fr_status fr_op_set_gemm_pipelining(int on);
fr_status fr_op_check(void* stream);

/* ------------------------------------------------------------------------
 * Host set-up of triangles, quadrilaterals, tetrahedra, prisms and hexahedra
 * for the per-operator path (host only, FP64, no GPU needed).
 *
 * What the reference's element classes compute before the time loop: point
 * sets, nodal bases and the dense operators (eles_tris / eles_quads /
 * eles_tets / eles_pris / eles_hexas::setup_ele_type_specific with
 * eles::set_opp_0 .. set_opp_6, src/eles.cpp:3620-4060,
 * src/eles_tris.cpp:66-648, src/eles_tets.cpp:68-1415,
 * src/eles_pris.cpp:51-1194), and for a mesh of those elements the metrics
 * (eles::set_transforms, src/eles.cpp:4557-4800) and the interface and
 * boundary tables (int_inters::set_interior, bdy_inters::set_boundary,
 * src/int_inters.cpp:95-178, src/bdy_inters.cpp:111-203).  Element types use
 * the reference's numbers.  Orders 1-5 (the reference's simplex point tables
 * end at 5); the SD-, HU-like and c+ simplex schemes exist for orders 2-5
 * (triangles 2-4), as in the reference.
 * ---------------------------------------------------------------------- */
enum { FR_ELE_TRI = 0, FR_ELE_QUAD = 1, FR_ELE_TET = 2, FR_ELE_PRISM = 3, FR_ELE_HEX = 4 };

typedef struct {
  int upts_type_tet;        /* 0 interior quadrature points, 1 alpha-optimised nodes      */
  int fpts_type_tet;        /* triangle flux points of tets: 0 interior, 1 alpha          */
  int vcjh_scheme_tet;      /* 0 user c_tet, 1 DG, 2 SD-like, 3 HU-like, 4 c+             */
  double c_tet;
  int upts_type_pri_tri;    /* prism triangle points: 0 interior, 1 alpha                 */
  int upts_type_pri_1d;     /* prism line points: 0 Gauss, 1 Gauss-Lobatto                */
  int vcjh_scheme_tri;      /* triangles and prisms' triangles, as vcjh_scheme_tet        */
  double c_tri;
  int vcjh_scheme_pri_1d;   /* prisms' line correction: 0 user eta_pri, 1 DG, 2 SD, 3 HU, 4 c+ */
  double eta_pri;
  int upts_type_hexa;       /* hexes: 0 Gauss, 1 Gauss-Lobatto                            */
  int vcjh_scheme_hexa;     /* as vcjh_scheme_pri_1d                                      */
  double eta_hexa;
  int upts_type_tri;        /* triangles: 0 interior, 1 alpha                             */
  int fpts_type_tri;        /* triangle edge points: 0 Gauss, 1 Gauss-Lobatto             */
  int upts_type_quad;       /* quads: 0 Gauss, 1 Gauss-Lobatto                            */
  int vcjh_scheme_quad;     /* as vcjh_scheme_pri_1d                                      */
  double eta_quad;
} fr_element_opts;

/* Sizes of one element type: solution and flux points, faces, flux points
 * of each face (n_fpts_per_face holds up to 6 entries).  NULL outputs are
 * skipped. */
fr_status fr_element_sizes(int ele_type, int order, int* n_upts, int* n_fpts, int* n_faces, int* n_fpts_per_face);

/* Point sets and dense operators of one element type in the reference's
 * layouts (first index fastest), D = 2 for triangles and quads, 3 otherwise:
 * loc_upts (D, n_upts), tloc_fpts and tnorm_fpts (D, n_fpts); opp_0
 * (n_fpts, n_upts); opp_1 (n_fpts, n_upts, D); opp_2 (n_upts, n_upts, D);
 * opp_3 (n_upts, n_fpts); opp_5 (n_upts, n_fpts, D).  The reference's opp_4
 * equals opp_2 and opp_6 equals opp_0.  opts NULL: every field 0 except
 * vcjh_scheme_hexa and vcjh_scheme_quad 1.  NULL outputs are skipped. */
fr_status fr_element_operators(int ele_type, int order, const fr_element_opts* opts, double* loc_upts,
                               double* tloc_fpts, double* tnorm_fpts, double* opp_0, double* opp_1, double* opp_2,
                               double* opp_3, double* opp_5);

/* A conforming mesh of one order: triangles and quads (dims 2) or tets,
 * prisms and hexes (dims 3).  xv (dims, n_verts); cell_type (n_cells)
 * element types; cell_verts (8, n_cells) vertex indices in the reference's
 * vertex order (tris 3; quads 4 in tensor order a + 2 b; tets 4; prisms 6;
 * hexes 8 in tensor order a + 2 b + 4 c; the rest of each column ignored);
 * period[dims] the periodic length of each axis (0: not periodic), NULL for
 * none; boundary faces (cell, local face, reference boundary type 1-7 or
 * 11-16).  Every other face must meet another face (directly or through a
 * periodic shift).  Elements of each type are numbered in cell order; the
 * element-type slots follow the type numbers (those present, at most three). */
typedef struct fr_mixed fr_mixed;
fr_status fr_mixed_create(int dims, int order, const fr_element_opts* opts, long long n_verts, const double* xv,
                          long long n_cells, const int* cell_type, const int* cell_verts, const double* period,
                          long long n_bfaces, const long long* bface_cell, const int* bface_face,
                          const int* bface_type, fr_mixed** out);
fr_status fr_mixed_destroy(fr_mixed* m);
/* ele_types and n_eles hold up to 3 entries (one per slot). */
fr_status fr_mixed_info(const fr_mixed* m, int* n_types, int* ele_types, long long* n_eles, int* n_inter_groups,
                        int* n_bdy_groups);
/* Metrics of slot `slot`: JGinv_upts (dims, dims, n_upts, n_eles),
 * detjac_upts (n_upts, n_eles), tdA_fpts (n_fpts, n_eles), norm_fpts
 * (n_fpts, n_eles, dims), pos_upts (n_upts, n_eles, dims), cell_of_ele
 * (n_eles) the mesh cell of each element.  NULL outputs are skipped. */
fr_status fr_mixed_metrics(const fr_mixed* m, int slot, double* JGinv_upts, double* detjac_upts, double* tdA_fpts,
                           double* norm_fpts, double* pos_upts, long long* cell_of_ele);
/* Interface group `group` (edges in 2-D; triangular faces first, then
 * quadrilateral, in 3-D):
 * table (6, n_fpts_per_inter, n_inters) of (element type, element, flux
 * point) of the left and the right side of every interface point, the lower
 * cell being the left side; flux points are paired by position.  Query the
 * sizes with table NULL first. */
fr_status fr_mixed_inters(const fr_mixed* m, int group, int* n_fpts_per_inter, long long* n_inters, int* table);
/* Boundary group `group` (triangular faces first): table (4, n_fpts_per_inter,
 * n_inters) of (element type, element, flux point, boundary type). */
fr_status fr_mixed_bdy_inters(const fr_mixed* m, int group, int* n_fpts_per_inter, long long* n_inters, int* table);

/* ------------------------------------------------------------------------
 * Fused RK stage for meshes of dense-operator element types.
 *
 * The per-operator sequence of CalcResidual (src/solver.cpp:65-225: for every
 * element type extrapolate_solution, calculate_gradient, evaluate_invFlux;
 * every interface type calculate_common_invFlux; correct_gradient,
 * extrapolate_corrected_gradient, evaluate_viscFlux, extrapolate_totalFlux,
 * calculate_divergence; calculate_common_viscFlux; calculate_corrected_divergence)
 * and AdvanceSolution (src/eles.cpp:1155-1178) -- Navier-Stokes (viscous 1;
 * Rusanov + LDG) or Euler (viscous 0; Rusanov, or Roe in 2-D with
 * riemann_solve_type 2), 2-D or 3-D -- in two kernels per element type and
 * stage whose operator
 * products run on the FP64 tensor cores.  Inputs are what the per-operator
 * entry points take: each type's operators and metrics as its eles object
 * holds them (host arrays, column-major, the layouts of the fr_op_* calls;
 * opp_1/2/4/5 one array per dimension), its state disu_upts and optional
 * output div_tconf_upts on the device (n_upts, n_eles, n_fields), and the
 * interface tables of fr_mixed_inters / fr_mixed_bdy_inters ((6 | 4,
 * n_fpts_per_inter, n_inters) int arrays of (type index, element, flux point)
 * per side, the boundary type last), on the host.  Every flux point must lie
 * on exactly one interface or boundary (FR_ERR_MESH otherwise).  Element
 * types with kernels: tets, prisms, triangles and quads of orders 1 to 4,
 * hexes of orders 1 to 3 (FR_ERR_UNSUPPORTED otherwise).  The stage keeps the RK register and the
 * flux-point traces on the device; disu_upts is advanced in place.
 * ---------------------------------------------------------------------- */
typedef struct {
  int n_upts, n_fpts;
  long long n_eles;
  const double* opp_0;       /* (n_fpts, n_upts)                      */
  const double* opp_1[3];    /* (n_fpts, n_upts) per dimension         */
  const double* opp_2[3];    /* (n_upts, n_upts) per dimension         */
  const double* opp_3;       /* (n_upts, n_fpts)                      */
  const double* opp_4[3];    /* (n_upts, n_upts) per dimension         */
  const double* opp_5[3];    /* (n_upts, n_fpts) per dimension         */
  const double* opp_6;       /* (n_fpts, n_upts); opp_4/5/6 may be NULL for Euler */
  const double* JGinv_upts;  /* (n_dims, n_dims, n_upts, n_eles)      */
  const double* detjac_upts; /* (n_upts, n_eles)                      */
  const double* tdA_fpts;    /* (n_fpts, n_eles)                      */
  const double* norm_fpts;   /* (n_fpts, n_eles, n_dims)              */
  double* disu_upts;         /* device (n_upts, n_eles, n_fields)     */
  double* div_tconf_upts;    /* device, or NULL if residual() is not called */
} fr_mixed_stage_type;

typedef struct fr_mixed_stage fr_mixed_stage;
fr_status fr_mixed_stage_create(int n_dims, int n_types, const fr_mixed_stage_type* types, int n_int_groups,
                                const int* const* int_tables, const int* int_nfpi, const long long* int_ni,
                                int n_bdy_groups, const int* const* bdy_tables, const int* bdy_nfpi,
                                const long long* bdy_ni, const double* bdy_params, double R_ref,
                                const fr_phys_desc* phys, int viscous, int riemann_solve_type,
                                fr_mixed_stage** out);
fr_status fr_mixed_stage_destroy(fr_mixed_stage* s);
/* div_tconf_upts of every type for the current state (one CalcResidual). */
fr_status fr_mixed_stage_residual(fr_mixed_stage* s, void* stream);
/* n_steps RK45 steps of dt (5 stages each) on the current state. */
fr_status fr_mixed_stage_advance(fr_mixed_stage* s, int n_steps, double dt, void* stream);
/* The same, then the L1 residual norms of the last step into res_norms
 * (n_fields host doubles): CalcNormResidual with res_norm_type 1
 * (src/output.cpp:1452-1520), sum over every type's solution points of
 * |div_tconf_upts / detjac_upts| of the last stage, over their number.
 * Synchronises the stream; FR_ERR_NONFINITE for a NaN norm. */
fr_status fr_mixed_stage_advance_norms(fr_mixed_stage* s, int n_steps, double dt, double* res_norms, void* stream);
/* Launch shapes of each type's two stage kernels: gradient 0 = 8 elements x
 * 256 threads, 1 = 4 x 128, 2 = 8 x 128, 3 = 4 x 128 with registers for 4
 * blocks per SM, 4 = 8 x 256 with registers for 2; update 0 = 8 x 256,
 * 1 = 4 x 128,
 * 2 = 8 x 128 (every shape gives the same bits; shapes whose shared memory
 * exceeds a block's return FR_ERR_UNSUPPORTED).  create() sets gradient 3
 * and update 1 (else the first shape that fits);
 * autotune() times every shape on the current state (the update kernels in
 * residual mode, into scratch memory; the state is not changed) and keeps
 * the fastest per type. */
fr_status fr_mixed_stage_set_launch(fr_mixed_stage* s, int type, int grad_shape, int update_shape);
fr_status fr_mixed_stage_get_launch(const fr_mixed_stage* s, int type, int* grad_shape, int* update_shape);
fr_status fr_mixed_stage_autotune(fr_mixed_stage* s, void* stream);
/* on (default): the kernels of element types after the first run on side
 * streams of the stage, forked from and joined back into the caller's stream
 * around each kernel of a stage, so small types overlap large ones; off: all
 * on the caller's stream.  Same bits either way. */
fr_status fr_mixed_stage_set_concurrent(fr_mixed_stage* s, int on);
/* Flux points over all types, boundary points, kernel launches per stage. */
fr_status fr_mixed_stage_info(const fr_mixed_stage* s, long long* n_flux_points, long long* n_boundary_points,
                              int* launches_per_stage);

/* ------------------------------------------------------------------------
 * Residual without device allocation.
 *
 * No counterpart in the reference.  For callers that cannot call cudaMalloc
 * when they need a residual: code in the middle of recording work for later
 * replay, code whose device memory comes from someone else's pool, hosts that
 * forbid allocation after start-up.  The caller passes every input and the
 * output; the scratch between the stage kernels (traces, viscous-flux
 * projections, normal discontinuous flux, divergence, common flux) lives in a
 * fixed 32 MiB array of device memory inside the library, which every GPU that
 * loads the library keeps until the process exits.  The first call on a
 * device looks up that array's device address, so make the first call before
 * any stream capture.  All calls share the array: calls whose work overlaps on
 * the GPU (different streams, different host threads) race and must be
 * serialised by the caller.  The looked-up address is kept for the life of
 * the process: do not use this entry point after cudaDeviceReset on that
 * device.  Meshes whose scratch would exceed 32 MiB are rejected with
 * FR_ERR_ARG (hex P=3: ~1950 Navier-Stokes or ~4350 Euler elements).
 * The mesh has no boundary points: every flux point is an interior point that
 * appears in face_lr, mate >= 0 everywhere, and side bits 2..7 are zero (they
 * are ignored).  Periodic meshes qualify; walled meshes go through the solver
 * object or the per-operator boundary entry points.
 * Output: div_tconf_upts of one CalcResidual, FP64, identical to
 * fr_solver_residual on the same mesh and state.
 * ---------------------------------------------------------------------- */
typedef struct {
  int dims, order, n_eles, viscous;   /* quads (P 1..5) or hexes (P 1..4)               */
  int upts_type, vcjh_scheme;         /* as in fr_scheme_desc (Gauss points only)       */
  double eta;
  fr_phys_desc phys;
  const double* disu_upts;            /* (n_upts, n_eles, F) state                      */
  const double* JGinv_upts;           /* (D, D, n_upts, n_eles)                         */
  const double* detjac_upts;          /* (n_upts, n_eles)                               */
  const double* norm_left;            /* (n_fpts, n_eles, D) unit normal of the
                                         interface's left side, at both sides' points  */
  const double* tdA_fpts;             /* (n_fpts, n_eles) own |J^-T n| dA               */
  const int* mate;                    /* (n_fpts, n_eles) matching point, flat index     */
  const unsigned char* side;          /* (n_fpts, n_eles) bit0 left side, bit1 negative
                                         LDG penalty                                    */
  long long n_int;                    /* interface points                               */
  const int* face_lr;                 /* (n_int, 2) left/right flat indices, 8-byte aligned */
  const unsigned char* face_sign;     /* (n_int) nonzero: negative LDG penalty           */
  double* div_tconf_upts;             /* output (n_upts, n_eles, F)                      */
} fr_residual_args;

fr_status fr_residual_noalloc(const fr_residual_args* args, void* stream);

#ifdef __cplusplus
}
#endif
#endif
