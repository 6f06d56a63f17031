// ref_harness.cpp -- test-infrastructure driver around the unmodified HiFiLES
// CPU objects (built by oracle/Makefile into oracle/_ref/).
//
// It reproduces the set-up sequence of the reference's main()
// (src/HiFiLES.cpp:90-101: input::setup -> SetInput -> GeoPreprocess ->
// InitSolution), optionally replaces the initial state by a closed-form field
// evaluated at the reference's own solution-point positions, and then
//   * dumps the per-type operator matrices opp_0..opp_6 (src/eles.cpp:3620-4052),
//     the metrics (src/eles.cpp:4557-4847) and the interior-interface wiring
//     decoded from the int_inters pointer tables (src/int_inters.cpp:95-178);
//   * with --stages, runs stage 0 of CalcResidual (src/solver.cpp:65-225) one
//     operator at a time and dumps every intermediate array;
//   * runs --steps RK45 steps exactly as main() does (src/HiFiLES.cpp:154-183)
//     and records the residual norms of CalcNormResidual (src/output.cpp:1452);
//   * with --integrals, evaluates the integral quantities of the initial state
//     on the reference's volume cubature and dumps them with that cubature.
// Output: one .npy per array (Fortran order = the reference's array<T> layout,
// first index fastest) plus params.txt with the non-dimensional constants.
//
// This file is compiled against the reference headers with protected members
// opened up; it is never linked into the product.

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <string>
#include <vector>
#include <iostream>
#include <fstream>
#include <time.h>

#define protected public
#include "global.h"
#include "array.h"
#include "funcs.h"
#include "input.h"
#include "flux.h"
#include "geometry.h"
#include "solver.h"
#include "output.h"
#include "solution.h"
#include "mesh.h"
#undef protected

using namespace std;

static string g_out;

static void write_npy(const string& name, const void* data, const char* descr,
                      size_t elsize, const vector<int>& shape)
{
  string path = g_out + "/" + name + ".npy";
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) { fprintf(stderr, "cannot write %s\n", path.c_str()); exit(3); }
  string hdr = string("{'descr': '") + descr + "', 'fortran_order': True, 'shape': (";
  size_t n = 1;
  for (size_t i = 0; i < shape.size(); i++) {
    char b[32]; snprintf(b, sizeof b, "%d,", shape[i]); hdr += b;
    if (i + 1 < shape.size()) hdr += " ";
    n *= (size_t)shape[i];
  }
  hdr += "), }";
  size_t total = 10 + hdr.size() + 1;
  size_t pad = (64 - total % 64) % 64;
  hdr.append(pad, ' ');
  hdr += '\n';
  unsigned char pre[10] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0, 0, 0};
  pre[8] = (unsigned char)(hdr.size() & 0xff);
  pre[9] = (unsigned char)(hdr.size() >> 8);
  fwrite(pre, 1, 10, f);
  fwrite(hdr.data(), 1, hdr.size(), f);
  fwrite(data, elsize, n, f);
  fclose(f);
}

static void dump(const string& name, array<double>& a, int ndim)
{
  vector<int> shape;
  for (int d = 0; d < ndim; d++) shape.push_back(a.get_dim(d));
  write_npy(name, a.get_ptr_cpu(), "<f8", 8, shape);
}

static void dump_ints(const string& name, const vector<int>& v, const vector<int>& shape)
{
  write_npy(name, v.data(), "<i4", 4, shape);
}

static const double PI_ = 3.14159265358979323846;

// Closed-form initial states evaluated at the reference's solution points.
//  vortex_u1v0 : isentropic vortex of strength 5 at the origin in a free
//                stream rho=1, u=1, v=0, p=1 (same vortex profile as
//                src/funcs.cpp:1646-1657, advected along x only).
//  tgv_mach01  : Taylor-Green vortex with rho0=1, U0=1 and p0=1/(gamma M^2),
//                M=0.1 (the 3-D initial field of src/eles.cpp:550-565 with the
//                background pressure changed from 100).
static void apply_ic(const string& ic, solution& S)
{
  double gamma = run_input.gamma;
  for (int t = 0; t < S.n_ele_types; t++) {
    eles* e = S.mesh_eles(t);
    if (e->n_eles == 0) continue;
    for (int i = 0; i < e->n_eles; i++)
      for (int j = 0; j < e->n_upts_per_ele; j++) {
        double x = e->pos_upts(j, i, 0), y = e->pos_upts(j, i, 1);
        double z = (e->n_dims == 3) ? e->pos_upts(j, i, 2) : 0.0;
        double q[5] = {0, 0, 0, 0, 0};
        if (ic == "vortex_u1v0") {
          double eps = 5.0, f = 1.0 - (x * x + y * y);
          double rho = pow(1.0 - eps * eps * (gamma - 1.0) / (8.0 * gamma * PI_ * PI_) * exp(f), 1.0 / (gamma - 1.0));
          double vx = 1.0 - eps * y / (2.0 * PI_) * exp(f / 2.0);
          double vy = eps * x / (2.0 * PI_) * exp(f / 2.0);
          double p = pow(rho, gamma);
          q[0] = rho; q[1] = rho * vx; q[2] = rho * vy;
          q[3] = p / (gamma - 1.0) + 0.5 * rho * (vx * vx + vy * vy);
        } else if (ic == "tgv_mach01") {
          double M = 0.1, p0 = 1.0 / (gamma * M * M), rho = 1.0;
          double p = p0 + rho / 16.0 * (cos(2.0 * x) + cos(2.0 * y)) * (cos(2.0 * z) + 2.0);
          double u = sin(x) * cos(y) * cos(z), v = -cos(x) * sin(y) * cos(z);
          q[0] = rho; q[1] = rho * u; q[2] = rho * v; q[3] = 0.0;
          q[4] = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v);
        } else if (ic == "channel_mach01") {
          // smooth non-uniform flow at the Mach 0.1 free stream of the
          // non-dimensionalisation (rho = 1, u = 1, p = 1/(gamma M^2))
          double M = 0.1, p0 = 1.0 / (gamma * M * M);
          double rho = 1.0 + 0.05 * sin(x) * cos(y);
          double u = 1.0 + 0.1 * sin(y), v = 0.1 * cos(x), w = 0.05 * sin(x + y + z);
          double p = p0 * (1.0 + 0.01 * cos(x + y));
          if (e->n_dims == 2) {
            q[0] = rho; q[1] = rho * u; q[2] = rho * v;
            q[3] = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v);
          } else {
            q[0] = rho; q[1] = rho * u; q[2] = rho * v; q[3] = rho * w;
            q[4] = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w);
          }
        } else {
          fprintf(stderr, "unknown --ic %s\n", ic.c_str()); exit(2);
        }
        for (int k = 0; k < e->n_fields; k++) e->disu_upts(0)(j, i, k) = q[k];
      }
  }
}

// Decode a pointer into some element type's array (fpt-major (n_fpts, n_eles, ...)).
static void locate(solution& S, double* p, bool grad, int& type, int& ele, int& fpt)
{
  for (int t = 0; t < S.n_ele_types; t++) {
    eles* e = S.mesh_eles(t);
    if (e->n_eles == 0) continue;
    array<double>& a = grad ? e->grad_disu_fpts : e->disu_fpts;
    double* b = a.get_ptr_cpu();
    size_t n = (size_t)e->n_fpts_per_ele * e->n_eles;
    if (p >= b && p < b + n) {
      size_t off = p - b;
      type = t; ele = off / e->n_fpts_per_ele; fpt = off % e->n_fpts_per_ele;
      return;
    }
  }
  fprintf(stderr, "pointer not found\n"); exit(4);
}

static void dump_setup(solution& S)
{
  FILE* f = fopen((g_out + "/params.txt").c_str(), "w");
  fprintf(f, "gamma %.17g\nmu_inf %.17g\nprandtl %.17g\nrt_inf %.17g\nc_sth %.17g\n"
             "fix_vis %.17g\ntau %.17g\npen_fact %.17g\ndt %.17g\nviscous %d\n"
             "order %d\nn_dims %d\nprandtl_t %.17g\n",
          run_input.gamma, run_input.mu_inf, run_input.prandtl, run_input.rt_inf,
          run_input.c_sth, run_input.fix_vis, run_input.tau, run_input.pen_fact,
          run_input.dt, run_input.viscous, run_input.order, S.n_dims, run_input.prandtl_t);
  fprintf(f, "R_ref %.17g\n", run_input.R_ref);
  if (S.n_bdy_inter_types > 0)
    for (int i = 0; i < 14; i++) fprintf(f, "bdy%d %.17g\n", i, S.mesh_bdy_inters(0).bdy_params(i));
  for (int t = 0; t < S.n_ele_types; t++) {
    eles* e = S.mesh_eles(t);
    fprintf(f, "type %d ele_type %d n_eles %d n_upts %d n_fpts %d\n", t, e->ele_type,
            e->n_eles, e->n_eles ? e->n_upts_per_ele : 0, e->n_eles ? e->n_fpts_per_ele : 0);
  }
  fclose(f);

  for (int t = 0; t < S.n_ele_types; t++) {
    eles* e = S.mesh_eles(t);
    if (e->n_eles == 0) continue;
    char pre[16]; snprintf(pre, sizeof pre, "t%d_", e->ele_type);
    string P(pre);
    int D = e->n_dims;
    dump(P + "loc_upts", e->loc_upts, 2);
    dump(P + "tloc_fpts", e->tloc_fpts, 2);
    dump(P + "tnorm_fpts", e->tnorm_fpts, 2);
    dump(P + "opp_0", e->opp_0, 2);
    dump(P + "opp_3", e->opp_3, 2);
    for (int d = 0; d < D; d++) {
      char b[8]; snprintf(b, sizeof b, "%d", d);
      dump(P + "opp_1_" + b, e->opp_1(d), 2);
      dump(P + "opp_2_" + b, e->opp_2(d), 2);
      if (e->viscous) {
        dump(P + "opp_4_" + b, e->opp_4(d), 2);
        dump(P + "opp_5_" + b, e->opp_5(d), 2);
      }
    }
    if (e->viscous) dump(P + "opp_6", e->opp_6, 2);
    dump(P + "detjac_upts", e->detjac_upts, 2);
    dump(P + "JGinv_upts", e->JGinv_upts, 4);
    dump(P + "tdA_fpts", e->tdA_fpts, 2);
    dump(P + "norm_fpts", e->norm_fpts, 3);
    dump(P + "pos_upts", e->pos_upts, 3);
    dump(P + "pos_fpts", e->pos_fpts, 3);
    dump(P + "disu_upts_init", e->disu_upts(0), 3);
  }

  // interior interfaces: (type, ele, fpt) of the left and right side of every
  // interface flux point, decoded from the pointer tables.
  for (int it = 0; it < S.n_int_inter_types; it++) {
    int_inters& I = S.mesh_int_inters(it);
    if (I.n_inters == 0) continue;
    vector<int> v;
    for (int i = 0; i < I.n_inters; i++)
      for (int j = 0; j < I.n_fpts_per_inter; j++) {
        int tl, el, fl, tr, er, fr;
        locate(S, I.disu_fpts_l(j, i, 0), false, tl, el, fl);
        locate(S, I.disu_fpts_r(j, i, 0), false, tr, er, fr);
        int row[6] = {tl, el, fl, tr, er, fr};
        v.insert(v.end(), row, row + 6);
      }
    char b[32]; snprintf(b, sizeof b, "int_inters_%d", it);
    vector<int> shape; shape.push_back(6); shape.push_back(I.n_fpts_per_inter); shape.push_back(I.n_inters);
    dump_ints(b, v, shape);
  }

  // boundary interfaces: (type, ele, fpt) of the owning side of every
  // boundary flux point and the interface's boundary type
  // (bdy_inters::set_boundary, src/bdy_inters.cpp:111-203).
  for (int it = 0; it < S.n_bdy_inter_types; it++) {
    bdy_inters& B = S.mesh_bdy_inters(it);
    if (B.n_inters == 0) continue;
    vector<int> v;
    for (int i = 0; i < B.n_inters; i++)
      for (int j = 0; j < B.n_fpts_per_inter; j++) {
        int tl, el, fl;
        locate(S, B.disu_fpts_l(j, i, 0), false, tl, el, fl);
        int row[4] = {tl, el, fl, B.boundary_type(i)};
        v.insert(v.end(), row, row + 4);
      }
    char b[32]; snprintf(b, sizeof b, "bdy_inters_%d", it);
    vector<int> shape; shape.push_back(4); shape.push_back(B.n_fpts_per_inter); shape.push_back(B.n_inters);
    dump_ints(b, v, shape);
  }
}

static void dump_stage(solution& S, const char* tag, const char* what)
{
  for (int t = 0; t < S.n_ele_types; t++) {
    eles* e = S.mesh_eles(t);
    if (e->n_eles == 0) continue;
    char pre[64]; snprintf(pre, sizeof pre, "t%d_%s_", e->ele_type, tag);
    string P(pre), W(what);
    if (W == "disu_fpts") dump(P + W, e->disu_fpts, 3);
    else if (W == "grad_disu_upts") dump(P + W, e->grad_disu_upts, 4);
    else if (W == "grad_disu_fpts") dump(P + W, e->grad_disu_fpts, 4);
    else if (W == "tdisf_upts") dump(P + W, e->tdisf_upts, 4);
    else if (W == "norm_tconf_fpts") dump(P + W, e->norm_tconf_fpts, 3);
    else if (W == "delta_disu_fpts") dump(P + W, e->delta_disu_fpts, 3);
    else if (W == "norm_tdisf_fpts") dump(P + W, e->norm_tdisf_fpts, 3);
    else if (W == "div_tconf_upts") dump(P + W, e->div_tconf_upts(0), 3);
    else if (W == "disu_upts0") dump(P + W, e->disu_upts(0), 3);
    else if (W == "disu_upts1") dump(P + W, e->disu_upts(1), 3);
    else if (W == "sgsf_upts") dump(P + W, e->sgsf_upts, 4);
    else if (W == "sgsf_fpts") dump(P + W, e->sgsf_fpts, 4);
  }
}

// Stage 0 of CalcResidual, operator by operator (src/solver.cpp:65-225 for a
// single rank with no shock capturing, no body force, no SA source; LES with
// an eddy-viscosity model, which needs no calc_sgs_terms, src/solver.cpp:72-76).
static void staged_residual(solution& S)
{
  int n = S.n_ele_types;
  for (int i = 0; i < n; i++) S.mesh_eles(i)->extrapolate_solution(0);
  dump_stage(S, "s01", "disu_fpts");
  if (S.viscous) {
    for (int i = 0; i < n; i++) S.mesh_eles(i)->calculate_gradient(0);
    dump_stage(S, "s02", "grad_disu_upts");
  }
  for (int i = 0; i < n; i++) S.mesh_eles(i)->evaluate_invFlux(0);
  dump_stage(S, "s03", "tdisf_upts");
  for (int i = 0; i < S.n_int_inter_types; i++) S.mesh_int_inters(i).calculate_common_invFlux();
  for (int i = 0; i < S.n_bdy_inter_types; i++) S.mesh_bdy_inters(i).evaluate_boundaryConditions_invFlux(S.time);
  dump_stage(S, "s04", "norm_tconf_fpts");
  if (S.viscous) {
    dump_stage(S, "s04", "delta_disu_fpts");
    for (int i = 0; i < n; i++) S.mesh_eles(i)->correct_gradient();
    dump_stage(S, "s05", "grad_disu_upts");
    for (int i = 0; i < n; i++) S.mesh_eles(i)->extrapolate_corrected_gradient();
    dump_stage(S, "s06", "grad_disu_fpts");
    for (int i = 0; i < n; i++) S.mesh_eles(i)->evaluate_viscFlux(0);
    dump_stage(S, "s07", "tdisf_upts");
  }
  if (run_input.LES) {
    dump_stage(S, "s07", "sgsf_upts");
    for (int i = 0; i < n; i++) S.mesh_eles(i)->evaluate_sgsFlux();
    dump_stage(S, "s07", "sgsf_fpts");
  }
  for (int i = 0; i < n; i++) S.mesh_eles(i)->extrapolate_totalFlux();
  dump_stage(S, "s08", "norm_tdisf_fpts");
  for (int i = 0; i < n; i++) S.mesh_eles(i)->calculate_divergence(0);
  dump_stage(S, "s09", "div_tconf_upts");
  if (S.viscous) {
    for (int i = 0; i < S.n_int_inter_types; i++) S.mesh_int_inters(i).calculate_common_viscFlux();
    for (int i = 0; i < S.n_bdy_inter_types; i++) S.mesh_bdy_inters(i).evaluate_boundaryConditions_viscFlux(S.time);
    dump_stage(S, "s10", "norm_tconf_fpts");
  }
  for (int i = 0; i < n; i++) S.mesh_eles(i)->calculate_corrected_divergence(0);
  dump_stage(S, "s11", "div_tconf_upts");
}

// The reference's integral quantities of the current state
// (output.cpp CalcIntegralQuantities -> eles::CalcIntegralQuantities,
// src/eles.cpp:6503-6641) after one residual evaluation (stage 0 of
// CalcResidual fills grad_disu_upts), and the volume cubature the reference
// integrates on: loc/weight_volume_cubpts, opp_volume_cubpts and
// vol_detjac_vol_cubpts (src/eles.cpp:4111-4130, 5320-5352).
static void dump_integrals(solution& S)
{
  CalcResidual(0, 0, &S);
  CalcIntegralQuantities(0, &S);
  vector<double> iq;
  for (int m = 0; m < run_input.n_integral_quantities; m++) iq.push_back(S.integral_quantities(m));
  vector<int> shape(1, (int)iq.size());
  write_npy("integral_quantities", iq.data(), "<f8", 8, shape);
  for (int t = 0; t < S.n_ele_types; t++) {
    eles* e = S.mesh_eles(t);
    if (e->n_eles == 0) continue;
    char pre[16]; snprintf(pre, sizeof pre, "t%d_", e->ele_type);
    string P(pre);
    dump(P + "loc_volume_cubpts", e->loc_volume_cubpts, 2);
    dump(P + "weight_volume_cubpts", e->weight_volume_cubpts, 1);
    dump(P + "opp_volume_cubpts", e->opp_volume_cubpts, 2);
    vector<double> dj;
    for (int i = 0; i < e->n_eles; i++)
      for (int j = 0; j < e->n_cubpts_per_ele; j++) dj.push_back(e->vol_detjac_vol_cubpts(j)(i));
    vector<int> sh; sh.push_back(e->n_cubpts_per_ele); sh.push_back(e->n_eles);
    write_npy(P + "vol_detjac_vol_cubpts", dj.data(), "<f8", 8, sh);
    dump(P + "grad_disu_upts_iq", e->grad_disu_upts, 4);
    dump(P + "disu_upts_iq", e->disu_upts(0), 3);
  }
}

int main(int argc, char** argv)
{
  if (argc < 3) {
    fprintf(stderr, "usage: ref_harness <input_file> <out_dir> [--ic NAME] [--steps N] [--stages] [--no-dump] [--integrals]"
                    " [--write-restart N]\n");
    return 2;
  }
  g_out = argv[2];
  string ic;
  int steps = 0;
  bool stages = false, nodump = false, integrals = false;
  int restart_out = -1;
  for (int a = 3; a < argc; a++) {
    if (!strcmp(argv[a], "--ic") && a + 1 < argc) ic = argv[++a];
    else if (!strcmp(argv[a], "--steps") && a + 1 < argc) steps = atoi(argv[++a]);
    else if (!strcmp(argv[a], "--stages")) stages = true;
    else if (!strcmp(argv[a], "--no-dump")) nodump = true;
    else if (!strcmp(argv[a], "--integrals")) integrals = true;
    else if (!strcmp(argv[a], "--write-restart") && a + 1 < argc) restart_out = atoi(argv[++a]);
    else { fprintf(stderr, "bad argument %s\n", argv[a]); return 2; }
  }

  static solution S;
  static mesh Mesh;
  run_input.setup(argv[1], 0);
  SetInput(&S);
  GeoPreprocess(&S, Mesh);
  InitSolution(&S);
  if (!ic.empty()) apply_ic(ic, S);

  S.norm_residual.setup(5);
  S.inv_force.setup(5);
  S.vis_force.setup(5);
  S.integral_quantities.setup(run_input.n_integral_quantities > 0 ? run_input.n_integral_quantities : 1);
  for (int i = 0; i < 5; i++) S.norm_residual(i) = 0.0;

  if (!nodump) dump_setup(S);
  if (integrals) {
    dump_integrals(S);
    printf("ref_harness done\n");
    return 0;
  }

  int first_stage = 0;
  if (stages) {
    staged_residual(S);
    for (int j = 0; j < S.n_ele_types; j++) S.mesh_eles(j)->AdvanceSolution(0, S.adv_type);
    dump_stage(S, "s12", "disu_upts0");
    dump_stage(S, "s12", "disu_upts1");
    first_stage = 1;
  }

  int nf = (S.n_dims == 2) ? 4 : 5;
  vector<double> hist;
  int RK = (S.adv_type == 3) ? 5 : 1;
  struct timespec t0, t1;
  clock_gettime(CLOCK_MONOTONIC, &t0);
  for (int s = 0; s < steps; s++) {
    for (int i = (s == 0 ? first_stage : 0); i < RK; i++) {
      CalcResidual(0, i, &S);
      for (int j = 0; j < S.n_ele_types; j++) S.mesh_eles(j)->AdvanceSolution(i, S.adv_type);
    }
    S.time += run_input.dt;
    CalcNormResidual(&S);
    for (int k = 0; k < nf; k++) hist.push_back(S.norm_residual(k));
  }
  clock_gettime(CLOCK_MONOTONIC, &t1);
  printf("step_loop_seconds %.9f\n", (t1.tv_sec - t0.tv_sec) + 1e-9 * (t1.tv_nsec - t0.tv_nsec));
  if (steps > 0 && !nodump) {
    vector<int> shape; shape.push_back(nf); shape.push_back(steps);
    write_npy("res_norms", hist.data(), "<f8", 8, shape);
    dump_stage(S, "final", "disu_upts0");
    dump_stage(S, "final", "div_tconf_upts");
  }
  if (restart_out >= 0) {
    // Rest_<N>_p0000.dat in the working directory (src/output.cpp:1057-1107)
    run_input.restart_mesh_out = 0;
    write_restart(restart_out, &S);
  }
  printf("ref_harness done\n");
  return 0;
}
