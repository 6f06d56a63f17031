// fr_physics.cuh -- pointwise Euler / Navier-Stokes physics of the FR path,
// device side, templated on the compute type T (double: FP64 form, float:
// FP32 form) and the number of dimensions D (F = D + 2 fields).
//
// The expressions repeat the reference's CPU routines term for term (true
// divisions, the same association order).  The translation units that include
// this header are compiled with -fmad=false, so nothing is contracted into an
// FMA behind the code's back: the FP64 form rounds exactly like the reference
// wherever it evaluates the same expression.  This matters: at low Mach
// number the flux terms are ~1e3-1e4 times larger than the residual they
// cancel to, so ulp-level differences in the fluxes show up at 1e-12 in the
// residual.
#pragma once

#include <cuda_runtime.h>

#include "fr_mlp.cuh"

namespace frb {

struct Phys {
  double gamma, prandtl, mu_inf, rt_inf, c_sth, fix_vis, tau, pen_fact;
  int sgs_model = 1;          // eddy-viscosity LES: 0 Smagorinsky, 1 WALE, 5 learned (fr_mlp.cuh)
  double filter_ratio = 1.0;  // LES filter width over the element's point spacing
  const float* mlp = nullptr; // device parameters of the learned closure (sgs_model 5)
  double bdy[14] = {};        // boundary values (bdy_inters::set_bdy_params order)
  double R_ref = 1.0;
};

template <typename T>
struct PhysT {
  T gamma, gm1, prandtl, mu_inf, rt_inf, c_sth, fix_vis, tau, pen_fact, filter_ratio;
  int sgs_model;
  const float* mlp;
  T bdy[14], R_ref;
  __host__ __device__ static PhysT make(const Phys& p) {
    PhysT q;
    q.gamma = (T)p.gamma; q.gm1 = (T)(p.gamma - 1.0); q.prandtl = (T)p.prandtl; q.mu_inf = (T)p.mu_inf;
    q.rt_inf = (T)p.rt_inf; q.c_sth = (T)p.c_sth; q.fix_vis = (T)p.fix_vis; q.tau = (T)p.tau;
    q.pen_fact = (T)p.pen_fact; q.filter_ratio = (T)p.filter_ratio; q.sgs_model = p.sgs_model;
    q.mlp = p.mlp;
    for (int i = 0; i < 14; i++) q.bdy[i] = (T)p.bdy[i];
    q.R_ref = (T)p.R_ref;
    return q;
  }
};

template <typename T> __device__ __forceinline__ T fr_sqrt(T x);
template <> __device__ __forceinline__ double fr_sqrt<double>(double x) { return sqrt(x); }
template <> __device__ __forceinline__ float fr_sqrt<float>(float x) { return sqrtf(x); }
template <typename T> __device__ __forceinline__ T fr_abs(T x);
template <> __device__ __forceinline__ double fr_abs<double>(double x) { return fabs(x); }
template <> __device__ __forceinline__ float fr_abs<float>(float x) { return fabsf(x); }
template <typename T> __device__ __forceinline__ T fr_pow15(T x);
template <> __device__ __forceinline__ double fr_pow15<double>(double x) { return pow(x, 1.5); }
template <> __device__ __forceinline__ float fr_pow15<float>(float x) { return powf(x, 1.5f); }

// Inviscid flux f[k][l] (field k, direction l): calc_invf_2d / calc_invf_3d,
// src/flux.cpp:36-128.
template <int D, typename T>
__device__ __forceinline__ void inv_flux(const PhysT<T>& ph, const T* u, T (*f)[D])
{
  constexpr int F = D + 2;
  T v[D];
#pragma unroll
  for (int l = 0; l < D; l++) v[l] = u[l + 1] / u[0];
  T ke = v[0] * v[0];
#pragma unroll
  for (int l = 1; l < D; l++) ke = ke + v[l] * v[l];
  T p = ph.gm1 * (u[F - 1] - (T(0.5) * u[0] * ke));
#pragma unroll
  for (int l = 0; l < D; l++) {
    f[0][l] = u[l + 1];
#pragma unroll
    for (int m = 0; m < D; m++) f[m + 1][l] = (m == l) ? p + (u[m + 1] * v[l]) : u[m + 1] * v[l];
    f[F - 1][l] = v[l] * (u[F - 1] + p);
  }
}

// Viscous flux, no turbulence model: calc_visf_2d / calc_visf_3d,
// src/flux.cpp:132-431.  With fix_vis == 1 the viscosity is mu_inf (the value
// mu + fix_vis*(mu_inf - mu) takes whenever the Sutherland value is within a
// factor 2 of mu_inf); otherwise Sutherland's law.
template <int D, typename T>
__device__ __forceinline__ void vis_flux(const PhysT<T>& ph, const T* u, T (*g)[D], T (*f)[D])
{
  constexpr int F = D + 2;
  const T rho = u[0];
  T v[D];
#pragma unroll
  for (int l = 0; l < D; l++) v[l] = u[l + 1] / rho;
  T ke = v[0] * v[0];
#pragma unroll
  for (int l = 1; l < D; l++) ke = ke + v[l] * v[l];
  T inte = u[F - 1] / rho - T(0.5) * ke;
  T mu;
  if (ph.fix_vis == T(1)) {
    mu = ph.mu_inf;
  } else {
    T rt = ph.gm1 * inte / ph.rt_inf;
    mu = ph.mu_inf * fr_pow15<T>(rt) * (T(1) + ph.c_sth) / (rt + ph.c_sth);
    mu = mu + ph.fix_vis * (ph.mu_inf - mu);
  }
  T dv[D][D];   // dv[m][l] = d v_m / d x_l
#pragma unroll
  for (int m = 0; m < D; m++)
#pragma unroll
    for (int l = 0; l < D; l++) dv[m][l] = (g[m + 1][l] - g[0][l] * v[m]) / rho;
  T de[D];
#pragma unroll
  for (int l = 0; l < D; l++) {
    T vdv = v[0] * dv[0][l];
#pragma unroll
    for (int m = 1; m < D; m++) vdv = vdv + v[m] * dv[m][l];
    T dke = T(0.5) * ke * g[0][l] + rho * vdv;
    de[l] = (g[F - 1][l] - dke - g[0][l] * inte) / rho;
  }
  T dsum = dv[0][0];
#pragma unroll
  for (int l = 1; l < D; l++) dsum = dsum + dv[l][l];
  const T diag = dsum / T(3.0);
  const T kt = mu / ph.prandtl;   // (mu/prandtl + mu_t/prandtl_t) with mu_t = 0
  T tau[D][D];
#pragma unroll
  for (int m = 0; m < D; m++)
#pragma unroll
    for (int l = 0; l < D; l++)
      tau[m][l] = (m == l) ? T(2.0) * mu * (dv[m][m] - diag) : mu * (dv[m][l] + dv[l][m]);
#pragma unroll
  for (int l = 0; l < D; l++) {
    f[0][l] = T(0);
    T w = v[0] * tau[0][l];
#pragma unroll
    for (int m = 0; m < D; m++) {
      f[m + 1][l] = -tau[m][l];
      if (m > 0) w = w + v[m] * tau[m][l];
    }
    f[F - 1][l] = -(w + kt * ph.gamma * de[l]);
  }
}

// The same viscous flux with one reciprocal of rho and explicit FMAs.  Used
// where the result only enters through the viscous terms, whose size is
// ~1/Re of the inviscid flux they are added to: its ulp-level differences from
// the reference's division form stay far below the rounding of the total flux.
__device__ __forceinline__ double fr_fma(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float fr_fma(float a, float b, float c) { return fmaf(a, b, c); }

// Shared part of the viscous flux: velocity v, stress tau and the heat-flux
// term q[l] = (mu gamma / Pr) de/dx_l of calc_visf_3d (src/flux.cpp:263-431).
template <int D, typename T>
__device__ __forceinline__ void vis_core(const PhysT<T>& ph, const T* u, T (*g)[D], T (&v)[D], T (&tau)[D][D],
                                         T (&q)[D])
{
  constexpr int F = D + 2;
  const T rho = u[0], ri = T(1) / rho;
#pragma unroll
  for (int l = 0; l < D; l++) v[l] = u[l + 1] * ri;
  T ke = v[0] * v[0];
#pragma unroll
  for (int l = 1; l < D; l++) ke = fr_fma(v[l], v[l], ke);
  T inte = fr_fma(T(-0.5), ke, u[F - 1] * ri);
  T mu;
  if (ph.fix_vis == T(1)) {
    mu = ph.mu_inf;
  } else {
    T rt = ph.gm1 * inte / ph.rt_inf;
    mu = ph.mu_inf * fr_pow15<T>(rt) * (T(1) + ph.c_sth) / (rt + ph.c_sth);
    mu = mu + ph.fix_vis * (ph.mu_inf - mu);
  }
  T dv[D][D];
#pragma unroll
  for (int m = 0; m < D; m++)
#pragma unroll
    for (int l = 0; l < D; l++) dv[m][l] = fr_fma(-g[0][l], v[m], g[m + 1][l]) * ri;
  T de[D];
#pragma unroll
  for (int l = 0; l < D; l++) {
    T vdv = v[0] * dv[0][l];
#pragma unroll
    for (int m = 1; m < D; m++) vdv = fr_fma(v[m], dv[m][l], vdv);
    T dke = fr_fma(T(0.5) * ke, g[0][l], rho * vdv);
    de[l] = fr_fma(-g[0][l], inte, g[F - 1][l] - dke) * ri;
  }
  T dsum = dv[0][0];
#pragma unroll
  for (int l = 1; l < D; l++) dsum = dsum + dv[l][l];
  const T diag = dsum * T(1.0 / 3.0);
  const T kg = mu / ph.prandtl * ph.gamma, mu2 = T(2) * mu;
#pragma unroll
  for (int m = 0; m < D; m++)
#pragma unroll
    for (int l = 0; l < D; l++)
      tau[m][l] = (m == l) ? mu2 * (dv[m][m] - diag) : mu * (dv[m][l] + dv[l][m]);
#pragma unroll
  for (int l = 0; l < D; l++) q[l] = kg * de[l];
}

template <int D, typename T>
__device__ __forceinline__ void vis_flux_fast(const PhysT<T>& ph, const T* u, T (*g)[D], T (*f)[D])
{
  constexpr int F = D + 2;
  T v[D], tau[D][D], q[D];
  vis_core<D, T>(ph, u, g, v, tau, q);
#pragma unroll
  for (int l = 0; l < D; l++) {
    f[0][l] = T(0);
    T w = q[l];
#pragma unroll
    for (int m = 0; m < D; m++) {
      f[m + 1][l] = -tau[m][l];
      w = fr_fma(v[m], tau[m][l], w);
    }
    f[F - 1][l] = -w;
  }
}

// The viscous flux projected on n, pr[k - 1] = project(f, k, n) for the
// components k = 1 .. F-1, without holding all of f.
template <int D, typename T>
__device__ __forceinline__ void vis_flux_proj(const PhysT<T>& ph, const T* u, T (*g)[D], const T* n, T* pr)
{
  T v[D], tau[D][D], q[D];
  vis_core<D, T>(ph, u, g, v, tau, q);
#pragma unroll
  for (int l = 0; l < D; l++) {
    T w = q[l];
#pragma unroll
    for (int m = 0; m < D; m++) {
      const T fm = -tau[m][l];
      pr[m] = l == 0 ? fm * n[0] : fr_fma(fm, n[l], pr[m]);
      w = fr_fma(v[m], tau[m][l], w);
    }
    const T fe = -w;
    pr[D] = l == 0 ? fe * n[0] : fr_fma(fe, n[l], pr[D]);
  }
}

// Rusanov common normal flux, static mesh: inters::rusanov_flux,
// src/inters.cpp:311-365 (the grid-velocity term v_g . n is zero).
template <int D, typename T>
__device__ __forceinline__ void rusanov(const PhysT<T>& ph, const T* ul, const T* ur, const T* n, T* fn)
{
  constexpr int F = D + 2;
  T fl[F][D], fr[F][D];
  inv_flux<D, T>(ph, ul, fl);
  inv_flux<D, T>(ph, ur, fr);
  T vl[D], vr[D];
#pragma unroll
  for (int l = 0; l < D; l++) { vl[l] = ul[l + 1] / ul[0]; vr[l] = ur[l + 1] / ur[0]; }
  T vnl = vl[0] * n[0], vnr = vr[0] * n[0], kl = vl[0] * vl[0], kr = vr[0] * vr[0];
#pragma unroll
  for (int l = 1; l < D; l++) {
    vnl = vnl + vl[l] * n[l]; vnr = vnr + vr[l] * n[l];
    kl = kl + vl[l] * vl[l]; kr = kr + vr[l] * vr[l];
  }
  T pl = ph.gm1 * (ul[F - 1] - (T(0.5) * ul[0] * kl));
  T pr = ph.gm1 * (ur[F - 1] - (T(0.5) * ur[0] * kr));
  T vav = fr_sqrt<T>(T(0.25) * (vnl + vnr) * (vnl + vnr));
  T cav = fr_sqrt<T>((ph.gamma * (pl + pr)) / (ul[0] + ur[0]));
  T eig = fr_abs<T>(vav + cav);
#pragma unroll
  for (int k = 0; k < F; k++) {
    T a = fl[k][0] * n[0], b = fr[k][0] * n[0];
#pragma unroll
    for (int l = 1; l < D; l++) { a = a + fl[k][l] * n[l]; b = b + fr[k][l] * n[l]; }
    fn[k] = T(0.5) * ((a + b) - eig * (ur[k] - ul[k]));
  }
}

// Roe common normal flux with the entropy fix of inters::roe_flux,
// src/inters.cpp:390-508, static mesh (v_g = 0).  2-D only, as in the
// reference ("Roe not implemented in 3D").
template <typename T>
__device__ __forceinline__ void roe(const PhysT<T>& ph, const T* ul, const T* ur, const T* n, T* fn)
{
  const T g = ph.gamma, gm1 = g - T(1.0);
  const T vl0 = ul[1] / ul[0], vl1 = ul[2] / ul[0], vr0 = ur[1] / ur[0], vr1 = ur[2] / ur[0];
  const T pl = gm1 * (ul[3] - (T(0.5) * ul[0] * ((vl0 * vl0) + (vl1 * vl1))));
  const T pr = gm1 * (ur[3] - (T(0.5) * ur[0] * ((vr0 * vr0) + (vr1 * vr1))));
  const T hl = (ul[3] + pl) / ul[0], hr = (ur[3] + pr) / ur[0];
  const T sq = fr_sqrt<T>(ur[0] / ul[0]);
  const T rr = T(1.) / (sq + T(1.));
  const T um0 = rr * (vl0 + sq * vr0), um1 = rr * (vl1 + sq * vr1);
  const T hm = rr * (hl + sq * hr);
  T usq = T(0.);
  usq = usq + T(0.5) * um0 * um0;
  usq = usq + T(0.5) * um1 * um1;
  const T am2 = gm1 * (hm - usq);
  const T am = fr_sqrt<T>(am2);
  T unm = T(0.), vgn = T(0.), rl = T(0.), rrn = T(0.);
  unm = unm + um0 * n[0]; unm = unm + um1 * n[1];
  vgn = vgn + T(0.0) * n[0]; vgn = vgn + T(0.0) * n[1];
  rl = rl + ul[1] * n[0]; rl = rl + ul[2] * n[1];
  rrn = rrn + ur[1] * n[0]; rrn = rrn + ur[2] * n[1];
  T f0 = rl + rrn;
  T f1 = rl * vl0 + rrn * vr0 + (pl + pr) * n[0];
  T f2 = rl * vl1 + rrn * vr1 + (pl + pr) * n[1];
  T f3 = rl * hl + rrn * hr;
  const T du0 = ur[0] - ul[0], du1 = ur[1] - ul[1], du2 = ur[2] - ul[2], du3 = ur[3] - ul[3];
  T l0 = fr_abs<T>(unm - vgn), lP = fr_abs<T>(unm - vgn + am), lM = fr_abs<T>(unm - vgn - am);
  const T eps = T(0.5) * (fr_abs<T>(rl / ul[0] - rrn / ur[0]) +
                          fr_abs<T>(fr_sqrt<T>(g * pl / ul[0]) - fr_sqrt<T>(g * pr / ur[0])));
  if (l0 < T(2.) * eps) l0 = T(0.25) * l0 * l0 / eps + eps;
  if (lP < T(2.) * eps) lP = T(0.25) * lP * lP / eps + eps;
  if (lM < T(2.) * eps) lM = T(0.25) * lM * lM / eps + eps;
  const T a2 = T(0.5) * (lP + lM) - l0;
  const T a3 = T(0.5) * (lP - lM) / am;
  const T a1 = a2 * gm1 / am2;
  const T a4 = a3 * gm1;
  const T a5 = usq * du0 - um0 * du1 - um1 * du2 + du3;
  const T a6 = unm * du0 - n[0] * du1 - n[1] * du2;
  const T aL1 = a1 * a5 - a3 * a6, bL1 = a4 * a5 - a2 * a6;
  f0 = f0 - (l0 * du0 + aL1);
  f1 = f1 - (l0 * du1 + aL1 * um0 + bL1 * n[0]);
  f2 = f2 - (l0 * du2 + aL1 * um1 + bL1 * n[1]);
  f3 = f3 - (l0 * du3 + aL1 * hm + bL1 * unm);
  fn[0] = T(0.5) * f0 - T(0.5) * vgn * (ur[0] + ul[0]);
  fn[1] = T(0.5) * f1 - T(0.5) * vgn * (ur[1] + ul[1]);
  fn[2] = T(0.5) * f2 - T(0.5) * vgn * (ur[2] + ul[2]);
  fn[3] = T(0.5) * f3 - T(0.5) * vgn * (ur[3] + ul[3]);
}

template <typename T> __device__ __forceinline__ T fr_pow(T x, T y);
template <> __device__ __forceinline__ double fr_pow<double>(double x, double y) { return pow(x, y); }
template <> __device__ __forceinline__ float fr_pow<float>(float x, float y) { return powf(x, y); }

// Ghost state of a boundary flux point: bdy_inters::set_inv_boundary_conditions
// for the Euler/Navier-Stokes types, src/bdy_inters.cpp:391-860; static mesh
// (grid velocity 0), no turbulence model.  Types (get_bc_number,
// src/geometry.cpp:121-148): 1 sub_in_simp, 2 sub_out_simp, 3 sub_in_char,
// 4 sub_out_char, 5 sup_in, 6 sup_out, 7 slip_wall, 11 isotherm_fix,
// 12 adiabat_fix, 13 isotherm_move, 14 adiabat_move, 15 char,
// 16 slip_wall_dual.  ph.bdy holds rho_bound, v_bound[3], p_bound,
// v_wall[3], T_wall, p_total_bound, T_total_bound, n_free_stream[3].
template <int D, typename T>
__device__ __forceinline__ void bc_ghost(const PhysT<T>& ph, int type, const T* ul, const T* n, T* ur)
{
  const T g = ph.gamma, R_ref = ph.R_ref;
  const T rho_bound = ph.bdy[0], p_bound = ph.bdy[4], T_wall = ph.bdy[8];
  const T rho_l = ul[0], e_l = ul[D + 1];
  T v_l[D], v_r[D], v_sq = T(0.), rho_r = T(0), e_r = T(0), p_r, vn_l;
#pragma unroll
  for (int i = 0; i < D; i++) { v_l[i] = ul[i + 1] / ul[0]; v_r[i] = T(0); }
#pragma unroll
  for (int i = 0; i < D; i++) v_sq = v_sq + (v_l[i] * v_l[i]);
  const T p_l = (g - T(1.0)) * (e_l - T(0.5) * rho_l * v_sq);
  auto energy = [&](void) {
    T s = T(0.);
#pragma unroll
    for (int i = 0; i < D; i++) s = s + (v_r[i] * v_r[i]);
    e_r = (p_r / (g - T(1.0))) + T(0.5) * rho_r * s;
  };
  switch (type) {
    case 1:                                   // sub_in_simp
      rho_r = rho_bound;
#pragma unroll
      for (int i = 0; i < D; i++) v_r[i] = ph.bdy[1 + i];
      p_r = p_l;
      energy();
      break;
    case 2:                                   // sub_out_simp
      rho_r = rho_l;
#pragma unroll
      for (int i = 0; i < D; i++) v_r[i] = v_l[i];
      p_r = p_bound;
      energy();
      break;
    case 3: {                                 // sub_in_char
      const T p_total_bound = ph.bdy[9], T_total_bound = ph.bdy[10];
      vn_l = T(0.);
#pragma unroll
      for (int i = 0; i < D; i++) vn_l = vn_l + v_l[i] * n[i];
      const T c_l = fr_sqrt<T>(g * p_l / rho_l);
      const T R_plus = vn_l + T(2.0) * c_l / (g - T(1.0));
      const T h_total = g * R_ref / (g - T(1.0)) * T_total_bound;
      T vs = T(0.);
#pragma unroll
      for (int i = 0; i < D; i++) vs = vs + v_l[i] * v_l[i];
      const T c_total_sq = (g - T(1.0)) * (h_total - (e_l / rho_l + p_l / rho_l) + T(0.5) * vs) + c_l * c_l;
      T alpha = T(0.);
#pragma unroll
      for (int i = 0; i < D; i++) alpha = alpha + n[i] * ph.bdy[11 + i];
      const T aa = T(1.0) + T(0.5) * (g - T(1.0)) * alpha * alpha;
      const T bb = -(g - T(1.0)) * alpha * R_plus;
      const T cc = T(0.5) * (g - T(1.0)) * R_plus * R_plus - T(2.0) * c_total_sq / (g - T(1.0));
      T dd = bb * bb - T(4.0) * aa * cc;
      dd = fr_sqrt<T>(dd > T(0.0) ? dd : T(0.0));
      T V_r = (-bb + dd) / (T(2.0) * aa);
      V_r = V_r > T(0.0) ? V_r : T(0.0);
      vs = V_r * V_r;
      T c_r_sq = c_total_sq - T(0.5) * (g - T(1.0)) * vs;
      T Mach_sq = vs / (c_r_sq);
      Mach_sq = Mach_sq < T(1.0) ? Mach_sq : T(1.0);
      vs = Mach_sq * c_r_sq;
      V_r = fr_sqrt<T>(vs);
      c_r_sq = c_total_sq - T(0.5) * (g - T(1.0)) * vs;
#pragma unroll
      for (int i = 0; i < D; i++) v_r[i] = V_r * ph.bdy[11 + i];
      const T T_r = c_r_sq / (g * R_ref);
      p_r = p_total_bound * fr_pow<T>(T_r / T_total_bound, g / (g - T(1.0)));
      rho_r = p_r / (R_ref * T_r);
      e_r = (p_r / (g - T(1.0))) + T(0.5) * rho_r * vs;
      break;
    }
    case 4: {                                 // sub_out_char
      vn_l = T(0.);
#pragma unroll
      for (int i = 0; i < D; i++) vn_l = vn_l + v_l[i] * n[i];
      const T c_l = fr_sqrt<T>(g * p_l / rho_l);
      const T R_plus = vn_l + T(2.0) * c_l / (g - T(1.0));
      const T s = p_l / fr_pow<T>(rho_l, g);
      p_r = p_bound;
      rho_r = fr_pow<T>(p_r / s, T(1.0) / g);
      const T c_r = fr_sqrt<T>(g * p_r / rho_r);
      const T vn_r = R_plus - T(2.0) * c_r / (g - T(1.0));
      T vs = T(0.);
#pragma unroll
      for (int i = 0; i < D; i++) {
        v_r[i] = v_l[i] + (vn_r - vn_l) * n[i];
        vs = vs + (v_r[i] * v_r[i]);
      }
      e_r = (p_r / (g - T(1.0))) + T(0.5) * rho_r * vs;
      break;
    }
    case 5:                                   // sup_in
      rho_r = rho_bound;
#pragma unroll
      for (int i = 0; i < D; i++) v_r[i] = ph.bdy[1 + i];
      p_r = p_bound;
      energy();
      break;
    case 6:                                   // sup_out
      rho_r = rho_l;
#pragma unroll
      for (int i = 0; i < D; i++) v_r[i] = v_l[i];
      e_r = e_l;
      break;
    case 7:                                   // slip_wall
      rho_r = rho_l;
      vn_l = T(0.);
#pragma unroll
      for (int i = 0; i < D; i++) vn_l = vn_l + (v_l[i] - T(0.0)) * n[i];
#pragma unroll
      for (int i = 0; i < D; i++) v_r[i] = v_l[i] - T(2.0) * vn_l * n[i];
      e_r = e_l;
      break;
    case 11: case 13:                         // isotherm_fix, isotherm_move
      p_r = p_l;
      rho_r = p_r / (R_ref * T_wall);
#pragma unroll
      for (int i = 0; i < D; i++) v_r[i] = type == 11 ? T(0.0) : ph.bdy[5 + i] + T(0.0);
      energy();
      break;
    case 12: case 14:                         // adiabat_fix, adiabat_move
      rho_r = rho_l;
      p_r = p_l;
#pragma unroll
      for (int i = 0; i < D; i++) v_r[i] = type == 12 ? T(0.0) : ph.bdy[5 + i] + T(0.0);
      energy();
      break;
    case 15: {                                // char
      vn_l = T(0.);
#pragma unroll
      for (int i = 0; i < D; i++) vn_l = vn_l + v_l[i] * n[i];
      T vn_bound = T(0);
#pragma unroll
      for (int i = 0; i < D; i++) vn_bound = vn_bound + ph.bdy[1 + i] * n[i];
      const T r_plus = vn_l + T(2.) / (g - T(1.)) * fr_sqrt<T>(g * p_l / rho_l);
      const T r_minus = vn_bound - T(2.) / (g - T(1.)) * fr_sqrt<T>(g * p_bound / rho_bound);
      const T c_star = T(0.25) * (g - T(1.)) * (r_plus - r_minus);
      const T vn_star = T(0.5) * (r_plus + r_minus);
      if (vn_l < T(0)) {
        const T one_over_s = fr_pow<T>(rho_bound, g) / p_bound;
        T vs = T(0.);
#pragma unroll
        for (int i = 0; i < D; i++) vs = vs + ph.bdy[1 + i] * ph.bdy[1 + i];
        const T h_free_stream = g / (g - T(1.)) * p_bound / rho_bound + T(0.5) * vs;
        rho_r = fr_pow<T>(T(1.) / g * (one_over_s * c_star * c_star), T(1.) / (g - T(1.)));
#pragma unroll
        for (int i = 0; i < D; i++) v_r[i] = vn_star * n[i] + (ph.bdy[1 + i] - vn_bound * n[i]);
        p_r = rho_r / g * c_star * c_star;
        e_r = rho_r * h_free_stream - p_r;
      } else {
        const T one_over_s = fr_pow<T>(rho_l, g) / p_l;
        rho_r = fr_pow<T>(T(1.) / g * (one_over_s * c_star * c_star), T(1.) / (g - T(1.)));
#pragma unroll
        for (int i = 0; i < D; i++) v_r[i] = vn_star * n[i] + (v_l[i] - vn_l * n[i]);
        p_r = rho_r / g * c_star * c_star;
        energy();
      }
      break;
    }
    default:                                  // 16 slip_wall_dual
      rho_r = rho_l;
      vn_l = T(0.);
#pragma unroll
      for (int i = 0; i < D; i++) vn_l = vn_l + v_l[i] * n[i];
#pragma unroll
      for (int i = 0; i < D; i++) v_r[i] = v_l[i] - vn_l * n[i];
      e_r = e_l;
      break;
  }
  ur[0] = rho_r;
#pragma unroll
  for (int i = 0; i < D; i++) ur[i + 1] = rho_r * v_r[i];
  ur[D + 1] = e_r;
}

// Energy gradient of the ghost side at adiabatic walls (12, 14): no
// temperature gradient, bdy_inters::set_vis_boundary_conditions,
// src/bdy_inters.cpp:1062-1113.  g[k][d]: copy of the own gradient, changed in place.
template <int D, typename T>
__device__ __forceinline__ void bc_vis_gradient(const PhysT<T>& ph, const T* ul, const T* ur, T (*g)[D])
{
  T v_sq = T(0.);
#pragma unroll
  for (int i = 0; i < D; i++) v_sq = v_sq + (ul[i + 1] * ul[i + 1]);
  const T p_l = (ph.gamma - T(1.0)) * (ul[D + 1] - T(0.5) * v_sq / ul[0]);
  const T inte = p_l / ((ph.gamma - T(1.0)) * ur[0]);
  T gv[D][D];
#pragma unroll
  for (int j = 0; j < D; j++)
#pragma unroll
    for (int i = 0; i < D; i++) gv[j][i] = (g[j + 1][i] - g[0][i] * ur[j + 1] / ur[0]) / ur[0];
  T ke = ur[1] * ur[1];
#pragma unroll
  for (int j = 1; j < D; j++) ke = ke + ur[j + 1] * ur[j + 1];
#pragma unroll
  for (int i = 0; i < D; i++) {
    T w = (ur[1] / ur[0]) * gv[0][i];
#pragma unroll
    for (int j = 1; j < D; j++) w = w + (ur[j + 1] / ur[0]) * gv[j][i];
    g[D + 1][i] = inte * g[0][i] + T(0.5) * (ke / (ur[0] * ur[0])) * g[0][i] + ur[0] * w;
  }
}

// Sign of the LDG penalty: one fixed direction per interface point, taken
// from the left normal (src/inters.cpp:555-564, 651-660).
template <int D, typename T>
__device__ __forceinline__ T ldg_beta(T pen, const T* n)
{
  T s = (D == 2) ? (n[0] + n[1]) : (n[0] + n[1] + T(1.4142135623730951) * n[2]);
  return s < T(0) ? -pen : pen;
}

// Projection of a viscous flux on the left normal: a_k = f_k . n.
template <int D, typename T>
__device__ __forceinline__ T project(T (*f)[D], int k, const T* n)
{
  T a = f[k][0] * n[0];
#pragma unroll
  for (int l = 1; l < D; l++) a = fr_fma(f[k][l], n[l], a);
  return a;
}

// LDG common normal viscous flux of an interior interface point from the two
// sides' normal projections aL = fL.n, aR = fR.n (inters::ldg_flux with
// flux_spec 0, src/inters.cpp:550-641):
//   f_c.n = (fL+fR)/2 . n + pen (n.n) (fL-fR).n + tau (n.n) (uL-uR)
// which is the reference's component form summed against n.
template <typename T>
__device__ __forceinline__ T ldg_normal(T aL, T aR, T uL, T uR, T pen, T tau, T nn)
{
  return fr_fma(fr_fma(pen, aL - aR, tau * (uL - uR)), nn, T(0.5) * (aL + aR));
}

// LDG common normal viscous flux from full fluxes (component form), for the
// per-operator path where both sides' gradients are at hand.
template <int D, typename T>
__device__ __forceinline__ void ldg_flux(const PhysT<T>& ph, T pen, const T* ul, const T* ur, T (*fl)[D],
                                         T (*fr)[D], const T* n, T* fn)
{
  constexpr int F = D + 2;
#pragma unroll
  for (int k = 0; k < F; k++) {
    T jump = n[0] * (fl[k][0] - fr[k][0]);
#pragma unroll
    for (int l = 1; l < D; l++) jump = jump + n[l] * (fl[k][l] - fr[k][l]);
    T du = ul[k] - ur[k];
    T acc = T(0);
#pragma unroll
    for (int l = 0; l < D; l++) {
      T fc = T(0.5) * (fl[k][l] + fr[k][l]) + pen * n[l] * (jump) + ph.tau * n[l] * du;
      acc = (l == 0) ? fc * n[0] : acc + fc * n[l];
    }
    fn[k] = acc;
  }
}

// Subgrid-scale flux of the eddy-viscosity LES models at a solution point
// (eles::calc_sgsf_upts with sgs_model 0 = Smagorinsky, Cs = 0.1, or 1 =
// WALE, Cw = 0.5; no wall model; src/eles.cpp:2456-2778), physical
// components fs[k][l].  g is the physical gradient g[k][l] = d q_k / d x_l,
// detjac the Jacobian determinant at the point, n1 = order + 1.
// sgs_model 5 is the learned closure of fr_mlp.cuh (no reference counterpart).
//
// Two index choices of the reference are kept as it evaluates them: its
// "velocity" vector is u_i = q_i / rho for i < D, so u_0 = rho / rho
// (src/eles.cpp:2483), and its velocity gradient subtracts u_j drho_j
// (src/eles.cpp:2656).  Both enter only the energy flux through the
// kinetic-energy gradient (the first also the internal energy); the strain
// rate and hence the eddy viscosity see the second alone.  The filter width
// is delta = filter_ratio vol^(1/D) / (order + 1) with vol = 2^D detjac
// (eles_quads / eles_hexas::calc_ele_vol); the turbulent Prandtl number 0.5.
// The WALE powers x^2.5, x^1.25, x^1.5 are taken through square roots.
template <int D, typename T>
__device__ __forceinline__ void sgs_flux(const PhysT<T>& ph, const T* q, const T (*g)[D], T detjac, T n1,
                                         T (*fs)[D])
{
  if (ph.sgs_model == 5) {
    sgs_flux_learned<D, T>(ph.mlp, ph.gamma, q, g, detjac, n1, ph.filter_ratio, fs);
    return;
  }
  constexpr int F = D + 2;
  const T rho = q[0];
  T u[D], ke = T(0);
#pragma unroll
  for (int i = 0; i < D; i++) {
    u[i] = q[i] / rho;
    ke = ke + T(0.5) * (u[i] * u[i]);
  }
  const T inte = q[F - 1] / rho - ke;
  const T vol = detjac * T(D == 3 ? 8 : 4);
  T root;
  if (D == 3) root = (T)cbrt(vol);
  else root = fr_sqrt<T>(vol);
  const T delta = ph.filter_ratio * root / n1;
  T du[D][D], de[D];
#pragma unroll
  for (int i = 0; i < D; i++) {
    T dke = ke * g[0][i];
#pragma unroll
    for (int j = 0; j < D; j++) {
      du[i][j] = (g[j + 1][i] - u[j] * g[0][j]) / rho;
      dke = dke + rho * u[j] * du[i][j];
    }
    de[i] = (g[F - 1][i] - dke - g[0][i] * inte) / rho;
  }
  T S[D][D], diag = T(0);
#pragma unroll
  for (int i = 0; i < D; i++) {
#pragma unroll
    for (int j = 0; j < D; j++) S[i][j] = (du[i][j] + du[j][i]) / T(2);
    diag = diag + S[i][i] / T(3);
  }
#pragma unroll
  for (int i = 0; i < D; i++) S[i][i] = S[i][i] - diag;
  T mu_t;
  if (ph.sgs_model == 0) {
    T s2 = T(0);
#pragma unroll
    for (int i = 0; i < D; i++)
#pragma unroll
      for (int j = 0; j < D; j++) s2 = s2 + T(2) * S[i][j] * S[i][j];
    const T Cs = T(0.1);
    mu_t = rho * Cs * Cs * delta * delta * fr_sqrt<T>(s2);
  } else {
    T Sq[D][D], dg = T(0);
#pragma unroll
    for (int i = 0; i < D; i++)
#pragma unroll
      for (int j = 0; j < D; j++) {
        T a = T(0);
#pragma unroll
        for (int k = 0; k < D; k++) a = a + (du[i][k] * du[k][j] + du[j][k] * du[k][i]) / T(2);
        Sq[i][j] = a;
        dg = dg + du[i][j] * du[j][i] / T(3);
      }
#pragma unroll
    for (int i = 0; i < D; i++) Sq[i][i] = Sq[i][i] - dg;
    T num = T(0), den = T(0);
#pragma unroll
    for (int i = 0; i < D; i++)
#pragma unroll
      for (int j = 0; j < D; j++) {
        num = num + Sq[i][j] * Sq[i][j];
        den = den + S[i][j] * S[i][j];
      }
    const T sn = fr_sqrt<T>(num);
    const T denom = den * den * fr_sqrt<T>(den) + num * fr_sqrt<T>(sn);
    const T Cs = T(0.5);
    mu_t = rho * Cs * Cs * delta * delta * (num * sn) / (denom + T(1.e-12));
  }
  const T Pr = T(0.5);
#pragma unroll
  for (int j = 0; j < D; j++) {
    fs[0][j] = T(0);
    fs[F - 1][j] = -ph.gamma * mu_t / Pr * de[j];
#pragma unroll
    for (int i = 1; i < F - 1; i++) fs[i][j] = T(-2) * mu_t * S[i - 1][j];
  }
}

}  // namespace frb
