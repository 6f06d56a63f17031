// fr_physics.cuh -- pointwise Euler / Navier-Stokes physics of the FR path,
// device side.  Templated on the compute type T (double for the FP64 form,
// float for the FP32 form) and the number of dimensions D (F = D + 2 fields).
//
// Formulas follow the reference's CPU routines; the operation order is kept
// where it is cheap to keep, so the FP64 form agrees with the reference to a
// few ulp (contractions into FMA are allowed).
#pragma once

#include <cuda_runtime.h>

namespace frb {

struct Phys {
  double gamma, prandtl, mu_inf, rt_inf, c_sth, fix_vis, tau, pen_fact;
};

template <typename T>
struct PhysT {
  T gamma, gm1, prandtl, mu_inf, rt_inf, c_sth, fix_vis, tau, pen_fact;
  __host__ __device__ static PhysT make(const Phys& p) {
    PhysT q;
    q.gamma = (T)p.gamma; q.gm1 = (T)(p.gamma - 1.0); q.prandtl = (T)p.prandtl; q.mu_inf = (T)p.mu_inf;
    q.rt_inf = (T)p.rt_inf; q.c_sth = (T)p.c_sth; q.fix_vis = (T)p.fix_vis; q.tau = (T)p.tau;
    q.pen_fact = (T)p.pen_fact;
    return q;
  }
};

__device__ __forceinline__ double ffma(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float ffma(float a, float b, float c) { return fmaf(a, b, c); }

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
  T rinv = T(1) / u[0];
  T v[D];
#pragma unroll
  for (int l = 0; l < D; l++) v[l] = u[l + 1] * rinv;
  T ke = T(0);
#pragma unroll
  for (int l = 0; l < D; l++) ke += v[l] * v[l];
  T p = ph.gm1 * (u[F - 1] - (T(0.5) * u[0] * ke));
#pragma unroll
  for (int l = 0; l < D; l++) {
    f[0][l] = u[l + 1];
#pragma unroll
    for (int m = 0; m < D; m++) f[m + 1][l] = u[m + 1] * v[l] + (m == l ? p : T(0));
    f[F - 1][l] = v[l] * (u[F - 1] + p);
  }
}

// Viscous flux (no turbulence model): calc_visf_2d / calc_visf_3d,
// src/flux.cpp:132-431.  With fix_vis == 1 the Sutherland value is replaced by
// mu_inf, which is what mu + fix_vis*(mu_inf - mu) evaluates to.
template <int D, typename T>
__device__ __forceinline__ void vis_flux(const PhysT<T>& ph, const T* u, T (*g)[D], T (*f)[D])
{
  constexpr int F = D + 2;
  T rho = u[0], rinv = T(1) / rho;
  T v[D];
#pragma unroll
  for (int l = 0; l < D; l++) v[l] = u[l + 1] * rinv;
  T ke = T(0);
#pragma unroll
  for (int l = 0; l < D; l++) ke += v[l] * v[l];
  T inte = u[F - 1] * rinv - T(0.5) * ke;
  T mu;
  if (ph.fix_vis == T(1)) {
    mu = ph.mu_inf;
  } else {
    T rt = ph.gm1 * inte / ph.rt_inf;
    mu = ph.mu_inf * fr_pow15<T>(rt) * (T(1) + ph.c_sth) / (rt + ph.c_sth);
    mu = mu + ph.fix_vis * (ph.mu_inf - mu);
  }
  // velocity gradients dv[m][l] = d v_m / d x_l
  T dv[D][D];
#pragma unroll
  for (int m = 0; m < D; m++)
#pragma unroll
    for (int l = 0; l < D; l++) dv[m][l] = (g[m + 1][l] - g[0][l] * v[m]) * rinv;
  T de[D];
#pragma unroll
  for (int l = 0; l < D; l++) {
    T vdv = T(0);
#pragma unroll
    for (int m = 0; m < D; m++) vdv += v[m] * dv[m][l];
    T dke = T(0.5) * ke * g[0][l] + rho * vdv;
    de[l] = (g[F - 1][l] - dke - g[0][l] * inte) * rinv;
  }
  T div = T(0);
#pragma unroll
  for (int l = 0; l < D; l++) div += dv[l][l];
  T diag = div / T(3);
  T kt = (mu / ph.prandtl) * ph.gamma;
  T tau[D][D];
#pragma unroll
  for (int m = 0; m < D; m++)
#pragma unroll
    for (int l = 0; l < D; l++)
      tau[m][l] = (m == l) ? T(2) * mu * (dv[m][m] - diag) : mu * (dv[m][l] + dv[l][m]);
#pragma unroll
  for (int l = 0; l < D; l++) {
    f[0][l] = T(0);
    T w = T(0);
#pragma unroll
    for (int m = 0; m < D; m++) {
      f[m + 1][l] = -tau[m][l];
      w += v[m] * tau[m][l];
    }
    f[F - 1][l] = -(w + kt * de[l]);
  }
}

// Rusanov common normal flux for a static mesh: inters::rusanov_flux,
// src/inters.cpp:311-365.
template <int D, typename T>
__device__ __forceinline__ void rusanov(const PhysT<T>& ph, const T* ul, const T* ur, const T* n, T* fn)
{
  constexpr int F = D + 2;
  T fl[F][D], fr[F][D];
  inv_flux<D, T>(ph, ul, fl);
  inv_flux<D, T>(ph, ur, fr);
  T vnl = T(0), vnr = T(0), kl = T(0), kr = T(0);
  T il = T(1) / ul[0], ir = T(1) / ur[0];
#pragma unroll
  for (int l = 0; l < D; l++) {
    T a = ul[l + 1] * il, b = ur[l + 1] * ir;
    vnl += a * n[l]; vnr += b * n[l]; kl += a * a; kr += b * b;
  }
  T pl = ph.gm1 * (ul[F - 1] - T(0.5) * ul[0] * kl);
  T pr = ph.gm1 * (ur[F - 1] - T(0.5) * ur[0] * kr);
  T vav = fr_sqrt<T>(T(0.25) * (vnl + vnr) * (vnl + vnr));
  T cav = fr_sqrt<T>((ph.gamma * (pl + pr)) / (ul[0] + ur[0]));
  T eig = fr_abs<T>(vav + cav);
#pragma unroll
  for (int k = 0; k < F; k++) {
    T a = T(0), b = T(0);
#pragma unroll
    for (int l = 0; l < D; l++) { a += fl[k][l] * n[l]; b += fr[k][l] * n[l]; }
    fn[k] = T(0.5) * ((a + b) - eig * (ur[k] - ul[k]));
  }
}

// LDG sign switch of the penalty: a fixed direction per interface point taken
// from the left normal, src/inters.cpp:555-564, 651-660.
template <int D, typename T>
__device__ __forceinline__ T ldg_beta(T pen, const T* n)
{
  T s = (D == 2) ? (n[0] + n[1]) : (n[0] + n[1] + T(1.4142135623730951) * n[2]);
  return s < T(0) ? -pen : pen;
}

// LDG common normal viscous flux for an interior interface: inters::ldg_flux
// (flux_spec 0), src/inters.cpp:550-641.  pen is the signed penalty of
// ldg_beta, passed in so both sides of an interface use the same sign.
template <int D, typename T>
__device__ __forceinline__ void ldg_flux(const PhysT<T>& ph, T pen, const T* ul, const T* ur, T (*fl)[D],
                                         T (*fr)[D], const T* n, T* fn)
{
  constexpr int F = D + 2;
#pragma unroll
  for (int k = 0; k < F; k++) {
    T jump = T(0);
#pragma unroll
    for (int l = 0; l < D; l++) jump += n[l] * (fl[k][l] - fr[k][l]);
    T du = ul[k] - ur[k];
    T acc = T(0);
#pragma unroll
    for (int l = 0; l < D; l++) {
      T fc = T(0.5) * (fl[k][l] + fr[k][l]) + pen * n[l] * jump + ph.tau * n[l] * du;
      acc += fc * n[l];
    }
    fn[k] = acc;
  }
}

}  // namespace frb
