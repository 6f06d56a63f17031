// fr_mlp.cuh -- the learned subgrid-scale closure: a 6-64-64-1 multilayer
// perceptron (tanh, tanh, softplus) in FP32 that gives the eddy-viscosity
// coefficient c >= 0 of mu_t = rho * Delta^2 * |S| * c from five invariants of
// the resolved velocity gradient and the filter width.  The reference has no
// such model: its eddy-viscosity models are Smagorinsky and WALE
// (eles::calc_sgsf_upts, src/eles.cpp:2456-2778); this one plugs into the
// same flux, with the same turbulent Prandtl number (0.5) and the same
// filter width Delta = filter_ratio * vol^(1/D) / (order + 1).
//
// Parameter vector (floats), in this order:
//   W1[64][6], b1[64], W2[64][64], b2[64], w3[64], b3      (trained, 4673)
//   xmean[6], xscale[6]    input normalisation x_n = (x - xmean) * xscale
#pragma once

#include <cuda_runtime.h>

namespace frb {

constexpr int kMlpIn = 6, kMlpH = 64;
constexpr int kMlpW1 = 0;
constexpr int kMlpB1 = kMlpW1 + kMlpH * kMlpIn;
constexpr int kMlpW2 = kMlpB1 + kMlpH;
constexpr int kMlpB2 = kMlpW2 + kMlpH * kMlpH;
constexpr int kMlpW3 = kMlpB2 + kMlpH;
constexpr int kMlpB3 = kMlpW3 + kMlpH;
constexpr int kMlpTrain = kMlpB3 + 1;            // 4673 trained parameters
constexpr int kMlpXm = kMlpTrain;
constexpr int kMlpXs = kMlpXm + kMlpIn;
constexpr int kMlpN = kMlpXs + kMlpIn;           // 4685 floats in all

__device__ __forceinline__ float mlp_softplus(float o) { return o > 20.f ? o : log1pf(expf(o)); }

// c = softplus(w3 . tanh(W2 tanh(W1 x_n + b1) + b2) + b3); every thread of a
// warp reads the same weights, so the loads are broadcasts.
__device__ __forceinline__ float mlp_eval(const float* __restrict__ w, const float* xr)
{
  float x[kMlpIn];
#pragma unroll
  for (int k = 0; k < kMlpIn; k++) x[k] = (xr[k] - __ldg(w + kMlpXm + k)) * __ldg(w + kMlpXs + k);
  float h1[kMlpH];
#pragma unroll
  for (int i = 0; i < kMlpH; i++) {
    float a = __ldg(w + kMlpB1 + i);
#pragma unroll
    for (int k = 0; k < kMlpIn; k++) a = fmaf(__ldg(w + kMlpW1 + i * kMlpIn + k), x[k], a);
    h1[i] = tanhf(a);
  }
  float o = __ldg(w + kMlpB3);
  for (int j = 0; j < kMlpH; j++) {
    float a = __ldg(w + kMlpB2 + j);
#pragma unroll
    for (int i = 0; i < kMlpH; i++) a = fmaf(__ldg(w + kMlpW2 + j * kMlpH + i), h1[i], a);
    o = fmaf(__ldg(w + kMlpW3 + j), tanhf(a), o);
  }
  return mlp_softplus(o);
}

// Inputs of the closure at one point from the conserved state q and its
// physical gradient g[k][l] = d q_k / d x_l.  With A_ij = d u_i / d x_j,
// S the deviatoric symmetric part and W the antisymmetric part of A, and
// a2 = sum A_ij^2:
//   x = ( tr S^2 / a2, tr W^2 / a2, tr S^3 / a2^1.5, tr S W^2 / a2^1.5,
//         tr S^2 W^2 / a2^2, log Delta )
// Also returns Delta, the deviatoric strain S, |S| = sqrt(2 S:S) and the
// internal-energy gradient de (for the SGS heat flux).
template <int D, typename T>
__device__ __forceinline__ void sgs_learned_inputs(const T* q, const T (*g)[D], T detjac, T n1, T filter_ratio,
                                                   float* x, T& delta, T (*S)[D], T& smag, T* de)
{
  constexpr int F = D + 2;
  const T rho = q[0];
  T u[D], ke = T(0);
#pragma unroll
  for (int i = 0; i < D; i++) {
    u[i] = q[i + 1] / rho;
    ke = ke + T(0.5) * u[i] * u[i];
  }
  const T inte = q[F - 1] / rho - ke;
  T A[D][D];
#pragma unroll
  for (int i = 0; i < D; i++)
#pragma unroll
    for (int j = 0; j < D; j++) A[i][j] = (g[i + 1][j] - u[i] * g[0][j]) / rho;
#pragma unroll
  for (int j = 0; j < D; j++) {
    T ud = T(0);
#pragma unroll
    for (int i = 0; i < D; i++) ud = ud + u[i] * A[i][j];
    de[j] = (g[F - 1][j] - ke * g[0][j] - rho * ud - g[0][j] * inte) / rho;
  }
  T W[D][D], tr = T(0), a2 = T(0);
#pragma unroll
  for (int i = 0; i < D; i++) tr = tr + A[i][i];
#pragma unroll
  for (int i = 0; i < D; i++)
#pragma unroll
    for (int j = 0; j < D; j++) {
      S[i][j] = T(0.5) * (A[i][j] + A[j][i]) - (i == j ? tr / T(3) : T(0));
      W[i][j] = T(0.5) * (A[i][j] - A[j][i]);
      a2 = a2 + A[i][j] * A[i][j];
    }
  a2 = a2 + T(1e-30);
  T S2[D][D], W2[D][D];
#pragma unroll
  for (int i = 0; i < D; i++)
#pragma unroll
    for (int j = 0; j < D; j++) {
      T s = T(0), w = T(0);
#pragma unroll
      for (int k = 0; k < D; k++) { s = s + S[i][k] * S[k][j]; w = w + W[i][k] * W[k][j]; }
      S2[i][j] = s; W2[i][j] = w;
    }
  T trS2 = T(0), trW2 = T(0), trS3 = T(0), trSW2 = T(0), trS2W2 = T(0);
#pragma unroll
  for (int i = 0; i < D; i++)
#pragma unroll
    for (int j = 0; j < D; j++) {
      trS2 = trS2 + S[i][j] * S[j][i];
      trW2 = trW2 + W[i][j] * W[j][i];
      trS3 = trS3 + S2[i][j] * S[j][i];
      trSW2 = trSW2 + S[i][j] * W2[j][i];
      trS2W2 = trS2W2 + S2[i][j] * W2[j][i];
    }
  const T ra = T(1) / a2, ra15 = ra / sqrt(a2);
  x[0] = (float)(trS2 * ra);
  x[1] = (float)(trW2 * ra);
  x[2] = (float)(trS3 * ra15);
  x[3] = (float)(trSW2 * ra15);
  x[4] = (float)(trS2W2 * ra * ra);
  const T vol = detjac * T(D == 3 ? 8 : 4);
  const T root = D == 3 ? (T)cbrt(vol) : (T)sqrt(vol);
  delta = filter_ratio * root / n1;
  x[5] = (float)log(delta);
  smag = sqrt(T(2) * trS2);
}

// SGS flux of the learned closure: mu_t = rho Delta^2 |S| c(x); momentum
// -2 mu_t S, energy -gamma mu_t / 0.5 de (the flux form of calc_sgsf_upts).
template <int D, typename T>
__device__ __forceinline__ void sgs_flux_learned(const float* __restrict__ w, T gamma, const T* q, const T (*g)[D],
                                                 T detjac, T n1, T filter_ratio, T (*fs)[D])
{
  constexpr int F = D + 2;
  float x[kMlpIn];
  T delta, S[D][D], smag, de[D];
  sgs_learned_inputs<D, T>(q, g, detjac, n1, filter_ratio, x, delta, S, smag, de);
  const T c = (T)mlp_eval(w, x);
  const T mu_t = q[0] * delta * delta * smag * c;
#pragma unroll
  for (int j = 0; j < D; j++) {
    fs[0][j] = T(0);
    fs[F - 1][j] = -gamma * mu_t / T(0.5) * de[j];
#pragma unroll
    for (int i = 1; i < F - 1; i++) fs[i][j] = T(-2) * mu_t * S[i - 1][j];
  }
}

}  // namespace frb
