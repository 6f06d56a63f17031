// fr_diag.cu -- integral diagnostics on the device: the quantities of
// eles::CalcIntegralQuantities (src/eles.cpp:6503-6641) -- kinetic energy,
// enstrophy (the reference's "vorticity": rho |w|^2 / 2), pressure
// dilatation, strain colon product and its deviatoric form -- on the
// reference's volume cubature: the state and its corrected gradient are
// interpolated to each cubature point with the dense nodal-basis rows
// opp_volume_cubpts (column order, as the reference's loop), the quantities
// are formed with the reference's expressions, and weight x detJ at the
// cubature point integrates them.  One thread per (element, cubature point)
// writes per-block partial sums; fr_diag_finalize adds them in block order,
// so the result does not depend on scheduling.
#include <cuda_runtime.h>

namespace frb {

constexpr int kDiagQ = 5;

// NQ 5: all five quantities (G, the corrected gradient (nu, E, F, D), is
// read); NQ 1: the kinetic energy alone (G unused).
template <int D, typename TG, int NQ>
__global__ void __launch_bounds__(256)
fr_diag_kernel(const double* __restrict__ U, const TG* __restrict__ G, const double* __restrict__ opp,
               const double* __restrict__ W, const double* __restrict__ detj, long long E, int nu, int nc,
               double gamma, double* __restrict__ partial)
{
  constexpr int F = D + 2;
  __shared__ double red[NQ][256 / 32];
  double acc[NQ];
#pragma unroll
  for (int q = 0; q < NQ; q++) acc[q] = 0.0;
  const long long npts = E * nc;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < npts; i += (long long)gridDim.x * blockDim.x) {
    const long long e = i / nc;
    const int j = (int)(i - e * nc);
    double u[F], g[F][D];
#pragma unroll
    for (int m = 0; m < F; m++) {
      double s = 0.;
      for (int k = 0; k < nu; k++) s += opp[j + (size_t)nc * k] * U[k + nu * (e + E * m)];
      u[m] = s;
    }
    if (NQ > 1) {
#pragma unroll
      for (int m = 0; m < F; m++)
#pragma unroll
        for (int n = 0; n < D; n++) {
          double s = 0.;
          for (int k = 0; k < nu; k++) s += opp[j + (size_t)nc * k] * (double)G[k + nu * (e + E * (m + (long long)F * n))];
          g[m][n] = s;
        }
    }
    const double wj = W[j], dj = detj[j + (size_t)nc * e];
    const double irho = 1. / u[0];
    double tke = 0.0;
#pragma unroll
    for (int n = 1; n < F - 1; n++) tke += 0.5 * u[n] * u[n];
    acc[0] += irho * tke * wj * dj;
    if (NQ > 1) {
      const double dudx = irho * (g[1][0] - u[1] * irho * g[0][0]);
      const double dudy = irho * (g[1][1] - u[1] * irho * g[0][1]);
      const double dvdx = irho * (g[2][0] - u[2] * irho * g[0][0]);
      const double dvdy = irho * (g[2][1] - u[2] * irho * g[0][1]);
      double dudz = 0, dvdz = 0, dwdx = 0, dwdy = 0, dwdz = 0;
      if (D == 3) {
        dudz = irho * (g[1][D - 1] - u[1] * irho * g[0][D - 1]);
        dvdz = irho * (g[2][D - 1] - u[2] * irho * g[0][D - 1]);
        dwdx = irho * (g[D][0] - u[D] * irho * g[0][0]);
        dwdy = irho * (g[D][1] - u[D] * irho * g[0][1]);
        dwdz = irho * (g[D][D - 1] - u[D] * irho * g[0][D - 1]);
      }
      // vorticity: rho |w|^2 / 2
      const double wz = dvdx - dudy;
      double vort = wz * wz;
      if (D == 3) {
        const double wx = dwdy - dvdz, wy = dudz - dwdx;
        vort += wx * wx + wy * wy;
      }
      vort *= 0.5 / irho;
      // pressure dilatation
      const double pressure = (gamma - 1.0) * (u[F - 1] - irho * tke);
      const double pd = D == 2 ? pressure * (dudx + dvdy) : pressure * (dudx + dvdy + dwdz);
      // strain-rate colon products
      double S[3][3];
      S[0][0] = dudx;
      S[0][1] = (dudy + dvdx) / 2.0;
      S[1][0] = S[0][1];
      S[1][1] = dvdy;
      double diag = (S[0][0] + S[1][1]) / 3.0;
      if (D == 3) {
        S[0][2] = (dudz + dwdx) / 2.0;
        S[1][2] = (dvdz + dwdy) / 2.0;
        S[2][0] = S[0][2];
        S[2][1] = S[1][2];
        S[2][2] = dwdz;
        diag += S[2][2] / 3.0;
      }
      double sc = 0.0, dsc = 0.0;
#pragma unroll
      for (int a = 0; a < D; a++)
#pragma unroll
        for (int b = 0; b < D; b++) sc += S[a][b] * S[a][b];
#pragma unroll
      for (int a = 0; a < D; a++) S[a][a] -= diag;
#pragma unroll
      for (int a = 0; a < D; a++)
#pragma unroll
        for (int b = 0; b < D; b++) dsc += S[a][b] * S[a][b];
      acc[1] += vort * wj * dj;
      acc[2 % NQ] += pd * wj * dj;
      acc[3 % NQ] += sc * wj * dj;
      acc[4 % NQ] += dsc * wj * dj;
    }
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NQ; q++) {
    double v = acc[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[q][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < NQ) {
    double v = 0.0;
    for (int w = 0; w < 256 / 32; w++) v += red[threadIdx.x][w];
    partial[(size_t)blockIdx.x * NQ + threadIdx.x] = v;
  }
}

__global__ void fr_diag_finalize(const double* __restrict__ partial, int nblk, int nq, double* __restrict__ out)
{
  if (threadIdx.x >= nq) return;
  double v = 0.0;
  for (int b = 0; b < nblk; b++) v += partial[(size_t)b * nq + threadIdx.x];
  out[threadIdx.x] = v;
}

// G null: the kinetic energy alone (out[0]); otherwise all five quantities.
cudaError_t launch_diagnostics(int dims, int tc_size, const double* U, const void* G, const double* opp,
                               const double* W, const double* detj, long long E, int nu, int nc, double gamma,
                               double* partial, int nblk, double* out, cudaStream_t st)
{
  if (!G) {
    if (dims == 2) fr_diag_kernel<2, double, 1><<<nblk, 256, 0, st>>>(U, nullptr, opp, W, detj, E, nu, nc, gamma, partial);
    else fr_diag_kernel<3, double, 1><<<nblk, 256, 0, st>>>(U, nullptr, opp, W, detj, E, nu, nc, gamma, partial);
    fr_diag_finalize<<<1, 32, 0, st>>>(partial, nblk, 1, out);
    return cudaGetLastError();
  }
  if (dims == 2 && tc_size == 8)
    fr_diag_kernel<2, double, 5><<<nblk, 256, 0, st>>>(U, (const double*)G, opp, W, detj, E, nu, nc, gamma, partial);
  else if (dims == 2)
    fr_diag_kernel<2, float, 5><<<nblk, 256, 0, st>>>(U, (const float*)G, opp, W, detj, E, nu, nc, gamma, partial);
  else if (tc_size == 8)
    fr_diag_kernel<3, double, 5><<<nblk, 256, 0, st>>>(U, (const double*)G, opp, W, detj, E, nu, nc, gamma, partial);
  else
    fr_diag_kernel<3, float, 5><<<nblk, 256, 0, st>>>(U, (const float*)G, opp, W, detj, E, nu, nc, gamma, partial);
  fr_diag_finalize<<<1, 32, 0, st>>>(partial, nblk, kDiagQ, out);
  return cudaGetLastError();
}

}  // namespace frb
