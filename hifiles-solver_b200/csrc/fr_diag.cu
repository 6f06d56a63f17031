// fr_diag.cu -- integral diagnostics on the device: the quantities of
// eles::CalcIntegralQuantities (src/eles.cpp:6503-6641) -- kinetic energy,
// enstrophy (the reference's "vorticity": rho |w|^2 / 2), pressure
// dilatation, strain colon product and its deviatoric form -- integrated with
// the tensor Gauss rule of the solution points (weights w_a w_b (w_c) times
// detJ), from the current state and its corrected gradient.  One pass over
// the points writes per-block partial sums; fr_diag_finalize adds them in
// block order, so the result does not depend on scheduling.
#include <cuda_runtime.h>

namespace frb {

constexpr int kDiagQ = 5;

template <int D, typename TG>
__global__ void __launch_bounds__(256) fr_diag_kernel(const double* __restrict__ U, const TG* __restrict__ G,
                                                      const double* __restrict__ detj,
                                                      const double* __restrict__ W, long long npts, int nu,
                                                      double gamma, double* __restrict__ partial)
{
  constexpr int F = D + 2;
  __shared__ double red[kDiagQ][256 / 32];
  double acc[kDiagQ] = {0, 0, 0, 0, 0};
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < npts; i += (long long)gridDim.x * blockDim.x) {
    double q[F], g[F][D];
#pragma unroll
    for (int k = 0; k < F; k++) {
      q[k] = U[i + npts * k];
#pragma unroll
      for (int d = 0; d < D; d++) g[k][d] = (double)G[i + npts * (k + (long long)F * d)];
    }
    const double irho = 1. / q[0];
    double A[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};   // A[i][j] = d u_i / d x_j
#pragma unroll
    for (int a = 0; a < D; a++)
#pragma unroll
      for (int b = 0; b < D; b++) A[a][b] = irho * (g[a + 1][b] - q[a + 1] * irho * g[0][b]);
    double tke = 0.0;
#pragma unroll
    for (int n = 1; n < F - 1; n++) tke += 0.5 * q[n] * q[n];
    const double ke = irho * tke;
    double wz = A[1][0] - A[0][1], en = wz * wz;
    if (D == 3) {
      const double wx = A[2][1] - A[1][2], wy = A[0][2] - A[2][0];
      en += wx * wx + wy * wy;
    }
    en *= 0.5 / irho;
    const double pressure = (gamma - 1.0) * (q[F - 1] - irho * tke);
    double div = A[0][0] + A[1][1];
    if (D == 3) div += A[2][2];
    const double pd = pressure * div;
    double S[3][3], sc = 0.0, dsc = 0.0;
#pragma unroll
    for (int a = 0; a < D; a++)
#pragma unroll
      for (int b = 0; b < D; b++) S[a][b] = a == b ? A[a][a] : (A[a][b] + A[b][a]) / 2.0;
    double diag = 0.0;
#pragma unroll
    for (int a = 0; a < D; a++) diag += S[a][a] / 3.0;
#pragma unroll
    for (int a = 0; a < D; a++)
#pragma unroll
      for (int b = 0; b < D; b++) {
        sc += S[a][b] * S[a][b];
        const double s = a == b ? S[a][b] - diag : S[a][b];
        dsc += s * s;
      }
    const double wj = W[i % nu] * detj[i];
    acc[0] += ke * wj;
    acc[1] += en * wj;
    acc[2] += pd * wj;
    acc[3] += sc * wj;
    acc[4] += dsc * wj;
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < kDiagQ; q++) {
    double v = acc[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[q][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < kDiagQ) {
    double v = 0.0;
    for (int w = 0; w < 256 / 32; w++) v += red[threadIdx.x][w];
    partial[(size_t)blockIdx.x * kDiagQ + threadIdx.x] = v;
  }
}

__global__ void fr_diag_finalize(const double* __restrict__ partial, int nblk, double* __restrict__ out)
{
  if (threadIdx.x >= kDiagQ) return;
  double v = 0.0;
  for (int b = 0; b < nblk; b++) v += partial[(size_t)b * kDiagQ + threadIdx.x];
  out[threadIdx.x] = v;
}

cudaError_t launch_diagnostics(int dims, int tc_size, const double* U, const void* G, const double* detj,
                               const double* W, long long npts, int nu, double gamma, double* partial, int nblk,
                               double* out, cudaStream_t st)
{
  if (dims == 2 && tc_size == 8)
    fr_diag_kernel<2, double><<<nblk, 256, 0, st>>>(U, (const double*)G, detj, W, npts, nu, gamma, partial);
  else if (dims == 2)
    fr_diag_kernel<2, float><<<nblk, 256, 0, st>>>(U, (const float*)G, detj, W, npts, nu, gamma, partial);
  else if (tc_size == 8)
    fr_diag_kernel<3, double><<<nblk, 256, 0, st>>>(U, (const double*)G, detj, W, npts, nu, gamma, partial);
  else
    fr_diag_kernel<3, float><<<nblk, 256, 0, st>>>(U, (const float*)G, detj, W, npts, nu, gamma, partial);
  fr_diag_finalize<<<1, 32, 0, st>>>(partial, nblk, out);
  return cudaGetLastError();
}

}  // namespace frb
