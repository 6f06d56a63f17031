// fr_mlp.cu -- training and standalone inference of the learned SGS closure
// (parameter layout and the per-point model in fr_mlp.cuh), and the kernel
// that evaluates the closure's inputs from a solver's state and gradient.
//
// Training step on a batch of N samples (x_n, c*_n, weight s_n; s_n = 1 when
// no weights are given):
//   loss = (1/N) sum_n s_n (c(x_n) - c*_n)^2
// fr_mlp_loss_grad_kernel: one CTA per tile of 128 samples; forward pass with
// the activations kept in shared memory, then the backward pass as
// tile-local sums over the samples in a fixed order -> one partial gradient
// per CTA; fr_mlp_reduce_kernel sums the partials in CTA order, so a gradient
// is the same bit for bit on every run.  fr_mlp_adam_kernel applies Adam.
#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "fr_b200.h"
#include "fr_mlp.cuh"

namespace frb {

extern thread_local std::string g_err;

namespace {

constexpr int kTile = 128;
constexpr size_t kGradSmem = sizeof(float) * (kMlpIn + 2 * kMlpH + 2) * kTile;

fr_status mlp_fail(fr_status s, const std::string& m)
{
  g_err = m;
  return s;
}

__global__ void __launch_bounds__(256) fr_mlp_forward_kernel(const float* __restrict__ w, const float* __restrict__ X,
                                                             long long n, float* __restrict__ out)
{
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float x[kMlpIn];
#pragma unroll
  for (int k = 0; k < kMlpIn; k++) x[k] = X[i * kMlpIn + k];
  out[i] = mlp_eval(w, x);
}

__global__ void __launch_bounds__(kTile) fr_mlp_loss_grad_kernel(const float* __restrict__ w,
                                                                 const float* __restrict__ X,
                                                                 const float* __restrict__ Y,
                                                                 const float* __restrict__ SW, long long n,
                                                                 float inv_n, float* __restrict__ partial)
{
  // activations sample-minor ([unit][sample]) so that a warp's 32 samples
  // sit in 32 banks; 68 KB of dynamic shared memory
  extern __shared__ float mlp_smem[];
  auto sX = reinterpret_cast<float (*)[kTile]>(mlp_smem);
  auto sH1 = reinterpret_cast<float (*)[kTile]>(mlp_smem + kMlpIn * kTile);            // h1, then d loss / d a1
  auto sH2 = reinterpret_cast<float (*)[kTile]>(mlp_smem + (kMlpIn + kMlpH) * kTile);  // h2, then d loss / d a2
  float* sDo = mlp_smem + (kMlpIn + 2 * kMlpH) * kTile;
  float* sLoss = sDo + kTile;
  const int t = threadIdx.x;
  const long long s = (long long)blockIdx.x * kTile + t;
  const bool live = s < n;
  // ---- forward, one sample per thread
  float x[kMlpIn];
#pragma unroll
  for (int k = 0; k < kMlpIn; k++) {
    x[k] = live ? (X[s * kMlpIn + k] - w[kMlpXm + k]) * w[kMlpXs + k] : 0.f;
    sX[k][t] = x[k];
  }
  for (int i = 0; i < kMlpH; i++) {
    float a = w[kMlpB1 + i];
#pragma unroll
    for (int k = 0; k < kMlpIn; k++) a = fmaf(w[kMlpW1 + i * kMlpIn + k], x[k], a);
    sH1[i][t] = tanhf(a);
  }
  float o = w[kMlpB3];
  for (int j = 0; j < kMlpH; j++) {
    float a = w[kMlpB2 + j];
    for (int i = 0; i < kMlpH; i++) a = fmaf(w[kMlpW2 + j * kMlpH + i], sH1[i][t], a);
    const float h = tanhf(a);
    sH2[j][t] = h;
    o = fmaf(w[kMlpW3 + j], h, o);
  }
  const float c = mlp_softplus(o);
  const float r = live ? c - Y[s] : 0.f;
  const float sw = (live && SW) ? SW[s] : 1.f;
  const float sig = 1.f / (1.f + expf(-o));
  sDo[t] = 2.f * sw * r * sig * inv_n;  // d loss / d o
  sLoss[t] = sw * r * r;
  __syncthreads();

  float* P = partial + (size_t)blockIdx.x * (kMlpTrain + 1);
  // ---- output layer: dw3_j = sum_s do h2_j, db3 = sum_s do
  if (t < kMlpH) {
    float acc = 0.f;
    for (int q = 0; q < kTile; q++) acc = fmaf(sDo[q], sH2[t][q], acc);
    P[kMlpW3 + t] = acc;
  }
  if (t == kMlpH) {
    float acc = 0.f, l = 0.f;
    for (int q = 0; q < kTile; q++) { acc += sDo[q]; l += sLoss[q]; }
    P[kMlpB3] = acc;
    P[kMlpTrain] = l;
  }
  __syncthreads();
  // ---- d loss / d a2 = do w3_j (1 - h2_j^2), in place
  for (int j = 0; j < kMlpH; j++) {
    const float h = sH2[j][t];
    sH2[j][t] = sDo[t] * w[kMlpW3 + j] * (1.f - h * h);
  }
  __syncthreads();
  // ---- dW2[j][i] = sum_s da2_j h1_i, db2_j = sum_s da2_j
  for (int e = t; e < kMlpH * kMlpH; e += kTile) {
    const int j = e / kMlpH, i = e - j * kMlpH;
    float acc = 0.f;
    for (int q = 0; q < kTile; q++) acc = fmaf(sH2[j][q], sH1[i][q], acc);
    P[kMlpW2 + e] = acc;
  }
  if (t < kMlpH) {
    float acc = 0.f;
    for (int q = 0; q < kTile; q++) acc += sH2[t][q];
    P[kMlpB2 + t] = acc;
  }
  __syncthreads();
  // ---- d loss / d a1_i = (sum_j W2[j][i] da2_j) (1 - h1_i^2), in place
  for (int i = 0; i < kMlpH; i++) {
    float acc = 0.f;
    for (int j = 0; j < kMlpH; j++) acc = fmaf(w[kMlpW2 + j * kMlpH + i], sH2[j][t], acc);
    const float h = sH1[i][t];
    sH1[i][t] = acc * (1.f - h * h);
  }
  __syncthreads();
  // ---- dW1[i][k] = sum_s da1_i x_k, db1_i = sum_s da1_i
  for (int e = t; e < kMlpH * kMlpIn; e += kTile) {
    const int i = e / kMlpIn, k = e - i * kMlpIn;
    float acc = 0.f;
    for (int q = 0; q < kTile; q++) acc = fmaf(sH1[i][q], sX[k][q], acc);
    P[kMlpW1 + e] = acc;
  }
  if (t < kMlpH) {
    float acc = 0.f;
    for (int q = 0; q < kTile; q++) acc += sH1[t][q];
    P[kMlpB1 + t] = acc;
  }
}

// grad[p] = sum over CTAs of partial[b][p] (CTA order); loss = sum of the
// per-CTA squared residuals / n.
__global__ void fr_mlp_reduce_kernel(const float* __restrict__ partial, int nblk, float inv_n,
                                     float* __restrict__ grad, float* __restrict__ loss)
{
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p > kMlpTrain) return;
  float acc = 0.f;
  for (int b = 0; b < nblk; b++) acc += partial[(size_t)b * (kMlpTrain + 1) + p];
  if (p < kMlpTrain) grad[p] = acc;
  else if (loss) *loss = acc * inv_n;
}

__global__ void fr_mlp_adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                                   float* __restrict__ v, float lr, float b1, float b2, float eps, float c1,
                                   float c2)
{
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kMlpTrain) return;
  const float gp = g[p];
  const float mp = b1 * m[p] + (1.f - b1) * gp;
  const float vp = b2 * v[p] + (1.f - b2) * gp * gp;
  m[p] = mp;
  v[p] = vp;
  w[p] -= lr * (mp / c1) / (sqrtf(vp / c2) + eps);
}

template <int D, typename TC>
__global__ void fr_sgs_inputs_kernel(const double* __restrict__ U, const TC* __restrict__ G,
                                     const double* __restrict__ detj, long long npts, int nu, long long E, double n1,
                                     double filter_ratio, float* __restrict__ X)
{
  constexpr int F = D + 2;
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npts) return;
  double q[F], g[F][D];
#pragma unroll
  for (int k = 0; k < F; k++) {
    q[k] = U[i + npts * k];
#pragma unroll
    for (int d = 0; d < D; d++) g[k][d] = (double)G[i + npts * (k + (long long)F * d)];
  }
  float x[kMlpIn];
  double delta, S[D][D], smag, de[D];
  sgs_learned_inputs<D, double>(q, g, detj[i], n1, filter_ratio, x, delta, S, smag, de);
#pragma unroll
  for (int k = 0; k < kMlpIn; k++) X[i * kMlpIn + k] = x[k];
  (void)nu; (void)E;
}

}  // namespace

// Host launcher used by fr_solver_sgs_features (fr_solver.cu).
cudaError_t launch_sgs_inputs(int dims, int tc_size, const double* U, const void* G, const double* detj, long long npts,
                              int nu, long long E, int order, double filter_ratio, float* X, cudaStream_t st)
{
  unsigned g = (unsigned)((npts + 255) / 256);
  if (dims == 2 && tc_size == 8)
    fr_sgs_inputs_kernel<2, double><<<g, 256, 0, st>>>(U, (const double*)G, detj, npts, nu, E, order + 1.0,
                                                       filter_ratio, X);
  else if (dims == 2)
    fr_sgs_inputs_kernel<2, float><<<g, 256, 0, st>>>(U, (const float*)G, detj, npts, nu, E, order + 1.0,
                                                      filter_ratio, X);
  else if (tc_size == 8)
    fr_sgs_inputs_kernel<3, double><<<g, 256, 0, st>>>(U, (const double*)G, detj, npts, nu, E, order + 1.0,
                                                       filter_ratio, X);
  else
    fr_sgs_inputs_kernel<3, float><<<g, 256, 0, st>>>(U, (const float*)G, detj, npts, nu, E, order + 1.0,
                                                      filter_ratio, X);
  return cudaGetLastError();
}

// Parameters of a closure that is switched off: zero weights, unit input
// scaling and b3 = -20, so c = softplus(-20) ~ 2e-9.
void mlp_default_params(float* w)
{
  for (int p = 0; p < kMlpN; p++) w[p] = 0.f;
  w[kMlpB3] = -20.f;
  for (int k = 0; k < kMlpIn; k++) w[kMlpXs + k] = 1.f;
}

}  // namespace frb

using namespace frb;

int fr_mlp_n_params(void) { return kMlpN; }
int fr_mlp_n_trained(void) { return kMlpTrain; }

long long fr_mlp_scratch_floats(long long n) { return ((n + kTile - 1) / kTile) * (long long)(kMlpTrain + 1); }

fr_status fr_mlp_forward(const float* w, const float* x, long long n, float* out, void* stream)
{
  if (!w || (n > 0 && (!x || !out)) || n < 0) return mlp_fail(FR_ERR_ARG, "bad argument");
  if (n == 0) return FR_OK;
  fr_mlp_forward_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(w, x, n, out);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? FR_OK : mlp_fail(FR_ERR_CUDA, cudaGetErrorString(e));
}

fr_status fr_mlp_loss_grad(const float* w, const float* x, const float* y, const float* sw, long long n, float* grad,
                           float* loss, float* scratch, long long scratch_floats, void* stream)
{
  if (!w || !x || !y || !grad || !scratch || n <= 0) return mlp_fail(FR_ERR_ARG, "bad argument");
  if (scratch_floats < fr_mlp_scratch_floats(n))
    return mlp_fail(FR_ERR_ARG, "scratch smaller than fr_mlp_scratch_floats(n)");
  const long long nblk = (n + kTile - 1) / kTile;
  if (nblk > 0x7fffffffLL) return mlp_fail(FR_ERR_ARG, "batch too large");
  cudaStream_t st = (cudaStream_t)stream;
  const float inv_n = (float)(1.0 / (double)n);
  static bool once = (cudaFuncSetAttribute(fr_mlp_loss_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)kGradSmem), true);
  (void)once;
  fr_mlp_loss_grad_kernel<<<(unsigned)nblk, kTile, kGradSmem, st>>>(w, x, y, sw, n, inv_n, scratch);
  fr_mlp_reduce_kernel<<<(kMlpTrain + 1 + 255) / 256, 256, 0, st>>>(scratch, (int)nblk, inv_n, grad, loss);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? FR_OK : mlp_fail(FR_ERR_CUDA, cudaGetErrorString(e));
}

fr_status fr_mlp_adam(float* w, const float* grad, float* m, float* v, int step, float lr, void* stream)
{
  if (!w || !grad || !m || !v || step < 1 || !(lr > 0.f)) return mlp_fail(FR_ERR_ARG, "bad argument");
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float c1 = (float)(1.0 - std::pow(0.9, step)), c2 = (float)(1.0 - std::pow(0.999, step));
  fr_mlp_adam_kernel<<<(kMlpTrain + 255) / 256, 256, 0, (cudaStream_t)stream>>>(w, grad, m, v, lr, b1, b2, eps, c1,
                                                                                 c2);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? FR_OK : mlp_fail(FR_ERR_CUDA, cudaGetErrorString(e));
}
