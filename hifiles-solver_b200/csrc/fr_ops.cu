// fr_ops.cu -- per-operator entry points: the reference's GPU seam, one call
// per method of class eles / int_inters, on caller-owned device arrays in the
// reference's own layouts.  Operators are the reference's dense matrices
// (opp_0 .. opp_6, any element type); interface data come through the same
// device tables of device pointers that int_inters builds
// (src/int_inters.cpp:95-178), so a caller can swap these in for the
// cublasDgemm / *_kernel_wrapper calls without touching its data.
#include <cuda_runtime.h>

#include <string>

#include "fr_b200.h"
#include "fr_physics.cuh"

namespace frb {
extern thread_local std::string g_err;
// BF16 3-term split operator product on the tensor cores (fr_tc_gemm.cu)
fr_status gemm_bf16x3(int m, int k, long long ncols, const double* A, const double* B, double* C, int beta,
                      cudaStream_t s, int terms);
fr_status gemm_bf16x3_check(cudaStream_t s);
void gemm_set_prefetch(int on);
}
using namespace frb;

namespace {

fr_status op_fail(fr_status s, const std::string& m)
{
  g_err = m;
  return s;
}

fr_status launched(const char* what)
{
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return op_fail(FR_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return FR_OK;
}

constexpr int kTileCols = 32;
constexpr int kTileStride = kTileCols + 1;  // staged B rows padded: the column-major copy-in is conflict-free
constexpr int kDenseThreads = 256;
constexpr int kMaxOps = 3;
constexpr int kSmallOps = 8192;             // operator entries (all nd) staged in shared memory
constexpr size_t kDenseSmem = 220 * 1024;
constexpr size_t kStageSmem = 64 * 1024;    // fused products stage their operators while a block stays within this
constexpr size_t kStageSmem1 = 112 * 1024;  // the same for a single product

struct OpSet {
  const double* a[kMaxOps];
  // selected without indexing the parameter array by a run-time value
  __device__ __forceinline__ const double* get(int d) const { return d == 0 ? a[0] : (d == 1 ? a[1] : a[2]); }
};

// Dense operator products over all ncols columns, nd <= 3 operators A_d
// (m x k, column major), the reference's cublasDgemm('N','N', m, ncols, k, 1,
// A_d, m, B, k, beta, C, m) calls of one method fused into one pass:
//   FAN = false:  C = beta C + sum_d A_d B_d        (B_d = B + d strideB),
//                 the d-loop of extrapolate_totalFlux / calculate_divergence
//                 (beta 1 for d > 0): each output is one fma chain over d, l;
//   FAN = true:   C_d = beta C_d + A_d B            (C_d = C + d strideC),
//                 calculate_gradient / correct_gradient: B is read once.
// A tile of 32 columns of every B_d and C_d is staged through shared memory so
// all global streams are contiguous.  Each thread keeps an RM x 4 register
// tile: rows r0 + 32 i (i < RM; r0 = lane, then lane + 32 RM ... while rows
// remain) and columns warp + 8 j (j < 4), so per term l a warp reads 4
// broadcast entries of B from shared memory and RM coalesced 32-row slices of
// A_d's column l, for 4 RM fused multiply-adds.  With SA the operators are
// copied to shared memory first, otherwise read through the read-only cache.
// Sums run over d, then l, in increasing order: the result equals nd separate
// single-operator products bit for bit.
template <int RM, bool SA, bool FAN, int LW>
__global__ void __launch_bounds__(kDenseThreads)
dense_apply_kernel(int m, int k, long long ncols, int nd, OpSet ops, const double* __restrict__ B,
                   long long strideB, double* __restrict__ Cm, long long strideC, int beta)
{
  extern __shared__ double sm[];
  const int nb = FAN ? 1 : nd, ncs = FAN ? nd : 1;
  double* sB = sm;                                          // [nb][k][kTileStride]
  double* sC = sB + (size_t)nb * k * kTileStride;           // [ncs][kTileCols][m]
  double* sA = sC + (size_t)ncs * kTileCols * m;            // [nd][k][m] when SA
  if (SA)
    for (int d = 0; d < nd; d++)
      for (int i = threadIdx.x; i < m * k; i += kDenseThreads) sA[(size_t)d * m * k + i] = __ldg(ops.get(d) + i);
  const long long c0 = (long long)blockIdx.x * kTileCols;
  const int nc = (int)min((long long)kTileCols, ncols - c0);
  for (int b = 0; b < nb; b++) {
    const double* Bt = B + b * strideB + (size_t)c0 * k;
    double* sb = sB + (size_t)b * k * kTileStride;
    for (int i = threadIdx.x; i < nc * k; i += kDenseThreads) {
      int c = i / k, l = i - c * k;
      sb[l * kTileStride + c] = Bt[i];
    }
  }
  if (beta)
    for (int t = 0; t < ncs; t++) {
      const double* Ct = Cm + t * strideC + (size_t)c0 * m;
      double* sc = sC + (size_t)t * kTileCols * m;
      for (int i = threadIdx.x; i < nc * m; i += kDenseThreads) sc[i] = Ct[i];
    }
  __syncthreads();
  // LW lanes of a warp share a column and take LW consecutive rows; the
  // 32 / LW lane groups, the 8 warps and RC register columns cover the tile
  constexpr int RC = LW == 32 ? 4 : 2, CW = 32 / LW;
  static_assert(CW * 8 * RC == kTileCols, "column tile");
  const int lane = threadIdx.x & 31, wc = threadIdx.x >> 5;
  const int cbase = lane / LW + CW * wc;
  for (int r0 = lane & (LW - 1); r0 < m; r0 += LW * RM) {
    double acc[RM][RC];
    for (int d = 0; d < nd; d++) {
      double* sc = sC + (FAN ? (size_t)d * kTileCols * m : 0);
      if (FAN || d == 0) {
#pragma unroll
        for (int i = 0; i < RM; i++)
#pragma unroll
          for (int j = 0; j < RC; j++) {
            const int r = r0 + LW * i, c = cbase + 8 * CW * j;
            acc[i][j] = (beta && r < m && c < nc) ? sc[c * m + r] : 0.0;
          }
      }
      const double* sb = sB + (FAN ? 0 : (size_t)d * k * kTileStride);
      const double* Ar = (SA ? sA + (size_t)d * m * k : ops.get(d)) + r0;
      for (int l = 0; l < k; l++) {
        double bv[RC], a[RM];
#pragma unroll
        for (int j = 0; j < RC; j++) bv[j] = sb[l * kTileStride + cbase + 8 * CW * j];
#pragma unroll
        for (int i = 0; i < RM; i++)
          a[i] = (r0 + LW * i < m) ? (SA ? Ar[LW * i + (size_t)m * l] : __ldg(Ar + LW * i + (size_t)m * l)) : 0.0;
#pragma unroll
        for (int i = 0; i < RM; i++)
#pragma unroll
          for (int j = 0; j < RC; j++) acc[i][j] = fma(bv[j], a[i], acc[i][j]);
      }
      if (FAN || d == nd - 1) {
#pragma unroll
        for (int i = 0; i < RM; i++)
#pragma unroll
          for (int j = 0; j < RC; j++) {
            const int r = r0 + LW * i, c = cbase + 8 * CW * j;
            if (r < m && c < nc) sc[c * m + r] = acc[i][j];
          }
      }
    }
  }
  __syncthreads();
  for (int t = 0; t < ncs; t++) {
    double* Ct = Cm + t * strideC + (size_t)c0 * m;
    const double* sc = sC + (size_t)t * kTileCols * m;
    for (int i = threadIdx.x; i < nc * m; i += kDenseThreads) Ct[i] = sc[i];
  }
}

// FP64 tensor-core form of the same products (mma.sync m8n8k4 f64): a block
// stages a tile of 64-512 columns (the widest within 100 kB) of every B_d in
// shared memory by asynchronous copies (column-major,
// leading dimension ldk = 4 or 12 mod 16 doubles, rows k .. ceil4(k) zeroed),
// and each warp unit computes 8 rows x 32 columns: the accumulator starts at
// beta C, then runs over d and the k-steps in increasing order, so fused and
// separate products agree bit for bit, and every column's result is the same
// in any tiling.  Operator fragments are read from the column-major A_d
// through the read-only cache (entries beyond m x k read as zero).
constexpr int kMmaThreads = 256;
constexpr int kMmaTN = 4;  // 8-column tiles per warp unit

__device__ __forceinline__ void dmma8(double (&c)[2], double a, double b)
{
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
      : "+d"(c[0]), "+d"(c[1])
      : "d"(a), "d"(b));
}

__device__ __forceinline__ void cp_async8(void* dst, const void* src)
{
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}

template <bool FAN, int NCT>
__global__ void __launch_bounds__(kMmaThreads)
dense_mma_kernel(int m, int k, long long ncols, int nd, OpSet ops, const double* __restrict__ B,
                 long long strideB, double* __restrict__ Cm, long long strideC, int beta, int ldk)
{
  extern __shared__ __align__(16) double sm[];
  const int nb = FAN ? 1 : nd;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int NW = kMmaThreads / 32;
  const long long c0 = (long long)blockIdx.x * NCT;
  const int nc = (int)min((long long)NCT, ncols - c0);
  const int kp = (k + 3) & ~3;
  // B tile: asynchronous copies, one column per warp pass with the lanes
  // along k (contiguous in global memory), many columns in flight
  for (int b = 0; b < nb; b++) {
    const double* Bt = B + b * strideB + (size_t)c0 * k;
    double* sb = sm + (size_t)b * NCT * ldk;
    for (int c = warp; c < NCT; c += NW) {
      if (c < nc)
        for (int l = lane; l < k; l += 32) cp_async8(&sb[c * ldk + l], Bt + (size_t)c * k + l);
      for (int l = k + lane; l < kp; l += 32) sb[c * ldk + l] = 0.0;
    }
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncthreads();
  const int MT = (m + 7) / 8, KS = kp / 4;
  constexpr int NB = NCT / 8 / kMmaTN;
  const int g = lane >> 2, t = lane & 3;
  for (int u = warp; u < MT * NB; u += NW) {
    const int mt = u / NB, nt0 = (u - mt * NB) * kMmaTN;
    const int r = mt * 8 + g;
    for (int o = 0; o < (FAN ? nd : 1); o++) {
      double* Co = Cm + (FAN ? o * strideC : 0);
      double acc[kMmaTN][2];
#pragma unroll
      for (int j = 0; j < kMmaTN; j++)
#pragma unroll
        for (int i = 0; i < 2; i++) {
          const int n = (nt0 + j) * 8 + 2 * t + i;
          acc[j][i] = (beta && r < m && n < nc) ? Co[r + (size_t)m * (c0 + n)] : 0.0;
        }
      const int d0 = FAN ? o : 0, d1 = FAN ? o + 1 : nd;
      for (int d = d0; d < d1; d++) {
        const double* A = ops.get(d);
        const double* sb = sm + (size_t)(FAN ? 0 : d) * NCT * ldk;
        const double* bp[kMmaTN];
#pragma unroll
        for (int j = 0; j < kMmaTN; j++) bp[j] = sb + ((nt0 + j) * 8 + g) * ldk + t;
        // operator fragments fetched 8 k-steps ahead of their MMAs
        for (int k0 = 0; k0 < KS; k0 += 8) {
          double af[8];
#pragma unroll
          for (int i = 0; i < 8; i++) {
            const int c = (k0 + i) * 4 + t;
            af[i] = (k0 + i < KS && r < m && c < k) ? __ldg(A + r + (size_t)m * c) : 0.0;
          }
#pragma unroll
          for (int i = 0; i < 8; i++)
            if (k0 + i < KS)
#pragma unroll
              for (int j = 0; j < kMmaTN; j++) dmma8(acc[j], af[i], bp[j][(k0 + i) * 4]);
        }
      }
#pragma unroll
      for (int j = 0; j < kMmaTN; j++)
#pragma unroll
        for (int i = 0; i < 2; i++) {
          const int n = (nt0 + j) * 8 + 2 * t + i;
          if (r < m && n < nc) Co[r + (size_t)m * (c0 + n)] = acc[j][i];
        }
    }
  }
}

int mma_ld(int k)
{
  int x = (k + 3) & ~3;
  while (x % 16 != 4 && x % 16 != 12) x++;
  return x;
}

size_t mma_smem(int k, int nb, int nct) { return (size_t)nb * nct * mma_ld(k) * sizeof(double); }

// the column tile of every B_d fits one block's shared memory (128 columns, else 64)
bool mma_fits(int k, int nb) { return mma_smem(k, nb, 64) <= 200 * 1024; }

fr_status dense_mma_launch(int m, int k, long long ncols, int nd, const OpSet& ops, const double* B, long long sB,
                           double* Cm, long long sC, int beta, bool fan, cudaStream_t s)
{
  const int ldk = mma_ld(k), nb = fan ? 1 : nd;
  // the widest column tile within 100 kB (short operators get wide tiles, so
  // a block's staging is spread over enough products), narrowed while the
  // grid would not give every SM two blocks
  int nct = 64;
  for (int c : {512, 256, 128})
    if (mma_smem(k, nb, c) <= 100 * 1024) {
      nct = c;
      break;
    }
  while (nct > 64 && (ncols + nct - 1) / nct < 2 * 148) nct /= 2;
  const size_t smem = mma_smem(k, nb, nct);
  auto pick = [&](auto kt, auto kf) { return fan ? kt : kf; };
  auto kern = nct == 512   ? pick(dense_mma_kernel<true, 512>, dense_mma_kernel<false, 512>)
              : nct == 256 ? pick(dense_mma_kernel<true, 256>, dense_mma_kernel<false, 256>)
              : nct == 128 ? pick(dense_mma_kernel<true, 128>, dense_mma_kernel<false, 128>)
                           : pick(dense_mma_kernel<true, 64>, dense_mma_kernel<false, 64>);
  // every instantiation may use up to 100 kB: set once per device
  static unsigned long long attr_set = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !(attr_set >> dev & 1ull)) {
    const void* all[] = {(const void*)dense_mma_kernel<true, 512>, (const void*)dense_mma_kernel<false, 512>,
                         (const void*)dense_mma_kernel<true, 256>, (const void*)dense_mma_kernel<false, 256>,
                         (const void*)dense_mma_kernel<true, 128>, (const void*)dense_mma_kernel<false, 128>,
                         (const void*)dense_mma_kernel<true, 64>, (const void*)dense_mma_kernel<false, 64>};
    for (const void* f : all) {
      cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
      if (e != cudaSuccess) return op_fail(FR_ERR_CUDA, cudaGetErrorString(e));
    }
    attr_set |= 1ull << dev;
  } else if (dev >= 64 && smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return op_fail(FR_ERR_CUDA, cudaGetErrorString(e));
  }
  const long long blocks = (ncols + nct - 1) / nct;
  if (blocks > 2147483647LL) return op_fail(FR_ERR_ARG, "too many columns");
  kern<<<(unsigned)blocks, kMmaThreads, smem, s>>>(m, k, ncols, nd, ops, B, sB, Cm, sC, beta, ldk);
  return launched("dense_mma_kernel");
}

template <int RM, int LW = 32>
fr_status dense_launch(int m, int k, long long ncols, int nd, const OpSet& ops, const double* B, long long sB,
                       double* Cm, long long sC, int beta, bool fan, cudaStream_t s, size_t smem, unsigned blocks)
{
  const size_t a_bytes = (size_t)nd * m * k * sizeof(double);
  const bool sa = (long long)nd * m * k <= kSmallOps && smem + a_bytes <= (nd == 1 ? kStageSmem1 : kStageSmem);
  if (sa) smem += a_bytes;
  auto kern = fan ? (sa ? dense_apply_kernel<RM, true, true, LW> : dense_apply_kernel<RM, false, true, LW>)
                  : (sa ? dense_apply_kernel<RM, true, false, LW> : dense_apply_kernel<RM, false, false, LW>);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return op_fail(FR_ERR_CUDA, cudaGetErrorString(e));
  }
  kern<<<blocks, kDenseThreads, smem, s>>>(m, k, ncols, nd, ops, B, sB, Cm, sC, beta);
  return launched("dense_apply_kernel");
}

// Precision of the operator products of this seam: 0 = FP64 on the FP64
// tensor cores (dense_mma_kernel; dense_apply_kernel when a column tile does
// not fit shared memory), 1 = BF16x3 and 2 = BF16x6 split products on the
// tcgen05 tensor cores, FP32 accumulation (fr_tc_gemm.cu), 3 = FP64 on the
// CUDA cores (dense_apply_kernel).
static int g_gemm_mode = 0;

// nd operator products of one method (see dense_apply_kernel); FAN selects
// C_d = beta C_d + A_d B, otherwise C = beta C + sum_d A_d B_d.  The tensor-
// core forms and shapes whose staged tiles exceed shared memory run as nd
// single products in the same order.
fr_status dense_apply_nd(int m, int k, long long ncols, int nd, const double* const* A, const double* B,
                         long long strideB, double* Cm, long long strideC, int beta, bool fan, cudaStream_t s)
{
  if (m <= 0 || k <= 0 || ncols < 0 || nd < 1 || nd > kMaxOps || !A || !B || !Cm)
    return op_fail(FR_ERR_ARG, "bad operator arguments");
  for (int d = 0; d < nd; d++)
    if (!A[d]) return op_fail(FR_ERR_ARG, "bad operator arguments");
  if (ncols == 0) return FR_OK;
  const int nb = fan ? 1 : nd, ncs = fan ? nd : 1;
  size_t smem = ((size_t)nb * k * kTileStride + (size_t)ncs * kTileCols * m) * sizeof(double);
  const size_t a1 = (size_t)m * k * sizeof(double);
  const size_t smem1 = ((size_t)k * kTileStride + (size_t)kTileCols * m) * sizeof(double);
  // fused unless one operator could sit in shared memory but all nd cannot:
  // then nd single products with a staged operator are faster
  const bool split = nd > 1 && (long long)m * k <= kSmallOps && smem1 + a1 <= kStageSmem1 &&
                     !((long long)nd * m * k <= kSmallOps && smem + nd * a1 <= kStageSmem);
  // FP64 products with short operators (k < 16) stay on the CUDA cores, where
  // they measured faster; both forms give the same bits
  if (g_gemm_mode == 0 && k >= 16 && mma_fits(k, fan ? 1 : nd)) {
    OpSet ops{};
    for (int d = 0; d < nd; d++) ops.a[d] = A[d];
    return dense_mma_launch(m, k, ncols, nd, ops, B, strideB, Cm, strideC, beta, fan, s);
  }
  const bool tc = g_gemm_mode == 1 || g_gemm_mode == 2;
  if (tc || split || (nd > 1 && smem > kDenseSmem)) {
    for (int d = 0; d < nd; d++) {
      const double* Bd = B + (fan ? 0 : d * strideB);
      double* Cd = Cm + (fan ? d * strideC : 0);
      const int bd = fan ? beta : (d > 0 ? 1 : beta);
      fr_status st = tc ? gemm_bf16x3(m, k, ncols, A[d], Bd, Cd, bd, s, g_gemm_mode == 2 ? 6 : 3)
                        : dense_apply_nd(m, k, ncols, 1, A + d, Bd, 0, Cd, 0, bd, false, s);
      if (st) return st;
    }
    return FR_OK;
  }
  if (smem > kDenseSmem) return op_fail(FR_ERR_UNSUPPORTED, "operator too large for one column tile");
  long long blocks = (ncols + kTileCols - 1) / kTileCols;
  if (blocks > 2147483647LL) return op_fail(FR_ERR_ARG, "too many columns");
  const unsigned nbk = (unsigned)blocks;
  OpSet ops{};
  for (int d = 0; d < nd; d++) ops.a[d] = A[d];
  // operators of at most 16 rows: 16 rows per warp, half the padding (for
  // taller ones the extra operator loads per fma measured slower)
  if (m <= 16) return dense_launch<1, 16>(m, k, ncols, nd, ops, B, strideB, Cm, strideC, beta, fan, s, smem, nbk);
  switch ((m + 31) / 32) {
    case 1: return dense_launch<1>(m, k, ncols, nd, ops, B, strideB, Cm, strideC, beta, fan, s, smem, nbk);
    case 2: return dense_launch<2>(m, k, ncols, nd, ops, B, strideB, Cm, strideC, beta, fan, s, smem, nbk);
    case 3: return dense_launch<3>(m, k, ncols, nd, ops, B, strideB, Cm, strideC, beta, fan, s, smem, nbk);
    case 4: return dense_launch<4>(m, k, ncols, nd, ops, B, strideB, Cm, strideC, beta, fan, s, smem, nbk);
    case 5: return dense_launch<5>(m, k, ncols, nd, ops, B, strideB, Cm, strideC, beta, fan, s, smem, nbk);
    case 6: return dense_launch<6>(m, k, ncols, nd, ops, B, strideB, Cm, strideC, beta, fan, s, smem, nbk);
    case 7: return dense_launch<7>(m, k, ncols, nd, ops, B, strideB, Cm, strideC, beta, fan, s, smem, nbk);
    default: return dense_launch<8>(m, k, ncols, nd, ops, B, strideB, Cm, strideC, beta, fan, s, smem, nbk);
  }
}

fr_status dense_apply(int m, int k, long long ncols, const double* A, const double* B, double* Cm, int beta,
                      cudaStream_t s)
{
  return dense_apply_nd(m, k, ncols, 1, &A, B, 0, Cm, 0, beta, false, s);
}

// bespoke_SPMV's product (src/cuda_kernels.cu, bespoke_SPMV_kernel) on the
// ELL operators of array_to_ellpack (src/funcs.cpp:961-1011): row i keeps
// nnz_per_row slots s, entry data[i + m s] at column idx[i + m s] (padding
// slots hold 0 at column 0).  c = q or c + q (add_flag) with q summed from 0
// over the slots in order.  A tile of 32 columns of B is staged through
// shared memory as in dense_apply_kernel; each thread keeps rows lane + 32 i
// and columns warp + 8 j.
template <int RM>
__global__ void __launch_bounds__(kDenseThreads)
spmv_ell_kernel(int m, int k, long long ncols, const double* __restrict__ data, const int* __restrict__ idx,
                int nnz, const double* __restrict__ B, double* __restrict__ Cm, int add)
{
  extern __shared__ double sm[];
  double* sB = sm;  // [k][kTileStride]
  const long long c0 = (long long)blockIdx.x * kTileCols;
  const int nc = (int)min((long long)kTileCols, ncols - c0);
  const double* Bt = B + (size_t)c0 * k;
  for (int i = threadIdx.x; i < nc * k; i += kDenseThreads) {
    int c = i / k, l = i - c * k;
    sB[l * kTileStride + c] = Bt[i];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, wc = threadIdx.x >> 5;
  double* Ct = Cm + (size_t)c0 * m;
  for (int r0 = lane; r0 < m; r0 += 32 * RM) {
    double q[RM][4];
#pragma unroll
    for (int i = 0; i < RM; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) q[i][j] = 0.0;
    for (int s = 0; s < nnz; s++) {
#pragma unroll
      for (int i = 0; i < RM; i++) {
        const int r = r0 + 32 * i;
        if (r >= m) continue;
        const double a = __ldg(data + r + (size_t)m * s);
        const int l = __ldg(idx + r + (size_t)m * s);
        if ((unsigned)l >= (unsigned)k) continue;  // a column outside the operator is never read
#pragma unroll
        for (int j = 0; j < 4; j++) q[i][j] = fma(a, sB[l * kTileStride + wc + 8 * j], q[i][j]);
      }
    }
#pragma unroll
    for (int i = 0; i < RM; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int r = r0 + 32 * i, c = wc + 8 * j;
        if (r < m && c < nc) {
          double* p = Ct + (size_t)c * m + r;
          *p = add ? *p + q[i][j] : q[i][j];
        }
      }
  }
}

// ------------------------------------------------------------ pointwise kernels

template <int D>
__global__ void inv_flux_kernel(int nu, long long E, const double* __restrict__ U, const double* __restrict__ JG,
                                double* __restrict__ TF, PhysT<double> ph)
{
  constexpr int F = D + 2;
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)nu * E) return;
  size_t NE = (size_t)nu * E;
  double q[F], f[F][D];
#pragma unroll
  for (int k = 0; k < F; k++) q[k] = U[i + NE * k];
  inv_flux<D, double>(ph, q, f);
  const double* G = JG + (size_t)D * D * i;
#pragma unroll
  for (int k = 0; k < F; k++)
#pragma unroll
    for (int l = 0; l < D; l++) {
      double acc = 0.0;
#pragma unroll
      for (int mm = 0; mm < D; mm++) acc = fma(G[l + D * mm], f[k][mm], acc);
      TF[i + NE * (k + (size_t)F * l)] = acc;
    }
}

template <int D>
__global__ void vis_flux_kernel(int nu, long long E, const double* __restrict__ U, const double* __restrict__ GU,
                                const double* __restrict__ JG, double* __restrict__ TF, PhysT<double> ph)
{
  constexpr int F = D + 2;
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)nu * E) return;
  size_t NE = (size_t)nu * E;
  double q[F], g[F][D], f[F][D];
#pragma unroll
  for (int k = 0; k < F; k++) {
    q[k] = U[i + NE * k];
#pragma unroll
    for (int d = 0; d < D; d++) g[k][d] = GU[i + NE * (k + (size_t)F * d)];
  }
  vis_flux<D, double>(ph, q, g, f);
  const double* G = JG + (size_t)D * D * i;
#pragma unroll
  for (int k = 0; k < F; k++)
#pragma unroll
    for (int l = 0; l < D; l++) {
      double acc = TF[i + NE * (k + (size_t)F * l)];
#pragma unroll
      for (int mm = 0; mm < D; mm++) acc = fma(G[l + D * mm], f[k][mm], acc);
      TF[i + NE * (k + (size_t)F * l)] = acc;
    }
}

// The viscous flux with the eddy-viscosity SGS flux of eles::evaluate_viscFlux
// with LES (src/eles.cpp:2369-2409): f = F_visc + F_sgs transformed and added
// to tdisf_upts, and the SGS flux alone transformed into sgsf_upts
// (sgsf_upts(j,i,k,l) = sum_m JGinv(l,m) F_sgs(k,m), summed from zero).
template <int D>
__global__ void vis_flux_les_kernel(int nu, long long E, const double* __restrict__ U, const double* __restrict__ GU,
                                    const double* __restrict__ JG, const double* __restrict__ detj,
                                    double* __restrict__ TF, double* __restrict__ SGS, PhysT<double> ph, double n1)
{
  constexpr int F = D + 2;
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)nu * E) return;
  size_t NE = (size_t)nu * E;
  double q[F], g[F][D], f[F][D], fs[F][D];
#pragma unroll
  for (int k = 0; k < F; k++) {
    q[k] = U[i + NE * k];
#pragma unroll
    for (int d = 0; d < D; d++) g[k][d] = GU[i + NE * (k + (size_t)F * d)];
  }
  vis_flux<D, double>(ph, q, g, f);
#pragma unroll
  for (int k = 0; k < F; k++)
#pragma unroll
    for (int d = 0; d < D; d++) fs[k][d] = 0.0;
  sgs_flux<D, double>(ph, q, g, detj[i], n1, fs);
#pragma unroll
  for (int k = 0; k < F; k++)
#pragma unroll
    for (int l = 0; l < D; l++) f[k][l] = f[k][l] + fs[k][l];
  const double* G = JG + (size_t)D * D * i;
#pragma unroll
  for (int k = 0; k < F; k++)
#pragma unroll
    for (int l = 0; l < D; l++) {
      double sg = 0.0;
#pragma unroll
      for (int mm = 0; mm < D; mm++) sg = sg + G[l + D * mm] * fs[k][mm];
      SGS[i + NE * (k + (size_t)F * l)] = sg;
      double acc = TF[i + NE * (k + (size_t)F * l)];
#pragma unroll
      for (int mm = 0; mm < D; mm++) acc = fma(G[l + D * mm], f[k][mm], acc);
      TF[i + NE * (k + (size_t)F * l)] = acc;
    }
}

// reference gradient -> physical gradient in place (src/eles.cpp:1822-1878)
template <int D>
__global__ void grad_transform_kernel(int nu, long long E, int F, double* __restrict__ GU,
                                      const double* __restrict__ JG, const double* __restrict__ detj)
{
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)nu * E) return;
  size_t NE = (size_t)nu * E;
  double inv = 1.0 / detj[i];
  const double* G = JG + (size_t)D * D * i;
  double Gm[D][D];
#pragma unroll
  for (int r = 0; r < D; r++)
#pragma unroll
    for (int c = 0; c < D; c++) Gm[r][c] = G[r + D * c] * inv;
  for (int k = 0; k < F; k++) {
    double gr[D];
#pragma unroll
    for (int d = 0; d < D; d++) gr[d] = GU[i + NE * (k + (size_t)F * d)];
#pragma unroll
    for (int c = 0; c < D; c++) {
      double acc = 0.0;
#pragma unroll
      for (int r = 0; r < D; r++) acc = fma(gr[r], Gm[r][c], acc);
      GU[i + NE * (k + (size_t)F * c)] = acc;
    }
  }
}

__global__ void axpy_kernel(long long n, double a, const double* __restrict__ x, double* __restrict__ y)
{
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = fma(a, x[i], y[i]);
}

// RK45 stage update (RK45_update_kernel of the reference, src/cuda_kernels.cu:2654-2690;
// CPU form src/eles.cpp:1155-1178) for fixed time steps.
__global__ void rk45_kernel(int nu, long long E, int F, double* __restrict__ u0, double* __restrict__ u1,
                            const double* __restrict__ div, const double* __restrict__ detj,
                            const double* __restrict__ src, double a, double b, double dt, double const_src)
{
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n = (long long)nu * E;
  if (i >= n * F) return;
  long long p = i % n;
  double rhs = -div[i] / detj[p] + const_src + (src ? src[i] : 0.0);
  double res = fma(a, u1[i], dt * rhs);
  u1[i] = res;
  u0[i] = fma(b, res, u0[i]);
}

// ---------------------------------------------------------- interface kernels
// Tables follow int_inters (src/int_inters.cpp:95-178): *_l / *_r are
// (n_fpts_per_inter, n_inters, n_fields[, n_dims]) arrays of pointers into the
// elements' flux-point arrays; tdA_l/_r (n_fpts_per_inter, n_inters); norm
// (n_fpts_per_inter, n_inters, n_dims) points at the left element's normals.

template <int D>
__global__ void common_inv_kernel(int nfpi, int ni, double* const* __restrict__ ul_p, double* const* __restrict__ ur_p,
                                  double* const* __restrict__ tl_p, double* const* __restrict__ tr_p,
                                  double* const* __restrict__ al_p, double* const* __restrict__ ar_p,
                                  double* const* __restrict__ n_p, double* const* __restrict__ dl_p,
                                  double* const* __restrict__ dr_p, PhysT<double> ph, int riemann, int viscous)
{
  constexpr int F = D + 2;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n = (long long)nfpi * ni;
  if (t >= n) return;
  double ul[F], ur[F], nn[D], fn[F];
#pragma unroll
  for (int k = 0; k < F; k++) { ul[k] = *ul_p[t + n * k]; ur[k] = *ur_p[t + n * k]; }
#pragma unroll
  for (int d = 0; d < D; d++) nn[d] = *n_p[t + n * d];
  if (D == 2 && riemann == 2) roe<double>(ph, ul, ur, nn, fn);
  else rusanov<D, double>(ph, ul, ur, nn, fn);
  double tal = *al_p[t], tar = *ar_p[t];
#pragma unroll
  for (int k = 0; k < F; k++) { *tl_p[t + n * k] = fn[k] * tal; *tr_p[t + n * k] = -fn[k] * tar; }
  if (viscous) {
    double pen = ldg_beta<D, double>(ph.pen_fact, nn);
#pragma unroll
    for (int k = 0; k < F; k++) {
      double uc = 0.5 * (ul[k] + ur[k]) - pen * (ul[k] - ur[k]);
      *dl_p[t + n * k] = uc - ul[k];
      *dr_p[t + n * k] = uc - ur[k];
    }
  }
}

// sl_p / sr_p (LES): the two sides' SGS flux at the flux points, added to
// their viscous fluxes before the LDG flux (src/int_inters.cpp:414-427); null
// without LES.
template <int D>
__global__ void common_vis_kernel(int nfpi, int ni, double* const* __restrict__ ul_p, double* const* __restrict__ ur_p,
                                  double* const* __restrict__ gl_p, double* const* __restrict__ gr_p,
                                  double* const* __restrict__ tl_p, double* const* __restrict__ tr_p,
                                  double* const* __restrict__ al_p, double* const* __restrict__ ar_p,
                                  double* const* __restrict__ n_p, PhysT<double> ph,
                                  double* const* __restrict__ sl_p = nullptr, double* const* __restrict__ sr_p = nullptr)
{
  constexpr int F = D + 2;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n = (long long)nfpi * ni;
  if (t >= n) return;
  double ul[F], ur[F], gl[F][D], gr[F][D], fl[F][D], fr[F][D], nn[D], fn[F];
#pragma unroll
  for (int k = 0; k < F; k++) {
    ul[k] = *ul_p[t + n * k]; ur[k] = *ur_p[t + n * k];
#pragma unroll
    for (int d = 0; d < D; d++) {
      gl[k][d] = *gl_p[t + n * (k + (long long)F * d)];
      gr[k][d] = *gr_p[t + n * (k + (long long)F * d)];
    }
  }
#pragma unroll
  for (int d = 0; d < D; d++) nn[d] = *n_p[t + n * d];
  vis_flux<D, double>(ph, ul, gl, fl);
  vis_flux<D, double>(ph, ur, gr, fr);
  if (sl_p) {
#pragma unroll
    for (int d = 0; d < D; d++)
#pragma unroll
      for (int k = 0; k < F; k++) {
        fl[k][d] += *sl_p[t + n * (k + (long long)F * d)];
        fr[k][d] += *sr_p[t + n * (k + (long long)F * d)];
      }
  }
  ldg_flux<D, double>(ph, ldg_beta<D, double>(ph.pen_fact, nn), ul, ur, fl, fr, nn, fn);
  double tal = *al_p[t], tar = *ar_p[t];
#pragma unroll
  for (int k = 0; k < F; k++) { *tl_p[t + n * k] += fn[k] * tal; *tr_p[t + n * k] += -fn[k] * tar; }
}

// --------------------------------------------------------- boundary kernels
// Tables follow bdy_inters (src/bdy_inters.cpp:111-203): only the owning
// (left) side; boundary_type[i] is the type of boundary interface i and
// bdy_params the 14 boundary values of bdy_inters::set_bdy_params
// (src/bdy_inters.cpp:78-108), both in device memory as the reference keeps
// them.  The ghost state, the central boundary flux and the viscous wall flux
// are the ones of the fused interface kernel's boundary points.

__device__ __forceinline__ void load_bdy(PhysT<double>& ph, const double* __restrict__ bp)
{
#pragma unroll
  for (int i = 0; i < 14; i++) ph.bdy[i] = bp[i];
}

// bdy_inters::evaluate_boundaryConditions_invFlux (src/bdy_inters.cpp:245-389):
// norm_tconf_l = f_n tdA with f_n the central flux of own and ghost state
// (the own flux alone at dual-consistent slip walls, Roe in 2-D when asked),
// and, viscous, the LDG common solution delta_l = (u_ghost + u_l)/2 - u_l.
template <int D>
__global__ void bdy_inv_kernel(int nfpi, int ni, double* const* __restrict__ ul_p, double* const* __restrict__ tl_p,
                               double* const* __restrict__ al_p, double* const* __restrict__ n_p,
                               double* const* __restrict__ dl_p, const int* __restrict__ btype,
                               const double* __restrict__ bp, PhysT<double> ph, int riemann, int viscous)
{
  constexpr int F = D + 2;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n = (long long)nfpi * ni;
  if (t >= n) return;
  load_bdy(ph, bp);
  const int type = btype[t / nfpi];
  double ul[F], ug[F], nn[D], fn[F], fl[F][D], fr[F][D];
#pragma unroll
  for (int k = 0; k < F; k++) ul[k] = *ul_p[t + n * k];
#pragma unroll
  for (int d = 0; d < D; d++) nn[d] = *n_p[t + n * d];
  bc_ghost<D, double>(ph, type, ul, nn, ug);
  inv_flux<D, double>(ph, ul, fl);
  inv_flux<D, double>(ph, ug, fr);
  if (type == 16) {
#pragma unroll
    for (int k = 0; k < F; k++) {
      double s = fl[k][0] * nn[0];
#pragma unroll
      for (int l = 1; l < D; l++) s = s + fl[k][l] * nn[l];
      fn[k] = s;
    }
  } else if (D == 2 && riemann == 2) {
    roe<double>(ph, ul, ug, nn, fn);
  } else {
#pragma unroll
    for (int k = 0; k < F; k++) {
      double s = fl[k][0] * nn[0], q = fr[k][0] * nn[0];
#pragma unroll
      for (int l = 1; l < D; l++) { s = s + fl[k][l] * nn[l]; q = q + fr[k][l] * nn[l]; }
      fn[k] = 0.5 * (s + q);
    }
  }
  const double tal = *al_p[t];
#pragma unroll
  for (int k = 0; k < F; k++) *tl_p[t + n * k] = fn[k] * tal;
  if (viscous) {
#pragma unroll
    for (int k = 0; k < F; k++) *dl_p[t + n * k] = 0.5 * (ug[k] + ul[k]) - ul[k];
  }
}

// bdy_inters::evaluate_boundaryConditions_viscFlux (src/bdy_inters.cpp:905-1057):
// norm_tconf_l += (f_v + tau n (u_l - u_ghost)) . n tdA, f_v the own viscous
// flux, or the ghost side's with no wall-normal temperature gradient at
// adiabatic walls (types 12 and 14).
template <int D>
__global__ void bdy_vis_kernel(int nfpi, int ni, double* const* __restrict__ ul_p, double* const* __restrict__ gl_p,
                               double* const* __restrict__ tl_p, double* const* __restrict__ al_p,
                               double* const* __restrict__ n_p, const int* __restrict__ btype,
                               const double* __restrict__ bp, PhysT<double> ph)
{
  constexpr int F = D + 2;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n = (long long)nfpi * ni;
  if (t >= n) return;
  load_bdy(ph, bp);
  const int type = btype[t / nfpi];
  double ul[F], ug[F], nn[D], g[F][D], fv[F][D];
#pragma unroll
  for (int k = 0; k < F; k++) {
    ul[k] = *ul_p[t + n * k];
#pragma unroll
    for (int d = 0; d < D; d++) g[k][d] = *gl_p[t + n * (k + (long long)F * d)];
  }
#pragma unroll
  for (int d = 0; d < D; d++) nn[d] = *n_p[t + n * d];
  vis_flux_fast<D, double>(ph, ul, g, fv);
  bc_ghost<D, double>(ph, type, ul, nn, ug);
  if (type == 12 || type == 14) {
    bc_vis_gradient<D, double>(ph, ul, ug, g);
    vis_flux_fast<D, double>(ph, ug, g, fv);
  }
  const double tal = *al_p[t];
#pragma unroll
  for (int k = 0; k < F; k++) {
    double fnk = (fv[k][0] + ph.tau * nn[0] * (ul[k] - ug[k])) * nn[0];
#pragma unroll
    for (int d = 1; d < D; d++) fnk = fnk + (fv[k][d] + ph.tau * nn[d] * (ul[k] - ug[k])) * nn[d];
    *tl_p[t + n * k] += fnk * tal;
  }
}

inline unsigned grid_for(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

PhysT<double> phys_of(const fr_phys_desc* p)
{
  Phys q{p->gamma, p->prandtl, p->mu_inf, p->rt_inf, p->c_sth, p->fix_vis, p->tau, p->pen_fact};
  return PhysT<double>::make(q);
}

bool dims_ok(int d, int F) { return (d == 2 && F == 4) || (d == 3 && F == 5); }

}  // namespace

#define ST(stream) ((cudaStream_t)(stream))

extern "C" {

fr_status fr_op_set_gemm_precision(int mode)
{
  if (mode < 0 || mode > 3)
    return op_fail(FR_ERR_ARG,
                   "GEMM precision: 0 (FP64 tensor cores), 1 (BF16x3), 2 (BF16x6) or 3 (FP64 CUDA cores)");
  g_gemm_mode = mode;
  return FR_OK;
}

int fr_op_gemm_precision(void) { return g_gemm_mode; }

fr_status fr_op_set_gemm_pipelining(int on)
{
  gemm_set_prefetch(on);
  return FR_OK;
}

fr_status fr_op_check(void* stream)
{
  cudaError_t e = cudaStreamSynchronize(ST(stream));
  if (e != cudaSuccess) return op_fail(FR_ERR_CUDA, cudaGetErrorString(e));
  return gemm_bf16x3_check(ST(stream));
}

fr_status fr_op_extrapolate_solution(int n_fpts, int n_upts, int n_fields, int n_eles, const double* opp_0,
                                     const double* disu_upts, double* disu_fpts, void* stream)
{
  return dense_apply(n_fpts, n_upts, (long long)n_fields * n_eles, opp_0, disu_upts, disu_fpts, 0, ST(stream));
}

fr_status fr_op_evaluate_invFlux(int n_upts, int n_dims, int n_fields, int n_eles, const double* disu_upts,
                                 const double* JGinv_upts, double* tdisf_upts, const fr_phys_desc* phys,
                                 void* stream)
{
  if (!phys || !disu_upts || !JGinv_upts || !tdisf_upts || !dims_ok(n_dims, n_fields))
    return op_fail(FR_ERR_ARG, "bad arguments");
  long long n = (long long)n_upts * n_eles;
  if (n == 0) return FR_OK;
  if (n_dims == 2) inv_flux_kernel<2><<<grid_for(n, 128), 128, 0, ST(stream)>>>(n_upts, n_eles, disu_upts, JGinv_upts, tdisf_upts, phys_of(phys));
  else inv_flux_kernel<3><<<grid_for(n, 128), 128, 0, ST(stream)>>>(n_upts, n_eles, disu_upts, JGinv_upts, tdisf_upts, phys_of(phys));
  return launched("inv_flux_kernel");
}

fr_status fr_op_calculate_gradient(int n_upts, int n_dims, int n_fields, int n_eles, const double* const* opp_4,
                                   const double* disu_upts, double* grad_disu_upts, void* stream)
{
  if (!opp_4 || n_dims < 2 || n_dims > 3) return op_fail(FR_ERR_ARG, "bad arguments");
  long long cols = (long long)n_fields * n_eles;
  return dense_apply_nd(n_upts, n_upts, cols, n_dims, opp_4, disu_upts, 0, grad_disu_upts, (long long)n_upts * cols,
                        0, true, ST(stream));
}

fr_status fr_op_correct_gradient(int n_upts, int n_fpts, int n_dims, int n_fields, int n_eles,
                                 const double* const* opp_5, const double* delta_disu_fpts, const double* JGinv_upts,
                                 const double* detjac_upts, double* grad_disu_upts, void* stream)
{
  if (!opp_5 || n_dims < 2 || n_dims > 3 || !JGinv_upts || !detjac_upts) return op_fail(FR_ERR_ARG, "bad arguments");
  long long cols = (long long)n_fields * n_eles;
  fr_status st = dense_apply_nd(n_upts, n_fpts, cols, n_dims, opp_5, delta_disu_fpts, 0, grad_disu_upts,
                                (long long)n_upts * cols, 1, true, ST(stream));
  if (st) return st;
  long long n = (long long)n_upts * n_eles;
  if (n_dims == 2) grad_transform_kernel<2><<<grid_for(n, 128), 128, 0, ST(stream)>>>(n_upts, n_eles, n_fields, grad_disu_upts, JGinv_upts, detjac_upts);
  else grad_transform_kernel<3><<<grid_for(n, 128), 128, 0, ST(stream)>>>(n_upts, n_eles, n_fields, grad_disu_upts, JGinv_upts, detjac_upts);
  return launched("grad_transform_kernel");
}

fr_status fr_op_extrapolate_corrected_gradient(int n_fpts, int n_upts, int n_dims, int n_fields, int n_eles,
                                               const double* opp_6, const double* grad_disu_upts,
                                               double* grad_disu_fpts, void* stream)
{
  long long cols = (long long)n_fields * n_eles;
  for (int d = 0; d < n_dims; d++) {
    fr_status st = dense_apply(n_fpts, n_upts, cols, opp_6, grad_disu_upts + (size_t)n_upts * cols * d,
                               grad_disu_fpts + (size_t)n_fpts * cols * d, 0, ST(stream));
    if (st) return st;
  }
  return FR_OK;
}

fr_status fr_op_evaluate_viscFlux(int n_upts, int n_dims, int n_fields, int n_eles, const double* disu_upts,
                                  const double* grad_disu_upts, const double* JGinv_upts, double* tdisf_upts,
                                  const fr_phys_desc* phys, void* stream)
{
  if (!phys || !disu_upts || !grad_disu_upts || !JGinv_upts || !tdisf_upts || !dims_ok(n_dims, n_fields))
    return op_fail(FR_ERR_ARG, "bad arguments");
  long long n = (long long)n_upts * n_eles;
  if (n == 0) return FR_OK;
  if (n_dims == 2) vis_flux_kernel<2><<<grid_for(n, 128), 128, 0, ST(stream)>>>(n_upts, n_eles, disu_upts, grad_disu_upts, JGinv_upts, tdisf_upts, phys_of(phys));
  else vis_flux_kernel<3><<<grid_for(n, 128), 128, 0, ST(stream)>>>(n_upts, n_eles, disu_upts, grad_disu_upts, JGinv_upts, tdisf_upts, phys_of(phys));
  return launched("vis_flux_kernel");
}

fr_status fr_op_evaluate_viscFlux_les(int n_upts, int n_dims, int n_fields, int n_eles, const double* disu_upts,
                                      const double* grad_disu_upts, const double* JGinv_upts,
                                      const double* detjac_upts, double* tdisf_upts, double* sgsf_upts,
                                      const fr_phys_desc* phys, int sgs_model, double filter_ratio, int order,
                                      void* stream)
{
  if (!phys || !disu_upts || !grad_disu_upts || !JGinv_upts || !detjac_upts || !tdisf_upts || !sgsf_upts ||
      !dims_ok(n_dims, n_fields) || order < 1)
    return op_fail(FR_ERR_ARG, "bad arguments");
  if (sgs_model != 0 && sgs_model != 1)
    return op_fail(FR_ERR_UNSUPPORTED, "SGS models at the per-operator boundary: 0 (Smagorinsky), 1 (WALE)");
  if (!(filter_ratio > 0.0)) return op_fail(FR_ERR_ARG, "filter_ratio must be positive");
  long long n = (long long)n_upts * n_eles;
  if (n == 0) return FR_OK;
  PhysT<double> ph = phys_of(phys);
  ph.sgs_model = sgs_model;
  ph.filter_ratio = filter_ratio;
  if (n_dims == 2)
    vis_flux_les_kernel<2><<<grid_for(n, 128), 128, 0, ST(stream)>>>(n_upts, n_eles, disu_upts, grad_disu_upts, JGinv_upts, detjac_upts, tdisf_upts, sgsf_upts, ph, (double)(order + 1));
  else
    vis_flux_les_kernel<3><<<grid_for(n, 128), 128, 0, ST(stream)>>>(n_upts, n_eles, disu_upts, grad_disu_upts, JGinv_upts, detjac_upts, tdisf_upts, sgsf_upts, ph, (double)(order + 1));
  return launched("vis_flux_les_kernel");
}

fr_status fr_op_evaluate_sgsFlux(int n_fpts, int n_upts, int n_dims, int n_fields, int n_eles, const double* opp_0,
                                 const double* sgsf_upts, double* sgsf_fpts, void* stream)
{
  if (!opp_0 || !sgsf_upts || !sgsf_fpts || n_dims < 1 || n_dims > 3) return op_fail(FR_ERR_ARG, "bad arguments");
  const long long cols = (long long)n_fields * n_eles;
  for (int d = 0; d < n_dims; d++) {
    fr_status st = dense_apply(n_fpts, n_upts, cols, opp_0, sgsf_upts + (size_t)n_upts * cols * d,
                               sgsf_fpts + (size_t)n_fpts * cols * d, 0, ST(stream));
    if (st) return st;
  }
  return FR_OK;
}

fr_status fr_op_int_inters_common_viscFlux_les(int n_fpts_per_inter, int n_dims, int n_fields, int n_inters,
                                               double* const* disu_fpts_l, double* const* disu_fpts_r,
                                               double* const* grad_disu_fpts_l, double* const* grad_disu_fpts_r,
                                               double* const* norm_tconf_fpts_l, double* const* norm_tconf_fpts_r,
                                               double* const* tdA_fpts_l, double* const* tdA_fpts_r,
                                               double* const* norm_fpts, double* const* sgsf_fpts_l,
                                               double* const* sgsf_fpts_r, const fr_phys_desc* phys, void* stream)
{
  if (!phys || !sgsf_fpts_l || !sgsf_fpts_r || !dims_ok(n_dims, n_fields)) return op_fail(FR_ERR_ARG, "bad arguments");
  long long n = (long long)n_fpts_per_inter * n_inters;
  if (n == 0) return FR_OK;
  if (n_dims == 2)
    common_vis_kernel<2><<<grid_for(n, 128), 128, 0, ST(stream)>>>(n_fpts_per_inter, n_inters, disu_fpts_l, disu_fpts_r, grad_disu_fpts_l, grad_disu_fpts_r, norm_tconf_fpts_l, norm_tconf_fpts_r, tdA_fpts_l, tdA_fpts_r, norm_fpts, phys_of(phys), sgsf_fpts_l, sgsf_fpts_r);
  else
    common_vis_kernel<3><<<grid_for(n, 128), 128, 0, ST(stream)>>>(n_fpts_per_inter, n_inters, disu_fpts_l, disu_fpts_r, grad_disu_fpts_l, grad_disu_fpts_r, norm_tconf_fpts_l, norm_tconf_fpts_r, tdA_fpts_l, tdA_fpts_r, norm_fpts, phys_of(phys), sgsf_fpts_l, sgsf_fpts_r);
  return launched("common_vis_kernel");
}

fr_status fr_op_extrapolate_totalFlux(int n_fpts, int n_upts, int n_dims, int n_fields, int n_eles,
                                      const double* const* opp_1, const double* tdisf_upts, double* norm_tdisf_fpts,
                                      void* stream)
{
  if (!opp_1 || n_dims < 1 || n_dims > 3) return op_fail(FR_ERR_ARG, "bad arguments");
  long long cols = (long long)n_fields * n_eles;
  return dense_apply_nd(n_fpts, n_upts, cols, n_dims, opp_1, tdisf_upts, (long long)n_upts * cols, norm_tdisf_fpts, 0,
                        0, false, ST(stream));
}

fr_status fr_op_calculate_divergence(int n_upts, int n_dims, int n_fields, int n_eles, const double* const* opp_2,
                                     const double* tdisf_upts, double* div_tconf_upts, void* stream)
{
  if (!opp_2 || n_dims < 1 || n_dims > 3) return op_fail(FR_ERR_ARG, "bad arguments");
  long long cols = (long long)n_fields * n_eles;
  return dense_apply_nd(n_upts, n_upts, cols, n_dims, opp_2, tdisf_upts, (long long)n_upts * cols, div_tconf_upts, 0,
                        0, false, ST(stream));
}

fr_status fr_op_calculate_corrected_divergence(int n_upts, int n_fpts, int n_fields, int n_eles, const double* opp_3,
                                               const double* norm_tdisf_fpts, double* norm_tconf_fpts,
                                               double* div_tconf_upts, void* stream)
{
  long long n = (long long)n_fpts * n_fields * n_eles;
  if (n > 0) {
    axpy_kernel<<<grid_for(n, 256), 256, 0, ST(stream)>>>(n, -1.0, norm_tdisf_fpts, norm_tconf_fpts);
    fr_status st = launched("axpy_kernel");
    if (st) return st;
  }
  return dense_apply(n_upts, n_fpts, (long long)n_fields * n_eles, opp_3, norm_tconf_fpts, div_tconf_upts, 1,
                     ST(stream));
}

fr_status fr_op_int_inters_common_invFlux(int n_fpts_per_inter, int n_dims, int n_fields, int n_inters,
                                          double* const* disu_fpts_l, double* const* disu_fpts_r,
                                          double* const* norm_tconf_fpts_l, double* const* norm_tconf_fpts_r,
                                          double* const* tdA_fpts_l, double* const* tdA_fpts_r,
                                          double* const* norm_fpts, double* const* delta_disu_fpts_l,
                                          double* const* delta_disu_fpts_r, const fr_phys_desc* phys,
                                          int riemann_solve_type, int viscous, void* stream)
{
  if (!phys || !dims_ok(n_dims, n_fields)) return op_fail(FR_ERR_ARG, "bad arguments");
  if (riemann_solve_type != 0 && riemann_solve_type != 2)
    return op_fail(FR_ERR_UNSUPPORTED, "common flux: riemann_solve_type 0 (Rusanov) or 2 (Roe, 2-D)");
  if (riemann_solve_type == 2 && n_dims != 2) return op_fail(FR_ERR_UNSUPPORTED, "Roe flux is 2-D only");
  if (viscous && (!delta_disu_fpts_l || !delta_disu_fpts_r)) return op_fail(FR_ERR_ARG, "viscous needs delta tables");
  long long n = (long long)n_fpts_per_inter * n_inters;
  if (n == 0) return FR_OK;
  if (n_dims == 2)
    common_inv_kernel<2><<<grid_for(n, 128), 128, 0, ST(stream)>>>(n_fpts_per_inter, n_inters, disu_fpts_l, disu_fpts_r, norm_tconf_fpts_l, norm_tconf_fpts_r, tdA_fpts_l, tdA_fpts_r, norm_fpts, delta_disu_fpts_l, delta_disu_fpts_r, phys_of(phys), riemann_solve_type, viscous);
  else
    common_inv_kernel<3><<<grid_for(n, 128), 128, 0, ST(stream)>>>(n_fpts_per_inter, n_inters, disu_fpts_l, disu_fpts_r, norm_tconf_fpts_l, norm_tconf_fpts_r, tdA_fpts_l, tdA_fpts_r, norm_fpts, delta_disu_fpts_l, delta_disu_fpts_r, phys_of(phys), riemann_solve_type, viscous);
  return launched("common_inv_kernel");
}

fr_status fr_op_int_inters_common_viscFlux(int n_fpts_per_inter, int n_dims, int n_fields, int n_inters,
                                           double* const* disu_fpts_l, double* const* disu_fpts_r,
                                           double* const* grad_disu_fpts_l, double* const* grad_disu_fpts_r,
                                           double* const* norm_tconf_fpts_l, double* const* norm_tconf_fpts_r,
                                           double* const* tdA_fpts_l, double* const* tdA_fpts_r,
                                           double* const* norm_fpts, const fr_phys_desc* phys, void* stream)
{
  if (!phys || !dims_ok(n_dims, n_fields)) return op_fail(FR_ERR_ARG, "bad arguments");
  long long n = (long long)n_fpts_per_inter * n_inters;
  if (n == 0) return FR_OK;
  if (n_dims == 2)
    common_vis_kernel<2><<<grid_for(n, 128), 128, 0, ST(stream)>>>(n_fpts_per_inter, n_inters, disu_fpts_l, disu_fpts_r, grad_disu_fpts_l, grad_disu_fpts_r, norm_tconf_fpts_l, norm_tconf_fpts_r, tdA_fpts_l, tdA_fpts_r, norm_fpts, phys_of(phys));
  else
    common_vis_kernel<3><<<grid_for(n, 128), 128, 0, ST(stream)>>>(n_fpts_per_inter, n_inters, disu_fpts_l, disu_fpts_r, grad_disu_fpts_l, grad_disu_fpts_r, norm_tconf_fpts_l, norm_tconf_fpts_r, tdA_fpts_l, tdA_fpts_r, norm_fpts, phys_of(phys));
  return launched("common_vis_kernel");
}

fr_status fr_op_bdy_inters_common_invFlux(int n_fpts_per_inter, int n_dims, int n_fields, int n_inters,
                                          double* const* disu_fpts_l, double* const* norm_tconf_fpts_l,
                                          double* const* tdA_fpts_l, double* const* norm_fpts,
                                          const int* boundary_type, const double* bdy_params,
                                          double* const* delta_disu_fpts_l, const fr_phys_desc* phys, double R_ref,
                                          int riemann_solve_type, int viscous, void* stream)
{
  if (!phys || !dims_ok(n_dims, n_fields) || n_fpts_per_inter < 0 || n_inters < 0)
    return op_fail(FR_ERR_ARG, "bad arguments");
  if (riemann_solve_type != 0 && riemann_solve_type != 2)
    return op_fail(FR_ERR_UNSUPPORTED, "boundary fluxes: riemann_solve_type 0 (Rusanov) or 2 (Roe, 2-D)");
  if (riemann_solve_type == 2 && n_dims != 2) return op_fail(FR_ERR_UNSUPPORTED, "Roe flux is 2-D only");
  long long n = (long long)n_fpts_per_inter * n_inters;
  if (n == 0) return FR_OK;
  if (!disu_fpts_l || !norm_tconf_fpts_l || !tdA_fpts_l || !norm_fpts || !boundary_type || !bdy_params ||
      (viscous && !delta_disu_fpts_l))
    return op_fail(FR_ERR_ARG, "missing boundary table");
  PhysT<double> ph = phys_of(phys);
  ph.R_ref = R_ref;
  if (n_dims == 2)
    bdy_inv_kernel<2><<<grid_for(n, 128), 128, 0, ST(stream)>>>(n_fpts_per_inter, n_inters, disu_fpts_l, norm_tconf_fpts_l, tdA_fpts_l, norm_fpts, delta_disu_fpts_l, boundary_type, bdy_params, ph, riemann_solve_type, viscous);
  else
    bdy_inv_kernel<3><<<grid_for(n, 128), 128, 0, ST(stream)>>>(n_fpts_per_inter, n_inters, disu_fpts_l, norm_tconf_fpts_l, tdA_fpts_l, norm_fpts, delta_disu_fpts_l, boundary_type, bdy_params, ph, riemann_solve_type, viscous);
  return launched("bdy_inv_kernel");
}

fr_status fr_op_bdy_inters_common_viscFlux(int n_fpts_per_inter, int n_dims, int n_fields, int n_inters,
                                           double* const* disu_fpts_l, double* const* grad_disu_fpts_l,
                                           double* const* norm_tconf_fpts_l, double* const* tdA_fpts_l,
                                           double* const* norm_fpts, const int* boundary_type,
                                           const double* bdy_params, const fr_phys_desc* phys, double R_ref,
                                           void* stream)
{
  if (!phys || !dims_ok(n_dims, n_fields) || n_fpts_per_inter < 0 || n_inters < 0)
    return op_fail(FR_ERR_ARG, "bad arguments");
  long long n = (long long)n_fpts_per_inter * n_inters;
  if (n == 0) return FR_OK;
  if (!disu_fpts_l || !grad_disu_fpts_l || !norm_tconf_fpts_l || !tdA_fpts_l || !norm_fpts || !boundary_type ||
      !bdy_params)
    return op_fail(FR_ERR_ARG, "missing boundary table");
  PhysT<double> ph = phys_of(phys);
  ph.R_ref = R_ref;
  if (n_dims == 2)
    bdy_vis_kernel<2><<<grid_for(n, 128), 128, 0, ST(stream)>>>(n_fpts_per_inter, n_inters, disu_fpts_l, grad_disu_fpts_l, norm_tconf_fpts_l, tdA_fpts_l, norm_fpts, boundary_type, bdy_params, ph);
  else
    bdy_vis_kernel<3><<<grid_for(n, 128), 128, 0, ST(stream)>>>(n_fpts_per_inter, n_inters, disu_fpts_l, grad_disu_fpts_l, norm_tconf_fpts_l, tdA_fpts_l, norm_fpts, boundary_type, bdy_params, ph);
  return launched("bdy_vis_kernel");
}

fr_status fr_op_spmv_ell(int m, int n, int n_fields, int n_eles, const double* ell_data, const int* ell_indices,
                         int nnz_per_row, const double* b, double* c, int cell_type, int order, int add_flag,
                         void* stream)
{
  (void)cell_type;
  (void)order;
  if (m <= 0 || n <= 0 || n_fields <= 0 || n_eles < 0 || nnz_per_row < 0 || (add_flag != 0 && add_flag != 1) ||
      !ell_data || !ell_indices || !b || !c)
    return op_fail(FR_ERR_ARG, "bad arguments");
  const long long cols = (long long)n_fields * n_eles;
  if (cols == 0) return FR_OK;
  const size_t smem = (size_t)n * kTileStride * sizeof(double);
  if (smem > kDenseSmem || m > 32 * 8) return op_fail(FR_ERR_UNSUPPORTED, "sparse operator too large");
  const long long blocks = (cols + kTileCols - 1) / kTileCols;
  if (blocks > 2147483647LL) return op_fail(FR_ERR_ARG, "too many columns");
  const int rm = (m + 31) / 32;
  auto kern = rm == 1 ? spmv_ell_kernel<1> : rm == 2 ? spmv_ell_kernel<2> : rm == 3 ? spmv_ell_kernel<3>
            : rm == 4 ? spmv_ell_kernel<4> : rm == 5 ? spmv_ell_kernel<5> : rm == 6 ? spmv_ell_kernel<6>
            : rm == 7 ? spmv_ell_kernel<7> : spmv_ell_kernel<8>;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return op_fail(FR_ERR_CUDA, cudaGetErrorString(e));
  }
  kern<<<(unsigned)blocks, kDenseThreads, smem, ST(stream)>>>(m, n, cols, ell_data, ell_indices, nnz_per_row, b, c,
                                                             add_flag);
  return launched("spmv_ell_kernel");
}

fr_status fr_op_advance_rk45(int n_upts, int n_fields, int n_eles, int stage, double dt, double const_src,
                             double* disu_upts_0, double* disu_upts_1, const double* div_tconf_upts,
                             const double* detjac_upts, const double* src_upts, void* stream)
{
  static const double A[5] = {0.0, -0.417890474499852, -1.192151694642677, -1.697784692471528, -1.514183444257156};
  static const double B[5] = {0.149659021999229, 0.379210312999627, 0.822955029386982, 0.699450455949122,
                              0.153057247968152};
  if (stage < 0 || stage > 4 || !disu_upts_0 || !disu_upts_1 || !div_tconf_upts || !detjac_upts)
    return op_fail(FR_ERR_ARG, "bad arguments");
  long long n = (long long)n_upts * n_eles * n_fields;
  if (n == 0) return FR_OK;
  rk45_kernel<<<grid_for(n, 256), 256, 0, ST(stream)>>>(n_upts, n_eles, n_fields, disu_upts_0, disu_upts_1,
                                                       div_tconf_upts, detjac_upts, src_upts, A[stage], B[stage], dt,
                                                       const_src);
  return launched("rk45_kernel");
}

}  // extern "C"
