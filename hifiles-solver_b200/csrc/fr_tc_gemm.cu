// fr_tc_gemm.cu -- the dense operator product of the per-operator seam,
// C = A B (+ C), on the fifth-generation tensor cores in BF16 with a 3-term
// split and FP32 accumulation: the GEMM precision form of the reference's
// cublasDgemm('N','N', m, ncols, k, 1, opp, m, B, k, beta, C, m) calls
// (eles::extrapolate_solution, calculate_gradient, ... , src/eles.cpp).
//
// Each column j of B is split after subtracting its first entry c_j: A B =
// A (B - c 1^T) + (A 1) c^T, with the row sums A 1 and the second term in
// FP64, so the BF16 parts carry only the variation inside an element's column
// (the state's free-stream level needs no BF16 bits).
// Split: x = x0 + x1 + x2 with x0 = bf16(x), x1 = bf16(x - x0),
// x2 = bf16(x - x0 - x1).  TERMS = 3 (BF16x3) keeps x0y0 + x0y1 + x1y0, about
// 16 bits; TERMS = 6 (BF16x6) adds x0y2 + x1y1 + x2y0, about 24 bits (FP32
// level).  Either is one accumulation over K' = TERMS KP:
//   BF16x3:  A' = [A0 | A0 | A1],            B' = [B0 ; B1 ; B0]
//   BF16x6:  A' = [A0 | A0 | A1 | A0 | A1 | A2],  B' = [B0 ; B1 ; B0 ; B2 ; B1 ; B0]
// Shared memory holds each distinct part once (2 or 3 of A and of B); the
// descriptors of each K-copy point at its parts.
// KP is k rounded up to 16 (zeros); MT = 1 or 2 MMA tiles of 128 rows cover
// the operator's m <= 256 rows (zero rows beyond m); TN = 64 or 32 columns
// per tile, the larger that fits shared memory.  Inputs and outputs stay FP64
// in HBM.
//
// One block of 128 threads per tile pass, persistent over column tiles:
// the threads stage A' once and B' per tile into shared memory in the
// K-major, no-swizzle canonical layout (8 x 16-byte core matrices), one
// thread issues the MT K'/16 tcgen05.mma instructions into MT TMEM
// accumulators (128 lanes x TN columns each) and commits them to an
// mbarrier; the four warps read their 32 lanes of each back with tcgen05.ld
// and write C.  Every mbarrier wait
// is bounded: on expiry the kernel sets the error flag and waits once more
// (bounded) for its MMAs; it frees its TMEM only when they have completed
// (otherwise the allocation is left held rather than released under MMAs that
// may still write it).
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include <mutex>
#include <string>

#include "fr_b200.h"

namespace frb {
extern thread_local std::string g_err;

namespace {

constexpr int kTM = 128;          // rows of one MMA tile (operator rows, zero-padded)
constexpr int kThreads = 128;
constexpr uint32_t kTmemCols = 64;    // MT x TN accumulator columns (64 in both shapes)
constexpr long long kWaitLimit = 1LL << 20;   // x 1 us suspend hint: about a second

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor, K-major, no swizzle (layout type 0),
// descriptor version 1; offsets in bytes (16-byte units in the descriptor)
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N >> 3 at bit 17, M >> 4 at bit 24
template <int TN>
__host__ __device__ constexpr uint32_t idesc_bf16()
{
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN >> 3) << 17) | ((uint32_t)(kTM >> 4) << 24);
}

template <int TN>
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate)
{
  constexpr uint32_t kIdesc = idesc_bf16<TN>();
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
      "}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity)
{
  uint32_t ok;
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t"
      "}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(1000u)
      : "memory");
  return ok != 0;
}

// bounded wait on an mbarrier phase; false when the limit ran out
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity)
{
  for (long long i = 0; i < kWaitLimit; i++)
    if (mbar_try(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32])
{
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// 8 values -> 16-byte chunks of their three BF16 parts (x0 + x1 + x2 = x to
// about 24 bits; each residual is formed in FP64)
__device__ __forceinline__ void split8(const double (&x)[8], uint4 (&q)[3])
{
  uint32_t w[3][4];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    uint32_t lo16[3], hi16[3];
#pragma unroll
    for (int h = 0; h < 2; h++) {
      double r = x[2 * i + h];
#pragma unroll
      for (int t = 0; t < 3; t++) {
        const __nv_bfloat16 b = __double2bfloat16(r);
        r -= (double)__bfloat162float(b);
        (h ? hi16 : lo16)[t] = __bfloat16_as_ushort(b);
      }
    }
#pragma unroll
    for (int t = 0; t < 3; t++) w[t][i] = lo16[t] | (hi16[t] << 16);
  }
#pragma unroll
  for (int t = 0; t < 3; t++) q[t] = make_uint4(w[t][0], w[t][1], w[t][2], w[t][3]);
}

// part of A' (a = 1) or B' (a = 0) in K-copy j of the split product
__host__ __device__ constexpr int part_of(int j, int a)
{
  // BF16x3: A 0 0 1, B 0 1 0; BF16x6: A 0 0 1 0 1 2, B 0 1 0 2 1 0
  constexpr int PA[6] = {0, 0, 1, 0, 1, 2}, PB[6] = {0, 1, 0, 2, 1, 0};
  return a ? PA[j] : PB[j];
}

// distinct parts kept of each operand: 2 (BF16x3) or 3 (BF16x6)
__host__ __device__ constexpr int n_parts(int terms) { return terms == 6 ? 3 : 2; }

// byte offset of 16-byte chunk (row, kchunk) of a K-major tile of R rows
__device__ __forceinline__ uint32_t chunk_off(int row, int kc, int R)
{
  return (uint32_t)((kc * (R / 8) + row / 8) * 128 + (row % 8) * 16);
}

// PF > 0: software-pipelined B.  Each thread holds the raw FP64 chunks it
// splits for the next column tile in registers (at most PF chunks of 8
// values: TN * KP / 8 <= PF * kThreads), loaded right after the current
// tile's split, so the loads of tile t + 1 are in flight while tile t's MMAs
// run and its accumulators are read back.  The arithmetic is the same as with
// PF = 0 (B read at the split), so both give identical results.
template <int TERMS, int MT, int TN, int PF = 0>
__global__ void __launch_bounds__(kThreads)
fr_gemm_bf16x3_kernel(int m, int k, int KP, long long ncols, const double* __restrict__ A,
                      const double* __restrict__ B, double* __restrict__ C, int beta, int* __restrict__ err)
{
  static_assert(MT * TN == (int)kTmemCols, "accumulator columns");
  constexpr int RA = MT * kTM;             // rows of A'
  constexpr int NP = n_parts(TERMS);
  extern __shared__ __align__(1024) unsigned char sm[];
  const int KC = KP / 8;                   // 16-byte chunks of one part (KP values)
  const size_t tileA = (size_t)kTM * KC * 16, partA = (size_t)MT * tileA, partB = (size_t)TN * KC * 16;
  unsigned char* sA = sm;                  // NP parts x MT tiles of kTM x KP bf16
  unsigned char* sB = sm + NP * partA;     // NP parts of TN x KP bf16
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_slot;
  __shared__ double rowsum[RA];            // A 1 (FP64, column order)
  __shared__ double cB[TN];                // first entry of each B column of the tile
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // A' once: rows r (fastest) x chunks c of A; tile mt holds rows 128 mt ..
  for (int w = tid; w < RA * KC; w += kThreads) {
    const int r = w % RA, c = w / RA, mt = r / kTM, rr = r % kTM;
    double x[8];
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int kk = 8 * c + i;
      x[i] = (r < m && kk < k) ? __ldg(A + r + (size_t)m * kk) : 0.0;
    }
    uint4 q[3];
    split8(x, q);
#pragma unroll
    for (int pp = 0; pp < NP; pp++)
      *reinterpret_cast<uint4*>(sA + pp * partA + mt * tileA + chunk_off(rr, c, kTM)) = q[pp];
  }
  for (int r = tid; r < RA; r += kThreads) {
    double acc = 0.0;
    if (r < m)
      for (int kk = 0; kk < k; kk++) acc += __ldg(A + r + (size_t)m * kk);
    rowsum[r] = acc;
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = tmem_slot;
  bool drained = true;                     // no MMA of this block may still be running
  const long long ntiles = (ncols + TN - 1) / TN;
  uint32_t parity = 0;
  constexpr int PFW = PF > 0 ? PF : 1;
  double xn[PFW][8];                       // PF: the next tile's raw chunks (w = tid + q kThreads)
  auto load_next = [&](long long tt) {
    const long long jn = tt * TN;
#pragma unroll
    for (int q = 0; q < PFW; q++) {
      const int w = tid + q * kThreads, n = w % TN, c = w / TN;
      const long long j = jn + n;
#pragma unroll
      for (int i = 0; i < 8; i++) {
        const int kk = 8 * c + i;
        xn[q][i] = (w < TN * KC && j < ncols && kk < k) ? __ldg(B + (size_t)j * k + kk) : 0.0;
      }
    }
  };
  if (PF > 0 && blockIdx.x < ntiles) load_next(blockIdx.x);
  for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const long long j0 = t * TN;
    if constexpr (PF > 0) {
      // the column levels: the thread holding chunk 0 of column n
#pragma unroll
      for (int q = 0; q < PFW; q++) {
        const int w = tid + q * kThreads;
        if (w < TN) cB[w] = j0 + w < ncols ? xn[q][0] : 0.0;
      }
    } else {
      for (int n = tid; n < TN; n += kThreads) cB[n] = j0 + n < ncols ? __ldg(B + (size_t)(j0 + n) * k) : 0.0;
    }
    __syncthreads();
    // B' for columns j0 ..: columns n (fastest) x chunks c, less the column's first entry
    if constexpr (PF > 0) {
#pragma unroll
      for (int q = 0; q < PFW; q++) {
        const int w = tid + q * kThreads, n = w % TN, c = w / TN;
        if (w >= TN * KC) continue;
        const long long j = j0 + n;
        double x[8];
#pragma unroll
        for (int i = 0; i < 8; i++) {
          const int kk = 8 * c + i;
          x[i] = (j < ncols && kk < k) ? xn[q][i] - cB[n] : 0.0;
        }
        uint4 qq[3];
        split8(x, qq);
#pragma unroll
        for (int pp = 0; pp < NP; pp++) *reinterpret_cast<uint4*>(sB + pp * partB + chunk_off(n, c, TN)) = qq[pp];
      }
      // the next tile's loads stay in flight through this tile's MMAs and read-back
      if (t + gridDim.x < ntiles) load_next(t + gridDim.x);
    } else {
      for (int w = tid; w < TN * KC; w += kThreads) {
        const int n = w % TN, c = w / TN;
        const long long j = j0 + n;
        double x[8];
#pragma unroll
        for (int i = 0; i < 8; i++) {
          const int kk = 8 * c + i;
          x[i] = (j < ncols && kk < k) ? __ldg(B + (size_t)j * k + kk) - cB[n] : 0.0;
        }
        uint4 q[3];
        split8(x, q);
#pragma unroll
        for (int pp = 0; pp < NP; pp++) *reinterpret_cast<uint4*>(sB + pp * partB + chunk_off(n, c, TN)) = q[pp];
      }
    }
    // generic-proxy writes -> visible to the tensor cores' reads
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    fence_before();
    __syncthreads();
    fence_after();
    if (tid == 0) {
      // K-copy j multiplies A part part_of(j, 1) with B part part_of(j, 0)
#pragma unroll
      for (int j = 0; j < TERMS; j++) {
        const uint32_t b0 = smem_u32(sB + part_of(j, 0) * partB);
        for (int s = 0; s < KC / 2; s++) {
          const uint64_t bd = umma_desc(b0 + (uint32_t)(2 * s) * (TN / 8) * 128, (TN / 8) * 128, 128);
#pragma unroll
          for (int mt = 0; mt < MT; mt++) {
            const uint32_t a0 = smem_u32(sA + part_of(j, 1) * partA + mt * tileA);
            const uint64_t ad = umma_desc(a0 + (uint32_t)(2 * s) * (kTM / 8) * 128, (kTM / 8) * 128, 128);
            mma_bf16<TN>(tmem + (uint32_t)(mt * TN), ad, bd, (j > 0 || s > 0) ? 1u : 0u);
          }
        }
      }
      mma_commit(&bar);
    }
    // every thread waits (bounded); the block leaves together if any ran out
    if (!__syncthreads_and(mbar_wait(&bar, parity) ? 1 : 0)) {
      if (tid == 0) atomicExch(err, 1);
      // the MMAs may still be running: wait once more, and keep the TMEM
      // allocated unless they are known to have completed
      drained = __syncthreads_and(mbar_wait(&bar, parity) ? 1 : 0) != 0;
      break;
    }
    parity ^= 1u;
    fence_after();
    // accumulator mt, lanes 32 warp .. +31 -> rows 128 mt + 32 warp + lane of C
#pragma unroll
    for (int mt = 0; mt < MT; mt++) {
      const int r = mt * kTM + 32 * warp + lane;
#pragma unroll
      for (int h = 0; h < TN / 32; h++) {
        float v[32];
        tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(mt * TN + 32 * h), v);
        if (r < m) {
#pragma unroll
          for (int i = 0; i < 32; i++) {
            const long long j = j0 + 32 * h + i;
            if (j < ncols) {
              double* c = C + r + (size_t)m * j;
              const double ab = (double)v[i] + cB[32 * h + i] * rowsum[r];
              *c = beta ? *c + ab : ab;
            }
          }
        }
      }
    }
    fence_before();
    __syncthreads();
    fence_after();
  }
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 0 && drained)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

// the timeout flag of the products, one per device (allocated on that device)
constexpr int kMaxDevices = 64;
std::mutex g_gemm_err_mutex;
int* g_gemm_err[kMaxDevices] = {};

fr_status gemm_err_flag(int** out)
{
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess && (dev < 0 || dev >= kMaxDevices)) e = cudaErrorInvalidDevice;
  if (e != cudaSuccess) {
    g_err = cudaGetErrorString(e);
    return FR_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lock(g_gemm_err_mutex);
  if (!g_gemm_err[dev]) {
    e = cudaMalloc(&g_gemm_err[dev], sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(g_gemm_err[dev], 0, sizeof(int));
    if (e != cudaSuccess) {
      g_err = cudaGetErrorString(e);
      return FR_ERR_CUDA;
    }
  }
  *out = g_gemm_err[dev];
  return FR_OK;
}

}  // namespace

// Shared memory of one block: the distinct parts of A (mt tiles of 128 rows)
// and of the B tile.
static size_t gemm_split_smem(int k, int terms, int mt, int tn)
{
  const int KP = (k + 15) / 16 * 16;
  return (size_t)(mt * kTM + tn) * n_parts(terms) * KP * 2;
}

// chunks of 8 B values a thread holds for the next column tile (software
// pipelining; 0 turns it off); the pipelined form can be switched off for
// comparisons (fr_tc_gemm_set_prefetch)
constexpr int kPrefetchChunks = 4;
int g_gemm_prefetch = 1;

// dynamic shared memory a block may use (227 kB less the static part: the
// barrier, the TMEM slot, the row sums and the column shifts, under 3 kB)
static constexpr size_t kSmemMax = 232448 - 3072;

// tile shape for an m x k operator: {MT, TN}, or {0, 0} when none fits
static void gemm_split_shape(int m, int k, int terms, int& mt, int& tn)
{
  mt = m <= kTM ? 1 : (m <= 2 * kTM ? 2 : 0);
  tn = mt == 1 ? 64 : 32;
  if (mt == 0 || k < 1 || gemm_split_smem(k, terms, mt, tn) > kSmemMax) mt = tn = 0;
}

bool gemm_split_supported(int m, int k, int terms)
{
  int mt, tn;
  gemm_split_shape(m, k, terms, mt, tn);
  return m >= 1 && mt > 0;
}

template <int TERMS, int MT, int TN, int PF>
static fr_status launch_split(int m, int k, long long ncols, const double* A, const double* B, double* C, int beta,
                              cudaStream_t s)
{
  const size_t smem = gemm_split_smem(k, TERMS, MT, TN);
  const void* kfn = (const void*)fr_gemm_bf16x3_kernel<TERMS, MT, TN, PF>;
  cudaError_t e = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) {
    g_err = cudaGetErrorString(e);
    return FR_ERR_CUDA;
  }
  cudaFuncSetAttribute(kfn, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  int dev = 0, sms = 0, per = 0, smem_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kfn, kThreads, smem);
  // blocks that fit by shared memory (3 kB static and 1 kB reserved per block)
  const int by_smem = smem_sm > 0 ? (int)((size_t)smem_sm / (smem + 4096)) : 1;
  if (by_smem > per) per = by_smem;
  // each block holds kTmemCols of the SM's 512 TMEM columns: more blocks
  // would only wait in tcgen05.alloc
  if (per > (int)(512 / kTmemCols)) per = (int)(512 / kTmemCols);
  int* err = nullptr;
  fr_status fs = gemm_err_flag(&err);
  if (fs) return fs;
  const long long ntiles = (ncols + TN - 1) / TN;
  long long grid = (long long)(per > 0 ? per : 1) * (sms > 0 ? sms : 1);
  if (grid > ntiles) grid = ntiles;
  fr_gemm_bf16x3_kernel<TERMS, MT, TN, PF><<<(unsigned)grid, kThreads, smem, s>>>(m, k, (k + 15) / 16 * 16, ncols, A,
                                                                                  B, C, beta, err);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    g_err = std::string("fr_gemm_bf16x3_kernel: ") + cudaGetErrorString(e);
    return FR_ERR_CUDA;
  }
  return FR_OK;
}

fr_status gemm_bf16x3(int m, int k, long long ncols, const double* A, const double* B, double* C, int beta,
                      cudaStream_t s, int terms)
{
  if (terms != 3 && terms != 6) {
    g_err = "split products have 3 or 6 terms";
    return FR_ERR_ARG;
  }
  int mt, tn;
  gemm_split_shape(m, k, terms, mt, tn);
  if (m < 1 || mt == 0) {
    g_err = std::string(terms == 6 ? "BF16x6" : "BF16x3") + " operator product: " + std::to_string(m) + " x " +
            std::to_string(k) + " does not fit one block's shared memory";
    return FR_ERR_UNSUPPORTED;
  }
  if (ncols == 0) return FR_OK;
  // software-pipelined B when a thread's share of the column tile fits its
  // registers (kPrefetchChunks chunks of 8 values)
  const int kp = (k + 15) / 16 * 16;
  // (measured: 2 % faster for BF16x3, 6 % slower for BF16x6, whose six MMA
  // copies already overlap the loads of the other blocks)
  const bool pf = terms == 3 && (long long)tn * (kp / 8) <= (long long)kPrefetchChunks * kThreads && g_gemm_prefetch;
  if (terms == 3) {
    if (mt == 1) return pf ? launch_split<3, 1, 64, kPrefetchChunks>(m, k, ncols, A, B, C, beta, s)
                           : launch_split<3, 1, 64, 0>(m, k, ncols, A, B, C, beta, s);
    return pf ? launch_split<3, 2, 32, kPrefetchChunks>(m, k, ncols, A, B, C, beta, s)
              : launch_split<3, 2, 32, 0>(m, k, ncols, A, B, C, beta, s);
  }
  if (mt == 1) return pf ? launch_split<6, 1, 64, kPrefetchChunks>(m, k, ncols, A, B, C, beta, s)
                         : launch_split<6, 1, 64, 0>(m, k, ncols, A, B, C, beta, s);
  return pf ? launch_split<6, 2, 32, kPrefetchChunks>(m, k, ncols, A, B, C, beta, s)
            : launch_split<6, 2, 32, 0>(m, k, ncols, A, B, C, beta, s);
}

// FR_ERR_TIMEOUT if a tensor-core product gave up waiting for its MMAs since
// the last check (the flag is cleared); synchronises the stream.
void gemm_set_prefetch(int on) { g_gemm_prefetch = on ? 1 : 0; }

fr_status gemm_bf16x3_check(cudaStream_t s)
{
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices || !g_gemm_err[dev]) return FR_OK;
  int* flag = g_gemm_err[dev];
  int v = 0;
  cudaError_t e = cudaMemcpyAsync(&v, flag, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    g_err = cudaGetErrorString(e);
    return FR_ERR_CUDA;
  }
  if (v) {
    cudaMemsetAsync(flag, 0, sizeof(int), s);
    g_err = "tensor-core operator product: MMA completion wait ran out";
    return FR_ERR_TIMEOUT;
  }
  return FR_OK;
}

}  // namespace frb
