// fr_mixed_fused.cu -- fused RK stage for meshes of dense-operator element
// types (tetrahedra, prisms, hexahedra through their dense operators): the
// whole CalcResidual + RK45 update (src/solver.cpp:65-225, src/eles.cpp:
// 1155-1178) in two kernels per element type and stage, instead of the ~20
// calls of the per-operator path.
//
// Flux-point space: the flux points of every element type, numbered
// type by type (off_t + f + n_fpts_t e); traces UF (two buffers, read by the
// stage that follows the one that wrote them), viscous normal projections VF,
// left normals nL, own tdA, the neighbour of each point (mate, or -1 - the
// point's place in the boundary list) and its side bits (bit 0 left side,
// bits 2.. the boundary type) are stored over that space, so a neighbour of
// another element type is one index away.
//
// Kernel A (mixed_grad_kernel), per block of EPB elements, in shared memory:
//   own traces (read) -> LDG common solution delta at the flux points
//   (int_inters::calculate_common_invFlux's viscous part, bdy_inters'
//   boundary states) -> grad = opp_4 U + opp_5 delta (calculate_gradient,
//   correct_gradient) -> physical gradient (JGinv / detJ) -> opp_6 grad at the
//   flux points -> viscous normal projections VF / boundary viscous fluxes BV
//   -> transformed inviscid + viscous flux at the solution points ->
//   norm_tdisf = sum_d opp_1[d] f_d and div_tdisf = sum_d opp_2[d] f_d.
// Kernel B (mixed_update_kernel): Rusanov + LDG common normal fluxes at the
//   own flux points from both sides' traces and projections (both sides of
//   an interface evaluate the same expression on the same inputs, left side
//   first, so the two values are bit-identical), minus norm_tdisf ->
//   div = div_tdisf + opp_3 (norm_tconf - norm_tdisf) -> RK45 update of the
//   state and register (or div_tconf alone) -> traces of the new state,
//   opp_0 U, into the other trace buffer.
//
// Operator products run on the FP64 tensor cores (mma.sync m8n8k4 f64): each
// operator is stored in fragment order (8-row tiles x 4-column steps, 32
// entries per fragment in lane order), the element data in shared memory as
// column-major matrices, one column per (element, field[, dimension]), whose
// leading dimension is 4 or 12 mod 16 doubles so that a fragment load hits
// 16 distinct banks per half-warp.  Padding rows of the operators are zero
// and every padding row of the data that a product reads is set to zero, so
// padded products add exact zeros.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "fr_b200.h"
#include "fr_face_update.cuh"
#include "fr_physics.cuh"

namespace frb {
extern thread_local std::string g_err;
}
using namespace frb;

namespace {

fr_status mfail(fr_status s, const std::string& m)
{
  g_err = m;
  return s;
}

fr_status mlaunched(const char* what)
{
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return mfail(FR_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return FR_OK;
}

constexpr int kMixedEPB = 8;   // elements per block: 8 x (D + 2) columns fill whole 8-column tiles
constexpr int kMixedNT = 256;  // threads per block

__host__ __device__ constexpr int c4(int x) { return (x + 3) / 4 * 4; }
__host__ __device__ constexpr int c8(int x) { return (x + 7) / 8 * 8; }
__host__ __device__ constexpr int cmax(int a, int b) { return a > b ? a : b; }
// smallest leading dimension >= x that is 4 or 12 mod 16
__host__ __device__ constexpr int bank_ld(int x) { return (x % 16 == 4 || x % 16 == 12) ? x : bank_ld(x + 1); }
// column tiles per warp unit: all of them up to 6, else a divisor
__host__ __device__ constexpr int tiles_per_unit(int ntl)
{
  return ntl <= 6 ? ntl : (ntl % 5 == 0 ? 5 : (ntl % 4 == 0 ? 4 : (ntl % 3 == 0 ? 3 : 4)));
}

// Shared-memory plan and product shapes of one element type (doubles).
constexpr size_t kMixedSmemMax = 227 * 1024;  // dynamic shared memory of one block
__host__ __device__ constexpr int r2(int x) { return (x + 1) / 2 * 2; }  // 16-byte region starts

template <int D, int NU, int NF, int EPB, int MINB = 1>
struct MPlan {
  static constexpr int F = D + 2, DD = D * D, EU = EPB * NU, EF = EPB * NF;
  static constexpr int N = EPB * F, NP = c8(N);          // (element, field) columns
  static constexpr int NG = N * D, NGP = c8(NG);         // (element, field, dimension) columns
  static constexpr int ldU = bank_ld(c4(NU));
  static constexpr int ldF = bank_ld(c8(NF));
  static constexpr int ldG = bank_ld(cmax(c8(D * NU), (D - 1) * NU + c4(NU)));
  static constexpr int ldT = bank_ld(c4(D * NU));
  static constexpr int MT_U = c8(NU) / 8, MT_F = c8(NF) / 8, MT_G = c8(D * NU) / 8;
  static constexpr int KS_U = c4(NU) / 4, KS_F = c4(NF) / 4, KS_T = c4(D * NU) / 4;
  static constexpr int NTL = NP / 8, NTLG = NGP / 8;
  static constexpr int TN = tiles_per_unit(NTL), TNG = tiles_per_unit(NTLG);
  // kernel A: the matrices U | own traces | gradient (the neighbours' traces
  // [F][EF] before it) | X (delta, then the gradient at the flux points, then
  // the transformed flux); then what the load phase stages: left normals
  // [D][EF], detJ [EU], JGinv [EPB][DD NU] (when it fits), mate and side [EF]
  // ints each
  static constexpr int oU = 0, oUF = oU + NP * ldU, oG = oUF + NP * ldF, oX = oG + NP * ldG;
  static constexpr int nX = cmax(cmax(NP * ldF, NGP * ldF), NP * ldT);
  static constexpr int oNL = oX + r2(nX), oDJ = oNL + r2(D * EF), oJG = oDJ + r2(EU);
  // JGinv is staged when MINB blocks with it fit in an SM's shared memory
  // (228 KB, 1 KB reserved per block), else read through the L1 cache
  static constexpr bool SJ = (size_t)MINB * (sizeof(double) * (size_t)(oJG + r2(DD * EU) + r2(EF)) + 1024) <=
                                 228 * 1024 &&
                             sizeof(double) * (size_t)(oJG + r2(DD * EU) + r2(EF)) <= kMixedSmemMax;
  static constexpr int oIA = oJG + (SJ ? r2(DD * EU) : 0);
  static constexpr int nA = oIA + r2(EF);
  // kernel B: the jump norm_tconf - norm_tdisf (norm_tdisf first) | own traces
  // [F][EF] (the new state [NP][ldU] after the flux phase) | neighbours'
  // traces | own and neighbours' viscous projections [F-1][EF] | left normals
  // [D][EF] | tdA [EF] | div_tdisf, RK register, state [F][EU] | detJ [EU] |
  // mate and side
  static constexpr int oJ = 0, oUo = r2(NP * ldF), oUN = oUo + r2(cmax(F * EF, NP * ldU));
  static constexpr int oVo = oUN + r2(F * EF), oVN = oVo + r2((F - 1) * EF), oNLb = oVN + r2((F - 1) * EF);
  static constexpr int oTA = oNLb + r2(D * EF), oDV = oTA + r2(EF), oRG = oDV + r2(F * EU), oUO = oRG + r2(F * EU);
  static constexpr int oDJb = oUO + r2(F * EU), oIB = oDJb + r2(EU);
  static constexpr int nB = oIB + r2(EF);
  // trace kernel: the state
  static constexpr int nC = NP * ldU;
  static_assert(ldT >= c4(D * NU) && ldG >= c8(D * NU) && ldF >= c8(NF) && ldU >= c4(NU), "plan");
  static_assert(F * EF <= NP * ldG, "the neighbours' traces fit in the gradient's place");
};

struct MixedType {
  int NU, NF;
  long long E, off;  // elements; first flux point in the flux-point space
  const double *A45u, *A45f, *A6, *A1, *A2, *A3, *A0;  // operators in fragment order
  const double *JG, *detj;
  double *U, *REG, *DIV, *ND, *DV;
};

struct MixedFpts {
  long long NT;  // flux points over all types
  const int* mate;
  const int* side;  // bit 0 left side, bits 2.. boundary type
  const double* nL;   // [D][NT]
  const double* tdA;  // [NT]
  double* VF;         // [F-1][NT]
  double* BV;         // [boundary points][F]
};

__device__ __forceinline__ void dmma(double (&c)[2], double a, double b)
{
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
      : "+d"(c[0]), "+d"(c[1])
      : "d"(a), "d"(b));
}

// One warp unit of C = A1 B1 (+ A2 B2): rows 8 mt .. 8 mt + 7 (u / NB) and TN
// column tiles from TN (u % NB).  A in fragment order, B's column n starts at
// b(n) (rows contiguous); epi(row, n, C[row][n], C[row][n + 1]) for n even.
template <int NTL, int TN, int KS1, int KS2, class B1, class B2, class Epi>
__device__ __forceinline__ void mma_unit(int u, const double* __restrict__ A1, B1 b1, const double* __restrict__ A2,
                                         B2 b2, Epi epi)
{
  constexpr int NB = (NTL + TN - 1) / TN;
  const int lane = threadIdx.x & 31, mt = u / NB, nt0 = (u - mt * NB) * TN;
  double acc[TN][2];
  const double* p1[TN];
  const double* p2[TN];
#pragma unroll
  for (int j = 0; j < TN; j++) {
    acc[j][0] = 0.0;
    acc[j][1] = 0.0;
    const int n = (nt0 + j < NTL ? nt0 + j : nt0) * 8 + (lane >> 2);
    p1[j] = b1(n) + (lane & 3);
    p2[j] = KS2 > 0 ? b2(n) + (lane & 3) : p1[j];
  }
  const double* a1 = A1 + (size_t)mt * KS1 * 32 + lane;
#pragma unroll 4
  for (int ks = 0; ks < KS1; ks++) {
    const double a = __ldg(a1 + ks * 32);
#pragma unroll
    for (int j = 0; j < TN; j++)
      if (nt0 + j < NTL) dmma(acc[j], a, p1[j][ks * 4]);
  }
  if constexpr (KS2 > 0) {
    const double* a2 = A2 + (size_t)mt * KS2 * 32 + lane;
#pragma unroll 4
    for (int ks = 0; ks < KS2; ks++) {
      const double a = __ldg(a2 + ks * 32);
#pragma unroll
      for (int j = 0; j < TN; j++)
        if (nt0 + j < NTL) dmma(acc[j], a, p2[j][ks * 4]);
    }
  }
#pragma unroll
  for (int j = 0; j < TN; j++)
    if (nt0 + j < NTL) epi(mt * 8 + (lane >> 2), (nt0 + j) * 8 + 2 * (lane & 3), acc[j][0], acc[j][1]);
}

template <int NTL, int TN>
__host__ __device__ constexpr int units(int mt)
{
  return mt * ((NTL + TN - 1) / TN);
}

// zero rows r0 .. r1 - 1 of the first ncol columns of a column-major matrix:
// the padding rows a product reads (times the operator's zero columns), which
// must hold finite values
template <int R0, int R1, int LD, int NCOL, int NTH>
__device__ __forceinline__ void zero_pad_rows(double* a)
{
  constexpr int W = R1 - R0;
  if constexpr (W > 0)
    for (int i = threadIdx.x; i < NCOL * W; i += NTH) a[(i / W) * LD + R0 + i % W] = 0.0;
}

// the block's state into columns (element, field) of sU (rows = solution points)
template <int F, int NU, int EPB, int ldU, int NTH>
__device__ __forceinline__ void load_state(double* sU, const double* __restrict__ U, long long e0, long long E,
                                           int nval)
{
  const int nuv = nval * NU;
  const size_t NUE = (size_t)NU * E;
  for (int r = threadIdx.x; r < nuv; r += NTH) {
    const int el = r / NU, p = r - el * NU;
    double* dst = sU + el * F * ldU + p;
    const double* src = U + (size_t)NU * e0 + r;
#pragma unroll
    for (int k = 0; k < F; k++) cp_async<8>(dst + k * ldU, src + NUE * k);
  }
}

// ------------------------------------------------------------------ kernel A
// A load phase issues every global read of the block (state, traces, the
// neighbours' traces through mate, normals, metrics, wiring) into shared
// memory, so the loads are in flight together; the compute phases that follow
// touch global memory only to write.
template <int D, int NU, int NF, int EPB, int NTH, int MINB>
__global__ void __launch_bounds__(NTH, MINB) mixed_grad_kernel(MixedType t, MixedFpts m,
                                                               const double* __restrict__ UFc, PhysT<double> ph)
{
  using Q = MPlan<D, NU, NF, EPB, MINB>;
  constexpr int F = D + 2, NW = NTH / 32, DD = D * D, EU = Q::EU, EF = Q::EF;
  extern __shared__ __align__(16) double msm[];
  double* sU = msm + Q::oU;
  double* sUF = msm + Q::oUF;
  double* sG = msm + Q::oG;
  double* sX = msm + Q::oX;
  double* sUN = sG;  // neighbours' traces, until the gradient product
  double* sNL = msm + Q::oNL;
  double* sDJ = msm + Q::oDJ;
  double* sJG = msm + Q::oJG;
  int* sMate = reinterpret_cast<int*>(msm + Q::oIA);
  int* sSide = sMate + EF;
  const int tid = threadIdx.x, warp = tid >> 5;
  const long long E = t.E, NT = m.NT, e0 = (long long)blockIdx.x * EPB;
  const int nval = (int)(E - e0 < EPB ? E - e0 : EPB), nuv = nval * NU, nfv = nval * NF;
  const long long gb = t.off + (long long)NF * e0;

  // load phase: asynchronous copies (cp.async), many in flight per thread;
  // first everything at known addresses, then the neighbours' traces through
  // the staged mate.  The matrices are not cleared: only the padding rows
  // the products read are zeroed (U here, delta and the flux before their
  // products); every other padding entry only reaches outputs that are not
  // written.
  zero_pad_rows<NU, c4(NU), Q::ldU, Q::NP, NTH>(sU);
  load_state<F, NU, EPB, Q::ldU, NTH>(sU, t.U, e0, E, nval);
  for (int r = tid; r < nfv; r += NTH) {
    const int el = r / NF, f = r - el * NF;
    const long long g = gb + r;
    double* dst = sUF + el * F * Q::ldF + f;
#pragma unroll
    for (int k = 0; k < F; k++) cp_async<8>(dst + k * Q::ldF, UFc + g + NT * k);
#pragma unroll
    for (int d = 0; d < D; d++) cp_async<8>(&sNL[d * EF + r], m.nL + g + NT * d);
    cp_async<4>(&sMate[r], m.mate + g);
    cp_async<4>(&sSide[r], m.side + g);
  }
  for (int i = tid; i < nuv; i += NTH) {
    cp_async<8>(&sDJ[i], t.detj + (size_t)NU * e0 + i);
    if constexpr (Q::SJ)
#pragma unroll
      for (int q = 0; q < DD; q++) cp_async<8>(&sJG[i + q * nuv], t.JG + (size_t)DD * NU * e0 + i + q * nuv);
  }
  cp_async_wait_all();
  __syncthreads();
  for (int r = tid; r < nfv; r += NTH) {
    const int mt = sMate[r];
    if (mt < 0) continue;
#pragma unroll
    for (int k = 0; k < F; k++) cp_async<8>(&sUN[k * EF + r], UFc + mt + NT * k);
  }
  zero_pad_rows<NF, c4(NF), Q::ldF, Q::NP, NTH>(sX);  // delta's padding rows
  cp_async_wait_all();
  __syncthreads();
  auto jg = [&](int i) { return Q::SJ ? sJG + DD * i : t.JG + (size_t)DD * ((size_t)NU * e0 + i); };

  // LDG common solution at the own flux points: delta = u_c - u_own into X
  for (int i = tid; i < nfv; i += NTH) {
    const int el = i / NF, f = i - el * NF;
    const int sd = sSide[i];
    double n[D], uo[F];
#pragma unroll
    for (int d = 0; d < D; d++) n[d] = sNL[d * EF + i];
#pragma unroll
    for (int k = 0; k < F; k++) uo[k] = sUF[(el * F + k) * Q::ldF + f];
    double* dx = sX + (el * F) * Q::ldF + f;
    if (sd >> 2) {
      BdyPoint<D, double> q;
#pragma unroll
      for (int k = 0; k < F; k++) q.u[k] = uo[k];
#pragma unroll
      for (int d = 0; d < D; d++) q.n[d] = n[d];
      ldg_boundary<D, double>(ph, sd >> 2, q, dx, sUF + (el * F) * Q::ldF + f, Q::ldF);
    } else {
      const bool left = sd & 1;
      const double pen = ldg_beta<D, double>(ph.pen_fact, n);
#pragma unroll
      for (int k = 0; k < F; k++) {
        const double un = sUN[k * EF + i];
        const double ul = left ? uo[k] : un, ur = left ? un : uo[k];
        const double uc = 0.5 * (ul + ur) - pen * (ul - ur);
        dx[k * Q::ldF] = uc - uo[k];
      }
    }
  }
  __syncthreads();

  // reference-space gradient: rows (d, point) of sG
  {
    auto bu = [&](int n) { return sU + n * Q::ldU; };
    auto bd = [&](int n) { return sX + n * Q::ldF; };
    auto epi = [&](int r, int n, double v0, double v1) {
      sG[n * Q::ldG + r] = v0;
      sG[(n + 1) * Q::ldG + r] = v1;
    };
    for (int u = warp; u < units<Q::NTL, Q::TN>(Q::MT_G); u += NW)
      mma_unit<Q::NTL, Q::TN, Q::KS_U, Q::KS_F>(u, t.A45u, bu, t.A45f, bd, epi);
  }
  __syncthreads();

  // physical gradient in place (transform_grad_disu_upts: JGinv / detJ)
  for (int i = tid; i < nuv; i += NTH) {
    const int el = i / NU, p = i - el * NU;
    const double inv = 1.0 / sDJ[i];
    const double* G = jg(i);
    double Gm[D][D];
#pragma unroll
    for (int r = 0; r < D; r++)
#pragma unroll
      for (int c = 0; c < D; c++) Gm[r][c] = G[r + D * c] * inv;
#pragma unroll
    for (int k = 0; k < F; k++) {
      double* s = sG + (el * F + k) * Q::ldG + p;
      double gr[D];
#pragma unroll
      for (int r = 0; r < D; r++) gr[r] = s[r * NU];
#pragma unroll
      for (int c = 0; c < D; c++) {
        double acc = 0.0;
#pragma unroll
        for (int r = 0; r < D; r++) acc = fma(gr[r], Gm[r][c], acc);
        s[c * NU] = acc;
      }
    }
  }
  __syncthreads();

  // gradient at the flux points: column d N + (element, field) of X for
  // dimension d (dimension-major, so the 8 columns of a fragment load are
  // consecutive columns of sG and hit distinct banks)
  {
    auto bg = [&](int n) {
      const int c = n < Q::NG ? n : Q::NG - 1, d = c / Q::N;
      return sG + (c - d * Q::N) * Q::ldG + d * NU;
    };
    auto epi = [&](int r, int n, double v0, double v1) {
      sX[n * Q::ldF + r] = v0;
      sX[(n + 1) * Q::ldF + r] = v1;
    };
    for (int u = warp; u < units<Q::NTLG, Q::TNG>(Q::MT_F); u += NW)
      mma_unit<Q::NTLG, Q::TNG, Q::KS_U, 0>(u, t.A6, bg, t.A6, bg, epi);
  }
  __syncthreads();

  // viscous normal projections (interior points) and boundary viscous fluxes
  for (int i = tid; i < nfv; i += NTH) {
    const int el = i / NF, f = i - el * NF;
    const long long g = gb + i;
    const int mt = sMate[i], sd = sSide[i];
    double n[D], uo[F], gf[F][D];
#pragma unroll
    for (int d = 0; d < D; d++) n[d] = sNL[d * EF + i];
#pragma unroll
    for (int k = 0; k < F; k++) {
      uo[k] = sUF[(el * F + k) * Q::ldF + f];
#pragma unroll
      for (int c = 0; c < D; c++) gf[k][c] = sX[(c * Q::N + el * F + k) * Q::ldF + f];
    }
    if (sd >> 2) {
      BdyPoint<D, double> q;
#pragma unroll
      for (int k = 0; k < F; k++) {
        q.u[k] = uo[k];
#pragma unroll
        for (int c = 0; c < D; c++) q.g[k][c] = gf[k][c];
      }
#pragma unroll
      for (int d = 0; d < D; d++) q.n[d] = n[d];
      vis_boundary<D, double, false>(ph, sd >> 2, q, m.BV + (size_t)(-1 - (long long)mt) * F);
    } else {
      double pr[F - 1];
      vis_flux_proj<D, double>(ph, uo, gf, n, pr);
#pragma unroll
      for (int k = 0; k < F - 1; k++) m.VF[g + NT * k] = pr[k];
    }
  }
  __syncthreads();

  zero_pad_rows<D * NU, c4(D * NU), Q::ldT, Q::NP, NTH>(sX);  // the flux's padding rows
  // transformed flux at the solution points (evaluate_invFlux, then
  // evaluate_viscFlux adding to it): rows (d, point) of X.  The viscous flux
  // takes one reciprocal of rho (vis_flux_fast): its terms are ~1/Re of the
  // inviscid flux they are added to, so its ulp-level differences from the
  // reference's divisions stay far below the rounding of the sum.
  for (int i = tid; i < nuv; i += NTH) {
    const int el = i / NU, p = i - el * NU;
    const double* G = jg(i);
    double q[F], tf[F][D];
    {
      double fi[F][D];
#pragma unroll
      for (int k = 0; k < F; k++) q[k] = sU[(el * F + k) * Q::ldU + p];
      inv_flux<D, double>(ph, q, fi);
#pragma unroll
      for (int k = 0; k < F; k++)
#pragma unroll
        for (int l = 0; l < D; l++) {
          double acc = 0.0;
#pragma unroll
          for (int mm = 0; mm < D; mm++) acc = fma(G[l + D * mm], fi[k][mm], acc);
          tf[k][l] = acc;
        }
    }
    {
      double gq[F][D], fv[F][D];
#pragma unroll
      for (int k = 0; k < F; k++)
#pragma unroll
        for (int c = 0; c < D; c++) gq[k][c] = sG[(el * F + k) * Q::ldG + c * NU + p];
      vis_flux_fast<D, double>(ph, q, gq, fv);
#pragma unroll
      for (int k = 0; k < F; k++)
#pragma unroll
        for (int l = 0; l < D; l++) {
          double acc = tf[k][l];
#pragma unroll
          for (int mm = 0; mm < D; mm++) acc = fma(G[l + D * mm], fv[k][mm], acc);
          sX[(el * F + k) * Q::ldT + l * NU + p] = acc;
        }
    }
  }
  __syncthreads();

  // norm_tdisf = sum_d opp_1[d] f_d and div_tdisf = sum_d opp_2[d] f_d
  {
    auto bt = [&](int n) { return sX + n * Q::ldT; };
    const size_t NFE = (size_t)NF * E, NUE = (size_t)NU * E;
    auto put = [&](double* out, int rows, size_t stride, int r, int n, double v) {
      const int el = n / F, k = n - el * F;
      if (r < rows && el < nval) out[r + (size_t)rows * (e0 + el) + stride * k] = v;
    };
    auto epi_nd = [&](int r, int n, double v0, double v1) {
      put(t.ND, NF, NFE, r, n, v0);
      put(t.ND, NF, NFE, r, n + 1, v1);
    };
    auto epi_dv = [&](int r, int n, double v0, double v1) {
      put(t.DV, NU, NUE, r, n, v0);
      put(t.DV, NU, NUE, r, n + 1, v1);
    };
    constexpr int U1 = units<Q::NTL, Q::TN>(Q::MT_F), U2 = units<Q::NTL, Q::TN>(Q::MT_U);
    for (int u = warp; u < U1 + U2; u += NW) {
      if (u < U1) mma_unit<Q::NTL, Q::TN, Q::KS_T, 0>(u, t.A1, bt, t.A1, bt, epi_nd);
      else mma_unit<Q::NTL, Q::TN, Q::KS_T, 0>(u - U1, t.A2, bt, t.A2, bt, epi_dv);
    }
  }
}

// ------------------------------------------------------------------ kernel B
// MODE 1: RK45 stage update (rk_a, rk_b, dt) and the new traces into UFn;
// MODE 0: div_tconf_upts into t.DIV only.  Like kernel A, a load phase first
// stages every global read of the block in shared memory.
template <int D, int NU, int NF, int EPB, int NTH, int MINB, int MODE>
__global__ void __launch_bounds__(NTH, MINB) mixed_update_kernel(MixedType t, MixedFpts m,
                                                                 const double* __restrict__ UFc,
                                                                 double* __restrict__ UFn, PhysT<double> ph,
                                                                 double rk_a, double rk_b, double dt)
{
  using Q = MPlan<D, NU, NF, EPB>;
  constexpr int F = D + 2, NW = NTH / 32, EU = Q::EU, EF = Q::EF;
  extern __shared__ __align__(16) double msm[];
  double* sJ = msm + Q::oJ;
  double* sUo = msm + Q::oUo;
  double* sUn = sUo;  // the new state, after the flux phase
  double* sUN = msm + Q::oUN;
  double* sVo = msm + Q::oVo;
  double* sVN = msm + Q::oVN;
  double* sNL = msm + Q::oNLb;
  double* sTA = msm + Q::oTA;
  double* sDV = msm + Q::oDV;
  double* sRG = msm + Q::oRG;
  double* sUO = msm + Q::oUO;
  double* sDJ = msm + Q::oDJb;
  int* sMate = reinterpret_cast<int*>(msm + Q::oIB);
  int* sSide = sMate + EF;
  const int tid = threadIdx.x, warp = tid >> 5;
  const long long E = t.E, NT = m.NT, e0 = (long long)blockIdx.x * EPB;
  const int nval = (int)(E - e0 < EPB ? E - e0 : EPB), nuv = nval * NU, nfv = nval * NF;
  const long long gb = t.off + (long long)NF * e0;
  const size_t NFE = (size_t)NF * E, NUE = (size_t)NU * E;

  // load phase: asynchronous copies, as in the gradient kernel
  zero_pad_rows<NF, c4(NF), Q::ldF, Q::NP, NTH>(sJ);
  for (int r = tid; r < nfv; r += NTH) {
    const int el = r / NF, f = r - el * NF;
    const long long g = gb + r;
    double* dj = sJ + el * F * Q::ldF + f;
    const double* nd = t.ND + (size_t)NF * e0 + r;
#pragma unroll
    for (int k = 0; k < F; k++) {
      cp_async<8>(&sUo[k * EF + r], UFc + g + NT * k);
      cp_async<8>(dj + k * Q::ldF, nd + NFE * k);
    }
#pragma unroll
    for (int k = 0; k < F - 1; k++) cp_async<8>(&sVo[k * EF + r], m.VF + g + NT * k);
#pragma unroll
    for (int d = 0; d < D; d++) cp_async<8>(&sNL[d * EF + r], m.nL + g + NT * d);
    cp_async<4>(&sMate[r], m.mate + g);
    cp_async<4>(&sSide[r], m.side + g);
    cp_async<8>(&sTA[r], m.tdA + g);
  }
  for (int r = tid; r < nuv; r += NTH) {
    const size_t ix = (size_t)NU * e0 + r;
#pragma unroll
    for (int k = 0; k < F; k++) {
      cp_async<8>(&sDV[k * EU + r], t.DV + ix + NUE * k);
      if (MODE == 1) {
        cp_async<8>(&sRG[k * EU + r], t.REG + ix + NUE * k);
        cp_async<8>(&sUO[k * EU + r], t.U + ix + NUE * k);
      }
    }
    if (MODE == 1) cp_async<8>(&sDJ[r], t.detj + ix);
  }
  cp_async_wait_all();
  __syncthreads();
  for (int r = tid; r < nfv; r += NTH) {
    const int mt = sMate[r];
    if (mt < 0) continue;
#pragma unroll
    for (int k = 0; k < F; k++) cp_async<8>(&sUN[k * EF + r], UFc + mt + NT * k);
#pragma unroll
    for (int k = 0; k < F - 1; k++) cp_async<8>(&sVN[k * EF + r], m.VF + mt + NT * k);
  }
  cp_async_wait_all();
  __syncthreads();

  // common normal fluxes times the own tdA, minus norm_tdisf
  for (int i = tid; i < nfv; i += NTH) {
    const int el = i / NF, f = i - el * NF;
    const int mt = sMate[i], sd = sSide[i];
    double n[D], uo[F], c[F];
#pragma unroll
    for (int d = 0; d < D; d++) n[d] = sNL[d * EF + i];
#pragma unroll
    for (int k = 0; k < F; k++) uo[k] = sUo[k * EF + i];
    const double tl = sTA[i];
    if (sd >> 2) {
      FUBdy<D, double> q;
#pragma unroll
      for (int k = 0; k < F; k++) {
        q.ul[k] = uo[k];
        q.bv[k] = m.BV[(size_t)(-1 - (long long)mt) * F + k];
      }
#pragma unroll
      for (int d = 0; d < D; d++) q.n[d] = n[d];
      q.tl = tl;
      fu_boundary<D, 1, double, 0>(ph, sd >> 2, q, c, 1);
    } else {
      const bool left = sd & 1;
      double ul[F], ur[F], fn[F];
#pragma unroll
      for (int k = 0; k < F; k++) {
        const double v = sUN[k * EF + i];
        ul[k] = left ? uo[k] : v;
        ur[k] = left ? v : uo[k];
      }
      rusanov<D, double>(ph, ul, ur, n, fn);
#pragma unroll
      for (int k = 0; k < F; k++) c[k] = left ? fn[k] * tl : -fn[k] * tl;
      double nn = n[0] * n[0];
#pragma unroll
      for (int d = 1; d < D; d++) nn = fma(n[d], n[d], nn);
      const double pen = ldg_beta<D, double>(ph.pen_fact, n);
#pragma unroll
      for (int k = 0; k < F; k++) {
        const double ao = k ? sVo[(k - 1) * EF + i] : 0.0, an = k ? sVN[(k - 1) * EF + i] : 0.0;
        const double fv = ldg_normal<double>(left ? ao : an, left ? an : ao, ul[k], ur[k], pen, ph.tau, nn);
        c[k] = left ? c[k] + fv * tl : c[k] + (-fv) * tl;
      }
    }
#pragma unroll
    for (int k = 0; k < F; k++) {
      double* p = sJ + (el * F + k) * Q::ldF + f;
      *p = c[k] - *p;
    }
  }
  __syncthreads();

  // div_tconf = div_tdisf + opp_3 jump, then the RK45 update
  // (RK45_update_kernel: rhs = -div / detJ)
  {
    if (MODE == 1)  // padding rows of the new state, read (times zero) by the trace product
      for (int i = tid; i < Q::NP * (c4(NU) - NU); i += NTH) {
        const int n = i / (c4(NU) - NU), r = NU + i % (c4(NU) - NU);
        sUn[n * Q::ldU + r] = 0.0;
      }
    auto bj = [&](int n) { return sJ + n * Q::ldF; };
    auto one = [&](int r, int n, double v) {
      const int el = n / F, k = n - el * F;
      if (r >= NU || el >= nval) return;
      const int li = k * EU + el * NU + r;
      const size_t ix = (size_t)NU * e0 + (size_t)el * NU + r + NUE * k;
      const double div = v + sDV[li];
      if (MODE == 0) {
        t.DIV[ix] = div;
      } else {
        const double rhs = -div / sDJ[el * NU + r] + 0.0 + 0.0;
        const double res = fma(rk_a, sRG[li], dt * rhs);
        t.REG[ix] = res;
        const double un = fma(rk_b, res, sUO[li]);
        t.U[ix] = un;
        sUn[n * Q::ldU + r] = un;
      }
    };
    auto epi = [&](int r, int n, double v0, double v1) {
      one(r, n, v0);
      one(r, n + 1, v1);
    };
    for (int u = warp; u < units<Q::NTL, Q::TN>(Q::MT_U); u += NW)
      mma_unit<Q::NTL, Q::TN, Q::KS_F, 0>(u, t.A3, bj, t.A3, bj, epi);
  }
  if constexpr (MODE == 1) {
    __syncthreads();
    auto bu = [&](int n) { return sUn + n * Q::ldU; };
    auto one = [&](int r, int n, double v) {
      const int el = n / F, k = n - el * F;
      if (r < NF && el < nval) UFn[gb + r + (long long)NF * el + NT * k] = v;
    };
    auto epi = [&](int r, int n, double v0, double v1) {
      one(r, n, v0);
      one(r, n + 1, v1);
    };
    for (int u = warp; u < units<Q::NTL, Q::TN>(Q::MT_F); u += NW)
      mma_unit<Q::NTL, Q::TN, Q::KS_U, 0>(u, t.A0, bu, t.A0, bu, epi);
  }
}

// ------------------------------------------------------------ trace kernel
// UFn = opp_0 U (extrapolate_solution) with the update kernel's product, so
// the traces match the ones the update kernel writes bit for bit.
template <int D, int NU, int NF, int EPB, int NTH>
__global__ void __launch_bounds__(NTH) mixed_trace_kernel(MixedType t, long long NT, double* __restrict__ UFn)
{
  using Q = MPlan<D, NU, NF, EPB>;
  constexpr int F = D + 2, NW = NTH / 32;
  extern __shared__ __align__(16) double msm[];
  const int warp = threadIdx.x >> 5;
  const long long E = t.E, e0 = (long long)blockIdx.x * EPB;
  const int nval = (int)(E - e0 < EPB ? E - e0 : EPB);
  const long long gb = t.off + (long long)NF * e0;
  zero_pad_rows<NU, c4(NU), Q::ldU, Q::NP, NTH>(msm);
  load_state<F, NU, EPB, Q::ldU, NTH>(msm, t.U, e0, E, nval);
  cp_async_wait_all();
  __syncthreads();
  auto bu = [&](int n) { return msm + n * Q::ldU; };
  auto one = [&](int r, int n, double v) {
    const int el = n / F, k = n - el * F;
    if (r < NF && el < nval) UFn[gb + r + (long long)NF * el + NT * k] = v;
  };
  auto epi = [&](int r, int n, double v0, double v1) {
    one(r, n, v0);
    one(r, n + 1, v1);
  };
  for (int u = warp; u < units<Q::NTL, Q::TN>(Q::MT_F); u += NW)
    mma_unit<Q::NTL, Q::TN, Q::KS_U, 0>(u, t.A0, bu, t.A0, bu, epi);
}

// ------------------------------------------------------------ dispatch
// Launch shapes: elements per block, threads per block, blocks per SM the
// registers are capped for.  Gradient and update kernels pick theirs
// independently (fr_mixed_stage_autotune); the products give the same bits
// in every shape, since each output is the same chain of k-steps.
struct MixedShape {
  int epb, nth, minb;
};
constexpr MixedShape kGradShapes[] = {{8, 256, 1}, {4, 128, 3}, {8, 128, 2}, {4, 128, 4}, {8, 256, 2}};
constexpr MixedShape kUpdShapes[] = {{8, 256, 2}, {4, 128, 4}, {8, 128, 4}};
constexpr int kNGrad = sizeof(kGradShapes) / sizeof(kGradShapes[0]);
constexpr int kNUpd = sizeof(kUpdShapes) / sizeof(kUpdShapes[0]);

using GradFn = void (*)(MixedType, MixedFpts, const double*, PhysT<double>);
using UpdFn = void (*)(MixedType, MixedFpts, const double*, double*, PhysT<double>, double, double, double);
using TraceFn = void (*)(MixedType, long long, double*);

struct MixedKernels {
  int D, NU, NF;
  GradFn grad[kNGrad];
  size_t smem_a[kNGrad];
  UpdFn upd0[kNUpd], upd1[kNUpd];
  size_t smem_b[kNUpd];
  TraceFn trace;
  size_t smem_c;
};

template <int D, int NU, int NF, int V>
void fill_grad(MixedKernels& k)
{
  constexpr MixedShape g = kGradShapes[V];
  k.smem_a[V] = sizeof(double) * MPlan<D, NU, NF, g.epb, g.minb>::nA;
  k.grad[V] = k.smem_a[V] <= kMixedSmemMax ? mixed_grad_kernel<D, NU, NF, g.epb, g.nth, g.minb> : nullptr;
}

template <int D, int NU, int NF, int V>
void fill_upd(MixedKernels& k)
{
  constexpr MixedShape u = kUpdShapes[V];
  k.smem_b[V] = sizeof(double) * MPlan<D, NU, NF, u.epb>::nB;
  const bool fits = k.smem_b[V] <= kMixedSmemMax;
  k.upd0[V] = fits ? mixed_update_kernel<D, NU, NF, u.epb, u.nth, u.minb, 0> : nullptr;
  k.upd1[V] = fits ? mixed_update_kernel<D, NU, NF, u.epb, u.nth, u.minb, 1> : nullptr;
}

template <int D, int NU, int NF>
MixedKernels mixed_kernels()
{
  MixedKernels k;
  k.D = D;
  k.NU = NU;
  k.NF = NF;
  fill_grad<D, NU, NF, 0>(k);
  fill_grad<D, NU, NF, 1>(k);
  fill_grad<D, NU, NF, 2>(k);
  fill_grad<D, NU, NF, 3>(k);
  fill_grad<D, NU, NF, 4>(k);
  fill_upd<D, NU, NF, 0>(k);
  fill_upd<D, NU, NF, 1>(k);
  fill_upd<D, NU, NF, 2>(k);
  static_assert(kNGrad == 5 && kNUpd == 3, "one fill per shape");
  k.trace = mixed_trace_kernel<D, NU, NF, kMixedEPB, kMixedNT>;
  k.smem_c = sizeof(double) * MPlan<D, NU, NF, kMixedEPB>::nC;
  return k;
}

// (dims, solution points, flux points) with kernels: tets, prisms and hexes of
// orders 2 and 3
bool find_kernels(int D, int NU, int NF, MixedKernels* out)
{
  if (D != 3) return false;
#define FR_MIXED_SHAPE(nu, nf) \
  if (NU == nu && NF == nf) {  \
    *out = mixed_kernels<3, nu, nf>(); \
    return true;               \
  }
  FR_MIXED_SHAPE(10, 24)  // tet P2
  FR_MIXED_SHAPE(20, 40)  // tet P3
  FR_MIXED_SHAPE(18, 39)  // prism P2
  FR_MIXED_SHAPE(40, 68)  // prism P3
  FR_MIXED_SHAPE(27, 54)  // hex P2
  FR_MIXED_SHAPE(64, 96)  // hex P3
#undef FR_MIXED_SHAPE
  return false;
}

// operator A (rows x cols, row r column c at get(r, c)) in fragment order
template <class Get>
std::vector<double> fragments(int rows, int cols, Get get)
{
  const int MT = (rows + 7) / 8, KS = (cols + 3) / 4;
  std::vector<double> f((size_t)MT * KS * 32, 0.0);
  for (int mt = 0; mt < MT; mt++)
    for (int ks = 0; ks < KS; ks++)
      for (int lane = 0; lane < 32; lane++) {
        const int r = mt * 8 + lane / 4, c = ks * 4 + lane % 4;
        if (r < rows && c < cols) f[((size_t)mt * KS + ks) * 32 + lane] = get(r, c);
      }
  return f;
}

}  // namespace

struct fr_mixed_stage {
  int D = 3, F = 5, n_types = 0;
  PhysT<double> ph;
  long long NT = 0, n_bpts = 0;
  std::vector<MixedType> types;
  std::vector<MixedKernels> kern;
  std::vector<void*> allocs;
  std::vector<int> gv, uv;  // launch shape of each type's gradient and update kernels
  MixedFpts fp{};
  double* UF[2] = {nullptr, nullptr};
  int cur = 0;
  // element types after the first run on side streams, forked from and
  // joined to the caller's stream around each kernel of a stage
  bool concurrent = true;
  std::vector<cudaStream_t> side_streams;
  std::vector<cudaEvent_t> fork_ev, join_ev;
  ~fr_mixed_stage()
  {
    for (void* p : allocs) cudaFree(p);
    for (cudaStream_t q : side_streams) cudaStreamDestroy(q);
    for (cudaEvent_t e : fork_ev) cudaEventDestroy(e);
    for (cudaEvent_t e : join_ev) cudaEventDestroy(e);
  }
  template <class T>
  fr_status upload(const std::vector<T>& h, const T** out)
  {
    void* p = nullptr;
    if (h.empty()) {
      *out = nullptr;
      return FR_OK;
    }
    if (cudaMalloc(&p, h.size() * sizeof(T)) != cudaSuccess) return mfail(FR_ERR_CUDA, "device allocation failed");
    allocs.push_back(p);
    if (cudaMemcpy(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
      return mfail(FR_ERR_CUDA, "upload failed");
    *out = static_cast<const T*>(p);
    return FR_OK;
  }
  fr_status zeros(size_t n, double** out)
  {
    void* p = nullptr;
    if (cudaMalloc(&p, (n ? n : 1) * sizeof(double)) != cudaSuccess) return mfail(FR_ERR_CUDA, "device allocation failed");
    allocs.push_back(p);
    if (cudaMemset(p, 0, (n ? n : 1) * sizeof(double)) != cudaSuccess) return mfail(FR_ERR_CUDA, "memset failed");
    *out = static_cast<double*>(p);
    return FR_OK;
  }
};

namespace {

unsigned blocks_of(long long E, int epb) { return (unsigned)((E + epb - 1) / epb); }


fr_status launch_grad(fr_mixed_stage* s, int i, int v, const double* UFc, cudaStream_t st)
{
  const MixedType& t = s->types[i];
  const MixedShape& g = kGradShapes[v];
  s->kern[i].grad[v]<<<blocks_of(t.E, g.epb), g.nth, s->kern[i].smem_a[v], st>>>(t, s->fp, UFc, s->ph);
  return mlaunched("mixed_grad_kernel");
}

fr_status launch_upd(fr_mixed_stage* s, int i, int v, int mode, int stage, double dt, const double* UFc, double* UFn,
                     cudaStream_t st)
{
  static const double A[5] = {0.0, -0.417890474499852, -1.192151694642677, -1.697784692471528, -1.514183444257156};
  static const double B[5] = {0.149659021999229, 0.379210312999627, 0.822955029386982, 0.699450455949122,
                              0.153057247968152};
  const MixedType& t = s->types[i];
  const MixedShape& u = kUpdShapes[v];
  auto k = mode ? s->kern[i].upd1[v] : s->kern[i].upd0[v];
  k<<<blocks_of(t.E, u.epb), u.nth, s->kern[i].smem_b[v], st>>>(t, s->fp, UFc, UFn, s->ph, A[stage], B[stage], dt);
  return mlaunched("mixed_update_kernel");
}

// the kernels of every element type, types after the first on their side
// streams when concurrent (fork from st, join back into st)
template <class Launch>
fr_status for_types(fr_mixed_stage* s, cudaStream_t st, Launch launch)
{
  const bool par = s->concurrent && s->n_types > 1;
  if (par) {
    if (cudaEventRecord(s->fork_ev[0], st) != cudaSuccess) return mfail(FR_ERR_CUDA, "event record failed");
    for (size_t j = 0; j < s->side_streams.size(); j++)
      if (cudaStreamWaitEvent(s->side_streams[j], s->fork_ev[0], 0) != cudaSuccess)
        return mfail(FR_ERR_CUDA, "stream wait failed");
  }
  // the side-stream types go first, so their blocks are resident while the
  // first type's blocks fill the rest of the GPU
  for (int j = 1; j <= s->n_types; j++) {
    const int i = j % s->n_types;
    if (s->types[i].E == 0) continue;
    if (fr_status e = launch(i, par && i > 0 ? s->side_streams[i - 1] : st)) return e;
  }
  if (par)
    for (size_t j = 0; j < s->side_streams.size(); j++) {
      if (cudaEventRecord(s->join_ev[j], s->side_streams[j]) != cudaSuccess ||
          cudaStreamWaitEvent(st, s->join_ev[j], 0) != cudaSuccess)
        return mfail(FR_ERR_CUDA, "stream join failed");
    }
  return FR_OK;
}

fr_status launch_trace(fr_mixed_stage* s, cudaStream_t st)
{
  return for_types(s, st, [&](int i, cudaStream_t q) {
    const MixedType& t = s->types[i];
    s->kern[i].trace<<<blocks_of(t.E, kMixedEPB), kMixedNT, s->kern[i].smem_c, q>>>(t, s->NT, s->UF[s->cur]);
    return mlaunched("mixed_trace_kernel");
  });
}

// one CalcResidual (+ the RK45 update of stage `stage` when mode is 1)
fr_status launch_stage(fr_mixed_stage* s, int mode, int stage, double dt, cudaStream_t st)
{
  const double* UFc = s->UF[s->cur];
  double* UFn = s->UF[s->cur ^ 1];
  if (fr_status e = for_types(s, st, [&](int i, cudaStream_t q) { return launch_grad(s, i, s->gv[i], UFc, q); }))
    return e;
  if (fr_status e = for_types(
          s, st, [&](int i, cudaStream_t q) { return launch_upd(s, i, s->uv[i], mode, stage, dt, UFc, UFn, q); }))
    return e;
  if (mode) s->cur ^= 1;
  return FR_OK;
}

fr_status set_smem(const MixedKernels& k)
{
  std::vector<std::pair<const void*, size_t>> list;
  for (int v = 0; v < kNGrad; v++) list.push_back({(const void*)k.grad[v], k.smem_a[v]});
  for (int v = 0; v < kNUpd; v++) {
    list.push_back({(const void*)k.upd0[v], k.smem_b[v]});
    list.push_back({(const void*)k.upd1[v], k.smem_b[v]});
  }
  list.push_back({(const void*)k.trace, k.smem_c});
  bool any_grad = false, any_upd = false;
  for (int v = 0; v < kNGrad; v++) any_grad = any_grad || k.grad[v];
  for (int v = 0; v < kNUpd; v++) any_upd = any_upd || k.upd1[v];
  if (!any_grad || !any_upd || k.smem_c > kMixedSmemMax)
    return mfail(FR_ERR_UNSUPPORTED, "element type too large for one block of shared memory");
  for (auto& q : list) {
    if (!q.first) continue;  // a launch shape whose plan exceeds shared memory
    if (cudaFuncSetAttribute(q.first, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)q.second) != cudaSuccess)
      return mfail(FR_ERR_CUDA, "cudaFuncSetAttribute failed");
  }
  return FR_OK;
}

}  // namespace

extern "C" {

fr_status fr_mixed_stage_create(int n_dims, int n_types, const fr_mixed_stage_type* types, int n_int_groups,
                                const int* const* int_tables, const int* int_nfpi, const long long* int_ni,
                                int n_bdy_groups, const int* const* bdy_tables, const int* bdy_nfpi,
                                const long long* bdy_ni, const double* bdy_params, double R_ref,
                                const fr_phys_desc* phys, fr_mixed_stage** out)
{
  g_err.clear();
  if (!out || !types || !phys || n_types < 1) return mfail(FR_ERR_ARG, "bad arguments");
  *out = nullptr;
  if (n_dims != 3) return mfail(FR_ERR_UNSUPPORTED, "fused mixed stage: 3-D meshes only");
  if ((n_int_groups > 0 && (!int_tables || !int_nfpi || !int_ni)) ||
      (n_bdy_groups > 0 && (!bdy_tables || !bdy_nfpi || !bdy_ni)) || n_int_groups < 0 || n_bdy_groups < 0)
    return mfail(FR_ERR_ARG, "null interface table");
  const int D = n_dims, F = D + 2;
  auto s = new fr_mixed_stage();
  auto bail = [&](fr_status e) {
    delete s;
    return e;
  };
  s->D = D;
  s->F = F;
  s->n_types = n_types;
  {
    Phys q{phys->gamma, phys->prandtl, phys->mu_inf, phys->rt_inf, phys->c_sth, phys->fix_vis, phys->tau,
           phys->pen_fact};
    for (int i = 0; i < 14; i++) q.bdy[i] = bdy_params ? bdy_params[i] : 0.0;
    q.R_ref = R_ref;
    s->ph = PhysT<double>::make(q);
  }
  std::vector<long long> off(n_types + 1, 0);
  for (int i = 0; i < n_types; i++) {
    const fr_mixed_stage_type& ty = types[i];
    const int NU = ty.n_upts, NF = ty.n_fpts;
    if (NU <= 0 || NF <= 0 || ty.n_eles < 0 || !ty.disu_upts || !ty.opp_0 || !ty.opp_3 || !ty.opp_6 ||
        !ty.JGinv_upts || !ty.detjac_upts || !ty.tdA_fpts || !ty.norm_fpts)
      return bail(mfail(FR_ERR_ARG, "bad element type description"));
    for (int d = 0; d < D; d++)
      if (!ty.opp_1[d] || !ty.opp_2[d] || !ty.opp_4[d] || !ty.opp_5[d])
        return bail(mfail(FR_ERR_ARG, "missing operator"));
    MixedKernels k;
    if (!find_kernels(D, NU, NF, &k))
      return bail(mfail(FR_ERR_UNSUPPORTED, "fused mixed stage: no kernels for " + std::to_string(NU) +
                                                " solution / " + std::to_string(NF) + " flux points"));
    if (fr_status e = set_smem(k)) return bail(e);
    s->kern.push_back(k);
    int g0 = 0, u0 = 0;
    while (!k.grad[g0]) g0++;
    while (!k.upd1[u0]) u0++;
    s->gv.push_back(g0);
    s->uv.push_back(u0);
    off[i + 1] = off[i] + (long long)NF * ty.n_eles;
  }
  s->NT = off[n_types];
  const long long NT = s->NT;

  // operators in fragment order
  for (int i = 0; i < n_types; i++) {
    const fr_mixed_stage_type& ty = types[i];
    const int NU = ty.n_upts, NF = ty.n_fpts;
    const long long E = ty.n_eles;
    MixedType t{};
    t.NU = NU;
    t.NF = NF;
    t.E = E;
    t.off = off[i];
    auto cm = [](const double* a, int rows) { return [a, rows](int r, int c) { return a[r + (size_t)rows * c]; }; };
    std::vector<double> h;
    h = fragments(D * NU, NU, [&](int r, int c) { return ty.opp_4[r / NU][r % NU + (size_t)NU * c]; });
    if (fr_status e = s->upload(h, &t.A45u)) return bail(e);
    h = fragments(D * NU, NF, [&](int r, int c) { return ty.opp_5[r / NU][r % NU + (size_t)NU * c]; });
    if (fr_status e = s->upload(h, &t.A45f)) return bail(e);
    h = fragments(NF, NU, cm(ty.opp_6, NF));
    if (fr_status e = s->upload(h, &t.A6)) return bail(e);
    h = fragments(NF, D * NU, [&](int r, int c) { return ty.opp_1[c / NU][r + (size_t)NF * (c % NU)]; });
    if (fr_status e = s->upload(h, &t.A1)) return bail(e);
    h = fragments(NU, D * NU, [&](int r, int c) { return ty.opp_2[c / NU][r + (size_t)NU * (c % NU)]; });
    if (fr_status e = s->upload(h, &t.A2)) return bail(e);
    h = fragments(NU, NF, cm(ty.opp_3, NU));
    if (fr_status e = s->upload(h, &t.A3)) return bail(e);
    h = fragments(NF, NU, cm(ty.opp_0, NF));
    if (fr_status e = s->upload(h, &t.A0)) return bail(e);
    std::vector<double> jg(ty.JGinv_upts, ty.JGinv_upts + (size_t)D * D * NU * E);
    if (fr_status e = s->upload(jg, &t.JG)) return bail(e);
    std::vector<double> dj(ty.detjac_upts, ty.detjac_upts + (size_t)NU * E);
    if (fr_status e = s->upload(dj, &t.detj)) return bail(e);
    t.U = ty.disu_upts;
    t.DIV = ty.div_tconf_upts;
    if (fr_status e = s->zeros((size_t)NU * E * F, &t.REG)) return bail(e);
    if (fr_status e = s->zeros((size_t)NF * E * F, &t.ND)) return bail(e);
    if (fr_status e = s->zeros((size_t)NU * E * F, &t.DV)) return bail(e);
    s->types.push_back(t);
  }

  // flux-point space: neighbours, sides, left normals, own tdA
  std::vector<int> mate(NT, 0);
  std::vector<int> side(NT, 0);
  std::vector<unsigned char> seen(NT, 0);
  std::vector<double> nL((size_t)D * NT, 0.0), tdA(NT, 0.0);
  auto gidx = [&](int ty, long long e, int f, long long* g) {
    if (ty < 0 || ty >= n_types || e < 0 || e >= types[ty].n_eles || f < 0 || f >= types[ty].n_fpts) return false;
    *g = off[ty] + f + (long long)types[ty].n_fpts * e;
    return true;
  };
  auto normal = [&](int ty, long long e, int f, int d) {
    const fr_mixed_stage_type& q = types[ty];
    return q.norm_fpts[f + (size_t)q.n_fpts * (e + (size_t)q.n_eles * d)];
  };
  for (int gi = 0; gi < n_int_groups; gi++) {
    const int* w = int_tables[gi];
    const long long n = (long long)int_nfpi[gi] * int_ni[gi];
    if (n > 0 && !w) return bail(mfail(FR_ERR_ARG, "null interface table"));
    for (long long j = 0; j < n; j++) {
      const int* q = w + 6 * j;
      long long gl, gr;
      if (!gidx(q[0], q[1], q[2], &gl) || !gidx(q[3], q[4], q[5], &gr))
        return bail(mfail(FR_ERR_MESH, "interface table entry out of range"));
      if (seen[gl] || seen[gr] || gl == gr) return bail(mfail(FR_ERR_MESH, "flux point wired twice"));
      if (gl > 2147483647LL || gr > 2147483647LL) return bail(mfail(FR_ERR_ARG, "too many flux points"));
      seen[gl] = seen[gr] = 1;
      mate[gl] = (int)gr;
      mate[gr] = (int)gl;
      side[gl] = 1;
      side[gr] = 0;
      for (int d = 0; d < D; d++) nL[gl + NT * d] = nL[gr + NT * d] = normal(q[0], q[1], q[2], d);
    }
  }
  long long place = 0;
  for (int gi = 0; gi < n_bdy_groups; gi++) {
    const int* w = bdy_tables[gi];
    const long long n = (long long)bdy_nfpi[gi] * bdy_ni[gi];
    if (n > 0 && !w) return bail(mfail(FR_ERR_ARG, "null boundary table"));
    for (long long j = 0; j < n; j++) {
      const int* q = w + 4 * j;
      long long g;
      if (!gidx(q[0], q[1], q[2], &g)) return bail(mfail(FR_ERR_MESH, "boundary table entry out of range"));
      const int bt = q[3];
      if (!((bt >= 1 && bt <= 7) || (bt >= 11 && bt <= 16)))
        return bail(mfail(FR_ERR_UNSUPPORTED, "boundary type " + std::to_string(bt)));
      if (seen[g]) return bail(mfail(FR_ERR_MESH, "flux point wired twice"));
      seen[g] = 1;
      mate[g] = (int)(-1 - place);
      side[g] = bt << 2;
      for (int d = 0; d < D; d++) nL[g + NT * d] = normal(q[0], q[1], q[2], d);
      place++;
    }
  }
  for (long long g = 0; g < NT; g++)
    if (!seen[g]) return bail(mfail(FR_ERR_MESH, "flux point on no interface"));
  for (int i = 0; i < n_types; i++) {
    const fr_mixed_stage_type& q = types[i];
    for (long long e = 0; e < q.n_eles; e++)
      for (int f = 0; f < q.n_fpts; f++) tdA[off[i] + f + (long long)q.n_fpts * e] = q.tdA_fpts[f + (size_t)q.n_fpts * e];
  }
  s->n_bpts = place;
  s->fp.NT = NT;
  if (fr_status e = s->upload(mate, &s->fp.mate)) return bail(e);
  if (fr_status e = s->upload(side, &s->fp.side)) return bail(e);
  if (fr_status e = s->upload(nL, &s->fp.nL)) return bail(e);
  if (fr_status e = s->upload(tdA, &s->fp.tdA)) return bail(e);
  if (fr_status e = s->zeros((size_t)(F - 1) * NT, &s->fp.VF)) return bail(e);
  if (fr_status e = s->zeros((size_t)F * (place ? place : 1), &s->fp.BV)) return bail(e);
  if (fr_status e = s->zeros((size_t)F * NT, &s->UF[0])) return bail(e);
  if (fr_status e = s->zeros((size_t)F * NT, &s->UF[1])) return bail(e);
  s->fork_ev.resize(1, nullptr);
  if (cudaEventCreateWithFlags(&s->fork_ev[0], cudaEventDisableTiming) != cudaSuccess)
    return bail(mfail(FR_ERR_CUDA, "event creation failed"));
  for (int i = 1; i < n_types; i++) {
    cudaStream_t q;
    cudaEvent_t ev;
    if (cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking) != cudaSuccess)
      return bail(mfail(FR_ERR_CUDA, "stream creation failed"));
    s->side_streams.push_back(q);
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess)
      return bail(mfail(FR_ERR_CUDA, "event creation failed"));
    s->join_ev.push_back(ev);
  }
  *out = s;
  return FR_OK;
}

fr_status fr_mixed_stage_destroy(fr_mixed_stage* s)
{
  delete s;
  return FR_OK;
}

fr_status fr_mixed_stage_residual(fr_mixed_stage* s, void* stream)
{
  g_err.clear();
  if (!s) return mfail(FR_ERR_ARG, "null stage");
  for (const MixedType& t : s->types)
    if (!t.DIV && t.E > 0) return mfail(FR_ERR_ARG, "div_tconf_upts not given");
  cudaStream_t st = (cudaStream_t)stream;
  if (fr_status e = launch_trace(s, st)) return e;
  return launch_stage(s, 0, 0, 0.0, st);
}

fr_status fr_mixed_stage_advance(fr_mixed_stage* s, int n_steps, double dt, void* stream)
{
  g_err.clear();
  if (!s || n_steps < 0) return mfail(FR_ERR_ARG, "bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  if (n_steps == 0) return FR_OK;
  if (fr_status e = launch_trace(s, st)) return e;
  for (int n = 0; n < n_steps; n++)
    for (int k = 0; k < 5; k++)
      if (fr_status e = launch_stage(s, 1, k, dt, st)) return e;
  return FR_OK;
}

fr_status fr_mixed_stage_set_launch(fr_mixed_stage* s, int type, int grad_shape, int update_shape)
{
  g_err.clear();
  if (!s || type < 0 || type >= s->n_types || grad_shape < 0 || grad_shape >= kNGrad || update_shape < 0 ||
      update_shape >= kNUpd)
    return mfail(FR_ERR_ARG, "bad type or launch shape");
  if (!s->kern[type].grad[grad_shape] || !s->kern[type].upd1[update_shape])
    return mfail(FR_ERR_UNSUPPORTED, "launch shape exceeds shared memory for this element type");
  s->gv[type] = grad_shape;
  s->uv[type] = update_shape;
  return FR_OK;
}

fr_status fr_mixed_stage_set_concurrent(fr_mixed_stage* s, int on)
{
  g_err.clear();
  if (!s) return mfail(FR_ERR_ARG, "null stage");
  s->concurrent = on != 0;
  return FR_OK;
}

fr_status fr_mixed_stage_get_launch(const fr_mixed_stage* s, int type, int* grad_shape, int* update_shape)
{
  g_err.clear();
  if (!s || type < 0 || type >= s->n_types) return mfail(FR_ERR_ARG, "bad type");
  if (grad_shape) *grad_shape = s->gv[type];
  if (update_shape) *update_shape = s->uv[type];
  return FR_OK;
}

fr_status fr_mixed_stage_autotune(fr_mixed_stage* s, void* stream)
{
  g_err.clear();
  if (!s) return mfail(FR_ERR_ARG, "null stage");
  cudaStream_t st = (cudaStream_t)stream;
  // the update kernels are timed in residual mode, into a scratch output,
  // so the state is not touched
  size_t most = 1;
  for (const MixedType& t : s->types) most = std::max(most, (size_t)((long long)t.NU * t.E * s->F));
  double* scratch = nullptr;
  if (cudaMalloc(&scratch, most * sizeof(double)) != cudaSuccess) return mfail(FR_ERR_CUDA, "device allocation failed");
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  fr_status rc = launch_trace(s, st);
  const double* UFc = s->UF[s->cur];
  constexpr int reps = 3;
  for (int i = 0; i < s->n_types && rc == FR_OK; i++) {
    if (s->types[i].E == 0) continue;
    MixedType saved = s->types[i];
    s->types[i].DIV = scratch;
    for (int pass = 0; pass < 2 && rc == FR_OK; pass++) {
      const int nv = pass == 0 ? kNGrad : kNUpd;
      int pick = pass == 0 ? s->gv[i] : s->uv[i];
      float best = 0.f;
      bool have = false;
      for (int v = 0; v < nv && rc == FR_OK; v++) {
        if (pass == 0 ? !s->kern[i].grad[v] : !s->kern[i].upd0[v]) continue;
        // one untimed launch, then the timed ones
        for (int r = 0; r <= reps && rc == FR_OK; r++) {
          if (r == 1) cudaEventRecord(e0, st);
          rc = pass == 0 ? launch_grad(s, i, v, UFc, st) : launch_upd(s, i, v, 0, 0, 0.0, UFc, nullptr, st);
        }
        cudaEventRecord(e1, st);
        if (cudaEventSynchronize(e1) != cudaSuccess) rc = mfail(FR_ERR_CUDA, "autotune timing failed");
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (!have || ms < best) {
          best = ms;
          pick = v;
          have = true;
        }
      }
      (pass == 0 ? s->gv : s->uv)[i] = pick;
    }
    s->types[i] = saved;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(scratch);
  return rc;
}

fr_status fr_mixed_stage_info(const fr_mixed_stage* s, long long* n_flux_points, long long* n_boundary_points,
                              int* launches_per_stage)
{
  g_err.clear();
  if (!s) return mfail(FR_ERR_ARG, "null stage");
  if (n_flux_points) *n_flux_points = s->NT;
  if (n_boundary_points) *n_boundary_points = s->n_bpts;
  int n = 0;
  for (const MixedType& t : s->types) n += t.E > 0 ? 2 : 0;
  if (launches_per_stage) *launches_per_stage = n;
  return FR_OK;
}

}  // extern "C"
