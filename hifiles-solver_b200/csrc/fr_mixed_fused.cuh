// fr_mixed_fused.cuh -- kernels of the fused RK stage for dense-operator
// element types (fr_mixed_fused.cu has the design notes and the host side):
// shared-memory plans, the FP64 tensor-core product units, the gradient,
// update and trace kernels, and the table of launch shapes.  Included by
// fr_mixed_fused.cu (3-D element types) and fr_mixed_fused_2d.cu (2-D), so
// the two sets of template instances build in parallel.
#pragma once

#include <cuda_runtime.h>

#include "fr_face_update.cuh"
#include "fr_physics.cuh"

namespace frb_mixed {
using namespace frb;

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
  static_assert(F * EU <= oNLb - oUN, "residual terms fit in the neighbours' traces and projections");
};

struct MixedType {
  int NU, NF;
  long long E, off;  // elements; first flux point in the flux-point space
  const double *A45u, *A45f, *A6, *A1, *A2, *A3, *A0;  // operators in fragment order
  const double *JG, *detj;
  double *U, *REG, *DIV, *ND, *DV;
  double* partial;  // non-null on a stage whose residual norms are wanted: [block][F]
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
  // operator fragments are fetched CH k-steps ahead of their MMAs, so their
  // read-only-cache latency is paid once per CH steps
  constexpr int CH = 8;
  const double* a1 = A1 + (size_t)mt * KS1 * 32 + lane;
#pragma unroll
  for (int k0 = 0; k0 < KS1; k0 += CH) {
    double af[CH];
#pragma unroll
    for (int i = 0; i < CH; i++) af[i] = k0 + i < KS1 ? __ldg(a1 + (k0 + i) * 32) : 0.0;
#pragma unroll
    for (int i = 0; i < CH; i++)
      if (k0 + i < KS1)
#pragma unroll
        for (int j = 0; j < TN; j++)
          if (nt0 + j < NTL) dmma(acc[j], af[i], p1[j][(k0 + i) * 4]);
  }
  if constexpr (KS2 > 0) {
    const double* a2 = A2 + (size_t)mt * KS2 * 32 + lane;
#pragma unroll
    for (int k0 = 0; k0 < KS2; k0 += CH) {
      double af[CH];
#pragma unroll
      for (int i = 0; i < CH; i++) af[i] = k0 + i < KS2 ? __ldg(a2 + (k0 + i) * 32) : 0.0;
#pragma unroll
      for (int i = 0; i < CH; i++)
        if (k0 + i < KS2)
#pragma unroll
          for (int j = 0; j < TN; j++)
            if (nt0 + j < NTL) dmma(acc[j], af[i], p2[j][(k0 + i) * 4]);
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

// ------------------------------------------------------ kernel A, Euler form
// The inviscid stage needs no gradient: the transformed inviscid flux at the
// solution points (evaluate_invFlux), then norm_tdisf = sum_d opp_1[d] f_d
// and div_tdisf = sum_d opp_2[d] f_d.  JGinv is read through the L1 cache.
template <int D, int NU, int NF, int EPB>
struct MPlanInv {
  using Q = MPlan<D, NU, NF, EPB>;
  static constexpr int oU = 0, oT = Q::NP * Q::ldU, nI = oT + Q::NP * Q::ldT;
};

template <int D, int NU, int NF, int EPB, int NTH, int MINB>
__global__ void __launch_bounds__(NTH, MINB) mixed_inv_kernel(MixedType t, MixedFpts m,
                                                              const double* __restrict__ UFc, PhysT<double> ph)
{
  using Q = MPlan<D, NU, NF, EPB>;
  using I = MPlanInv<D, NU, NF, EPB>;
  constexpr int F = D + 2, NW = NTH / 32, DD = D * D;
  extern __shared__ __align__(16) double msm[];
  double* sU = msm + I::oU;
  double* sT = msm + I::oT;
  const int tid = threadIdx.x, warp = tid >> 5;
  const long long E = t.E, e0 = (long long)blockIdx.x * EPB;
  const int nval = (int)(E - e0 < EPB ? E - e0 : EPB), nuv = nval * NU;
  (void)m;
  (void)UFc;
  zero_pad_rows<NU, c4(NU), Q::ldU, Q::NP, NTH>(sU);
  zero_pad_rows<D * NU, c4(D * NU), Q::ldT, Q::NP, NTH>(sT);
  load_state<F, NU, EPB, Q::ldU, NTH>(sU, t.U, e0, E, nval);
  cp_async_wait_all();
  __syncthreads();
  for (int i = tid; i < nuv; i += NTH) {
    const int el = i / NU, p = i - el * NU;
    const double* G = t.JG + (size_t)DD * ((size_t)NU * e0 + i);
    double q[F], fi[F][D];
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
        sT[(el * F + k) * Q::ldT + l * NU + p] = acc;
      }
  }
  __syncthreads();
  auto bt = [&](int n) { return sT + n * Q::ldT; };
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

// ------------------------------------------------------------------ kernel B
// MODE 1: RK45 stage update (rk_a, rk_b, dt) and the new traces into UFn;
// MODE 0: div_tconf_upts into t.DIV only.  Like kernel A, a load phase first
// stages every global read of the block in shared memory.
template <int D, int NU, int NF, int EPB, int NTH, int MINB, int MODE, int VISC = 1, int RIEMANN = 0>
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
  double* sRes = sUN;  // |div/detJ| [F][EU] for residual norms, after the flux phase
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
    if constexpr (VISC != 0)
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
    if constexpr (VISC != 0)
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
        q.bv[k] = VISC ? m.BV[(size_t)(-1 - (long long)mt) * F + k] : 0.0;
      }
#pragma unroll
      for (int d = 0; d < D; d++) q.n[d] = n[d];
      q.tl = tl;
      fu_boundary<D, VISC, double, RIEMANN>(ph, sd >> 2, q, c, 1);
    } else {
      const bool left = sd & 1;
      double ul[F], ur[F], fn[F];
#pragma unroll
      for (int k = 0; k < F; k++) {
        const double v = sUN[k * EF + i];
        ul[k] = left ? uo[k] : v;
        ur[k] = left ? v : uo[k];
      }
      if constexpr (RIEMANN == 2 && D == 2) roe<double>(ph, ul, ur, n, fn);
      else rusanov<D, double>(ph, ul, ur, n, fn);
#pragma unroll
      for (int k = 0; k < F; k++) c[k] = left ? fn[k] * tl : -fn[k] * tl;
      if constexpr (VISC != 0) {
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
        // |div/detJ - const_src - src| of compute_res_upts (src/eles.cpp:6086-6115)
        if (t.partial) sRes[li] = fabs(div / sDJ[el * NU + r] - 0.0 - 0.0);
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
    if (t.partial && tid < F) {
      // the block's L1 residual sum of field tid: cell by cell, points in
      // order within a cell, as compute_res_upts adds them
      double bs = 0.0;
      for (int el = 0; el < nval; el++) {
        double cs = 0.0;
        for (int r = 0; r < NU; r++) cs += sRes[tid * EU + el * NU + r];
        bs += cs;
      }
      t.partial[(size_t)blockIdx.x * F + tid] = bs;
    }
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

// Physics forms: 0 Navier-Stokes (Rusanov + LDG), 1 Euler with Rusanov,
// 2 Euler with Roe (2-D).  The Euler forms have one launch shape (gradient
// slot 1: the flux kernel of 4 elements x 128 threads; update 1).
constexpr int kNForms = 3;

struct MixedKernels {
  int D, NU, NF;
  GradFn grad[kNForms][kNGrad];
  size_t smem_a[kNForms][kNGrad];
  UpdFn upd0[kNForms][kNUpd], upd1[kNForms][kNUpd];
  size_t smem_b[kNUpd];
  TraceFn trace;
  size_t smem_c;
};

template <int D, int NU, int NF, int V>
void fill_grad(MixedKernels& k)
{
  constexpr MixedShape g = kGradShapes[V];
  k.smem_a[0][V] = sizeof(double) * MPlan<D, NU, NF, g.epb, g.minb>::nA;
  k.grad[0][V] = k.smem_a[0][V] <= kMixedSmemMax ? mixed_grad_kernel<D, NU, NF, g.epb, g.nth, g.minb> : nullptr;
}

template <int D, int NU, int NF, int V>
void fill_upd(MixedKernels& k)
{
  constexpr MixedShape u = kUpdShapes[V];
  k.smem_b[V] = sizeof(double) * MPlan<D, NU, NF, u.epb>::nB;
  const bool fits = k.smem_b[V] <= kMixedSmemMax;
  k.upd0[0][V] = fits ? mixed_update_kernel<D, NU, NF, u.epb, u.nth, u.minb, 0> : nullptr;
  k.upd1[0][V] = fits ? mixed_update_kernel<D, NU, NF, u.epb, u.nth, u.minb, 1> : nullptr;
}

template <int D, int NU, int NF>
void fill_euler(MixedKernels& k)
{
  constexpr MixedShape g = kGradShapes[1], u = kUpdShapes[1];
  const size_t sa = sizeof(double) * MPlanInv<D, NU, NF, g.epb>::nI;
  const bool fa = sa <= kMixedSmemMax, fb = k.smem_b[1] <= kMixedSmemMax;
  for (int f = 1; f < kNForms; f++) {
    k.smem_a[f][1] = sa;
    k.grad[f][1] = fa ? mixed_inv_kernel<D, NU, NF, g.epb, g.nth, g.minb> : nullptr;
  }
  k.upd0[1][1] = fb ? mixed_update_kernel<D, NU, NF, u.epb, u.nth, u.minb, 0, 0, 0> : nullptr;
  k.upd1[1][1] = fb ? mixed_update_kernel<D, NU, NF, u.epb, u.nth, u.minb, 1, 0, 0> : nullptr;
  if constexpr (D == 2) {
    k.upd0[2][1] = fb ? mixed_update_kernel<D, NU, NF, u.epb, u.nth, u.minb, 0, 0, 2> : nullptr;
    k.upd1[2][1] = fb ? mixed_update_kernel<D, NU, NF, u.epb, u.nth, u.minb, 1, 0, 2> : nullptr;
  }
}

template <int D, int NU, int NF>
MixedKernels mixed_kernels()
{
  MixedKernels k{};
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
  fill_euler<D, NU, NF>(k);
  k.trace = mixed_trace_kernel<D, NU, NF, kMixedEPB, kMixedNT>;
  k.smem_c = sizeof(double) * MPlan<D, NU, NF, kMixedEPB>::nC;
  return k;
}


// the kernels of the 2-D element types of orders 2 and 3 (fr_mixed_fused_2d.cu)
bool find_kernels_2d(int NU, int NF, MixedKernels* out);
// the kernels of orders 1 and 4 (fr_mixed_fused_p14.cu)
bool find_kernels_p14(int D, int NU, int NF, MixedKernels* out);

}  // namespace frb_mixed
