// fr_face_update.cuh -- the last part of an RK stage in one element-blocked
// kernel: the common interface fluxes of the element's own flux points
// (int_inters::calculate_common_invFlux, src/int_inters.cpp:225-354, and
// calculate_common_viscFlux, src/int_inters.cpp:359-470; boundary points as
// bdy_inters::evaluate_boundaryConditions_invFlux, src/bdy_inters.cpp:245-389),
// norm_tconf - norm_tdisf, the VCJH correction
// (calculate_corrected_divergence, src/eles.cpp:1594-1661) and the RK45 stage
// update (eles::AdvanceSolution, src/eles.cpp:1155-1178) with the next
// stage's flux-point traces.
//
// Both elements of an interface evaluate its common flux, each for its own
// flux point, from the same two traces (the left side's and the right
// side's), the same left normal and their own dA, so the two copies are the
// ones a separate interface pass writes for the two sides.  The element's own
// trace is interpolated here from the state it holds (the arithmetic that
// produced the stored traces, so the values agree bit for bit); the
// neighbour's trace and viscous projection come from its flux-point arrays.
//
// Inputs reach shared memory as one-dimensional bulk copies (cp.async.bulk,
// the TMA unit; fr_tma.cuh): per field, the element block's contiguous runs
// of the state, RK register, inverse Jacobian, discontinuous normal flux,
// divergence, own viscous projection, normals and dA; per interface face, the
// neighbour's run of flux points on that face (its traces and viscous
// projections), found from the mate index of the face's first point.  This
// needs every run to be a multiple of 16 bytes (fu_bulk_ok); other shapes use
// fr_face_kernel + fr_update_kernel.
#pragma once

#include <cuda_runtime.h>

#include "fr_fused.cuh"
#include "fr_tma.cuh"

namespace frb {

// Shared-memory order of the state: point (a, b, c) at a + N1 b + PS c.
// Hexahedra of P = 3 pad each z-plane of 16 points to 18 words, which keeps
// every plane copy 16-byte aligned and limits the flux-point line reads (16
// threads per face) to 2-way bank conflicts on x- and y-faces (4-way in the
// unpadded order).
template <int DIM, int P>
struct UPad {
  static constexpr int N1 = P + 1;
  static constexpr int PS = (DIM == 3 && N1 == 4) ? 18 : N1 * N1;
  static constexpr int SU = DIM == 3 ? PS * N1 : N1 * N1;
  static constexpr bool PAD = DIM == 3 && PS != N1 * N1;
};

// Whether the bulk-copy kernel applies: every per-element run (state, point
// and flux-point arrays, one face of flux points, the state's z-planes) is a
// multiple of 16 bytes.
template <int DIM, int P, typename TC>
__host__ __device__ constexpr bool fu_bulk_ok()
{
  using S = Shape<DIM, P>;
  return (S::NU * 8) % 16 == 0 && (S::NU * sizeof(TC)) % 16 == 0 && (S::NF * sizeof(TC)) % 16 == 0 &&
         (S::NFPF * sizeof(TC)) % 16 == 0 && (DIM == 2 || ((P + 1) * (P + 1) * 8) % 16 == 0) &&
         (S::NF * 4) % 16 == 0;
}

// Per-block operator copy: derivative rows, correction derivatives, and for
// every flux point its line in the natural point order (code) and in the
// padded state order (pcode): start | stride << 8 | axis << 16 | plus << 18.
template <typename T, int NF>
struct FUOps {
  T D[kMaxN1][kMaxN1];
  T gL[kMaxN1], gR[kMaxN1];
  int code[NF], pcode[NF];
};

template <int DIM, int P, typename TC, int VISC, int MODE, int EPB, int NT>
struct FUPlan {
  using S = Shape<DIM, P>;
  using UP = UPad<DIM, P>;
  static constexpr int F = S::F, NU = S::NU, NF = S::NF, NFACE = S::NFACE, NFPF = S::NFPF, D = DIM;
  __host__ __device__ static constexpr size_t r16(size_t b) { return (b + 15) / 16 * 16; }
  static constexpr size_t bBar = 16;
  static constexpr size_t bOps = r16(sizeof(FUOps<TC, NF>));
  static constexpr size_t bU = r16(8 * (size_t)F * EPB * UP::SU);
  static constexpr size_t bREG = MODE == 1 ? r16(8 * (size_t)F * EPB * NU) : 0;
  static constexpr size_t bIDJ = MODE == 1 ? r16(8 * (size_t)EPB * NU) : 0;
  static constexpr size_t bC = r16(sizeof(TC) * F * EPB * NF);            // ND, then norm_tconf - norm_tdisf
  static constexpr size_t bDV = VISC ? r16(sizeof(TC) * F * EPB * NU) : 0;
  static constexpr size_t bVF = VISC ? r16(sizeof(TC) * (F - 1) * EPB * NF) : 0;
  static constexpr size_t bVN = VISC ? r16(sizeof(TC) * EPB * NFACE * (F - 1) * NFPF) : 0;
  static constexpr size_t bUN = r16(sizeof(TC) * EPB * NFACE * F * NFPF);
  static constexpr size_t bNL = r16(sizeof(TC) * D * EPB * NF);
  static constexpr size_t bTDA = r16(sizeof(TC) * EPB * NF);
  static constexpr size_t bJ = VISC ? 0 : r16(sizeof(TC) * EPB * D * D * NU);
  static constexpr size_t bFL = VISC ? 0 : r16(sizeof(TC) * EPB * D * F * NU);
  static constexpr size_t bRED = r16(sizeof(double) * (NT / 32) * F);
  static constexpr size_t oBar = 0, oOps = oBar + bBar, oU = oOps + bOps, oREG = oU + bU, oIDJ = oREG + bREG,
                          oC = oIDJ + bIDJ, oDV = oC + bC, oVF = oDV + bDV, oVN = oVF + bVF, oUN = oVN + bVN,
                          oNL = oUN + bUN, oTDA = oNL + bNL, oJ = oTDA + bTDA, oFL = oJ + bJ, oRED = oFL + bFL,
                          total = oRED + bRED;
};

template <int DIM, int P, typename TC, int VISC, int MODE, int EPB, int NT>
__host__ __device__ constexpr size_t face_update_smem_bytes()
{
  return FUPlan<DIM, P, TC, VISC, MODE, EPB, NT>::total;
}

// Common normal flux (times the own dA) of a boundary flux point:
// bdy_inters::evaluate_boundaryConditions_invFlux (src/bdy_inters.cpp:245-389):
// ghost state, then the central flux of the two states
// (convective_flux_boundary, src/inters.cpp:368-387), Roe in 2-D with
// RIEMANN 2, the own flux for slip_wall_dual (right_flux,
// src/inters.cpp:299-308); plus the viscous part from the gradient kernel.
template <int DIM, typename TC>
struct FUBdy {
  TC ul[DIM + 2], n[DIM], tl, bv[DIM + 2];
};
template <int DIM, int VISC, typename TC, int RIEMANN>
__device__ __noinline__ void fu_boundary(PhysT<TC> ph, int type, FUBdy<DIM, TC> q, TC* c, int cst)
{
  constexpr int F = DIM + 2, D = DIM;
  TC ug[F], fn[F];
  bc_ghost<D, TC>(ph, type, q.ul, q.n, ug);
  TC fl[F][D], fr[F][D];
  inv_flux<D, TC>(ph, q.ul, fl);
  inv_flux<D, TC>(ph, ug, fr);
  if (type == 16) {
    for (int k = 0; k < F; k++) {
      TC s = fl[k][0] * q.n[0];
      for (int l = 1; l < D; l++) s = s + fl[k][l] * q.n[l];
      fn[k] = s;
    }
  } else if (RIEMANN == 2 && DIM == 2) {
    roe<TC>(ph, q.ul, ug, q.n, fn);
  } else {
    for (int k = 0; k < F; k++) {
      TC s = fl[k][0] * q.n[0], r = fr[k][0] * q.n[0];
      for (int l = 1; l < D; l++) { s = s + fl[k][l] * q.n[l]; r = r + fr[k][l] * q.n[l]; }
      fn[k] = TC(0.5) * (s + r);
    }
  }
  for (int k = 0; k < F; k++) {
    TC v = fn[k] * q.tl;
    if (VISC) v = v + q.bv[k] * q.tl;
    c[k * cst] = v;
  }
}

// One RK stage after the gradient kernel (VISC 1), or the whole stage of the
// Euler path (VISC 0): common fluxes, correction, update (MODE 1) or the
// residual div_tconf (MODE 0, written to DIV).  idetj holds 1/detJ at the
// solution points (the update multiplies by it).  BV is the viscous normal
// flux of boundary points from the gradient kernel (side bits 2.. hold the
// boundary type there, and mate = -1 - the point's place in the boundary
// list).  err is set when a bounded wait for the bulk copies gives up.
// MINB: CTAs per SM the registers are capped for.  The body serves element
// block blk (fr_face_update_kernel: blockIdx.x; merged batch launches: their
// share of the grid).
template <int DIM, int P, int EPB, int NT, int VISC, int MODE, typename TC, int RIEMANN = 0>
__device__ __forceinline__ void
fr_face_update_body(long long blk, double* __restrict__ U, double* __restrict__ REG, TC* __restrict__ UFn,
                    const TC* __restrict__ UF, const int* __restrict__ mate, const unsigned char* __restrict__ side,
                    const TC* __restrict__ VF, const TC* __restrict__ ND, const TC* __restrict__ DV,
                    const TC* __restrict__ JG, const TC* __restrict__ nL, const TC* __restrict__ tdA,
                    const double* __restrict__ idetj, const TC* __restrict__ BV, double* __restrict__ DIV,
                    double* __restrict__ partial, long long E, const Line<TC>& L, const PhysT<TC>& ph, double rk_a,
                    double rk_b, double dt, int first_stage, int* __restrict__ err)
{
  static_assert(fu_bulk_ok<DIM, P, TC>(), "bulk-copy face/update kernel needs 16-byte runs");
  using S = Shape<DIM, P>;
  using UP = UPad<DIM, P>;
  using Q = FUPlan<DIM, P, TC, VISC, MODE, EPB, NT>;
  constexpr int NU = S::NU, NF = S::NF, F = S::F, D = DIM, DD = DIM * DIM, N1 = P + 1, NFACE = S::NFACE,
                NFPF = S::NFPF, SU = UP::SU;
  extern __shared__ __align__(16) unsigned char fr_smem[];
  auto bar = reinterpret_cast<unsigned long long*>(fr_smem + Q::oBar);
  auto B = reinterpret_cast<FUOps<TC, NF>*>(fr_smem + Q::oOps);
  double* sU = reinterpret_cast<double*>(fr_smem + Q::oU);        // [F][EPB][SU]
  double* sREG = reinterpret_cast<double*>(fr_smem + Q::oREG);    // [F][EPB][NU]
  double* sIDJ = reinterpret_cast<double*>(fr_smem + Q::oIDJ);    // [EPB][NU]
  TC* sC = reinterpret_cast<TC*>(fr_smem + Q::oC);                // [F][EPB][NF]
  TC* sDV = reinterpret_cast<TC*>(fr_smem + Q::oDV);              // [F][EPB][NU]
  TC* sVF = reinterpret_cast<TC*>(fr_smem + Q::oVF);              // [F-1][EPB][NF]
  TC* sVN = reinterpret_cast<TC*>(fr_smem + Q::oVN);              // [EPB][NFACE][F-1][NFPF]
  TC* sUN = reinterpret_cast<TC*>(fr_smem + Q::oUN);              // [EPB][NFACE][F][NFPF]
  TC* sNL = reinterpret_cast<TC*>(fr_smem + Q::oNL);              // [D][EPB][NF]
  TC* sTDA = reinterpret_cast<TC*>(fr_smem + Q::oTDA);            // [EPB][NF]
  TC* sJ = reinterpret_cast<TC*>(fr_smem + Q::oJ);                // [EPB][DD*NU]
  TC* sFl = reinterpret_cast<TC*>(fr_smem + Q::oFL);              // [EPB][D][F][NU]
  auto sRed = reinterpret_cast<double (*)[F]>(fr_smem + Q::oRED);

  const int tid = threadIdx.x;
  const long long e0 = blk * EPB;
  const int nval = (int)(E - e0 < EPB ? E - e0 : EPB);
  const long long NFE = (long long)NF * E, NUE = (long long)NU * E;
  const bool want_reg = MODE == 1 && !first_stage;

  // operator copy (the flux-point line codes, natural and padded)
  for (int i = tid; i < kMaxN1 * kMaxN1; i += NT) B->D[i / kMaxN1][i % kMaxN1] = L.D[i / kMaxN1][i % kMaxN1];
  for (int i = tid; i < kMaxN1; i += NT) { B->gL[i] = L.gL[i]; B->gR[i] = L.gR[i]; }
  for (int f = tid; f < NF; f += NT) {
    int u0, st, ax; bool plus;
    fpt_line<DIM, P>(f, u0, st, ax, plus);
    int a, b, c;
    upt_abc<DIM, P>(u0, a, b, c);
    const int pu0 = a + N1 * b + UP::PS * c;
    const int pst = ax == 0 ? 1 : (ax == 1 ? N1 : UP::PS);
    B->code[f] = u0 | (st << 8) | (ax << 16) | ((plus ? 1 : 0) << 18);
    B->pcode[f] = pu0 | (pst << 8) | (ax << 16) | ((plus ? 1 : 0) << 18);
  }

  // --- bulk copies: bar[0] the element block's own runs (one arrival by
  // thread 0 with the byte count), bar[1] the neighbours' face runs (one
  // arrival per face of the block)
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], EPB * NFACE);
    mbar_fence_init();
  }
  __syncthreads();
  if (tid < 32) {
    const int lane = tid;
    if (lane == 0) {
      unsigned bytes = 8u * nval * NU * F;
      if (want_reg) bytes += 8u * nval * NU * F;
      if (MODE == 1) bytes += 8u * nval * NU;
      if (VISC) bytes += (unsigned)sizeof(TC) * nval * (NF * F + NU * F + NF * (F - 1));
      bytes += (unsigned)sizeof(TC) * nval * NF * (D + 1);
      if (!VISC) bytes += (unsigned)sizeof(TC) * nval * DD * NU;
      mbar_arrive_tx(&bar[0], bytes);
    }
    __syncwarp();
    // the state: one copy per (field, element, z-plane) when padded, else per field
    constexpr int NQU = UP::PAD ? F * EPB * N1 : F;
    for (int q = lane; q < NQU; q += 32) {
      if (UP::PAD) {
        const int k = q / (EPB * N1), r = q - k * EPB * N1, el = r / N1, c = r - el * N1;
        if (el < nval)
          bulk_load(sU + (k * EPB + el) * SU + UP::PS * c, U + NU * (e0 + el + E * k) + N1 * N1 * c,
                    8u * N1 * N1, &bar[0]);
      } else {
        bulk_load(sU + q * EPB * SU, U + NU * (e0 + E * q), 8u * nval * NU, &bar[0]);
      }
    }
    // the remaining runs, one per (array, component)
    constexpr int NQ = (MODE == 1 ? F + 1 : 0) + (VISC ? F + F + (F - 1) : 0) + D + 1 + (VISC ? 0 : 1);
    for (int q = lane; q < NQ; q += 32) {
      int j = q;
      if (MODE == 1) {
        if (j < F) {
          if (want_reg) bulk_load(sREG + j * EPB * NU, REG + NU * (e0 + E * j), 8u * nval * NU, &bar[0]);
          continue;
        }
        j -= F;
        if (j == 0) { bulk_load(sIDJ, idetj + NU * e0, 8u * nval * NU, &bar[0]); continue; }
        j -= 1;
      }
      if (VISC) {
        if (j < F) { bulk_load(sC + j * EPB * NF, ND + NF * e0 + NFE * j, sizeof(TC) * nval * NF, &bar[0]); continue; }
        j -= F;
        if (j < F) { bulk_load(sDV + j * EPB * NU, DV + NU * e0 + NUE * j, sizeof(TC) * nval * NU, &bar[0]); continue; }
        j -= F;
        if (j < F - 1) { bulk_load(sVF + j * EPB * NF, VF + NF * e0 + NFE * j, sizeof(TC) * nval * NF, &bar[0]); continue; }
        j -= F - 1;
      }
      if (j < D) { bulk_load(sNL + j * EPB * NF, nL + NF * e0 + NFE * j, sizeof(TC) * nval * NF, &bar[0]); continue; }
      j -= D;
      if (j == 0) { bulk_load(sTDA, tdA + NF * e0, sizeof(TC) * nval * NF, &bar[0]); continue; }
      j -= 1;
      if (!VISC && j == 0) bulk_load(sJ, JG + (size_t)DD * NU * e0, sizeof(TC) * nval * DD * NU, &bar[0]);
    }
  } else if (tid < 64) {
    // neighbour face runs: face (el, fc) of the block, traces and viscous projections
    for (int q = tid - 32; q < EPB * NFACE; q += 32) {
      const int el = q / NFACE, fc = q - el * NFACE;
      int m = -1;
      if (el < nval) m = mate[NF * (e0 + el) + NFPF * fc];
      if (m < 0) {
        mbar_arrive_tx(&bar[1], 0u);
        continue;
      }
      const int run = m - m % NFPF;
      mbar_arrive_tx(&bar[1], (unsigned)sizeof(TC) * NFPF * (F + (VISC ? F - 1 : 0)));
#pragma unroll
      for (int k = 0; k < F; k++)
        bulk_load(sUN + ((el * NFACE + fc) * F + k) * NFPF, UF + run + NFE * k, sizeof(TC) * NFPF, &bar[1]);
      if (VISC)
#pragma unroll
        for (int k = 0; k < F - 1; k++)
          bulk_load(sVN + ((el * NFACE + fc) * (F - 1) + k) * NFPF, VF + run + NFE * k, sizeof(TC) * NFPF,
                    &bar[1]);
    }
  }
  static_assert(NT >= 64 || EPB * NFACE <= 0, "the face/update kernel needs at least two warps");

  // the thread's flux points: mate and side (plain loads, in flight during the copies)
  constexpr int IF = Items<NT, EPB * NF>::N, IU = Items<NT, EPB * NU>::N;
  int mt[IF];
  unsigned char sd[IF];
#pragma unroll
  for (int it = 0; it < IF; it++) {
    const int w = tid + it * NT, el = w / NF, f = w - el * NF;
    mt[it] = -1;
    sd[it] = 0;
    if (w < EPB * NF && el < nval) {
      mt[it] = mate[f + NF * (e0 + el)];
      sd[it] = side[f + NF * (e0 + el)];
    }
  }
  {
    const bool ok0 = mbar_wait(&bar[0], 0, err);
    const bool ok1 = mbar_wait(&bar[1], 0, err);
    (void)ok0; (void)ok1;
  }
  __syncthreads();

  // --- Euler path: transformed inviscid flux at the solution points
  // (evaluate_invFlux, src/eles.cpp:1331-1418)
  if constexpr (!VISC) {
#pragma unroll
    for (int it = 0; it < IU; it++) {
      const int w = tid + it * NT, el = w / NU, u = w - el * NU;
      if (w >= EPB * NU || el >= nval) continue;
      int a, b, c;
      upt_abc<DIM, P>(u, a, b, c);
      const int pu = a + N1 * b + UP::PS * c;
      TC g[DD];
#pragma unroll
      for (int q = 0; q < DD; q++) g[q] = sJ[el * DD * NU + DD * u + q];
      TC qv[F], fi[F][D];
#pragma unroll
      for (int k = 0; k < F; k++) qv[k] = (TC)sU[(k * EPB + el) * SU + pu];
      inv_flux<D, TC>(ph, qv, fi);
#pragma unroll
      for (int l = 0; l < D; l++)
#pragma unroll
        for (int k = 0; k < F; k++) {
          TC acc = g[l] * fi[k][0];
#pragma unroll
          for (int m = 1; m < D; m++) acc = acc + g[l + D * m] * fi[k][m];
          sFl[((el * D + l) * F + k) * NU + u] = acc;
        }
    }
    __syncthreads();
  }

  // --- common fluxes at the own flux points, minus the discontinuous normal flux
#pragma unroll
  for (int it = 0; it < IF; it++) {
    const int w = tid + it * NT, el = w / NF, f = w - el * NF;
    if (w >= EPB * NF || el >= nval) continue;
    const int pc = B->pcode[f];
    const int pu0 = code_u0(pc), pst = code_st(pc);
    const bool plus = code_plus(pc);
    TC Lc[P + 1];
#pragma unroll
    for (int m = 0; m <= P; m++) Lc[m] = plus ? L.Lp[m] : L.Lm[m];
    // own trace: the opp_0 row of f in column order, (((0 + t0) + t1) + ...)
    TC uo[F];
#pragma unroll
    for (int k = 0; k < F; k++) {
      const double* s = sU + (k * EPB + el) * SU + pu0;
      TC acc = TC(0);
#pragma unroll
      for (int m = 0; m <= P; m++) acc = acc + (TC)s[m * pst] * Lc[m];
      uo[k] = acc;
    }
    TC n[D];
#pragma unroll
    for (int d = 0; d < D; d++) n[d] = sNL[(d * EPB + el) * NF + f];
    const TC tl = sTDA[el * NF + f];
    TC c[F];
    if (sd[it] >> 2) {
      FUBdy<DIM, TC> q;
#pragma unroll
      for (int k = 0; k < F; k++) {
        q.ul[k] = uo[k];
        q.bv[k] = VISC ? BV[(-1 - (long long)mt[it]) * F + k] : TC(0);
      }
#pragma unroll
      for (int d = 0; d < D; d++) q.n[d] = n[d];
      q.tl = tl;
      fu_boundary<DIM, VISC, TC, RIEMANN>(ph, sd[it] >> 2, q, c, 1);
    } else {
      const int fc = f / NFPF, loc = mt[it] % NFPF;
      const TC* un = sUN + (el * NFACE + fc) * F * NFPF + loc;
      const bool left = sd[it] & 1;
      TC ul[F], ur[F];
#pragma unroll
      for (int k = 0; k < F; k++) {
        const TC v = un[k * NFPF];
        ul[k] = left ? uo[k] : v;
        ur[k] = left ? v : uo[k];
      }
      TC fn[F];
      if constexpr (RIEMANN == 2 && DIM == 2) roe<TC>(ph, ul, ur, n, fn);
      else rusanov<D, TC>(ph, ul, ur, n, fn);
#pragma unroll
      for (int k = 0; k < F; k++) c[k] = left ? fn[k] * tl : -fn[k] * tl;
      if constexpr (VISC != 0) {
        TC nn = n[0] * n[0];
#pragma unroll
        for (int d = 1; d < D; d++) nn = fr_fma(n[d], n[d], nn);
        const TC pen = (sd[it] & 2) ? -ph.pen_fact : ph.pen_fact;
        const TC* vn = sVN + (el * NFACE + fc) * (F - 1) * NFPF + loc;
        // every field, density included, takes the tau (u_l - u_r) penalty;
        // the density's viscous projections are zero
#pragma unroll
        for (int k = 0; k < F; k++) {
          const TC ao = k ? sVF[((k - 1) * EPB + el) * NF + f] : TC(0), an = k ? vn[(k - 1) * NFPF] : TC(0);
          const TC fv = ldg_normal<TC>(left ? ao : an, left ? an : ao, ul[k], ur[k], pen, ph.tau, nn);
          c[k] = left ? c[k] + fv * tl : c[k] + (-fv) * tl;
        }
      }
    }
    if constexpr (VISC != 0) {
#pragma unroll
      for (int k = 0; k < F; k++) {
        TC* p = sC + (k * EPB + el) * NF + f;
        *p = c[k] - *p;                               // daxpy(-1, norm_tdisf, norm_tconf)
      }
    } else {
      // norm_tdisf from the transformed flux (extrapolate_totalFlux), then norm_tconf - norm_tdisf
      const int cd = B->code[f];
      const int ax = code_ax(cd);
#pragma unroll
      for (int k = 0; k < F; k++) {
        const TC v = interp_code<P, TC, TC>(L, cd, sFl + ((el * D + ax) * F + k) * NU);
        sC[(k * EPB + el) * NF + f] = c[k] - (plus ? v : -v);
      }
    }
  }
  __syncthreads();

  // --- correction and update at the solution points
  double red[F];
#pragma unroll
  for (int k = 0; k < F; k++) red[k] = 0.0;
#pragma unroll
  for (int it = 0; it < IU; it++) {
    const int w = tid + it * NT, el = w / NU, u = w - el * NU;
    if (w >= EPB * NU || el >= nval) continue;
    const long long e = e0 + el;
    int abc[3];
    upt_abc<DIM, P>(u, abc[0], abc[1], abc[2]);
    const int pu = abc[0] + N1 * abc[1] + UP::PS * abc[2];
    // opp_3 row of u: one column per face, in flux-point order (the same for every field)
    int qf[S::NFACE];
    TC cf[S::NFACE];
#pragma unroll
    for (int fc = 0; fc < S::NFACE; fc++) {
      int al;
      qf[fc] = face_fpt<DIM, P>(fc, abc[0], abc[1], abc[2], al);
      cf[fc] = face_plus<DIM>(fc) ? B->gR[al] : -B->gL[al];
    }
    const double idj = MODE == 1 ? sIDJ[el * NU + u] : 1.0;
#pragma unroll
    for (int k = 0; k < F; k++) {
      const size_t gi = u + (size_t)NU * (e + E * k);
      TC acc;
      if constexpr (VISC != 0) {
        acc = sDV[(k * EPB + el) * NU + u];
      } else {
        acc = TC(0);
#pragma unroll
        for (int d = 0; d < D; d++) {
          const int st = upt_stride<DIM, P>(d), ub = u - abc[d] * st;
          const TC* s = sFl + ((el * D + d) * F + k) * NU;
#pragma unroll
          for (int m = 0; m <= P; m++) acc = acc + s[ub + m * st] * B->D[abc[d]][m];
        }
      }
      const TC* cc = sC + (k * EPB + el) * NF;
#pragma unroll
      for (int fc = 0; fc < S::NFACE; fc++) acc = acc + cc[qf[fc]] * cf[fc];
      const double R = (double)acc;
      if (MODE == 0) {
        DIV[gi] = R;
      } else {
        const double rhs = -R * idj;
        const double res = first_stage ? dt * rhs : rk_a * sREG[(k * EPB + el) * NU + u] + dt * rhs;
        REG[gi] = res;
        double* su = sU + (k * EPB + el) * SU + pu;
        const double un = *su + rk_b * res;
        U[gi] = un;
        *su = un;
        red[k] += fabs(rhs);
      }
    }
  }
  if (MODE == 1) {
    if (partial) {
      // deterministic per-block partial sums of |div/detjac| (CalcNormResidual)
      const int lane = tid & 31, wid = tid >> 5;
#pragma unroll
      for (int k = 0; k < F; k++) {
        double v = red[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sRed[wid][k] = v;
      }
    }
    __syncthreads();
    if (partial && tid < F) {
      double v = 0.0;
      for (int i = 0; i < NT / 32; i++) v += sRed[i][tid];
      partial[(size_t)blk * F + tid] = v;
    }
    // traces of the updated state for the next stage: the opp_0 row of f in column order
#pragma unroll
    for (int it = 0; it < IF; it++) {
      const int w = tid + it * NT, el = w / NF, f = w - el * NF;
      if (w >= EPB * NF || el >= nval) continue;
      const int pc = B->pcode[f];
      const int pu0 = code_u0(pc), pst = code_st(pc);
      const bool plus = code_plus(pc);
      TC Lc[P + 1];
#pragma unroll
      for (int m = 0; m <= P; m++) Lc[m] = plus ? L.Lp[m] : L.Lm[m];
#pragma unroll
      for (int k = 0; k < F; k++) {
        const double* s = sU + (k * EPB + el) * SU + pu0;
        TC acc = TC(0);
#pragma unroll
        for (int m = 0; m <= P; m++) acc = acc + (TC)s[m * pst] * Lc[m];
        UFn[f + NF * (e0 + el) + NFE * k] = acc;
      }
    }
  }
}

template <int DIM, int P, int EPB, int NT, int VISC, int MODE, typename TC, int RIEMANN = 0, int MINB = 1>
__global__ void __launch_bounds__(NT, MINB)
fr_face_update_kernel(double* __restrict__ U, double* __restrict__ REG, TC* __restrict__ UFn,
                      const TC* __restrict__ UF, const int* __restrict__ mate, const unsigned char* __restrict__ side,
                      const TC* __restrict__ VF, const TC* __restrict__ ND, const TC* __restrict__ DV,
                      const TC* __restrict__ JG, const TC* __restrict__ nL, const TC* __restrict__ tdA,
                      const double* __restrict__ idetj, const TC* __restrict__ BV, double* __restrict__ DIV,
                      double* __restrict__ partial, long long E, Line<TC> L, PhysT<TC> ph, double rk_a,
                      double rk_b, double dt, int first_stage, int* __restrict__ err)
{
  fr_face_update_body<DIM, P, EPB, NT, VISC, MODE, TC, RIEMANN>(blockIdx.x, U, REG, UFn, UF, mate, side, VF, ND, DV, JG,
                                                                nL, tdA, idetj, BV, DIV, partial, E, L, ph, rk_a, rk_b,
                                                                dt, first_stage, err);
}

}  // namespace frb
