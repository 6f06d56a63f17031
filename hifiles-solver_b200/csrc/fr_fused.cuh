// fr_fused.cuh -- fused, sum-factorised FR stage kernels for tensor-product
// elements (quadrilaterals D=2, hexahedra D=3) on sm_100a.
//
// One RK stage of the reference (CalcResidual, src/solver.cpp:65-225, then
// eles::AdvanceSolution, src/eles.cpp:1091-1188) runs as
//   viscous :  fr_grad_kernel -> fr_face_kernel -> fr_update_kernel
//   inviscid:                    fr_face_kernel -> fr_update_kernel
// The element kernels are element-blocked: a CTA owns EPB elements, stages their solution in
// shared memory, and applies the reference's operators as 1-D line
// contractions (every dense operator opp_0..opp_6 of a Gauss-point tensor
// element has exactly one non-trivial factor per line, so the contraction
// reproduces the dense product term by term).  Elements exchange data only
// through flux-point traces in HBM:
//   UF  (n_fpts, n_eles, F)      solution at the flux points, double-buffered
//                                across stages (written by the stage update)
//   VF  (n_fpts, n_eles, F-1)    own viscous flux at the flux points projected
//                                on the interface's left normal (viscous path)
//   ND  (n_fpts, n_eles, F)      normal discontinuous flux (norm_tdisf_fpts)
//   DV  (n_upts, n_eles, F)      divergence of the discontinuous flux
//   CF  (n_fpts, n_eles, F)      common normal flux times tdA (norm_tconf_fpts)
// mate[i] is the flat index (fpt + n_fpts*ele) of the matching point across
// the interface; side[i] bit 0 = this side is the left one, bit 1 = the LDG
// penalty sign is negative.  Both sides evaluate the common flux with the
// left/right roles and the left normal nL, so the two copies are identical.
#pragma once

#include <cuda_runtime.h>

#include "fr_physics.cuh"

namespace frb {

constexpr int kMaxN1 = 6;   // P <= 5 in the fused kernels

template <typename T>
struct Line {               // 1-D operator pieces (see Line1D in fr_host.hpp)
  T Lm[kMaxN1], Lp[kMaxN1], D[kMaxN1][kMaxN1], gL[kMaxN1], gR[kMaxN1], w[kMaxN1];
};

template <int DIM, int P>
struct Shape {
  static constexpr int N1 = P + 1;
  static constexpr int NU = DIM == 2 ? N1 * N1 : N1 * N1 * N1;
  static constexpr int NFPF = DIM == 2 ? N1 : N1 * N1;
  static constexpr int NFACE = 2 * DIM;
  static constexpr int NF = NFACE * NFPF;
  static constexpr int F = DIM + 2;
};

// Line through flux point f: first solution point, stride along the line,
// axis, and whether the face is at the +1 end.  Reference orderings:
// quads src/eles_quads.cpp:259-300, hexes src/eles_hexas.cpp:262-324.
template <int DIM, int P>
__device__ __forceinline__ void fpt_line(int f, int& u0, int& stride, int& axis, bool& plus)
{
  constexpr int N1 = P + 1;
  if (DIM == 2) {
    int fc = f / N1, j = f - fc * N1;
    switch (fc) {
      case 0: u0 = j; stride = N1; axis = 1; plus = false; break;
      case 1: u0 = N1 * j; stride = 1; axis = 0; plus = true; break;
      case 2: u0 = P - j; stride = N1; axis = 1; plus = true; break;
      default: u0 = N1 * (P - j); stride = 1; axis = 0; plus = false; break;
    }
  } else {
    constexpr int N2 = N1 * N1;
    int fc = f / N2, r = f - fc * N2, j = r / N1, k = r - j * N1;
    switch (fc) {
      case 0: u0 = (P - k) + N1 * j; stride = N2; axis = 2; plus = false; break;
      case 1: u0 = k + N2 * j; stride = N1; axis = 1; plus = false; break;
      case 2: u0 = N1 * k + N2 * j; stride = 1; axis = 0; plus = true; break;
      case 3: u0 = (P - k) + N2 * j; stride = N1; axis = 1; plus = true; break;
      case 4: u0 = N1 * (P - k) + N2 * j; stride = 1; axis = 0; plus = false; break;
      default: u0 = k + N1 * j; stride = N2; axis = 2; plus = true; break;
    }
  }
}

// Flux point of face fc on the line through solution point (a, b, c), and the
// index of that point along the face normal.
template <int DIM, int P>
__device__ __forceinline__ int face_fpt(int fc, int a, int b, int c, int& along)
{
  constexpr int N1 = P + 1;
  if (DIM == 2) {
    switch (fc) {
      case 0: along = b; return a;
      case 1: along = a; return N1 + b;
      case 2: along = b; return 2 * N1 + (P - a);
      default: along = a; return 3 * N1 + (P - b);
    }
  }
  constexpr int N2 = N1 * N1;
  switch (fc) {
    case 0: along = c; return (P - a) + N1 * b;
    case 1: along = b; return N2 + a + N1 * c;
    case 2: along = a; return 2 * N2 + b + N1 * c;
    case 3: along = b; return 3 * N2 + (P - a) + N1 * c;
    case 4: along = a; return 4 * N2 + (P - b) + N1 * c;
    default: along = c; return 5 * N2 + a + N1 * b;
  }
}

// axis and end of face fc (reference normals: quads f0 -y, f1 +x, f2 +y, f3 -x;
// hexes f0 -z, f1 -y, f2 +x, f3 +y, f4 -x, f5 +z)
template <int DIM>
__device__ __forceinline__ bool face_plus(int fc)
{
  if (DIM == 2) return fc == 1 || fc == 2;
  return fc == 2 || fc == 3 || fc == 5;
}
template <int DIM>
__device__ __forceinline__ int face_axis(int fc)
{
  if (DIM == 2) return (fc == 1 || fc == 3) ? 0 : 1;
  return (fc == 2 || fc == 4) ? 0 : ((fc == 1 || fc == 3) ? 1 : 2);
}

// Value at flux point f of a field stored point-major (s[u * sst]): the
// reference's opp_0 row of f applied in column order, (((0 + t0) + t1) + ...).
template <int DIM, int P, typename T, typename S>
__device__ __forceinline__ T line_interp(const Line<T>& L, const S* s, int sst, int f)
{
  int u0, st, ax; bool plus;
  fpt_line<DIM, P>(f, u0, st, ax, plus);
  T acc = T(0);
#pragma unroll
  for (int m = 0; m <= P; m++) acc = acc + (T)s[(u0 + m * st) * sst] * (plus ? L.Lp[m] : L.Lm[m]);
  return acc;
}

template <int DIM, int P>
__device__ __forceinline__ void upt_abc(int u, int& a, int& b, int& c)
{
  constexpr int N1 = P + 1;
  if (DIM == 2) { b = u / N1; a = u - b * N1; c = 0; }
  else { c = u / (N1 * N1); int r = u - c * N1 * N1; b = r / N1; a = r - b * N1; }
}

template <int DIM, int P>
__device__ __forceinline__ int upt_stride(int axis)
{
  constexpr int N1 = P + 1;
  return axis == 0 ? 1 : (axis == 1 ? N1 : N1 * N1);
}

// Sum over all axes of the 1-D derivative along each axis of a field stored
// point-major: the reference's sum_d opp_2[d] (or opp_4[d]) row of u, in
// column order per axis and axes in order.
template <int DIM, int P, typename T, typename S>
__device__ __forceinline__ T deriv_line(const Line<T>& L, const S* s, int sst, int u, int d, int i)
{
  const int st = upt_stride<DIM, P>(d), ub = u - i * st;
  T acc = T(0);
#pragma unroll
  for (int m = 0; m <= P; m++) acc = acc + (T)s[(ub + m * st) * sst] * L.D[i][m];
  return acc;
}

// Per-block copy of the operator pieces that threads index with their own
// (divergent) point indices, plus a table with the line of every flux point:
// code = u0 | stride << 8 | axis << 16 | plus << 18.  Reading these from
// shared memory avoids both serialised constant-bank loads and divergent
// branches on the face index.
template <typename T, int NF>
struct BlockOps {
  T D[kMaxN1][kMaxN1];
  T gL[kMaxN1], gR[kMaxN1];
  int code[NF];
};

template <typename T, int NF>
__host__ __device__ constexpr size_t blockops_bytes()
{
  return (sizeof(BlockOps<T, NF>) + 15) / 16 * 16;
}

template <int DIM, int P, typename T, int NF>
__device__ __forceinline__ void fill_blockops(BlockOps<T, NF>* B, const Line<T>& L, int tid, int nt)
{
  for (int i = tid; i < kMaxN1 * kMaxN1; i += nt) B->D[i / kMaxN1][i % kMaxN1] = L.D[i / kMaxN1][i % kMaxN1];
  for (int i = tid; i < kMaxN1; i += nt) { B->gL[i] = L.gL[i]; B->gR[i] = L.gR[i]; }
  for (int f = tid; f < NF; f += nt) {
    int u0, st, ax; bool plus;
    fpt_line<DIM, P>(f, u0, st, ax, plus);
    B->code[f] = u0 | (st << 8) | (ax << 16) | ((plus ? 1 : 0) << 18);
  }
}

__device__ __forceinline__ int code_u0(int c) { return c & 255; }
__device__ __forceinline__ int code_st(int c) { return (c >> 8) & 255; }
__device__ __forceinline__ int code_ax(int c) { return (c >> 16) & 3; }
__device__ __forceinline__ bool code_plus(int c) { return (c >> 18) & 1; }

// line_interp with the line taken from a flux-point code
template <int P, typename T, typename S>
__device__ __forceinline__ T interp_code(const Line<T>& L, int c, const S* s)
{
  const int u0 = code_u0(c), st = code_st(c);
  const bool plus = code_plus(c);
  T acc = T(0);
#pragma unroll
  for (int m = 0; m <= P; m++) acc = acc + (T)s[u0 + m * st] * (plus ? L.Lp[m] : L.Lm[m]);
  return acc;
}

// Dynamic shared-memory sizes of the stage kernels.
template <int DIM, int P, bool ALIAS> struct GradPlan;
template <int DIM, int P, int EPB, typename TC, int LES = 0, bool ALIAS = false>
__host__ __device__ constexpr size_t grad_smem_bytes();
template <int DIM, int P, int EPB, int NT, int VISC, int MODE, typename TC> struct UpdPlan;
template <int DIM, int P, int EPB, int NT, int VISC, int MODE, typename TC>
__host__ __device__ constexpr size_t update_smem_bytes();

template <int NT, int ITEMS>
struct Items {
  static constexpr int N = (ITEMS + NT - 1) / NT;
};

// ---------------------------------------------------------------------------
// Initial flux-point traces from the state (used once after the state is set).
template <int DIM, int P, typename TC>
__global__ void fr_trace_kernel(const double* __restrict__ U, TC* __restrict__ UF, long long E, Line<TC> L,
                                double* __restrict__ Uout = nullptr)
{
  using S = Shape<DIM, P>;
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  // with Uout, U is a staged state that the same pass copies into place
  // (the grid then covers max(NF, NU) points per element)
  if (Uout && i < E * S::NU)
#pragma unroll
    for (int k = 0; k < S::F; k++) Uout[i + (size_t)S::NU * E * k] = U[i + (size_t)S::NU * E * k];
  if (i >= E * S::NF) return;
  long long e = i / S::NF;
  int f = (int)(i - e * S::NF);
#pragma unroll
  for (int k = 0; k < S::F; k++) {
    const double* ue = U + (size_t)S::NU * (e + E * k);
    UF[f + (size_t)S::NF * (e + E * k)] = line_interp<DIM, P, TC, double>(L, ue, 1, f);
  }
}

// ---------------------------------------------------------------------------
// Asynchronous global -> shared copies (cp.async, sm_80 and later; no
// multicast).  Each thread copies its own elements; cp_async_wait_all plus a
// block barrier makes them visible to the block.
template <int N>
__device__ __forceinline__ void cp_async(void* dst, const void* src)
{
  static_assert(N == 4 || N == 8 || N == 16, "cp.async copies 4, 8 or 16 bytes");
  const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(s), "l"(src), "n"(N) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// N contiguous shared values, 16 bytes per load where N allows (s 16-byte aligned)
template <int N, typename T>
__device__ __forceinline__ void lds_line(const T* s, T (&v)[N])
{
  if constexpr (sizeof(T) == 8 && N % 2 == 0) {
#pragma unroll
    for (int i = 0; i < N; i += 2) {
      const double2 q = *reinterpret_cast<const double2*>(s + i);
      v[i] = q.x; v[i + 1] = q.y;
    }
  } else if constexpr (sizeof(T) == 4 && N % 4 == 0) {
#pragma unroll
    for (int i = 0; i < N; i += 4) {
      const float4 q = *reinterpret_cast<const float4*>(s + i);
      v[i] = q.x; v[i + 1] = q.y; v[i + 2] = q.z; v[i + 3] = q.w;
    }
  } else {
#pragma unroll
    for (int i = 0; i < N; i++) v[i] = s[i];
  }
}

// Shared-memory slot of solution point u in the gradient kernel's per-field
// point arrays.  Hexahedra of P = 3 in FP64 store point (a, b, c) at
// 16 c + 4 ((b + c) & 3) + ((a + c) & 3): every z-plane stays one 128-byte
// row, and the 16 points of any face plane (c, b or a fixed) fall in 16
// distinct 8-byte bank pairs, so the flux-point phases -- one thread per
// flux point, 16 threads per face, reading the line through their point --
// and the line reads of the solution-point phases are free of bank
// conflicts.  Other shapes, and 4-byte values (32 per bank row), keep the
// natural order.
template <int DIM, int P, typename TC>
__host__ __device__ constexpr bool swz_on()
{
  return DIM == 3 && P == 3 && sizeof(TC) == 8;
}
template <int DIM, int P, typename TC>
__device__ __forceinline__ int swz(int u)
{
  if constexpr (swz_on<DIM, P, TC>()) return (u & 48) | ((((u >> 2) + (u >> 4)) & 3) << 2) | ((u + (u >> 4)) & 3);
  else return u;
}

// Boundary points of the gradient kernel, out of line so that the hot loop
// bodies stay compact (most meshes have few or no boundary points).  The
// inputs travel by value, so no array of the calling thread has its address
// taken.
template <int D, typename TC>
struct BdyPoint {
  TC u[D + 2], n[D], g[D + 2][D], fv[D + 2][D];
};

// LDG common solution of a boundary point: ghost state from the boundary
// condition, then ldg_solution with flux_spec 1 or 2, u_c = (u_r + u_l)/2
// (bdy_inters::evaluate_boundaryConditions_invFlux, src/bdy_inters.cpp:245-389);
// writes delta = u_c - u_own and u_own at stride st.
template <int D, typename TC>
__device__ __noinline__ void ldg_boundary(PhysT<TC> ph, int type, BdyPoint<D, TC> q, TC* dx, TC* uf, int st)
{
  constexpr int F = D + 2;
  TC ug[F];
  bc_ghost<D, TC>(ph, type, q.u, q.n, ug);
  for (int k = 0; k < F; k++) {
    TC uc = TC(0.5) * (ug[k] + q.u[k]);
    dx[k * st] = uc - q.u[k];
    uf[k * st] = q.u[k];
  }
}

// Viscous normal flux of a boundary point, bdy_inters::evaluate_boundaryConditions_viscFlux
// (src/bdy_inters.cpp:905-1057): own flux q.fv (flux_spec 1) or the ghost
// side's with the adiabatic-wall energy gradient (flux_spec 2, types 12 and
// 14), plus tau n (u_l - u_r), on the normal.  q.g is the own gradient; with
// HAVE_FV = false the own flux is evaluated here from q.u and q.g.
template <int D, typename TC, bool HAVE_FV = true>
__device__ __noinline__ void vis_boundary(PhysT<TC> ph, int type, BdyPoint<D, TC> q, TC* bv)
{
  constexpr int F = D + 2;
  if (!HAVE_FV) vis_flux_fast<D, TC>(ph, q.u, q.g, q.fv);
  TC ug[F];
  bc_ghost<D, TC>(ph, type, q.u, q.n, ug);
  if (type == 12 || type == 14) {
    bc_vis_gradient<D, TC>(ph, q.u, ug, q.g);
    vis_flux_fast<D, TC>(ph, ug, q.g, q.fv);
  }
  for (int k = 0; k < F; k++) {
    TC fnk = (q.fv[k][0] + ph.tau * q.n[0] * (q.u[k] - ug[k])) * q.n[0];
    for (int d = 1; d < D; d++) fnk = fnk + (q.fv[k][d] + ph.tau * q.n[d] * (q.u[k] - ug[k])) * q.n[d];
    bv[k] = fnk;
  }
}

// side bytes of the block's flux points, after the operator copy
template <int EPB, int NF>
__host__ __device__ constexpr size_t grad_side_bytes()
{
  return (EPB * NF + 15) / 16 * 16;
}

// Shared-memory plan of fr_grad_kernel, per element, in units of TC:
//   sU  [F][NU]      solution
//   sX  [F][NF]      neighbour traces, then (in place) delta_disu_fpts
//   sUf [F][NF]      own solution at the flux points
//   sM  [R3N]        metrics JGinv (NU x D*D, the reference's per-element
//                    order) and detJ (NU) for the solution-point phase, then
//                    the left normals [D][NF] for the flux-point phase
//   sG  [F*D][NU]    physical gradient (component k + F*d)
//   sFl [D][F][NU]   transformed total flux
//   sS  [(F-1)*D][NU] transformed SGS flux (LES only)
// Every region size is rounded up to 4 words, so each region, and each
// element's block, starts on a 16-byte boundary whatever the point counts.
// With ALIAS the transformed flux sFl takes the place of sX and the metrics
// (both dead once every thread has finished its solution-point reads; the
// kernel puts a barrier there) and the left normals go to sU (dead after the
// solution-point phase): 25 % less shared memory per element.  oN is where
// the left normals [D][NF] live for the flux-point phase.
template <int DIM, int P, bool ALIAS>
struct GradPlan {
  using S = Shape<DIM, P>;
  __host__ __device__ static constexpr int r4(int n) { return (n + 3) / 4 * 4; }
  static constexpr int NM = (DIM * DIM + 1) * S::NU;        // metrics
  static constexpr int R3N = ALIAS ? NM : (NM > DIM * S::NF ? NM : DIM * S::NF);
  static constexpr int oX = r4(S::F * S::NU);
  static constexpr int oUf = ALIAS ? oX + r4(S::F * S::NF) + r4(R3N) : oX + r4(S::F * S::NF);
  static constexpr int oM = ALIAS ? oX + r4(S::F * S::NF) : oUf + r4(S::F * S::NF);
  static constexpr int oG = ALIAS ? oUf + r4(S::F * S::NF) : oM + r4(R3N);
  static constexpr int oFl = ALIAS ? oX : oG + r4(S::F * DIM * S::NU);
  static constexpr int oS = ALIAS ? oG + r4(S::F * DIM * S::NU) : oFl + r4(S::F * DIM * S::NU);
  static constexpr int oN = ALIAS ? 0 : oM;
  static_assert(!ALIAS || (S::F * DIM * S::NU <= oUf - oX && DIM * S::NF <= oX), "aliased regions too small");
  __host__ __device__ static constexpr int size(int les) { return oS + (les ? r4((S::F - 1) * DIM * S::NU) : 0); }
};

template <int DIM, int P, int EPB, typename TC, int LES, bool ALIAS>
__host__ __device__ constexpr size_t grad_smem_bytes()
{
  return blockops_bytes<TC, Shape<DIM, P>::NF>() + grad_side_bytes<EPB, Shape<DIM, P>::NF>() +
         sizeof(TC) * EPB * GradPlan<DIM, P, ALIAS>::size(LES);
}

// Whether an instantiation of fr_grad_kernel uses the aliased shared-memory
// plan: the FP64 hex P = 3 layout, no LES, not persistent, one solution
// point per thread (the in-phase barrier needs every thread's reads done).
template <int DIM, int P, int EPB, int NT, typename TC, int LES, int PERS>
__host__ __device__ constexpr bool grad_alias()
{
  return swz_on<DIM, P, TC>() && LES == 0 && PERS == 0 && Items<NT, EPB * Shape<DIM, P>::NU>::N == 1;
}

// Viscous stage, part 1 (per element):
//   LDG common solution at every own flux point (the delta_disu_fpts of
//   int_inters::calculate_common_invFlux, src/int_inters.cpp:331-350)
//   -> corrected reference gradient (calculate_gradient + correct_gradient,
//   src/eles.cpp:1667-1968) -> physical gradient
//   -> total discontinuous flux at the solution points (evaluate_invFlux +
//   evaluate_viscFlux) -> its divergence DV (calculate_divergence) and its
//   normal component at the flux points ND (extrapolate_totalFlux)
//   -> viscous flux at the own flux points from the extrapolated state and
//   gradient (what calculate_common_viscFlux evaluates for this side), kept
//   only as its projection on the interface's left normal: VF (F-1 values,
//   the mass component is zero).
// With LES = 1 the eddy-viscosity SGS flux joins the viscous flux at the
// solution points (evaluate_viscFlux, src/eles.cpp:2369-2380); its transformed
// components (sgsf_upts, src/eles.cpp:2382-2409) are extrapolated to the flux
// points (evaluate_sgsFlux, src/eles.cpp:3294-3368) and added there to the
// physical viscous flux before the projection, as calculate_common_viscFlux
// adds sgsf_fpts (src/int_inters.cpp:415-427).
// Inputs reach shared memory through cp.async, so no register holds a
// prefetched value across the phases; the left normals are fetched while the
// divergence is computed.  MINB is the CTAs per SM the registers are sized
// for; VEC = 0 keeps every global read element-sized (inputs only 8-byte
// aligned), VEC = 1 uses 16-byte copies where the per-element runs allow;
// PERS = 1 makes the blocks persistent (see the input staging below).
// Hexahedra of P = 3 in FP64 keep their per-point arrays in the order of swz
// (bank-conflict-free line reads), run the flux-point phase one line of
// solution points per task (both end flux points from one read), and, with
// one point per thread, use the aliased shared-memory plan of GradPlan.
// Outputs VF (n_fpts, n_eles, F-1), ND (n_fpts, n_eles, F), DV (n_upts, n_eles, F),
// BV (n_boundary_points, F) the viscous normal flux at boundary points (side
// bits 2.. hold the boundary type, mate = -1 - position in the boundary
// list; with BV null the mesh has no boundary points and those bits are
// ignored), and, when GRAD is not null, the corrected physical gradient
// grad_disu_upts (n_upts, n_eles, F, D).
// The body serves element block blk0 (and, with PERS, blk0 + k bstride);
// fr_grad_kernel runs it for blockIdx.x, merged batch launches for their
// share of the grid.
template <int DIM, int P, int EPB, int NT, typename TC, int LES = 0, int VEC = 1, int PERS = 0>
__device__ __forceinline__ void
fr_grad_body(long long blk0, long long bstride, const double* __restrict__ U, const TC* __restrict__ UF,
             const int* __restrict__ mate, const unsigned char* __restrict__ side, const TC* __restrict__ JG,
             const TC* __restrict__ detj, const TC* __restrict__ nL, TC* __restrict__ VF, TC* __restrict__ ND,
             TC* __restrict__ DV, long long E, const Line<TC>& L, const PhysT<TC>& ph, TC* __restrict__ GRAD,
             TC* __restrict__ BV)
{
  using S = Shape<DIM, P>;
  constexpr bool ALIAS = grad_alias<DIM, P, EPB, NT, TC, LES, PERS>();
  using G = GradPlan<DIM, P, ALIAS>;
  constexpr int NU = S::NU, NF = S::NF, F = S::F, D = DIM, DD = DIM * DIM;
  constexpr int IF = Items<NT, EPB * NF>::N, IU = Items<NT, EPB * NU>::N;
  constexpr int PE = G::size(LES);      // shared TC words per element
  extern __shared__ __align__(16) unsigned char fr_smem[];
  auto B = reinterpret_cast<BlockOps<TC, NF>*>(fr_smem);
  unsigned char* sSide = fr_smem + blockops_bytes<TC, NF>();
  TC* sm = reinterpret_cast<TC*>(fr_smem + blockops_bytes<TC, NF>() + grad_side_bytes<EPB, NF>());
#define FR_SU(el, k, u) sm[(el) * PE + (k) * NU + (u)]
#define FR_SX(el, k, f) sm[(el) * PE + G::oX + (k) * NF + (f)]
#define FR_SUF(el, k, f) sm[(el) * PE + G::oUf + (k) * NF + (f)]
#define FR_SM(el, i) sm[(el) * PE + G::oM + (i)]
#define FR_SG(el, c, u) sm[(el) * PE + G::oG + (c) * NU + (u)]
#define FR_SFL(el, l, k, u) sm[(el) * PE + G::oFl + ((l) * F + (k)) * NU + (u)]
#define FR_SS(el, c, u) sm[(el) * PE + G::oS + (c) * NU + (u)]
#define FR_SN(el, i) sm[(el) * PE + G::oN + (i)]
  fill_blockops<DIM, P, TC, NF>(B, L, threadIdx.x, NT);
  const long long NFE = (long long)NF * E;
  const long long nblk = (E + EPB - 1) / EPB;

  // --- inputs to shared memory: state, metrics, neighbour traces.  16-byte
  // copies where the per-element runs are whole 16-byte units (global bases
  // 16-byte aligned), element-sized otherwise.  With PERS = 1 a block walks
  // over element blocks blk0, + bstride, ...; the next block's state,
  // metrics and neighbour traces are fetched into their regions as soon as
  // the current block no longer reads them (after the solution-point phase),
  // so the copies overlap the divergence and flux-point phases, and the left
  // normals are read from global memory at the flux points.
  constexpr bool SWZ = swz_on<DIM, P, TC>();
  constexpr int VU = (VEC && !SWZ && sizeof(TC) == 8 && NU % 2 == 0) ? 2 : 1;
  constexpr int VJ = (VEC && (DD * NU * sizeof(TC)) % 16 == 0) ? 16 / sizeof(TC) : 1;
  constexpr int VD = (VEC && (NU * sizeof(TC)) % 16 == 0) ? 16 / sizeof(TC) : 1;
  // state (FP64 form: asynchronous; FP32 form: loaded and rounded here)
  auto stage_state = [&](long long eb, int nv) {
    for (int w = threadIdx.x; w < EPB * F * NU / VU; w += NT) {
      int el = w / (F * NU / VU), r = w * VU - el * F * NU, k = r / NU, u = r - k * NU;
      if (el < nv) {
        const double* src = U + u + (size_t)NU * (eb + el + E * k);
        const int su = swz<DIM, P, TC>(u);
        if constexpr (sizeof(TC) == 8) cp_async<8 * VU>(&FR_SU(el, k, su), src);
        else FR_SU(el, k, su) = (TC)*src;
      } else {
#pragma unroll
        for (int v = 0; v < VU; v++) {
          const int su = swz<DIM, P, TC>(u + v);
          FR_SU(el, k, su) = TC(1);
        }
      }
    }
  };
  auto stage_metrics = [&](long long eb, int nv) {
    for (int w = threadIdx.x; w < nv * DD * NU / VJ; w += NT) {
      int el = (w * VJ) / (DD * NU), r = w * VJ - el * DD * NU;
      cp_async<sizeof(TC) * VJ>(&FR_SM(el, r), JG + (size_t)DD * NU * eb + (size_t)w * VJ);
    }
    for (int w = threadIdx.x; w < nv * NU / VD; w += NT) {
      int el = (w * VD) / NU, u = w * VD - el * NU;
      cp_async<sizeof(TC) * VD>(&FR_SM(el, DD * NU + u), detj + (size_t)NU * eb + (size_t)w * VD);
    }
  };
  // wiring of the thread's flux points: mate index and side byte
  auto load_wiring = [&](long long eb, int nv, int (&mt)[IF], unsigned char (&sd)[IF]) {
#pragma unroll
    for (int it = 0; it < IF; it++) {
      int w = threadIdx.x + it * NT, el = w / NF, f = w - el * NF;
      mt[it] = -1;
      sd[it] = 0;
      if (w < EPB * NF && el < nv) {
        size_t own = f + (size_t)NF * (eb + el);
        mt[it] = mate[own];
        sd[it] = side[own];
      }
    }
  };
  // neighbour traces (boundary points, mate < 0, have none)
  auto stage_traces = [&](const int (&mt)[IF]) {
#pragma unroll
    for (int it = 0; it < IF; it++) {
      int w = threadIdx.x + it * NT, el = w / NF, f = w - el * NF;
      if (mt[it] >= 0) {
#pragma unroll
        for (int k = 0; k < F; k++) cp_async<sizeof(TC)>(&FR_SX(el, k, f), UF + mt[it] + NFE * k);
      }
    }
  };

  long long blk = blk0;
  int nval = (int)(E - blk * EPB < EPB ? E - blk * EPB : EPB);
  unsigned char psd[IF];
  {
    int mt[IF];
    stage_state(blk * EPB, nval);
    stage_metrics(blk * EPB, nval);
    load_wiring(blk * EPB, nval, mt, psd);
    stage_traces(mt);
    cp_async_commit();
  }
  for (;;) {
  const long long e0 = blk * EPB;
  cp_async_wait_all();
  __syncthreads();
#pragma unroll
  for (int it = 0; it < IF; it++) {
    const int w = threadIdx.x + it * NT;
    if (w < EPB * NF) sSide[w] = psd[it];
  }

  // --- LDG common solution u_c = (uL+uR)/2 - beta (uL-uR); delta = u_c - u_own (in place)
#pragma unroll
  for (int it = 0; it < IF; it++) {
    int w = threadIdx.x + it * NT, el = w / NF, f = w - el * NF;
    if (w >= EPB * NF || el >= nval) continue;
    const int cd = B->code[f];
    int sl[P + 1];
    TC Lc[P + 1];
#pragma unroll
    for (int m = 0; m <= P; m++) {
      sl[m] = swz<DIM, P, TC>(code_u0(cd) + m * code_st(cd));
      Lc[m] = code_plus(cd) ? L.Lp[m] : L.Lm[m];
    }
    // the reference's opp_0 row of f in column order, (((0 + t0) + t1) + ...)
    auto trace = [&](int k) {
      TC acc = TC(0);
#pragma unroll
      for (int m = 0; m <= P; m++) acc = acc + FR_SU(el, k, sl[m]) * Lc[m];
      return acc;
    };
    if (BV && (psd[it] >> 2)) {
      BdyPoint<D, TC> q;
#pragma unroll
      for (int k = 0; k < F; k++) q.u[k] = trace(k);
      const size_t own = f + (size_t)NF * (e0 + el);
#pragma unroll
      for (int d = 0; d < D; d++) q.n[d] = nL[own + NFE * d];
      ldg_boundary<D, TC>(ph, psd[it] >> 2, q, &FR_SX(el, 0, f), &FR_SUF(el, 0, f), NF);
      continue;
    }
    TC pen = (psd[it] & 2) ? -ph.pen_fact : ph.pen_fact;
#pragma unroll
    for (int k = 0; k < F; k++) {
      TC uo = trace(k);
      TC un = FR_SX(el, k, f);
      TC ul = (psd[it] & 1) ? uo : un, ur = (psd[it] & 1) ? un : uo;
      TC uc = TC(0.5) * (ul + ur) - pen * (ul - ur);
      FR_SX(el, k, f) = uc - uo;
      FR_SUF(el, k, f) = uo;
    }
  }
  __syncthreads();

  // --- gradient and total flux at the solution points
#pragma unroll
  for (int it = 0; it < IU; it++) {
    int w = threadIdx.x + it * NT, el = w / NU, u = w - el * NU;
    const bool valid = w < EPB * NU && el < nval;
    if (!ALIAS && !valid) continue;
    if (!valid) el = u = 0;                  // reads in bounds, results unused
    int abc[3];
    upt_abc<DIM, P>(u, abc[0], abc[1], abc[2]);
    TC gr[F][D];
#pragma unroll
    for (int d = 0; d < D; d++) {
      const int i = abc[d];
      int fm, fp, am, ap;
      if (DIM == 2) { fm = d == 0 ? 3 : 0; fp = d == 0 ? 1 : 2; }
      else { fm = d == 0 ? 4 : (d == 1 ? 1 : 0); fp = d == 0 ? 2 : (d == 1 ? 3 : 5); }
      int qm = face_fpt<DIM, P>(fm, abc[0], abc[1], abc[2], am);
      int qp = face_fpt<DIM, P>(fp, abc[0], abc[1], abc[2], ap);
      const int st = upt_stride<DIM, P>(d), ub = u - i * st;
      TC Dr[P + 1];
      int sl[P + 1];
#pragma unroll
      for (int m = 0; m <= P; m++) {
        Dr[m] = B->D[i][m];
        sl[m] = swz<DIM, P, TC>(ub + m * st);
      }
      const TC gm = B->gL[am], gpl = B->gR[ap];
#pragma unroll
      for (int k = 0; k < F; k++) {
        // the gradient only feeds the viscous flux: contracted with FMAs
        TC v[P + 1];
        if (!SWZ && d == 0) lds_line<P + 1, TC>(&FR_SU(el, k, ub), v);
        else {
#pragma unroll
          for (int m = 0; m <= P; m++) v[m] = FR_SU(el, k, sl[m]);
        }
        TC acc = v[0] * Dr[0];
#pragma unroll
        for (int m = 1; m <= P; m++) acc = fr_fma(v[m], Dr[m], acc);
        acc = fr_fma(FR_SX(el, k, qm), gm, acc);
        acc = fr_fma(FR_SX(el, k, qp), gpl, acc);
        gr[k][d] = acc;
      }
    }
    const int su = swz<DIM, P, TC>(u);
    TC g[DD];
#pragma unroll
    for (int q = 0; q < DD; q++) g[q] = FR_SM(el, DD * u + q);
    const TC dj = FR_SM(el, DD * NU + u);
    // physical gradient: d/dx_c = sum_r (JGinv(r,c)/detJ) d/dr (src/eles.cpp:1822-1878)
    TC inv = TC(1.0) / dj;
    TC gp[F][D];
#pragma unroll
    for (int c = 0; c < D; c++) {
      TC m0 = g[0 + D * c] * inv, m1 = g[1 + D * c] * inv, m2 = D == 3 ? g[2 + D * c] * inv : TC(0);
#pragma unroll
      for (int k = 0; k < F; k++) {
        TC acc = fr_fma(gr[k][1], m1, gr[k][0] * m0);
        if (D == 3) acc = fr_fma(gr[k][2], m2, acc);
        gp[k][c] = acc;
        if (valid) {
          FR_SG(el, k + F * c, su) = acc;
          if (GRAD) GRAD[u + (size_t)NU * (e0 + el + E * (k + (long long)F * c))] = acc;
        }
      }
    }
    TC q[F];
#pragma unroll
    for (int k = 0; k < F; k++) q[k] = FR_SU(el, k, su);
    if constexpr (ALIAS) {
      // sFl overwrites the neighbour traces and metrics: every thread's reads first
      __syncthreads();
      if (!valid) continue;
    }
    TC fi[F][D], fv[F][D];
    inv_flux<D, TC>(ph, q, fi);
    vis_flux_fast<D, TC>(ph, q, gp, fv);
    if constexpr (LES != 0) {
      TC fs[F][D];
      sgs_flux<D, TC>(ph, q, gp, dj, TC(P + 1), fs);
#pragma unroll
      for (int k = 1; k < F; k++)
#pragma unroll
        for (int l = 0; l < D; l++) {
          TC a = g[l] * fs[k][0];
#pragma unroll
          for (int m = 1; m < D; m++) a = a + g[l + D * m] * fs[k][m];
          FR_SS(el, (k - 1) + (F - 1) * l, su) = a;
          fv[k][l] = fv[k][l] + fs[k][l];
        }
    }
#pragma unroll
    for (int k = 0; k < F; k++)
#pragma unroll
      for (int l = 0; l < D; l++) {
        // inviscid part in the reference's rounding, viscous part added term by term
        TC acc = g[l] * fi[k][0];
#pragma unroll
        for (int m = 1; m < D; m++) acc = acc + g[l + D * m] * fi[k][m];
#pragma unroll
        for (int m = 0; m < D; m++) acc = fr_fma(g[l + D * m], fv[k][m], acc);
        FR_SFL(el, l, k, su) = acc;
      }
  }
  __syncthreads();

  // --- the next block's state, metrics and wiring (PERS), or the left
  // normals into the metric region, fetched while the divergence runs
  const long long nb = blk + bstride;
  const bool more = PERS && nb < nblk;
  const int nvn = more ? (int)(E - nb * EPB < EPB ? E - nb * EPB : EPB) : 0;
  int mtn[IF];
  unsigned char psn[IF];
  if (more) {
    if constexpr (sizeof(TC) == 8) stage_state(nb * EPB, nvn);
    stage_metrics(nb * EPB, nvn);
    load_wiring(nb * EPB, nvn, mtn, psn);
  }
  if (!PERS)
    for (int w = threadIdx.x; w < nval * D * NF; w += NT) {
      int el = w / (D * NF), r = w - el * D * NF, d = r / NF, f = r - d * NF;
      cp_async<sizeof(TC)>(&FR_SN(el, r), nL + f + (size_t)NF * (e0 + el) + NFE * d);
    }
  cp_async_commit();

  // --- divergence of the total discontinuous flux
#pragma unroll
  for (int it = 0; it < IU; it++) {
    int w = threadIdx.x + it * NT, el = w / NU, u = w - el * NU;
    if (w >= EPB * NU || el >= nval) continue;
    int abc[3];
    upt_abc<DIM, P>(u, abc[0], abc[1], abc[2]);
    TC Dm[D][P + 1];
#pragma unroll
    for (int d = 0; d < D; d++)
#pragma unroll
      for (int m = 0; m <= P; m++) Dm[d][m] = B->D[abc[d]][m];
    int sl[D][P + 1];
#pragma unroll
    for (int d = 0; d < D; d++)
#pragma unroll
      for (int m = 0; m <= P; m++) sl[d][m] = swz<DIM, P, TC>(u - abc[d] * upt_stride<DIM, P>(d) + m * upt_stride<DIM, P>(d));
#pragma unroll
    for (int k = 0; k < F; k++) {
      TC acc = TC(0);
#pragma unroll
      for (int d = 0; d < D; d++) {
        const int st = upt_stride<DIM, P>(d), ub = u - abc[d] * st;
        TC v[P + 1];
        if (!SWZ && d == 0) lds_line<P + 1, TC>(&FR_SFL(el, d, k, ub), v);
        else {
#pragma unroll
          for (int m = 0; m <= P; m++) v[m] = FR_SFL(el, d, k, sl[d][m]);
        }
#pragma unroll
        for (int m = 0; m <= P; m++) acc = acc + v[m] * Dm[d][m];
      }
      DV[u + (size_t)NU * (e0 + el + E * k)] = acc;
    }
  }
  if (more) {
    stage_traces(mtn);
    cp_async_commit();
  }
  if (!PERS) cp_async_wait_all();
  __syncthreads();

  if constexpr (SWZ) {
    // --- flux points, one line of solution points per task: the corrected
    // gradient (and SGS flux) and the transformed flux along the line are read
    // once and extrapolated to the flux points at both ends; each end then gets
    // its own viscous flux projected on the left normal (VF, or BV at a
    // boundary point) and its discontinuous normal flux ND.
    constexpr int NLN = NU / (P + 1);               // lines per axis
    constexpr int IL = Items<NT, EPB * D * NLN>::N;
#pragma unroll
    for (int it = 0; it < IL; it++) {
      const int w = threadIdx.x + it * NT, el = w / (D * NLN), r = w - el * (D * NLN), ax = r / NLN, j = r - ax * NLN;
      if (w >= EPB * D * NLN || el >= nval) continue;
      int a = 0, b = 0, c = 0;
      if (DIM == 2) {
        if (ax == 0) b = j; else a = j;
      } else {
        const int j0 = j % (P + 1), j1 = j / (P + 1);
        if (ax == 0) { b = j0; c = j1; } else if (ax == 1) { a = j0; c = j1; } else { a = j0; b = j1; }
      }
      const int st = upt_stride<DIM, P>(ax), ub = a + (P + 1) * (b + (P + 1) * c);
      const int fcm = DIM == 2 ? (ax == 0 ? 3 : 0) : (ax == 0 ? 4 : (ax == 1 ? 1 : 0));
      const int fcp = DIM == 2 ? (ax == 0 ? 1 : 2) : (ax == 0 ? 2 : (ax == 1 ? 3 : 5));
      int al;
      const int fe[2] = {face_fpt<DIM, P>(fcm, a, b, c, al), face_fpt<DIM, P>(fcp, a, b, c, al)};
      int sl[P + 1];
#pragma unroll
      for (int m = 0; m <= P; m++) sl[m] = swz<DIM, P, TC>(ub + m * st);
      // the own corrected gradient at both ends, opp_6 rows in column order with FMAs
      TC ge[2][F][D];
#pragma unroll
      for (int k = 0; k < F; k++)
#pragma unroll
        for (int d = 0; d < D; d++) {
          const TC* s = &FR_SG(el, k + F * d, 0);
          TC v[P + 1];
#pragma unroll
          for (int m = 0; m <= P; m++) v[m] = s[sl[m]];
          TC am = v[0] * L.Lm[0], ap = v[0] * L.Lp[0];
#pragma unroll
          for (int m = 1; m <= P; m++) {
            am = fr_fma(v[m], L.Lm[m], am);
            ap = fr_fma(v[m], L.Lp[m], ap);
          }
          ge[0][k][d] = am;
          ge[1][k][d] = ap;
        }
#pragma unroll
      for (int e = 0; e < 2; e++) {
        const int f = fe[e];
        const size_t own = f + (size_t)NF * (e0 + el);
        TC uf[F], n[D];
#pragma unroll
        for (int k = 0; k < F; k++) uf[k] = FR_SUF(el, k, f);
#pragma unroll
        for (int d = 0; d < D; d++) n[d] = PERS ? nL[own + NFE * d] : FR_SN(el, d * NF + f);
        const int btype = BV ? sSide[el * NF + f] >> 2 : 0;
        if constexpr (LES == 0) {
          // the projection is accumulated as the flux is formed (no full flux held)
          if (btype) {
            BdyPoint<D, TC> q;
#pragma unroll
            for (int k = 0; k < F; k++) {
              q.u[k] = uf[k];
#pragma unroll
              for (int d = 0; d < D; d++) q.g[k][d] = ge[e][k][d];
            }
#pragma unroll
            for (int d = 0; d < D; d++) q.n[d] = n[d];
            vis_boundary<D, TC, false>(ph, btype, q, &BV[(-1 - (long long)mate[own]) * F]);
          } else {
            TC pr[F - 1];
            vis_flux_proj<D, TC>(ph, uf, ge[e], n, pr);
#pragma unroll
            for (int k = 1; k < F; k++) VF[own + NFE * (k - 1)] = pr[k - 1];
          }
        } else {
          TC fv[F][D];
          vis_flux_fast<D, TC>(ph, uf, ge[e], fv);
#pragma unroll
          for (int k = 1; k < F; k++)
#pragma unroll
            for (int d = 0; d < D; d++) {
              const TC* s = &FR_SS(el, (k - 1) + (F - 1) * d, 0);
              const TC* Lc = e ? L.Lp : L.Lm;
              TC acc = s[sl[0]] * Lc[0];
#pragma unroll
              for (int m = 1; m <= P; m++) acc = fr_fma(s[sl[m]], Lc[m], acc);
              fv[k][d] = fv[k][d] + acc;
            }
          if (btype) {
            BdyPoint<D, TC> q;
#pragma unroll
            for (int k = 0; k < F; k++) {
              q.u[k] = uf[k];
#pragma unroll
              for (int d = 0; d < D; d++) { q.g[k][d] = ge[e][k][d]; q.fv[k][d] = fv[k][d]; }
            }
#pragma unroll
            for (int d = 0; d < D; d++) q.n[d] = n[d];
            vis_boundary<D, TC>(ph, btype, q, &BV[(-1 - (long long)mate[own]) * F]);
          } else {
#pragma unroll
            for (int k = 1; k < F; k++) VF[own + NFE * (k - 1)] = project<D, TC>(fv, k, n);
          }
        }
      }
      // the discontinuous normal flux at both ends, opp_1 rows in column order
      const size_t om = fe[0] + (size_t)NF * (e0 + el), op = fe[1] + (size_t)NF * (e0 + el);
#pragma unroll
      for (int k = 0; k < F; k++) {
        const TC* s = &FR_SFL(el, ax, k, 0);
        TC vm = TC(0), vp = TC(0);
#pragma unroll
        for (int m = 0; m <= P; m++) {
          const TC x = s[sl[m]];
          vm = vm + x * L.Lm[m];
          vp = vp + x * L.Lp[m];
        }
        ND[om + NFE * k] = -vm;
        ND[op + NFE * k] = vp;
      }
    }
  } else {
    // --- flux points, one thread per flux point: own viscous flux projected on
    //     the left normal, and the discontinuous normal flux
#pragma unroll
    for (int it = 0; it < IF; it++) {
      int w = threadIdx.x + it * NT, el = w / NF, f = w - el * NF;
      if (w >= EPB * NF || el >= nval) continue;
      size_t own = f + (size_t)NF * (e0 + el);
      TC uf[F], gf[F][D], n[D];
      const int cd = B->code[f];
      const int u0 = code_u0(cd), st = code_st(cd), ax = code_ax(cd);
      const bool plus = code_plus(cd);
      TC Lc[P + 1];
      int sl[P + 1];
#pragma unroll
      for (int m = 0; m <= P; m++) {
        Lc[m] = plus ? L.Lp[m] : L.Lm[m];
        sl[m] = swz<DIM, P, TC>(u0 + m * st);
      }
#pragma unroll
      for (int k = 0; k < F; k++) {
        uf[k] = FR_SUF(el, k, f);
#pragma unroll
        for (int d = 0; d < D; d++) {
          const TC* s = &FR_SG(el, k + F * d, 0);
          TC acc = s[sl[0]] * Lc[0];
#pragma unroll
          for (int m = 1; m <= P; m++) acc = fr_fma(s[sl[m]], Lc[m], acc);
          gf[k][d] = acc;
        }
      }
#pragma unroll
      for (int d = 0; d < D; d++) n[d] = PERS ? nL[own + NFE * d] : FR_SN(el, d * NF + f);
      const int btype = BV ? psd[it] >> 2 : 0;
      if constexpr (LES == 0) {
        // the projection is accumulated as the flux is formed (no full flux held)
        if (btype) {
          BdyPoint<D, TC> q;
#pragma unroll
          for (int k = 0; k < F; k++) {
            q.u[k] = uf[k];
#pragma unroll
            for (int d = 0; d < D; d++) q.g[k][d] = gf[k][d];
          }
#pragma unroll
          for (int d = 0; d < D; d++) q.n[d] = n[d];
          vis_boundary<D, TC, false>(ph, btype, q, &BV[(-1 - (long long)mate[own]) * F]);
        } else {
          TC pr[F - 1];
          vis_flux_proj<D, TC>(ph, uf, gf, n, pr);
#pragma unroll
          for (int k = 1; k < F; k++) VF[own + NFE * (k - 1)] = pr[k - 1];
        }
      } else {
        TC fv[F][D];
        vis_flux_fast<D, TC>(ph, uf, gf, fv);
#pragma unroll
        for (int k = 1; k < F; k++)
#pragma unroll
          for (int d = 0; d < D; d++) {
            const TC* s = &FR_SS(el, (k - 1) + (F - 1) * d, 0);
            TC acc = s[sl[0]] * Lc[0];
#pragma unroll
            for (int m = 1; m <= P; m++) acc = fr_fma(s[sl[m]], Lc[m], acc);
            fv[k][d] = fv[k][d] + acc;
          }
        if (btype) {
          BdyPoint<D, TC> q;
#pragma unroll
          for (int k = 0; k < F; k++) {
            q.u[k] = uf[k];
#pragma unroll
            for (int d = 0; d < D; d++) { q.g[k][d] = gf[k][d]; q.fv[k][d] = fv[k][d]; }
          }
#pragma unroll
          for (int d = 0; d < D; d++) q.n[d] = n[d];
          vis_boundary<D, TC>(ph, btype, q, &BV[(-1 - (long long)mate[own]) * F]);
        } else {
#pragma unroll
          for (int k = 1; k < F; k++) VF[own + NFE * (k - 1)] = project<D, TC>(fv, k, n);
        }
      }
#pragma unroll
      for (int k = 0; k < F; k++) {
        const TC* s = &FR_SFL(el, ax, k, 0);
        TC v = TC(0);
#pragma unroll
        for (int m = 0; m <= P; m++) v = v + s[sl[m]] * Lc[m];
        ND[own + NFE * k] = plus ? v : -v;
      }
    }
  }
  if (!more) break;
  blk = nb;
  nval = nvn;
#pragma unroll
  for (int it = 0; it < IF; it++) psd[it] = psn[it];
  if constexpr (sizeof(TC) != 8) stage_state(blk * EPB, nval);   // the state region is free after the solution-point phase
  }
#undef FR_SU
#undef FR_SX
#undef FR_SUF
#undef FR_SM
#undef FR_SG
#undef FR_SFL
#undef FR_SS
#undef FR_SN
}

template <int DIM, int P, int EPB, int NT, typename TC, int LES = 0, int MINB = 1, int VEC = 1, int PERS = 0>
__global__ void __launch_bounds__(NT, MINB)
fr_grad_kernel(const double* __restrict__ U, const TC* __restrict__ UF, const int* __restrict__ mate,
               const unsigned char* __restrict__ side, const TC* __restrict__ JG, const TC* __restrict__ detj,
               const TC* __restrict__ nL, TC* __restrict__ VF, TC* __restrict__ ND, TC* __restrict__ DV,
               long long E, Line<TC> L, PhysT<TC> ph, TC* __restrict__ GRAD, TC* __restrict__ BV)
{
  fr_grad_body<DIM, P, EPB, NT, TC, LES, VEC, PERS>(blockIdx.x, gridDim.x, U, UF, mate, side, JG, detj, nL, VF, ND,
                                                     DV, E, L, ph, GRAD, BV);
}

// Boundary point j of the interface kernel (flat own index bf[j], type
// bt[j]), out of line so that the interior path keeps few registers.
template <int DIM, int VISC, typename TC, int RIEMANN>
__device__ __noinline__ void face_boundary(PhysT<TC> ph, long long j, const TC* __restrict__ UF,
                                           const TC* __restrict__ nL, const TC* __restrict__ tdA, TC* __restrict__ CF,
                                           long long NFE, const int* __restrict__ bf,
                                           const unsigned char* __restrict__ bt, const TC* __restrict__ BV)
{
  constexpr int F = DIM + 2, D = DIM;
  const long long a = bf[j];
  const int type = bt[j];
  TC ul[F], ug[F], n[D], fn[F];
#pragma unroll
  for (int k = 0; k < F; k++) ul[k] = UF[a + NFE * k];
#pragma unroll
  for (int d = 0; d < D; d++) n[d] = nL[a + NFE * d];
  bc_ghost<D, TC>(ph, type, ul, n, ug);
  TC fl[F][D], fr[F][D];
  inv_flux<D, TC>(ph, ul, fl);
  inv_flux<D, TC>(ph, ug, fr);
  if (type == 16) {
#pragma unroll
    for (int k = 0; k < F; k++) {
      TC s = fl[k][0] * n[0];
#pragma unroll
      for (int l = 1; l < D; l++) s = s + fl[k][l] * n[l];
      fn[k] = s;
    }
  } else if (RIEMANN == 2 && DIM == 2) {
    roe<TC>(ph, ul, ug, n, fn);
  } else {
#pragma unroll
    for (int k = 0; k < F; k++) {
      TC s = fl[k][0] * n[0], q = fr[k][0] * n[0];
#pragma unroll
      for (int l = 1; l < D; l++) { s = s + fl[k][l] * n[l]; q = q + fr[k][l] * n[l]; }
      fn[k] = TC(0.5) * (s + q);
    }
  }
  const TC tl = tdA[a];
#pragma unroll
  for (int k = 0; k < F; k++) {
    TC c = fn[k] * tl;
    if (VISC) c = c + BV[j * F + k] * tl;
    CF[a + NFE * k] = c;
  }
}

// ---------------------------------------------------------------------------
// Common interface fluxes, once per interface flux point (one thread each):
// int_inters::calculate_common_invFlux (Rusanov, src/int_inters.cpp:225-354)
// and, viscous, calculate_common_viscFlux (LDG from the two sides' normal
// projections VF, src/int_inters.cpp:359-470).  Writes norm_tconf_fpts of
// both sides: +f_n tdA_l on the left, -f_n tdA_r on the right.
// face[i] = (left flat index, right flat index) of interface point i;
// fsign[i] != 0 when the LDG penalty sign is negative there.  RIEMANN is the
// reference's riemann_solve_type: 0 Rusanov, 2 Roe (2-D).
// Threads past nint take the boundary points: ghost state, inviscid common
// flux of bdy_inters::evaluate_boundaryConditions_invFlux (central flux of the
// two states, convective_flux_boundary, src/inters.cpp:368-387; Roe in 2-D
// with RIEMANN 2; the own flux for slip_wall_dual, right_flux,
// src/inters.cpp:299-308), plus the viscous part BV from the gradient kernel.
// Blocks of exactly 128 threads (one shared staging column per thread); the
// body serves block blk (fr_face_kernel: blockIdx.x; merged batch launches:
// their share of the grid).
template <int DIM, int VISC, typename TC, int RIEMANN = 0>
__device__ __forceinline__ void
fr_face_body(long long blk, const int2* __restrict__ face, const unsigned char* __restrict__ fsign, long long nint,
             const TC* __restrict__ UF, const TC* __restrict__ VF, const TC* __restrict__ nL,
             const TC* __restrict__ tdA, TC* __restrict__ CF, long long NFE, const PhysT<TC>& ph, long long nbdy,
             const int* __restrict__ bf, const unsigned char* __restrict__ bt, const TC* __restrict__ BV)
{
  constexpr int F = DIM + 2, D = DIM;
  long long i = blk * 128 + threadIdx.x;
  if (i >= nint) {
    if (i - nint < nbdy) face_boundary<DIM, VISC, TC, RIEMANN>(ph, i - nint, UF, nL, tdA, CF, NFE, bf, bt, BV);
    return;
  }
  // FP64: the point's inputs reach shared memory through cp.async (one
  // column per thread, field-major: no bank conflicts, no barrier), so they
  // are all in flight at once without holding registers; FP32 reads them
  // directly
  constexpr bool STAGE = sizeof(TC) == 8;
  constexpr int NV = 2 * F + D + 2 + (VISC ? 2 * (F - 1) : 0);
  __shared__ TC sv[STAGE ? NV : 1][STAGE ? 128 : 1];
  const int t = threadIdx.x;
  const int2 lr = face[i];
  const long long a = lr.x, b = lr.y;
  auto in = [&](int j, const TC* src) -> TC { return STAGE ? sv[j][t] : *src; };
  if constexpr (STAGE) {
    int j = 0;
#pragma unroll
    for (int k = 0; k < F; k++) cp_async<sizeof(TC)>(&sv[j++][t], UF + a + NFE * k);
#pragma unroll
    for (int k = 0; k < F; k++) cp_async<sizeof(TC)>(&sv[j++][t], UF + b + NFE * k);
#pragma unroll
    for (int d = 0; d < D; d++) cp_async<sizeof(TC)>(&sv[j++][t], nL + a + NFE * d);
    cp_async<sizeof(TC)>(&sv[j++][t], tdA + a);
    cp_async<sizeof(TC)>(&sv[j++][t], tdA + b);
    if (VISC) {
#pragma unroll
      for (int k = 1; k < F; k++) cp_async<sizeof(TC)>(&sv[j++][t], VF + a + NFE * (k - 1));
#pragma unroll
      for (int k = 1; k < F; k++) cp_async<sizeof(TC)>(&sv[j++][t], VF + b + NFE * (k - 1));
    }
    cp_async_commit();
    cp_async_wait_all();
  }
  TC ul[F], ur[F], n[D];
#pragma unroll
  for (int k = 0; k < F; k++) { ul[k] = in(k, UF + a + NFE * k); ur[k] = in(F + k, UF + b + NFE * k); }
#pragma unroll
  for (int d = 0; d < D; d++) n[d] = in(2 * F + d, nL + a + NFE * d);
  const TC tl = in(2 * F + D, tdA + a), tr = in(2 * F + D + 1, tdA + b);
  TC fn[F];
  if constexpr (RIEMANN == 2 && DIM == 2) roe<TC>(ph, ul, ur, n, fn);
  else rusanov<D, TC>(ph, ul, ur, n, fn);
  TC cl[F], cr[F];
#pragma unroll
  for (int k = 0; k < F; k++) { cl[k] = fn[k] * tl; cr[k] = -fn[k] * tr; }
  if (VISC) {
    TC nn = n[0] * n[0];
#pragma unroll
    for (int d = 1; d < D; d++) nn = fr_fma(n[d], n[d], nn);
    const TC pen = fsign[i] ? -ph.pen_fact : ph.pen_fact;
#pragma unroll
    for (int k = 0; k < F; k++) {
      TC al = k ? in(2 * F + D + 2 + (k - 1), VF + a + NFE * (k - 1)) : TC(0);
      TC ar = k ? in(2 * F + D + 2 + (F - 1) + (k - 1), VF + b + NFE * (k - 1)) : TC(0);
      TC fv = ldg_normal<TC>(al, ar, ul[k], ur[k], pen, ph.tau, nn);
      cl[k] = cl[k] + fv * tl;
      cr[k] = cr[k] + (-fv) * tr;
    }
  }
#pragma unroll
  for (int k = 0; k < F; k++) { CF[a + NFE * k] = cl[k]; CF[b + NFE * k] = cr[k]; }
}

template <int DIM, int VISC, typename TC, int RIEMANN = 0>
__global__ void __launch_bounds__(128)
fr_face_kernel(const int2* __restrict__ face, const unsigned char* __restrict__ fsign, long long nint,
               const TC* __restrict__ UF, const TC* __restrict__ VF, const TC* __restrict__ nL,
               const TC* __restrict__ tdA, TC* __restrict__ CF, long long NFE, PhysT<TC> ph,
               long long nbdy = 0, const int* __restrict__ bf = nullptr, const unsigned char* __restrict__ bt = nullptr,
               const TC* __restrict__ BV = nullptr)
{
  fr_face_body<DIM, VISC, TC, RIEMANN>(blockIdx.x, face, fsign, nint, UF, VF, nL, tdA, CF, NFE, ph, nbdy, bf, bt, BV);
}

// ---------------------------------------------------------------------------
// Stage, last part (per element): norm_tconf - norm_tdisf, the VCJH
// correction (calculate_corrected_divergence, src/eles.cpp:1594-1661), and
// either the residual (MODE 0) or the RK45 stage update
// (eles::AdvanceSolution, src/eles.cpp:1155-1178) followed by the next
// stage's traces (MODE 1).  The inviscid path (VISC 0) evaluates the flux,
// its divergence and its normal component here itself, in the reference's
// order; the viscous path takes DV and ND from fr_grad_kernel.
// Shared-memory plan of fr_update_kernel (byte offsets, every region
// rounded up to 16 bytes): state and RK register (FP64), detJ (FP64), common
// normal flux CF (overwritten in place by norm_tconf - norm_tdisf), ND and DV
// (viscous path), transformed flux and JGinv (inviscid path), norm partials.
template <int DIM, int P, int EPB, int NT, int VISC, int MODE, typename TC>
struct UpdPlan {
  using S = Shape<DIM, P>;
  __host__ __device__ static constexpr size_t r16(size_t b) { return (b + 15) / 16 * 16; }
  static constexpr size_t bU = r16(sizeof(double) * EPB * S::F * S::NU);
  static constexpr size_t bREG = MODE == 1 ? bU : 0;
  static constexpr size_t bDJ = MODE == 1 ? r16(sizeof(double) * EPB * S::NU) : 0;
  static constexpr size_t bCF = r16(sizeof(TC) * EPB * S::F * S::NF);
  static constexpr size_t bND = VISC ? bCF : 0;
  static constexpr size_t bDV = VISC ? r16(sizeof(TC) * EPB * S::F * S::NU) : 0;
  static constexpr size_t bFL = VISC ? 0 : r16(sizeof(TC) * EPB * DIM * S::F * S::NU);
  static constexpr size_t bJ = VISC ? 0 : r16(sizeof(TC) * EPB * DIM * DIM * S::NU);
  static constexpr size_t bRED = r16(sizeof(double) * (NT / 32) * S::F);
  static constexpr size_t oU = 0, oREG = oU + bU, oDJ = oREG + bREG, oCF = oDJ + bDJ, oND = oCF + bCF,
                          oDV = oND + bND, oFL = oDV + bDV, oJ = oFL + bFL, oRED = oJ + bJ, total = oRED + bRED;
};

template <int DIM, int P, int EPB, int NT, int VISC, int MODE, typename TC>
__host__ __device__ constexpr size_t update_smem_bytes()
{
  return blockops_bytes<TC, Shape<DIM, P>::NF>() + UpdPlan<DIM, P, EPB, NT, VISC, MODE, TC>::total;
}

// Stage, last part (per element): norm_tconf - norm_tdisf, the VCJH
// correction (calculate_corrected_divergence, src/eles.cpp:1594-1661), and
// either the residual (MODE 0) or the RK45 stage update
// (eles::AdvanceSolution, src/eles.cpp:1155-1178) followed by the next
// stage's traces (MODE 1).  The inviscid path (VISC 0) evaluates the flux,
// its divergence and its normal component here itself, in the reference's
// order; the viscous path takes DV and ND from fr_grad_kernel.  Every
// per-element input reaches shared memory through cp.async (16-byte copies
// where the element runs allow, VEC = 1; element-sized with VEC = 0 for
// inputs only 8-byte aligned), so all of a block's loads are in flight
// together.
// The body serves element block blk (fr_update_kernel: blockIdx.x; merged
// batch launches: their share of the grid).
template <int DIM, int P, int EPB, int NT, int VISC, int MODE, typename TC, int VEC = 1>
__device__ __forceinline__ void
fr_update_body(long long blk, double* __restrict__ U, double* __restrict__ REG, TC* __restrict__ UFn,
               const TC* __restrict__ CF, const TC* __restrict__ ND, const TC* __restrict__ DV,
               const TC* __restrict__ JG, const double* __restrict__ detj, double* __restrict__ DIV,
               double* __restrict__ partial, long long E, const Line<TC>& L, const PhysT<TC>& ph, double rk_a,
               double rk_b, double dt, int first_stage)
{
  using S = Shape<DIM, P>;
  using Q = UpdPlan<DIM, P, EPB, NT, VISC, MODE, TC>;
  constexpr int NU = S::NU, NF = S::NF, F = S::F, D = DIM, DD = DIM * DIM;
  extern __shared__ __align__(16) unsigned char fr_smem[];
  auto B = reinterpret_cast<BlockOps<TC, NF>*>(fr_smem);
  unsigned char* sm0 = fr_smem + blockops_bytes<TC, NF>();
  auto sU = reinterpret_cast<double (*)[F][NU]>(sm0 + Q::oU);
  auto sREG = reinterpret_cast<double (*)[F][NU]>(sm0 + Q::oREG);
  auto sDJ = reinterpret_cast<double (*)[NU]>(sm0 + Q::oDJ);
  auto sC = reinterpret_cast<TC (*)[F][NF]>(sm0 + Q::oCF);
  auto sND = reinterpret_cast<TC (*)[F][NF]>(sm0 + Q::oND);
  auto sDV = reinterpret_cast<TC (*)[F][NU]>(sm0 + Q::oDV);
  auto sFl = reinterpret_cast<TC (*)[D][F][NU]>(sm0 + Q::oFL);
  auto sJ = reinterpret_cast<TC (*)[DD * NU]>(sm0 + Q::oJ);
  auto sRed = reinterpret_cast<double (*)[F]>(sm0 + Q::oRED);
  fill_blockops<DIM, P, TC, NF>(B, L, threadIdx.x, NT);
  const long long e0 = blk * EPB;
  const int nval = (int)(E - e0 < EPB ? E - e0 : EPB);

  // --- inputs to shared memory
  constexpr int V8 = (VEC && NU % 2 == 0) ? 2 : 1;                                   // doubles per copy
  constexpr int VF = (VEC && (NF * sizeof(TC)) % 16 == 0) ? 16 / sizeof(TC) : 1;     // flux-point runs
  constexpr int VN = (VEC && (NU * sizeof(TC)) % 16 == 0) ? 16 / sizeof(TC) : 1;     // point runs
  constexpr int VJ = (VEC && (DD * NU * sizeof(TC)) % 16 == 0) ? 16 / sizeof(TC) : 1;
  // the state is kept in the bank-conflict-free point order of swz (read
  // along lines for the next stage's traces), so its copies are element-sized
  // where that order is not the natural one
  constexpr bool SWU = swz_on<DIM, P, double>();
  constexpr int V8U = SWU ? 1 : V8;
  const bool want_reg = MODE == 1 && !first_stage;
  for (int w = threadIdx.x; w < nval * F * NU / V8U; w += NT) {
    int el = w / (F * NU / V8U), r = w * V8U - el * F * NU, k = r / NU, u = r - k * NU;
    cp_async<8 * V8U>(&sU[el][k][swz<DIM, P, double>(u)], U + u + (size_t)NU * (e0 + el + E * k));
  }
  if (want_reg)
    for (int w = threadIdx.x; w < nval * F * NU / V8; w += NT) {
      int el = w / (F * NU / V8), r = w * V8 - el * F * NU, k = r / NU, u = r - k * NU;
      cp_async<8 * V8>(&sREG[el][k][u], REG + u + (size_t)NU * (e0 + el + E * k));
    }
  if (MODE == 1)
    for (int w = threadIdx.x; w < nval * NU / V8; w += NT) {
      int el = (w * V8) / NU, u = w * V8 - el * NU;
      cp_async<8 * V8>(&sDJ[el][u], detj + (size_t)NU * e0 + (size_t)w * V8);
    }
  for (int w = threadIdx.x; w < nval * F * NF / VF; w += NT) {
    int el = w / (F * NF / VF), r = w * VF - el * F * NF, k = r / NF, f = r - k * NF;
    size_t g = f + (size_t)NF * (e0 + el + E * k);
    cp_async<sizeof(TC) * VF>(&sC[el][k][f], CF + g);
    if (VISC) cp_async<sizeof(TC) * VF>(&sND[el][k][f], ND + g);
  }
  if (VISC)
    for (int w = threadIdx.x; w < nval * F * NU / VN; w += NT) {
      int el = w / (F * NU / VN), r = w * VN - el * F * NU, k = r / NU, u = r - k * NU;
      cp_async<sizeof(TC) * VN>(&sDV[el][k][u], DV + u + (size_t)NU * (e0 + el + E * k));
    }
  else
    for (int w = threadIdx.x; w < nval * DD * NU / VJ; w += NT) {
      int el = (w * VJ) / (DD * NU), r = w * VJ - el * DD * NU;
      cp_async<sizeof(TC) * VJ>(&sJ[el][r], JG + (size_t)DD * NU * e0 + (size_t)w * VJ);
    }
  cp_async_commit();
  cp_async_wait_all();
  __syncthreads();

  if (VISC) {
    for (int w = threadIdx.x; w < nval * F * NF; w += NT) {
      int el = w / (F * NF), r = w - el * F * NF, k = r / NF, f = r - k * NF;
      sC[el][k][f] = sC[el][k][f] - sND[el][k][f];      // daxpy(-1, norm_tdisf, norm_tconf)
    }
  } else {
    // transformed inviscid flux at the solution points (evaluate_invFlux, src/eles.cpp:1331-1418)
    for (int w = threadIdx.x; w < nval * NU; w += NT) {
      int el = w / NU, u = w - el * NU;
      TC g[DD];
#pragma unroll
      for (int q = 0; q < DD; q++) g[q] = sJ[el][DD * u + q];
      TC q[F], fi[F][D];
#pragma unroll
      for (int k = 0; k < F; k++) q[k] = (TC)sU[el][k][swz<DIM, P, double>(u)];
      inv_flux<D, TC>(ph, q, fi);
#pragma unroll
      for (int l = 0; l < D; l++)
#pragma unroll
        for (int k = 0; k < F; k++) {
          TC acc = g[l] * fi[k][0];
#pragma unroll
          for (int m = 1; m < D; m++) acc = acc + g[l + D * m] * fi[k][m];
          sFl[el][l][k][u] = acc;
        }
    }
    __syncthreads();
    // norm_tconf - norm_tdisf with the normal component extrapolated here (extrapolate_totalFlux)
    for (int w = threadIdx.x; w < nval * NF; w += NT) {
      int el = w / NF, f = w - el * NF;
      const int cd = B->code[f];
      const bool plus = code_plus(cd);
#pragma unroll
      for (int k = 0; k < F; k++) {
        TC v = interp_code<P, TC, TC>(L, cd, &sFl[el][code_ax(cd)][k][0]);
        sC[el][k][f] = sC[el][k][f] - (plus ? v : -v);
      }
    }
  }
  __syncthreads();

  double red[F];
#pragma unroll
  for (int k = 0; k < F; k++) red[k] = 0.0;
  constexpr int IU = Items<NT, EPB * NU>::N;
#pragma unroll
  for (int it = 0; it < IU; it++) {
    int w = threadIdx.x + it * NT, el = w / NU, u = w - el * NU;
    if (w >= EPB * NU || el >= nval) continue;
    const long long e = e0 + el;
    int abc[3];
    upt_abc<DIM, P>(u, abc[0], abc[1], abc[2]);
    // opp_3 row of u: one column per face, in flux-point order (the same for every field)
    int qf[S::NFACE];
    TC cf[S::NFACE];
#pragma unroll
    for (int fc = 0; fc < S::NFACE; fc++) {
      int al;
      qf[fc] = face_fpt<DIM, P>(fc, abc[0], abc[1], abc[2], al);
      cf[fc] = face_plus<DIM>(fc) ? B->gR[al] : -B->gL[al];
    }
    const double dj = MODE == 1 ? sDJ[el][u] : 1.0;
#pragma unroll
    for (int k = 0; k < F; k++) {
      size_t gi = u + (size_t)NU * (e + E * k);
      TC acc;
      if (VISC) {
        acc = sDV[el][k][u];
      } else {
        acc = TC(0);
#pragma unroll
        for (int d = 0; d < D; d++) {
          const int st = upt_stride<DIM, P>(d), ub = u - abc[d] * st;
#pragma unroll
          for (int m = 0; m <= P; m++) acc = acc + sFl[el][d][k][ub + m * st] * B->D[abc[d]][m];
        }
      }
#pragma unroll
      for (int fc = 0; fc < S::NFACE; fc++) acc = acc + sC[el][k][qf[fc]] * cf[fc];
      double R = (double)acc;
      if (MODE == 0) {
        DIV[gi] = R;
      } else {
        double rhs = -R / dj;
        double res = first_stage ? dt * rhs : rk_a * sREG[el][k][u] + dt * rhs;
        REG[gi] = res;
        const int su = swz<DIM, P, double>(u);
        double un = sU[el][k][su] + rk_b * res;
        U[gi] = un;
        sU[el][k][su] = un;
        red[k] += fabs(rhs);
      }
    }
  }
  if (MODE == 1) {
    if (partial) {
      // deterministic per-block partial sums of |div/detjac| (CalcNormResidual)
      const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
      for (int k = 0; k < F; k++) {
        double v = red[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sRed[wid][k] = v;
      }
    }
    __syncthreads();
    if (partial && threadIdx.x < F) {
      double v = 0.0;
      for (int i = 0; i < NT / 32; i++) v += sRed[i][threadIdx.x];
      partial[(size_t)blk * F + threadIdx.x] = v;
    }
    // traces of the updated state for the next stage
    for (int w = threadIdx.x; w < nval * NF; w += NT) {
      int el = w / NF, f = w - el * NF;
      long long e = e0 + el;
      const int cd = B->code[f];
      int sl[P + 1];
      TC Lc[P + 1];
#pragma unroll
      for (int m = 0; m <= P; m++) {
        sl[m] = swz<DIM, P, double>(code_u0(cd) + m * code_st(cd));
        Lc[m] = code_plus(cd) ? L.Lp[m] : L.Lm[m];
      }
      // the opp_0 row of f in column order, (((0 + t0) + t1) + ...)
#pragma unroll
      for (int k = 0; k < F; k++) {
        TC acc = TC(0);
#pragma unroll
        for (int m = 0; m <= P; m++) acc = acc + (TC)sU[el][k][sl[m]] * Lc[m];
        UFn[f + (size_t)NF * (e + E * k)] = acc;
      }
    }
  }
}

template <int DIM, int P, int EPB, int NT, int VISC, int MODE, typename TC, int VEC = 1>
__global__ void __launch_bounds__(NT)
fr_update_kernel(double* __restrict__ U, double* __restrict__ REG, TC* __restrict__ UFn, const TC* __restrict__ CF,
                 const TC* __restrict__ ND, const TC* __restrict__ DV, const TC* __restrict__ JG,
                 const double* __restrict__ detj, double* __restrict__ DIV, double* __restrict__ partial, long long E,
                 Line<TC> L, PhysT<TC> ph, double rk_a, double rk_b, double dt, int first_stage)
{
  fr_update_body<DIM, P, EPB, NT, VISC, MODE, TC, VEC>(blockIdx.x, U, REG, UFn, CF, ND, DV, JG, detj, DIV, partial, E,
                                                       L, ph, rk_a, rk_b, dt, first_stage);
}

// Block partial sums -> norms: one CTA of 256 threads per field; thread t
// sums partials t, t+256, ... in order, then a fixed shared-memory tree.  The
// order depends only on the number of partials, so results are reproducible.
static __global__ void __launch_bounds__(256)
fr_norm_finalize(const double* __restrict__ partial, int nblk, int F, double inv_n, double* __restrict__ out)
{
  __shared__ double s[256];
  const int k = blockIdx.x;
  double acc = 0.0;
  for (int b = threadIdx.x; b < nblk; b += 256) acc += partial[(size_t)b * F + k];
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[k] = s[0] * inv_n;
}

}  // namespace frb
