// fr_mixed_fused.cu -- fused RK stage for meshes of dense-operator element
// types (tetrahedra, prisms, hexahedra, triangles, quadrilaterals through
// their dense operators; the kernels are in fr_mixed_fused.cuh): the
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
// Euler form: kernel A is mixed_inv_kernel (the transformed inviscid flux and
//   norm_tdisf / div_tdisf alone); kernel B drops the viscous terms and takes
//   the Roe flux instead of Rusanov when asked (2-D).
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
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "fr_b200.h"
#include "fr_mixed_fused.cuh"

namespace frb {
extern thread_local std::string g_err;
}
using namespace frb;
using namespace frb_mixed;

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

// (dims, solution points, flux points) with kernels: tets, prisms and hexes of
// orders 2 and 3 here, triangles and quads of orders 2 and 3 in
// fr_mixed_fused_2d.cu, orders 1 and 4 in fr_mixed_fused_p14.cu
bool find_kernels(int D, int NU, int NF, MixedKernels* out)
{
  if (find_kernels_p14(D, NU, NF, out)) return true;
  if (D == 2) return find_kernels_2d(NU, NF, out);
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
  int pf = 0;  // physics form: 0 Navier-Stokes, 1 Euler (Rusanov), 2 Euler (Roe)
  std::vector<double*> partials;  // per type: [blocks of the smallest shape][F]
  double* norms_dev = nullptr;    // [F]
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

// L1 residual norms (CalcNormResidual with res_norm_type 1, src/output.cpp:
// 1452-1520): per type the block sums in block order, then the types in
// order, over the solution points of all types
struct NormParts {
  const double* p[8];
  int nb[8];
};
__global__ void mixed_norm_finalize(NormParts np, int n_types, int F, double n_upts, double* out)
{
  const int k = threadIdx.x;
  if (k >= F) return;
  double sum = 0.0;
  for (int i = 0; i < n_types; i++) {
    double ts = 0.0;
    for (int b = 0; b < np.nb[i]; b++) ts += np.p[i][(size_t)b * F + k];
    sum += ts;
  }
  out[k] = sum / n_upts;
}


fr_status launch_grad(fr_mixed_stage* s, int i, int v, const double* UFc, cudaStream_t st)
{
  const MixedType& t = s->types[i];
  const MixedShape& g = kGradShapes[v];
  s->kern[i].grad[s->pf][v]<<<blocks_of(t.E, g.epb), g.nth, s->kern[i].smem_a[s->pf][v], st>>>(t, s->fp, UFc,
                                                                                                 s->ph);
  return mlaunched("mixed_grad_kernel");
}

fr_status launch_upd(fr_mixed_stage* s, int i, int v, int mode, int stage, double dt, const double* UFc, double* UFn,
                     cudaStream_t st, bool norms = false)
{
  static const double A[5] = {0.0, -0.417890474499852, -1.192151694642677, -1.697784692471528, -1.514183444257156};
  static const double B[5] = {0.149659021999229, 0.379210312999627, 0.822955029386982, 0.699450455949122,
                              0.153057247968152};
  MixedType t = s->types[i];
  t.partial = norms ? s->partials[i] : nullptr;
  const MixedShape& u = kUpdShapes[v];
  auto k = mode ? s->kern[i].upd1[s->pf][v] : s->kern[i].upd0[s->pf][v];
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

// one CalcResidual (+ the RK45 update of stage `stage` when mode is 1; with
// norms, each block's residual sums into the partials)
fr_status launch_stage(fr_mixed_stage* s, int mode, int stage, double dt, cudaStream_t st, bool norms = false)
{
  const double* UFc = s->UF[s->cur];
  double* UFn = s->UF[s->cur ^ 1];
  if (fr_status e = for_types(s, st, [&](int i, cudaStream_t q) { return launch_grad(s, i, s->gv[i], UFc, q); }))
    return e;
  if (fr_status e = for_types(s, st, [&](int i, cudaStream_t q) {
        return launch_upd(s, i, s->uv[i], mode, stage, dt, UFc, UFn, q, norms);
      }))
    return e;
  if (mode) s->cur ^= 1;
  return FR_OK;
}

fr_status set_smem(const MixedKernels& k, int pf)
{
  std::vector<std::pair<const void*, size_t>> list;
  for (int v = 0; v < kNGrad; v++) list.push_back({(const void*)k.grad[pf][v], k.smem_a[pf][v]});
  for (int v = 0; v < kNUpd; v++) {
    list.push_back({(const void*)k.upd0[pf][v], k.smem_b[v]});
    list.push_back({(const void*)k.upd1[pf][v], k.smem_b[v]});
  }
  list.push_back({(const void*)k.trace, k.smem_c});
  bool any_grad = false, any_upd = false;
  for (int v = 0; v < kNGrad; v++) any_grad = any_grad || k.grad[pf][v];
  for (int v = 0; v < kNUpd; v++) any_upd = any_upd || k.upd1[pf][v];
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
                                const fr_phys_desc* phys, int viscous, int riemann_solve_type,
                                fr_mixed_stage** out)
{
  g_err.clear();
  if (!out || !types || !phys || n_types < 1) return mfail(FR_ERR_ARG, "bad arguments");
  *out = nullptr;
  if (n_dims != 2 && n_dims != 3) return mfail(FR_ERR_UNSUPPORTED, "fused mixed stage: 2-D or 3-D meshes");
  if (riemann_solve_type != 0 && riemann_solve_type != 2)
    return mfail(FR_ERR_UNSUPPORTED, "fused mixed stage: riemann_solve_type 0 (Rusanov) or 2 (Roe)");
  if (riemann_solve_type == 2 && (n_dims != 2 || viscous))
    return mfail(FR_ERR_UNSUPPORTED, "fused mixed stage: the Roe flux with 2-D Euler only");
  const int pf = viscous ? 0 : (riemann_solve_type == 2 ? 2 : 1);
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
  s->pf = pf;
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
    if (NU <= 0 || NF <= 0 || ty.n_eles < 0 || !ty.disu_upts || !ty.opp_0 || !ty.opp_3 ||
        (viscous && !ty.opp_6) || !ty.JGinv_upts || !ty.detjac_upts || !ty.tdA_fpts || !ty.norm_fpts)
      return bail(mfail(FR_ERR_ARG, "bad element type description"));
    for (int d = 0; d < D; d++)
      if (!ty.opp_1[d] || !ty.opp_2[d] || (viscous && (!ty.opp_4[d] || !ty.opp_5[d])))
        return bail(mfail(FR_ERR_ARG, "missing operator"));
    MixedKernels k;
    if (!find_kernels(D, NU, NF, &k))
      return bail(mfail(FR_ERR_UNSUPPORTED, "fused mixed stage: no kernels for " + std::to_string(NU) +
                                                " solution / " + std::to_string(NF) + " flux points"));
    s->kern.push_back(k);
    // defaults before any autotune: the shapes that measured fastest for
    // tets (4 elements x 128 threads), else the first that fits
    int g0 = 3, u0 = 1;
    if (!k.grad[pf][g0])
      for (g0 = 0; g0 < kNGrad - 1 && !k.grad[pf][g0];) g0++;
    if (!k.upd1[pf][u0])
      for (u0 = 0; u0 < kNUpd - 1 && !k.upd1[pf][u0];) u0++;
    if (!k.grad[pf][g0] || !k.upd1[pf][u0])
      return bail(mfail(FR_ERR_UNSUPPORTED, "element type too large for one block of shared memory"));
    s->gv.push_back(g0);
    s->uv.push_back(u0);
    off[i + 1] = off[i] + (long long)NF * ty.n_eles;
  }
  s->NT = off[n_types];
  const long long NT = s->NT;

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
  // every check above is on the host: device work starts here
  for (const MixedKernels& k : s->kern)
    if (fr_status e = set_smem(k, s->pf)) return bail(e);
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
    if (viscous) {  // the gradient's operators (opp_4, opp_5, opp_6)
      h = fragments(D * NU, NU, [&](int r, int c) { return ty.opp_4[r / NU][r % NU + (size_t)NU * c]; });
      if (fr_status e = s->upload(h, &t.A45u)) return bail(e);
      h = fragments(D * NU, NF, [&](int r, int c) { return ty.opp_5[r / NU][r % NU + (size_t)NU * c]; });
      if (fr_status e = s->upload(h, &t.A45f)) return bail(e);
      h = fragments(NF, NU, cm(ty.opp_6, NF));
      if (fr_status e = s->upload(h, &t.A6)) return bail(e);
    }
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
  if (n_types > 8) return bail(mfail(FR_ERR_ARG, "at most 8 element types"));
  for (int i = 0; i < n_types; i++) {
    double* p = nullptr;
    if (fr_status e = s->zeros((size_t)F * ((types[i].n_eles + 3) / 4 + 1), &p)) return bail(e);
    s->partials.push_back(p);
  }
  if (fr_status e = s->zeros((size_t)F, &s->norms_dev)) return bail(e);
  s->fork_ev.resize(1, nullptr);
  if (cudaEventCreateWithFlags(&s->fork_ev[0], cudaEventDisableTiming) != cudaSuccess)
    return bail(mfail(FR_ERR_CUDA, "event creation failed"));
  for (int i = 1; i < n_types; i++) {
    cudaStream_t q;
    cudaEvent_t ev;
    // the side streams get the highest priority, so the small types' blocks
    // take the SM slots that free up before the first type's remaining ones
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    if (cudaStreamCreateWithPriority(&q, cudaStreamNonBlocking, hi) != cudaSuccess)
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
  if (!s->kern[type].grad[s->pf][grad_shape] || !s->kern[type].upd1[s->pf][update_shape])
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
        if (pass == 0 ? !s->kern[i].grad[s->pf][v] : !s->kern[i].upd0[s->pf][v]) continue;
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

fr_status fr_mixed_stage_advance_norms(fr_mixed_stage* s, int n_steps, double dt, double* res_norms, void* stream)
{
  g_err.clear();
  if (!s || n_steps < 1 || !res_norms) return mfail(FR_ERR_ARG, "bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  if (fr_status e = launch_trace(s, st)) return e;
  for (int n = 0; n < n_steps; n++)
    for (int k = 0; k < 5; k++)
      if (fr_status e = launch_stage(s, 1, k, dt, st, n == n_steps - 1 && k == 4)) return e;
  NormParts np{};
  double n_upts = 0.0;
  for (int i = 0; i < s->n_types; i++) {
    np.p[i] = s->partials[i];
    np.nb[i] = s->types[i].E > 0 ? (int)blocks_of(s->types[i].E, kUpdShapes[s->uv[i]].epb) : 0;
    n_upts += (double)s->types[i].NU * (double)s->types[i].E;
  }
  mixed_norm_finalize<<<1, 32, 0, st>>>(np, s->n_types, s->F, n_upts, s->norms_dev);
  if (fr_status e = mlaunched("mixed_norm_finalize")) return e;
  if (cudaMemcpyAsync(res_norms, s->norms_dev, sizeof(double) * s->F, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return mfail(FR_ERR_CUDA, "norm read-back failed");
  for (int k = 0; k < s->F; k++)
    if (!std::isfinite(res_norms[k])) return mfail(FR_ERR_NONFINITE, "NaN residual encountered");
  return FR_OK;
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
