// fr_noalloc.cu -- a residual entry point that allocates no device memory.
//
// Who needs it: code that cannot call cudaMalloc at the point where it wants a
// residual -- e.g. a caller in the middle of recording work it will replay,
// a caller whose device memory is handed out by someone else's pool and may
// not grow, or an embedding host that forbids allocation after start-up.
// Such callers still own every input and output array; the scratch this
// residual needs between its kernels (flux-point traces, viscous-flux
// projections, the discontinuous normal flux, its divergence and the common
// interface flux) lives in one fixed array of device memory defined in this
// file.  Every GPU that loads the library keeps that array until the process
// exits.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <mutex>
#include <string>

#include "fr_b200.h"
#include "fr_fused.cuh"
#include "fr_host.hpp"

namespace frb {
extern thread_local std::string g_err;
}
using namespace frb;

namespace {

// 32 MiB of scratch (4 Mi doubles), shared by every call on a device.
constexpr size_t kScratchDoubles = size_t(4) << 20;
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double* g_scratch_ptr[kMaxDevices] = {};

fr_status na_fail(fr_status s, const char* m)
{
  g_err = m;
  return s;
}

// Set-up, once per device, with that device current: the device address of
// the scratch array (its name in host code is only a stand-in).  The address
// is kept for the life of the process, so the entry point must not be used
// after a cudaDeviceReset of that device (the module, and the array with it,
// is reloaded elsewhere).
fr_status scratch_for_device(int dev, double** out)
{
  if (dev < 0 || dev >= kMaxDevices) return na_fail(FR_ERR_ARG, "device index out of range");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      g_err = std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e);
      return FR_ERR_CUDA;
    }
    g_scratch_ptr[dev] = (double*)p;
  }
  *out = g_scratch_ptr[dev];
  return FR_OK;
}

// Default tiles (elements per CTA, threads per CTA) of the element kernels.
template <int DIM, int P> struct NaTile;
template <> struct NaTile<2, 1> { static constexpr int EPB = 32, NT = 128; };
template <> struct NaTile<2, 2> { static constexpr int EPB = 16, NT = 128; };
template <> struct NaTile<2, 3> { static constexpr int EPB = 8, NT = 128; };
template <> struct NaTile<2, 4> { static constexpr int EPB = 8, NT = 256; };
template <> struct NaTile<2, 5> { static constexpr int EPB = 4, NT = 160; };
template <> struct NaTile<3, 1> { static constexpr int EPB = 12, NT = 128; };
template <> struct NaTile<3, 2> { static constexpr int EPB = 4, NT = 128; };
template <> struct NaTile<3, 3> { static constexpr int EPB = 2, NT = 128; };
template <> struct NaTile<3, 4> { static constexpr int EPB = 1, NT = 128; };

bool make_line_noalloc(int P, int upts_type, int scheme, double eta_in, Line<double>& L)
{
  double loc[kMaxP + 1];
  if (!points_1d(P, upts_type, loc)) return false;
  double eta = vcjh_eta(scheme, P, eta_in);
  if (std::isnan(eta)) return false;
  int n = P + 1;
  for (int i = 0; i < kMaxN1; i++) {
    L.Lm[i] = L.Lp[i] = L.gL[i] = L.gR[i] = L.w[i] = 0.0;
    for (int j = 0; j < kMaxN1; j++) L.D[i][j] = 0.0;
  }
  for (int m = 0; m < n; m++) { L.Lm[m] = lagrange(-1.0, m, loc, n); L.Lp[m] = lagrange(1.0, m, loc, n); }
  for (int k = 0; k < n; k++) {
    for (int m = 0; m < n; m++) L.D[k][m] = dlagrange(loc[k], m, loc, n);
    L.gL[k] = dvcjh(loc[k], 0, P, eta);
    L.gR[k] = dvcjh(loc[k], 1, P, eta);
  }
  return true;
}

template <int DIM, int P>
fr_status run(const fr_residual_args* a, double* scratch, cudaStream_t s)
{
  using S = Shape<DIM, P>;
  constexpr int EPB = NaTile<DIM, P>::EPB, NT = NaTile<DIM, P>::NT;
  const long long E = a->n_eles, NFE = (long long)S::NF * E;
  const int F = S::F;
  const bool visc = a->viscous != 0;
  // UF and CF always; the divergence DV, viscous projections VF and normal
  // flux ND only on the viscous path (the Euler path forms them in the update)
  size_t need = (size_t)NFE * F * 2;
  if (visc) need += (size_t)S::NU * E * F + (size_t)NFE * (F - 1) + (size_t)NFE * F;
  if (need > kScratchDoubles) return na_fail(FR_ERR_ARG, "mesh too large for the fixed 32 MiB residual scratch");
  double* UF = scratch;
  double* CF = UF + NFE * F;
  double* DV = visc ? CF + NFE * F : nullptr;
  double* VF = visc ? DV + (size_t)S::NU * E * F : nullptr;
  double* ND = visc ? VF + NFE * (F - 1) : nullptr;
  Line<double> L;
  if (!make_line_noalloc(P, a->upts_type, a->vcjh_scheme, a->eta, L))
    return na_fail(FR_ERR_ARG, "unsupported point type or VCJH scheme for this order");
  Phys q{a->phys.gamma, a->phys.prandtl, a->phys.mu_inf, a->phys.rt_inf, a->phys.c_sth, a->phys.fix_vis,
         a->phys.tau, a->phys.pen_fact};
  PhysT<double> ph = PhysT<double>::make(q);
  // every flux point is written by the interface kernel when the interface list
  // covers the mesh; clearing keeps a partial list from reading an earlier call
  cudaError_t e = cudaMemsetAsync(CF, 0, sizeof(double) * NFE * F, s);
  if (e != cudaSuccess) return na_fail(FR_ERR_CUDA, cudaGetErrorString(e));
  fr_trace_kernel<DIM, P, double><<<(unsigned)((NFE + 255) / 256), 256, 0, s>>>(a->disu_upts, UF, E, L);
  const unsigned nblk = (unsigned)((E + EPB - 1) / EPB);
  if (visc) {
    constexpr size_t sm = grad_smem_bytes<DIM, P, EPB, double>();
    if (sm > 48 * 1024)
      cudaFuncSetAttribute(fr_grad_kernel<DIM, P, EPB, NT, double, 0, 1, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)sm);
    fr_grad_kernel<DIM, P, EPB, NT, double, 0, 1, 0><<<nblk, NT, sm, s>>>(a->disu_upts, UF, a->mate, a->side, a->JGinv_upts,
                                                                  a->detjac_upts, a->norm_left, VF, ND, DV, E, L, ph, nullptr, nullptr);
  }
  if (a->n_int > 0) {
    unsigned g = (unsigned)((a->n_int + 127) / 128);
    const int2* face = reinterpret_cast<const int2*>(a->face_lr);
    if (visc)
      fr_face_kernel<DIM, 1, double><<<g, 128, 0, s>>>(face, a->face_sign, a->n_int, UF, VF, a->norm_left,
                                                       a->tdA_fpts, CF, NFE, ph);
    else
      fr_face_kernel<DIM, 0, double><<<g, 128, 0, s>>>(face, a->face_sign, a->n_int, UF, nullptr, a->norm_left,
                                                       a->tdA_fpts, CF, NFE, ph);
  }
  if (visc) {
    constexpr size_t sm = update_smem_bytes<DIM, P, EPB, NT, 1, 0, double>();
    if (sm > 48 * 1024)
      cudaFuncSetAttribute(fr_update_kernel<DIM, P, EPB, NT, 1, 0, double, 0>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    fr_update_kernel<DIM, P, EPB, NT, 1, 0, double, 0><<<nblk, NT, sm, s>>>(
        const_cast<double*>(a->disu_upts), nullptr, nullptr, CF, ND, DV, a->JGinv_upts, a->detjac_upts, a->div_tconf_upts, nullptr, E, L, ph,
        0.0, 0.0, 0.0, 0);
  } else {
    constexpr size_t sm = update_smem_bytes<DIM, P, EPB, NT, 0, 0, double>();
    if (sm > 48 * 1024)
      cudaFuncSetAttribute(fr_update_kernel<DIM, P, EPB, NT, 0, 0, double, 0>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    fr_update_kernel<DIM, P, EPB, NT, 0, 0, double, 0><<<nblk, NT, sm, s>>>(
        const_cast<double*>(a->disu_upts), nullptr, nullptr, CF, nullptr, nullptr, a->JGinv_upts, a->detjac_upts,
        a->div_tconf_upts, nullptr, E, L, ph, 0.0, 0.0, 0.0, 0);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return na_fail(FR_ERR_CUDA, cudaGetErrorString(e));
  return FR_OK;
}

}  // namespace

extern "C" fr_status fr_residual_noalloc(const fr_residual_args* a, void* stream)
{
  if (!a || !a->disu_upts || !a->JGinv_upts || !a->detjac_upts || !a->norm_left || !a->tdA_fpts || !a->mate ||
      !a->side || !a->div_tconf_upts || (a->n_int > 0 && (!a->face_lr || !a->face_sign)))
    return na_fail(FR_ERR_ARG, "null argument");
  if (a->n_eles <= 0 || a->n_int < 0) return na_fail(FR_ERR_ARG, "bad sizes");
  if (((uintptr_t)a->face_lr) % 8 != 0) return na_fail(FR_ERR_ARG, "face_lr must be 8-byte aligned");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return na_fail(FR_ERR_CUDA, cudaGetErrorString(e));
  double* scratch = nullptr;
  fr_status st = scratch_for_device(dev, &scratch);
  if (st) return st;
  cudaStream_t s = (cudaStream_t)stream;
  if (a->dims == 2) {
    switch (a->order) {
      case 1: return run<2, 1>(a, scratch, s);
      case 2: return run<2, 2>(a, scratch, s);
      case 3: return run<2, 3>(a, scratch, s);
      case 4: return run<2, 4>(a, scratch, s);
      case 5: return run<2, 5>(a, scratch, s);
    }
  } else if (a->dims == 3) {
    switch (a->order) {
      case 1: return run<3, 1>(a, scratch, s);
      case 2: return run<3, 2>(a, scratch, s);
      case 3: return run<3, 3>(a, scratch, s);
      case 4: return run<3, 4>(a, scratch, s);
    }
  }
  return na_fail(FR_ERR_UNSUPPORTED, "no kernel for this (dims, order)");
}
