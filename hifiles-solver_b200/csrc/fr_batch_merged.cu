// fr_batch_merged.cu -- the merged stage kernels of a batch (see
// fr_batch_merged.cuh): one launch per stage kernel over the element blocks
// of every group, each block running its group's order.
#include <algorithm>
#include <string>

#include "fr_batch_merged.cuh"

namespace frb {

extern thread_local std::string g_err;

namespace {

template <int P, typename TC>
constexpr size_t merged_grad_smem()
{
  constexpr int EPB = MergedTile<P>::epb;
  return grad_smem_bytes<3, P, EPB, TC, 0, grad_alias<3, P, EPB, kMergedNT, TC, 0, 0>()>();
}

template <int P, typename TC>
constexpr size_t merged_upd_smem()
{
  constexpr int EPB = MergedTile<P>::epb;
  if constexpr (merged_fused<P, TC>()) return face_update_smem_bytes<3, P, TC, 1, 1, EPB, kMergedNT>();
  else return update_smem_bytes<3, P, EPB, kMergedNT, 1, 1, TC>();
}

template <int P, typename TC>
__device__ __forceinline__ void grad_slot(const MergedGrad<TC>& g, long long b)
{
  fr_grad_body<3, P, MergedTile<P>::epb, kMergedNT, TC, 0, 1, 0>(b, 0, g.U, g.UF, g.mate, g.side, g.JG, g.detj, g.nL,
                                                                 g.VF, g.ND, g.DV, g.E, g.L, g.ph, nullptr, g.BV);
}

template <int P, typename TC>
__device__ __forceinline__ void upd_slot(const MergedUpd<TC>& u, long long b)
{
  constexpr int EPB = MergedTile<P>::epb;
  if constexpr (merged_fused<P, TC>())
    fr_face_update_body<3, P, EPB, kMergedNT, 1, 1, TC, 0>(b, u.U, u.REG, u.UFn, u.UF, u.mate, u.side, u.VF, u.ND,
                                                           u.DV, u.JG, u.nL, u.tdA, u.idetj, u.BV, u.DIV, nullptr,
                                                           u.E, u.L, u.ph, u.rk_a, u.rk_b, u.dt, u.first_stage,
                                                           u.err);
  else
    fr_update_body<3, P, EPB, kMergedNT, 1, 1, TC>(b, u.U, u.REG, u.UFn, u.CF, u.ND, u.DV, u.JG, u.detj64, u.DIV,
                                                   nullptr, u.E, u.L, u.ph, u.rk_a, u.rk_b, u.dt, u.first_stage);
}

template <typename TC, int MINB>
__global__ void __launch_bounds__(kMergedNT, MINB) fr_merged_grad_kernel(const __grid_constant__ MergedGrads<TC> a)
{
  long long b = blockIdx.x;
  if (b < a.s[0].nblk) { grad_slot<2>(a.s[0], b); return; }
  b -= a.s[0].nblk;
  if (b < a.s[1].nblk) { grad_slot<3>(a.s[1], b); return; }
  b -= a.s[1].nblk;
  if (b < a.s[2].nblk) grad_slot<4>(a.s[2], b);
}

template <typename TC>
__global__ void __launch_bounds__(128) fr_merged_face_kernel(const __grid_constant__ MergedFaces<TC> a)
{
  long long b = blockIdx.x;
  for (int k = 0; k < 3; k++) {
    const MergedFace<TC>& f = a.s[k];
    if (b < f.nblk) {
      fr_face_body<3, 1, TC, 0>(b, f.face, f.fsign, f.nint, f.UF, f.VF, f.nL, f.tdA, f.CF, f.NFE, f.ph, f.nbdy, f.bf,
                                f.bt, f.BV);
      return;
    }
    b -= f.nblk;
  }
}

template <typename TC, int MINB>
__global__ void __launch_bounds__(kMergedNT, MINB) fr_merged_upd_kernel(const __grid_constant__ MergedUpds<TC> a)
{
  long long b = blockIdx.x;
  if (b < a.s[0].nblk) { upd_slot<2>(a.s[0], b); return; }
  b -= a.s[0].nblk;
  if (b < a.s[1].nblk) { upd_slot<3>(a.s[1], b); return; }
  b -= a.s[1].nblk;
  if (b < a.s[2].nblk) upd_slot<4>(a.s[2], b);
}

template <typename TC, int MINB>
fr_status launch_t(const void* grads, const void* faces, bool any_face, const void* upds, cudaStream_t s)
{
  const auto& G = *static_cast<const MergedGrads<TC>*>(grads);
  const auto& Fc = *static_cast<const MergedFaces<TC>*>(faces);
  const auto& U = *static_cast<const MergedUpds<TC>*>(upds);
  constexpr size_t smg = std::max({merged_grad_smem<2, TC>(), merged_grad_smem<3, TC>(), merged_grad_smem<4, TC>()});
  constexpr size_t smu = std::max({merged_upd_smem<2, TC>(), merged_upd_smem<3, TC>(), merged_upd_smem<4, TC>()});
  static bool once = [] {
    cudaFuncSetAttribute((const void*)fr_merged_grad_kernel<TC, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smg);
    cudaFuncSetAttribute((const void*)fr_merged_upd_kernel<TC, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smu);
    return true;
  }();
  (void)once;
  long long ng = G.s[0].nblk + G.s[1].nblk + G.s[2].nblk;
  long long nu = U.s[0].nblk + U.s[1].nblk + U.s[2].nblk;
  long long nf = Fc.s[0].nblk + Fc.s[1].nblk + Fc.s[2].nblk;
  if (ng > 2147483647LL || nu > 2147483647LL || nf > 2147483647LL) {
    g_err = "batch too large for one merged launch";
    return FR_ERR_ARG;
  }
  if (ng > 0) fr_merged_grad_kernel<TC, MINB><<<(unsigned)ng, kMergedNT, smg, s>>>(G);
  if (any_face && nf > 0) fr_merged_face_kernel<TC><<<(unsigned)nf, 128, 0, s>>>(Fc);
  if (nu > 0) fr_merged_upd_kernel<TC, MINB><<<(unsigned)nu, kMergedNT, smu, s>>>(U);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    g_err = std::string("merged stage kernels: ") + cudaGetErrorString(e);
    return FR_ERR_CUDA;
  }
  return FR_OK;
}

}  // namespace

fr_status merged_stage_launch(bool fp32, const void* grads, const void* faces, bool any_face, const void* upds,
                              int minb, cudaStream_t s)
{
  if (fp32) {
    if (minb >= 4) return launch_t<float, 4>(grads, faces, any_face, upds, s);
    if (minb == 3) return launch_t<float, 3>(grads, faces, any_face, upds, s);
    return launch_t<float, 1>(grads, faces, any_face, upds, s);
  }
  if (minb >= 4) return launch_t<double, 4>(grads, faces, any_face, upds, s);
  if (minb == 3) return launch_t<double, 3>(grads, faces, any_face, upds, s);
  return launch_t<double, 1>(grads, faces, any_face, upds, s);
}

}  // namespace frb
