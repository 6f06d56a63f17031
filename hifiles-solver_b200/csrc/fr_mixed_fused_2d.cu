// fr_mixed_fused_2d.cu -- the fused stage's kernels for triangles and
// quadrilaterals of orders 2 and 3 (the kernels are in fr_mixed_fused.cuh;
// this unit only instantiates them, beside the 3-D unit fr_mixed_fused.cu).
#include "fr_mixed_fused.cuh"

namespace frb_mixed {

bool find_kernels_2d(int NU, int NF, MixedKernels* out)
{
#define FR_MIXED_SHAPE(nu, nf) \
  if (NU == nu && NF == nf) {  \
    *out = mixed_kernels<2, nu, nf>(); \
    return true;               \
  }
  FR_MIXED_SHAPE(6, 9)    // triangle P2
  FR_MIXED_SHAPE(10, 12)  // triangle P3
  FR_MIXED_SHAPE(9, 12)   // quadrilateral P2
  FR_MIXED_SHAPE(16, 16)  // quadrilateral P3
#undef FR_MIXED_SHAPE
  return false;
}

}  // namespace frb_mixed
