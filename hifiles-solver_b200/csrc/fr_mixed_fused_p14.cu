// fr_mixed_fused_p14.cu -- the fused stage's kernels for orders 1 and 4:
// tets, prisms and hexes (hexes of order 4 exceed one block's shared memory
// and have none) and triangles and quads.  The kernels are in
// fr_mixed_fused.cuh; this unit only instantiates them, beside the units of
// orders 2 and 3.
#include "fr_mixed_fused.cuh"

namespace frb_mixed {

bool find_kernels_p14(int D, int NU, int NF, MixedKernels* out)
{
#define FR_MIXED_SHAPE(d, nu, nf)          \
  if (D == d && NU == nu && NF == nf) {    \
    *out = mixed_kernels<d, nu, nf>();     \
    return true;                           \
  }
  FR_MIXED_SHAPE(3, 4, 12)    // tet P1
  FR_MIXED_SHAPE(3, 35, 60)   // tet P4
  FR_MIXED_SHAPE(3, 6, 18)    // prism P1
  FR_MIXED_SHAPE(3, 75, 105)  // prism P4
  FR_MIXED_SHAPE(3, 8, 24)    // hex P1
  FR_MIXED_SHAPE(2, 3, 6)     // triangle P1
  FR_MIXED_SHAPE(2, 15, 15)   // triangle P4
  FR_MIXED_SHAPE(2, 4, 8)     // quadrilateral P1
  FR_MIXED_SHAPE(2, 25, 20)   // quadrilateral P4
#undef FR_MIXED_SHAPE
  return false;
}

}  // namespace frb_mixed
