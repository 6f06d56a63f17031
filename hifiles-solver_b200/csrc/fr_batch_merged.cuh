// fr_batch_merged.cuh -- one launch per stage kernel for a whole batch.
//
// A batch holds one merged mesh per (order, scheme) group.  Run group by
// group, a viscous RK stage launches the gradient kernel, the interface-flux
// kernel (orders whose runs are not 16-byte multiples) and the update kernel
// of every group: 2-3 launches per group and stage.  The merged launches
// below run each of those kernels once for all groups of hexahedra of orders
// 2, 3 and 4: the grid is the concatenation of the groups' element blocks,
// and each block runs the body of its group's order on that group's buffers
// (one body per block, chosen by the block index, so every barrier of a body
// is reached by the whole block).  All groups use 128-thread tiles (order 2:
// 4 elements per block, order 3: 2, order 4: 1); order 3 takes the fused
// interface/update body, orders 2 and 4 the interface-flux and update
// bodies.  No norms are formed (the batch reports none).
#pragma once

#include "fr_b200.h"
#include "fr_face_update.cuh"

namespace frb {

constexpr int kMergedNT = 128;
template <int P> struct MergedTile { static constexpr int epb = P == 2 ? 4 : P == 3 ? 2 : 1; };
// orders whose stage takes the fused interface/update kernel
template <int P, typename TC> __host__ __device__ constexpr bool merged_fused() { return fu_bulk_ok<3, P, TC>(); }

template <typename TC>
struct MergedGrad {
  const double* U; const TC* UF; const int* mate; const unsigned char* side; const TC* JG; const TC* detj;
  const TC* nL; TC* VF; TC* ND; TC* DV; TC* BV;
  long long E, nblk;
  Line<TC> L;
  PhysT<TC> ph;
};

template <typename TC>
struct MergedFace {
  const int2* face; const unsigned char* fsign; long long nint; const TC* UF; const TC* VF; const TC* nL;
  const TC* tdA; TC* CF; long long NFE, nbdy; const int* bf; const unsigned char* bt; const TC* BV;
  long long nblk;
  PhysT<TC> ph;
};

template <typename TC>
struct MergedUpd {
  double* U; double* REG; TC* UFn; const TC* UF; const TC* CF; const int* mate; const unsigned char* side;
  const TC* VF; const TC* ND; const TC* DV; const TC* JG; const TC* nL; const TC* tdA; const double* detj64;
  const double* idetj; const TC* BV; double* DIV; int* err;
  long long E, nblk;
  Line<TC> L;
  PhysT<TC> ph;
  double rk_a, rk_b, dt;
  int first_stage;
};

// Slot k of each launch holds the group of order k + 2 (nblk 0: no such group).
template <typename TC> struct MergedGrads { MergedGrad<TC> s[3]; };
template <typename TC> struct MergedFaces { MergedFace<TC> s[3]; };
template <typename TC> struct MergedUpds { MergedUpd<TC> s[3]; };

// Host: launch the three merged kernels of one stage (faces only when some
// group needs the separate interface kernel).  minb: CTAs per SM the
// registers are capped for (0: no cap).
fr_status merged_stage_launch(bool fp32, const void* grads, const void* faces, bool any_face, const void* upds,
                              int minb, cudaStream_t s);

}  // namespace frb
