// fr_runner.cuh -- the per-(dims, order, precision) launchers of the fused
// stage kernels behind fr_solver: compiled tile variants, the kernel-choice
// state the autotuner sets, and the launch of each stage kernel.  Each
// (dims, order, precision) runner is compiled in one of the fr_runner_*.cu
// translation units so the instantiations build in parallel.
#pragma once

#include <cuda_runtime.h>

#include "fr_batch_merged.cuh"
#include "fr_fused.cuh"
#include "fr_host.hpp"

namespace frb {

// RK45 coefficients (Carpenter-Kennedy low-storage, eles::AdvanceSolution,
// src/eles.cpp:1093-1113).
static const double kRK4A[5] = {0.0, -0.417890474499852, -1.192151694642677, -1.697784692471528,
                                -1.514183444257156};
static const double kRK4B[5] = {0.149659021999229, 0.379210312999627, 0.822955029386982, 0.699450455949122,
                                0.153057247968152};

struct Bufs {
  double *U = nullptr, *REG = nullptr, *DIV = nullptr, *detj64 = nullptr, *partial = nullptr, *norms = nullptr;
  void *UF[2] = {nullptr, nullptr}, *VF = nullptr, *ND = nullptr, *DV = nullptr, *CF = nullptr, *nL = nullptr,
       *tdA = nullptr, *JG = nullptr, *detj = nullptr, *GRAD = nullptr;
  int2* face = nullptr;
  unsigned char* fsign = nullptr;
  long long nint = 0;
  long long nbdy = 0;              // boundary flux points
  int* bf = nullptr;               // their flat indices
  unsigned char* bt = nullptr;     // their boundary types
  void* BV = nullptr;              // viscous boundary normal flux (nbdy, F), from the gradient kernel
  int* mate = nullptr;
  unsigned char* side = nullptr;
  double* idetj = nullptr;         // 1/detJ at the solution points (the update multiplies by it)
  int* err = nullptr;              // set by a kernel whose bounded wait gave up
};

struct Tile {
  int epb, nt, minb;   // elements per CTA, threads per CTA, CTAs per SM the registers are sized for (0: any)
  int pers = 0;        // gradient kernel only: 1 = persistent blocks that prefetch their next element block
};

struct Runner {
  virtual ~Runner() {}
  // traces of the state; with src, the state src is also copied into b.U
  virtual void trace(const Bufs& b, int cur, cudaStream_t s, const double* src = nullptr) = 0;
  virtual void grad(const Bufs& b, int cur, cudaStream_t s) = 0;
  virtual void face(const Bufs& b, int cur, cudaStream_t s) = 0;
  virtual void update(const Bufs& b, int cur, int mode, int stage, double dt, bool want_partial, cudaStream_t s) = 0;
  virtual int flux_blocks() const = 0;      // blocks of the update kernel (norm partials)
  virtual int max_flux_blocks() const = 0;  // over all update-kernel tiles
  virtual int launches_per_stage() const = 0;
  virtual void set_riemann(int rs) = 0;
  // tile variants of the two element kernels (autotuning)
  virtual int n_grad_tiles() const = 0;
  virtual int n_update_tiles() const = 0;
  virtual Tile grad_tile(int i) const = 0;
  virtual Tile update_tile(int i) const = 0;
  virtual void select(int g, int u) = 0;
  virtual int grad_sel() const = 0;
  virtual int update_sel() const = 0;
  // This group's slot of the merged batch launches (fr_batch_merged.cuh):
  // fills *grad, *face and *upd (MergedGrad / MergedFace / MergedUpd of the
  // runner's precision) for stage `stage` and returns the order, or 0 if the
  // group cannot join them.
  virtual int merged_args(const Bufs& b, int cur, int stage, double dt, void* grad, void* face, void* upd) const
  {
    (void)b; (void)cur; (void)stage; (void)dt; (void)grad; (void)face; (void)upd;
    return 0;
  }
};

// Compiled tile variants (elements per CTA, threads per CTA) of the gradient
// and update kernels per (dims, order); the first entry is the default, the
// autotuner may pick another.
template <int DIM, int P> struct Tiles;
#define FR_TILES(D_, P_, G, U) \
  template <> struct Tiles<D_, P_> { static constexpr Tile grad[] = G; static constexpr Tile upd[] = U; };
#define T_(...) {__VA_ARGS__}
FR_TILES(2, 1, T_({32, 128}), T_({32, 128}))
FR_TILES(2, 2, T_({16, 128}), T_({16, 128}))
FR_TILES(2, 3, T_({8, 128}, {4, 64}, {16, 256}), T_({8, 128}, {4, 64}, {16, 256}))
FR_TILES(2, 4, T_({8, 256}), T_({8, 256}))
FR_TILES(2, 5, T_({4, 160}), T_({4, 160}))
FR_TILES(3, 1, T_({12, 128}), T_({12, 128}))
FR_TILES(3, 2, T_({4, 128}, {2, 64}, {8, 256}), T_({4, 128}, {2, 64}, {8, 256}))
FR_TILES(3, 3, T_({2, 128, 4}, {1, 64, 8}, {2, 192, 2}, {2, 128, 3}, {1, 96, 0}, {4, 256, 2}, {1, 96, 5}, {1, 96, 6},
                  {1, 64, 8, 1}, {2, 128, 3, 1}, {1, 96, 10}), T_({1, 96, 7}, {1, 64, 8}, {1, 96}, {1, 64}, {2, 128}, {1, 96, 6}, {1, 64, 9}, {2, 192, 3}))
FR_TILES(3, 4, T_({1, 128}, {1, 160}, {2, 256}), T_({1, 128}, {2, 256}, {1, 160}))
#undef T_
#undef FR_TILES

static void set_smem(const void* k, size_t bytes)
{
  if (bytes > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <int DIM, int P, typename TC>
struct RunnerT : Runner {
  using S = Shape<DIM, P>;
  static constexpr int NG = sizeof(Tiles<DIM, P>::grad) / sizeof(Tile);
  static constexpr int NUP = sizeof(Tiles<DIM, P>::upd) / sizeof(Tile);
  long long E;
  int visc, les, riemann = 0;
  int gsel = 0, usel = 0;
  Line<TC> L;
  Line<double> L64;
  PhysT<TC> ph;
  RunnerT(long long E_, int visc_, int les_, const Line1D& l, const Phys& p) : E(E_), visc(visc_), les(les_)
  {
    for (int i = 0; i < kMaxN1; i++) {
      L.Lm[i] = L.Lp[i] = L.gL[i] = L.gR[i] = L.w[i] = TC(0);
      for (int j = 0; j < kMaxN1; j++) L.D[i][j] = TC(0);
    }
    for (int i = 0; i <= P; i++) {
      L.Lm[i] = (TC)l.Lm[i]; L.Lp[i] = (TC)l.Lp[i]; L.gL[i] = (TC)l.gL[i]; L.gR[i] = (TC)l.gR[i];
      L.w[i] = (TC)l.w[i];
      for (int j = 0; j <= P; j++) L.D[i][j] = (TC)l.D[i][j];
    }
    for (int i = 0; i < kMaxN1; i++) {
      L64.Lm[i] = i <= P ? l.Lm[i] : 0; L64.Lp[i] = i <= P ? l.Lp[i] : 0; L64.gL[i] = i <= P ? l.gL[i] : 0;
      L64.gR[i] = i <= P ? l.gR[i] : 0; L64.w[i] = i <= P ? l.w[i] : 0;
      for (int j = 0; j < kMaxN1; j++) L64.D[i][j] = (i <= P && j <= P) ? l.D[i][j] : 0;
    }
    ph = PhysT<TC>::make(p);
  }
  int n_grad_tiles() const override { return NG; }
  int n_update_tiles() const override { return NUP; }
  Tile grad_tile(int i) const override { return Tiles<DIM, P>::grad[i]; }
  Tile update_tile(int i) const override { return Tiles<DIM, P>::upd[i]; }
  void select(int g, int u) override { gsel = g; usel = u; }
  int grad_sel() const override { return gsel; }
  int update_sel() const override { return usel; }
  int flux_blocks() const override
  {
    int epb = Tiles<DIM, P>::upd[usel].epb;
    return (int)((E + epb - 1) / epb);
  }
  int max_flux_blocks() const override
  {
    int m = 1;
    for (int i = 0; i < NUP; i++) {
      int b = (int)((E + Tiles<DIM, P>::upd[i].epb - 1) / Tiles<DIM, P>::upd[i].epb);
      m = b > m ? b : m;
    }
    return m;
  }
  // the bulk-copy kernel folds the interface fluxes into the update (fr_face_update.cuh)
  static constexpr bool FU = fu_bulk_ok<DIM, P, TC>();
  int launches_per_stage() const override { return FU ? (visc ? 2 : 1) : (visc ? 3 : 2); }
  void set_riemann(int rs) override { riemann = rs; }
  void trace(const Bufs& b, int cur, cudaStream_t s, const double* src = nullptr) override
  {
    long long n = E * (src && S::NU > S::NF ? S::NU : S::NF);
    fr_trace_kernel<DIM, P, TC><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(src ? src : b.U, (TC*)b.UF[cur], E, L,
                                                                           src ? b.U : nullptr);
  }

  template <int I, int LES>
  void grad_i(const Bufs& b, int cur, cudaStream_t s)
  {
    if constexpr (I < NG) {
      if (I != gsel) return grad_i<I + 1, LES>(b, cur, s);
      constexpr int EPB = Tiles<DIM, P>::grad[I].epb, NT = Tiles<DIM, P>::grad[I].nt;
      constexpr int MINB = Tiles<DIM, P>::grad[I].minb > 0 ? Tiles<DIM, P>::grad[I].minb : 1;
      constexpr int PERS = Tiles<DIM, P>::grad[I].pers;
      constexpr size_t sm = grad_smem_bytes<DIM, P, EPB, TC, LES, grad_alias<DIM, P, EPB, NT, TC, LES, PERS>()>();
      const void* kfn = (const void*)fr_grad_kernel<DIM, P, EPB, NT, TC, LES, MINB, 1, PERS>;
      static bool once = (set_smem(kfn, sm), true);
      (void)once;
      long long grid = (E + EPB - 1) / EPB;
      if (PERS) {
        // persistent blocks: as many as are resident at once
        static int resident = [&] {
          int dev = 0, sms = 0, per = 0;
          cudaGetDevice(&dev);
          cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kfn, NT, sm);
          return (per > 0 ? per : 1) * (sms > 0 ? sms : 1);
        }();
        grid = grid < resident ? grid : resident;
      }
      fr_grad_kernel<DIM, P, EPB, NT, TC, LES, MINB, 1, PERS><<<(unsigned)grid, NT, sm, s>>>(
          b.U, (const TC*)b.UF[cur], b.mate, b.side, (const TC*)b.JG, (const TC*)b.detj, (const TC*)b.nL,
          (TC*)b.VF, (TC*)b.ND, (TC*)b.DV, E, L, ph, (TC*)b.GRAD, (TC*)b.BV);
    }
  }
  void grad(const Bufs& b, int cur, cudaStream_t s) override
  {
    if (les) grad_i<0, 1>(b, cur, s);
    else grad_i<0, 0>(b, cur, s);
  }

  template <int VISC, int RS>
  void face_t(const Bufs& b, int cur, cudaStream_t s)
  {
    unsigned g = (unsigned)((b.nint + b.nbdy + 127) / 128);
    fr_face_kernel<DIM, VISC, TC, RS><<<g, 128, 0, s>>>(b.face, b.fsign, b.nint, (const TC*)b.UF[cur],
                                                         VISC ? (const TC*)b.VF : nullptr, (const TC*)b.nL,
                                                         (const TC*)b.tdA, (TC*)b.CF, E * S::NF, ph, b.nbdy, b.bf,
                                                         b.bt, VISC ? (const TC*)b.BV : nullptr);
  }
  void face(const Bufs& b, int cur, cudaStream_t s) override
  {
    if (FU || b.nint + b.nbdy == 0) return;
    if (DIM == 2 && riemann == 2) {
      if (visc) face_t<1, 2>(b, cur, s);
      else face_t<0, 2>(b, cur, s);
    } else {
      if (visc) face_t<1, 0>(b, cur, s);
      else face_t<0, 0>(b, cur, s);
    }
  }

  template <int I, int VISC, int MODE>
  void update_i(const Bufs& b, int cur, int stage, double dt, bool want_partial, cudaStream_t s)
  {
    if constexpr (I < NUP) {
      if (I != usel) return update_i<I + 1, VISC, MODE>(b, cur, stage, dt, want_partial, s);
      constexpr int EPB = Tiles<DIM, P>::upd[I].epb, NT = Tiles<DIM, P>::upd[I].nt;
      if constexpr (FU) {
        constexpr int MB = Tiles<DIM, P>::upd[I].minb > 0 ? Tiles<DIM, P>::upd[I].minb : 1;
        if constexpr (DIM == 2) {
          if (riemann == 2) fu_launch<EPB, NT, VISC, MODE, 2, MB>(b, cur, stage, dt, want_partial, s);
          else fu_launch<EPB, NT, VISC, MODE, 0, MB>(b, cur, stage, dt, want_partial, s);
        } else {
          fu_launch<EPB, NT, VISC, MODE, 0, MB>(b, cur, stage, dt, want_partial, s);
        }
      } else {
        constexpr size_t sm = update_smem_bytes<DIM, P, EPB, NT, VISC, MODE, TC>();
        static bool once = (set_smem((const void*)fr_update_kernel<DIM, P, EPB, NT, VISC, MODE, TC>, sm), true);
        (void)once;
        fr_update_kernel<DIM, P, EPB, NT, VISC, MODE, TC><<<(unsigned)((E + EPB - 1) / EPB), NT, sm, s>>>(
            b.U, b.REG, (TC*)b.UF[cur ^ 1], (const TC*)b.CF, (const TC*)b.ND, (const TC*)b.DV, (const TC*)b.JG,
            b.detj64, b.DIV, want_partial ? b.partial : nullptr, E, L, ph, kRK4A[stage], kRK4B[stage], dt,
            stage == 0 ? 1 : 0);
      }
    }
  }
  template <int EPB, int NT, int VISC, int MODE, int RS, int MB>
  void fu_launch(const Bufs& b, int cur, int stage, double dt, bool want_partial, cudaStream_t s)
  {
    constexpr size_t sm = face_update_smem_bytes<DIM, P, TC, VISC, MODE, EPB, NT>();
    const void* kfn = (const void*)fr_face_update_kernel<DIM, P, EPB, NT, VISC, MODE, TC, RS, MB>;
    static bool once = (set_smem(kfn, sm), true);
    (void)once;
    fr_face_update_kernel<DIM, P, EPB, NT, VISC, MODE, TC, RS, MB><<<(unsigned)((E + EPB - 1) / EPB), NT, sm, s>>>(
        b.U, b.REG, (TC*)b.UF[cur ^ 1], (const TC*)b.UF[cur], b.mate, b.side, (const TC*)b.VF, (const TC*)b.ND,
        (const TC*)b.DV, (const TC*)b.JG, (const TC*)b.nL, (const TC*)b.tdA, b.idetj, (const TC*)b.BV, b.DIV,
        want_partial ? b.partial : nullptr, E, L, ph, kRK4A[stage], kRK4B[stage], dt, stage == 0 ? 1 : 0, b.err);
  }
  int merged_args(const Bufs& b, int cur, int stage, double dt, void* gv, void* fv, void* uv) const override
  {
    if constexpr (DIM == 3 && P >= 2 && P <= 4) {
      if (!visc || les || riemann != 0) return 0;
      constexpr int EPB = MergedTile<P>::epb;
      const long long nblk = (E + EPB - 1) / EPB;
      *static_cast<MergedGrad<TC>*>(gv) =
          MergedGrad<TC>{b.U, (const TC*)b.UF[cur], b.mate, b.side, (const TC*)b.JG, (const TC*)b.detj,
                         (const TC*)b.nL, (TC*)b.VF, (TC*)b.ND, (TC*)b.DV, (TC*)b.BV, E, nblk, L, ph};
      MergedFace<TC> f{};
      if constexpr (!merged_fused<P, TC>()) {
        const long long n = b.nint + b.nbdy;
        f = MergedFace<TC>{b.face, b.fsign, b.nint, (const TC*)b.UF[cur], (const TC*)b.VF, (const TC*)b.nL,
                           (const TC*)b.tdA, (TC*)b.CF, E * S::NF, b.nbdy, b.bf, b.bt, (const TC*)b.BV,
                           (n + 127) / 128, ph};
      }
      *static_cast<MergedFace<TC>*>(fv) = f;
      *static_cast<MergedUpd<TC>*>(uv) =
          MergedUpd<TC>{b.U, b.REG, (TC*)b.UF[cur ^ 1], (const TC*)b.UF[cur], (const TC*)b.CF, b.mate, b.side,
                        (const TC*)b.VF, (const TC*)b.ND, (const TC*)b.DV, (const TC*)b.JG, (const TC*)b.nL,
                        (const TC*)b.tdA, b.detj64, b.idetj, (const TC*)b.BV, b.DIV, b.err, E, nblk, L, ph,
                        kRK4A[stage], kRK4B[stage], dt, stage == 0 ? 1 : 0};
      return P;
    }
    (void)b; (void)cur; (void)stage; (void)dt; (void)gv; (void)fv; (void)uv;
    return 0;
  }
  void update(const Bufs& b, int cur, int mode, int stage, double dt, bool want_partial, cudaStream_t s) override
  {
    if (visc) {
      if (mode == 0) update_i<0, 1, 0>(b, cur, stage, dt, false, s);
      else update_i<0, 1, 1>(b, cur, stage, dt, want_partial, s);
    } else {
      if (mode == 0) update_i<0, 0, 0>(b, cur, stage, dt, false, s);
      else update_i<0, 0, 1>(b, cur, stage, dt, want_partial, s);
    }
  }
};

// One factory per (dims, order, precision), defined by FR_RUNNER in the
// fr_runner_*.cu translation units.
#define FR_RUNNER_NAME(D_, P_, T_) make_runner_##D_##_##P_##_##T_
#define FR_RUNNER(D_, P_, T_)                                                                          \
  Runner* FR_RUNNER_NAME(D_, P_, T_)(long long E, int visc, int les, const Line1D& l, const Phys& p) \
  {                                                                                                    \
    return new RunnerT<D_, P_, T_>(E, visc, les, l, p);                                                \
  }
#define FR_RUNNER_DECL(D_, P_, T_) \
  Runner* FR_RUNNER_NAME(D_, P_, T_)(long long E, int visc, int les, const Line1D& l, const Phys& p);
FR_RUNNER_DECL(2, 1, double) FR_RUNNER_DECL(2, 2, double) FR_RUNNER_DECL(2, 3, double)
FR_RUNNER_DECL(2, 4, double) FR_RUNNER_DECL(2, 5, double)
FR_RUNNER_DECL(3, 1, double) FR_RUNNER_DECL(3, 2, double) FR_RUNNER_DECL(3, 3, double)
FR_RUNNER_DECL(3, 4, double)
FR_RUNNER_DECL(2, 1, float) FR_RUNNER_DECL(2, 2, float) FR_RUNNER_DECL(2, 3, float)
FR_RUNNER_DECL(2, 4, float) FR_RUNNER_DECL(2, 5, float)
FR_RUNNER_DECL(3, 1, float) FR_RUNNER_DECL(3, 2, float) FR_RUNNER_DECL(3, 3, float)
FR_RUNNER_DECL(3, 4, float)

}  // namespace frb
