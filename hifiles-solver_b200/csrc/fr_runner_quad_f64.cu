// fr_runner_quad_f64.cu -- stage-kernel instantiations: quads P=1 FP64, quads P=2 FP64, quads P=3 FP64, quads P=4 FP64, quads P=5 FP64.
#include "fr_runner.cuh"

namespace frb {
FR_RUNNER(2, 1, double)
FR_RUNNER(2, 2, double)
FR_RUNNER(2, 3, double)
FR_RUNNER(2, 4, double)
FR_RUNNER(2, 5, double)
}  // namespace frb
