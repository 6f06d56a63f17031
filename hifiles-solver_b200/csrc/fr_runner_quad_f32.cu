// fr_runner_quad_f32.cu -- stage-kernel instantiations: quads P=1 FP32, quads P=2 FP32, quads P=3 FP32, quads P=4 FP32, quads P=5 FP32.
#include "fr_runner.cuh"

namespace frb {
FR_RUNNER(2, 1, float)
FR_RUNNER(2, 2, float)
FR_RUNNER(2, 3, float)
FR_RUNNER(2, 4, float)
FR_RUNNER(2, 5, float)
}  // namespace frb
