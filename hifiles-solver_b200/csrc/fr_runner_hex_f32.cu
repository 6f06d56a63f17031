// fr_runner_hex_f32.cu -- stage-kernel instantiations: hexes P=1 FP32, hexes P=2 FP32, hexes P=3 FP32, hexes P=4 FP32.
#include "fr_runner.cuh"

namespace frb {
FR_RUNNER(3, 1, float)
FR_RUNNER(3, 2, float)
FR_RUNNER(3, 3, float)
FR_RUNNER(3, 4, float)
}  // namespace frb
