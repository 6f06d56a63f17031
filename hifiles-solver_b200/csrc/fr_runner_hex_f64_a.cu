// fr_runner_hex_f64_a.cu -- stage-kernel instantiations: hexes P=1 FP64, hexes P=2 FP64.
#include "fr_runner.cuh"

namespace frb {
FR_RUNNER(3, 1, double)
FR_RUNNER(3, 2, double)
}  // namespace frb
