// fr_runner_hex_f64_p3.cu -- stage-kernel instantiations: hexes P=3 FP64.
#include "fr_runner.cuh"

namespace frb {
FR_RUNNER(3, 3, double)
}  // namespace frb
