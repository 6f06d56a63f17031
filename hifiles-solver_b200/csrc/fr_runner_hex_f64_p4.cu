// fr_runner_hex_f64_p4.cu -- stage-kernel instantiations: hexes P=4 FP64.
#include "fr_runner.cuh"

namespace frb {
FR_RUNNER(3, 4, double)
}  // namespace frb
