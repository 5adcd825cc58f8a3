// Stubs for the reference's GPU members in the CPU-only oracle build (libephref.so): the reference's
// CUDA integrator (src/integrators/RungeKutta.cu) is not compiled here.
#include "physics/mass.h"
#include "utils/logger.h"
#include <cstdlib>

void msystem::Cuda_RungeKutta12(fast_real, int_t) {
    LogCritical("reference CUDA path is not built into the CPU oracle library\n");
    abort();
}
void msystem::Cuda_accel() {
    LogCritical("reference CUDA path is not built into the CPU oracle library\n");
    abort();
}

