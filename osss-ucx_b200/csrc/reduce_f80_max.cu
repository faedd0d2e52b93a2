/*
 * reduce_f80_max.cu -- the reduce kernels instantiated for long double
 * (the x87 80-bit extended format, in software), op MAX: a running chain
 * with the exact replay of order-dependent elements.  Each long double op
 * has a translation unit of its own, since the software arithmetic makes
 * these the slowest instantiations to compile.
 */
#include "reduce_kernels.cuh"

namespace b200 {

int reduce_dispatch_f80_max(const RArgs &a, bool aligned, cudaStream_t s) {
  return run_float<f80, B200SHM_MAX>(a, aligned, s);
}

}  // namespace b200
