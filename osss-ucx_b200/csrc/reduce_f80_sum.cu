/*
 * reduce_f80_sum.cu -- the reduce kernels instantiated for long double
 * (the x87 80-bit extended format, in software), op SUM: the algorithm's
 * combine tree.  Each long double op has a translation unit of its own,
 * since the software arithmetic makes these the slowest instantiations to
 * compile.
 */
#include "reduce_kernels.cuh"

namespace b200 {

int reduce_dispatch_f80_sum(const RArgs &a, bool aligned, cudaStream_t s) {
  return run_float<f80, B200SHM_SUM>(a, aligned, s);
}

}  // namespace b200
