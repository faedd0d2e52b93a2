/*
 * reduce_f64.cu -- the reduce kernels instantiated for double:
 * MIN/MAX as a running chain with the exact replay of order-dependent
 * elements, SUM/PROD in the algorithm's combine tree.
 */
#include "reduce_kernels.cuh"

namespace b200 {

int reduce_dispatch_f64(int op, const RArgs &a, bool aligned, cudaStream_t s) {
  switch (op) {
  case B200SHM_MIN: return run_float<double, B200SHM_MIN>(a, aligned, s);
  case B200SHM_MAX: return run_float<double, B200SHM_MAX>(a, aligned, s);
  case B200SHM_SUM: return run_float<double, B200SHM_SUM>(a, aligned, s);
  default: return run_float<double, B200SHM_PROD>(a, aligned, s);
  }
}

}  // namespace b200
