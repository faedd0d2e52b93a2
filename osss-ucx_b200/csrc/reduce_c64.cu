/*
 * reduce_c64.cu -- the reduce kernels instantiated for complex double: SUM and
 * PROD (the only ops the reference defines on complex types) in the
 * algorithm's combine tree.
 */
#include "reduce_kernels.cuh"

namespace b200 {

int reduce_dispatch_c64(int op, const RArgs &a, bool aligned, cudaStream_t s) {
  return op == B200SHM_SUM ? run_cplx<cf64, B200SHM_SUM>(a, aligned, s)
                           : run_cplx<cf64, B200SHM_PROD>(a, aligned, s);
}

}  // namespace b200
