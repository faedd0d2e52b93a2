/*
 * reduce_int.cu -- the reduce kernels instantiated for the integer types
 * (8 to 64 bits, signed and unsigned).  Ops other than MIN/MAX give the
 * same bits on signed and unsigned views, so they run on the unsigned
 * type of the same width.
 */
#include "reduce_kernels.cuh"

namespace b200 {

int reduce_dispatch_int(int op, int dtype, const RArgs &a, bool aligned, cudaStream_t s) {
  switch (dtype) {
  case B200SHM_I8: return run_int<int8_t, uint8_t>(op, a, aligned, s);
  case B200SHM_I16: return run_int<int16_t, uint16_t>(op, a, aligned, s);
  case B200SHM_I32: return run_int<int32_t, uint32_t>(op, a, aligned, s);
  case B200SHM_I64: return run_int<int64_t, uint64_t>(op, a, aligned, s);
  case B200SHM_U8: return run_int<uint8_t, uint8_t>(op, a, aligned, s);
  case B200SHM_U16: return run_int<uint16_t, uint16_t>(op, a, aligned, s);
  case B200SHM_U32: return run_int<uint32_t, uint32_t>(op, a, aligned, s);
  case B200SHM_U64: return run_int<uint64_t, uint64_t>(op, a, aligned, s);
  default: return fail(B200SHM_ERR_ARG, "reduce: dtype %d is not an integer type", dtype);
  }
}

}  // namespace b200
