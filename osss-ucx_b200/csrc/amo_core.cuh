/*
 * amo_core.cuh -- one atomic memory operation on a word of the arena, the
 * element operation of the batched AMO kernel (amo.cu) and of the serving
 * loop (serve.cu).  Semantics of the reference's shmemc_ctx_{fadd,add,
 * swap,cswap,fetch,set,and,or,xor} (src/shmemc/ucx/comms.c:409-671).
 */
#pragma once
#include "internal.cuh"

namespace b200 {
namespace {

template <class W>
__device__ __forceinline__ W amo_one(int amo, W *p, W v, W c) {
  switch (amo) {
  case B200SHM_AMO_FETCH_ADD:
  case B200SHM_AMO_ADD: return atomicAdd(p, v);
  case B200SHM_AMO_FETCH_INC:
  case B200SHM_AMO_INC: return atomicAdd(p, (W)1);
  case B200SHM_AMO_SWAP:
  case B200SHM_AMO_SET: return atomicExch(p, v);
  case B200SHM_AMO_CSWAP: return atomicCAS(p, c, v);
  case B200SHM_AMO_FETCH: return atomicAdd(p, (W)0);
  case B200SHM_AMO_FETCH_AND:
  case B200SHM_AMO_AND: return atomicAnd(p, v);
  case B200SHM_AMO_FETCH_OR:
  case B200SHM_AMO_OR: return atomicOr(p, v);
  default: return atomicXor(p, v);
  }
}

}  // namespace
}  // namespace b200
