/*
 * amo.cu -- batched atomic memory operations on the symmetric heap.
 *
 * In the reference each shmem_<T>_atomic_<op> is a blocking UCX round trip
 * (shmemc_ctx_fadd -> helper_fetching_amo -> ucp_atomic_fetch_nb plus a
 * progress loop, src/shmemc/ucx/comms.c:265-292, 423-428), and AND/OR/XOR
 * are emulated with a compare-and-swap loop (comms.c:557-608).  Here a
 * batch of operations is one kernel, one thread per operation, each a
 * single L2 atomic at the target PE's slice.  Operations that hit the same
 * word are serialised by the hardware in an unspecified order, as
 * concurrent AMOs from different PEs are in OpenSHMEM.
 *
 * Targets are validated on the device (PE range, slice bounds, natural
 * alignment); an invalid one is skipped and sets the BADREQ status bit.
 */
#include <stdint.h>
#include <string.h>

#include <mutex>

#include "internal.cuh"
#include "amo_core.cuh"

namespace b200 {
namespace {

template <class W>
__global__ void __launch_bounds__(256) k_amo(int amo, uint64_t nops, const int32_t *pe,
                                             const uint64_t *off, const W *value, const W *cond,
                                             W *fetched, char *base, uint64_t slice, int npes,
                                             int *status) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nops;
       k += (uint64_t)gridDim.x * blockDim.x) {
    const int p = pe[k];
    const uint64_t o = off[k];
    if (p < 0 || p >= npes || o > slice - sizeof(W) || (o % sizeof(W)) != 0) {
      atomicOr(status, (int)B200SHM_STATUS_BADREQ);
      continue;
    }
    W *target = (W *)(base + (uint64_t)p * slice + o);
    const W v = value ? value[k] : (W)0;
    const W c = cond ? cond[k] : (W)0;
    const W old = amo_one<W>(amo, target, v, c);
    if (fetched) fetched[k] = old;
  }
}

/* one operation, operands by value; the old value goes to mapped host
 * memory so the caller reads it right after the stream synchronises */
template <class W>
__global__ void k_amo_one(int amo, W *target, W v, W c, W *fetched, int ok) {
  if (!ok) return;
  const W old = amo_one<W>(amo, target, v, c);
  if (fetched) *fetched = old;
}

}  // namespace

int amo_launch(int amo, int dtype, uint64_t nops, const int32_t *pe, const uint64_t *off,
               const void *value, const void *cond, void *fetched, cudaStream_t s) {
  if (!st().up) return fail(B200SHM_ERR_STATE, "b200shm is not initialised");
  if (amo < 0 || amo >= B200SHM_AMO_NOP) return fail(B200SHM_ERR_ARG, "amo: unknown op %d", amo);
  const bool w4 = dtype == B200SHM_I32 || dtype == B200SHM_U32 || dtype == B200SHM_F32;
  const bool w8 = dtype == B200SHM_I64 || dtype == B200SHM_U64 || dtype == B200SHM_F64;
  if (!w4 && !w8) return fail(B200SHM_ERR_UNSUPPORTED, "amo: dtype %d is not 4 or 8 bytes", dtype);
  const bool is_float = dtype == B200SHM_F32 || dtype == B200SHM_F64;
  if (is_float && amo != B200SHM_AMO_SWAP && amo != B200SHM_AMO_SET && amo != B200SHM_AMO_FETCH)
    return fail(B200SHM_ERR_UNSUPPORTED,
                "amo: floating types support only swap/set/fetch (extended AMO table)");
  const bool needs_value = !(amo == B200SHM_AMO_FETCH || amo == B200SHM_AMO_INC ||
                             amo == B200SHM_AMO_FETCH_INC);
  if (nops == 0) return B200SHM_OK;
  if (!pe || !off || (needs_value && !value) || (amo == B200SHM_AMO_CSWAP && !cond))
    return fail(B200SHM_ERR_ARG, "amo: missing operand array");
  const unsigned grid = grid_for(nops, 256, 8);
  if (w8)
    k_amo<unsigned long long><<<grid, 256, 0, s>>>(
        amo, nops, pe, off, (const unsigned long long *)value, (const unsigned long long *)cond,
        (unsigned long long *)fetched, st().base, st().slice, st().npes, st().d_status);
  else
    k_amo<unsigned int><<<grid, 256, 0, s>>>(amo, nops, pe, off, (const unsigned int *)value,
                                             (const unsigned int *)cond, (unsigned int *)fetched,
                                             st().base, st().slice, st().npes, st().d_status);
  count_launch();
  return B200SHM_OK;
}

/* One operation with its operands by value (the low 4 or 8 bytes of
 * value/cond), stream-ordered; the old value goes to `fetched` (a device or
 * mapped-host word, may be NULL).  The target is checked on the host. */
int amo_one_launch(int amo, int dtype, int pe, uint64_t off, uint64_t value, uint64_t cond,
                   void *fetched, cudaStream_t s) {
  if (!st().up) return fail(B200SHM_ERR_STATE, "b200shm is not initialised");
  if (amo < 0 || amo >= B200SHM_AMO_NOP) return fail(B200SHM_ERR_ARG, "amo: unknown op %d", amo);
  const bool w4 = dtype == B200SHM_I32 || dtype == B200SHM_U32 || dtype == B200SHM_F32;
  const bool w8 = dtype == B200SHM_I64 || dtype == B200SHM_U64 || dtype == B200SHM_F64;
  if (!w4 && !w8) return fail(B200SHM_ERR_UNSUPPORTED, "amo: dtype %d is not 4 or 8 bytes", dtype);
  const uint64_t w = w8 ? 8 : 4;
  if (pe < 0 || pe >= st().npes || off > st().slice - w || off % w)
    return fail(B200SHM_ERR_ARG, "amo: target (PE %d, offset %llu) is not a %llu-byte word of the heap",
                pe, (unsigned long long)off, (unsigned long long)w);
  char *target = st().base + (uint64_t)pe * st().slice + off;
  if (w8)
    k_amo_one<unsigned long long><<<1, 1, 0, s>>>(amo, (unsigned long long *)target, value, cond,
                                                  (unsigned long long *)fetched, 1);
  else
    k_amo_one<unsigned int><<<1, 1, 0, s>>>(amo, (unsigned int *)target, (unsigned int)value,
                                            (unsigned int)cond, (unsigned int *)fetched, 1);
  count_launch();
  return B200SHM_OK;
}

}  // namespace b200

extern "C" int b200shm_amo_batch(int amo, int dtype, uint64_t nops, const int32_t *pe,
                                 const uint64_t *off, const void *value, const void *cond,
                                 void *fetched, void *stream) {
  int rc = b200::amo_launch(amo, dtype, nops, pe, off, value, cond, fetched,
                            b200::pick_stream(stream));
  return rc ? rc : b200::finish(stream, "b200shm_amo_batch");
}

/* Per-thread slot of mapped pinned memory for b200shm_amo's fetched value. */
namespace b200 {
static int amo_slot(unsigned long long **host, unsigned long long **dev) {
  static std::mutex mu;
  static unsigned long long *h = nullptr, *d = nullptr;
  static int next = 0;
  static thread_local int mine = -1;
  constexpr int kSlots = 4096;
  std::lock_guard<std::mutex> lk(mu);
  if (h == nullptr) {
    cudaError_t e = cudaHostAlloc((void **)&h, kSlots * 64, cudaHostAllocMapped);
    if (e != cudaSuccess) return cuda_fail(e, "b200shm_amo slot");
    e = cudaHostGetDevicePointer((void **)&d, h, 0);
    if (e != cudaSuccess) return cuda_fail(e, "b200shm_amo slot");
  }
  if (mine < 0) mine = (next++) % kSlots;
  *host = h + (size_t)mine * 8;
  *dev = d + (size_t)mine * 8;
  return B200SHM_OK;
}
}  // namespace b200

extern "C" int b200shm_amo(int amo, int dtype, int pe, uint64_t off, const void *value,
                           const void *cond, void *fetched) {
  using namespace b200;
  if (!st().up) return fail(B200SHM_ERR_STATE, "b200shm is not initialised");
  if (amo < 0 || amo >= B200SHM_AMO_NOP) return fail(B200SHM_ERR_ARG, "amo: unknown op %d", amo);
  const bool w4 = dtype == B200SHM_I32 || dtype == B200SHM_U32 || dtype == B200SHM_F32;
  const bool w8 = dtype == B200SHM_I64 || dtype == B200SHM_U64 || dtype == B200SHM_F64;
  if (!w4 && !w8) return fail(B200SHM_ERR_UNSUPPORTED, "amo: dtype %d is not 4 or 8 bytes", dtype);
  const bool is_float = dtype == B200SHM_F32 || dtype == B200SHM_F64;
  if (is_float && amo != B200SHM_AMO_SWAP && amo != B200SHM_AMO_SET && amo != B200SHM_AMO_FETCH)
    return fail(B200SHM_ERR_UNSUPPORTED, "amo: floating types support only swap/set/fetch");
  const uint64_t w = w8 ? 8 : 4;
  if (pe < 0 || pe >= st().npes || off > st().slice - w || off % w)
    return fail(B200SHM_ERR_ARG, "amo: target (PE %d, offset %llu) is not a %llu-byte word of the heap",
                pe, (unsigned long long)off, (unsigned long long)w);
  unsigned long long *h = nullptr, *d = nullptr;
  int rc = amo_slot(&h, &d);
  if (rc) return rc;
  char *target = st().base + (uint64_t)pe * st().slice + off;
  cudaStream_t s = st().stream;
  if (w8) {
    unsigned long long v = 0, c = 0;
    if (value) memcpy(&v, value, 8);
    if (cond) memcpy(&c, cond, 8);
    k_amo_one<unsigned long long><<<1, 1, 0, s>>>(amo, (unsigned long long *)target, v, c, d, 1);
  } else {
    unsigned int v = 0, c = 0;
    if (value) memcpy(&v, value, 4);
    if (cond) memcpy(&c, cond, 4);
    k_amo_one<unsigned int><<<1, 1, 0, s>>>(amo, (unsigned int *)target, v, c, (unsigned int *)d, 1);
  }
  count_launch();
  rc = finish(nullptr, "b200shm_amo");
  if (rc) return rc;
  if (fetched) memcpy(fetched, (const void *)h, w);
  return B200SHM_OK;
}
