/*
 * reduce.cu -- the reduce entry points: argument checks, the per-call
 * reduce, the host-row pipeline (b200shm_reduce_host) and the reduce on
 * caller buffers (b200shm_reduce_noalloc).  The kernels and their launch
 * sequences are in reduce_kernels.cuh, instantiated per element-type
 * family in reduce_{int,f32,f64,c32,c64}.cu and
 * reduce_f80_{min,max,sum,prod}.cu, and reached through the
 * reduce_dispatch_<family> functions declared in reduce_core.cuh.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <mutex>
#include <unordered_map>
#include <vector>
#include <type_traits>

#include "internal.cuh"
#include "reduce_core.cuh"

namespace b200 {


/* Host side of b200shm_reduce, also used by the batched and serving paths. */
/* Checks shared by every reduce entry point: the (op, dtype, algo) triple
 * exists in the reference's type tables, and the team size fits the
 * combine trees of the GPU kernels. */
static int reduce_check(int op, int dtype, int algo, int pe_size) {
  if (op < 0 || op >= B200SHM_NOP || dtype < 0 || dtype >= B200SHM_NDTYPE || algo < 0 ||
      algo >= B200SHM_NALGO)
    return fail(B200SHM_ERR_ARG, "reduce: bad op %d / dtype %d / algo %d", op, dtype, algo);
  const bool is_int = dtype <= B200SHM_U64;
  const bool is_cpx = dtype == B200SHM_C32 || dtype == B200SHM_C64;
  if ((op <= B200SHM_XOR && !is_int) || ((op == B200SHM_MIN || op == B200SHM_MAX) && is_cpx))
    return fail(B200SHM_ERR_UNSUPPORTED, "reduce: op %d is not defined on dtype %d", op, dtype);
  if (pe_size < 1) return fail(B200SHM_ERR_ARG, "reduce: team size %d < 1", pe_size);
  int p2s = 1;
  while (p2s * 2 <= pe_size) p2s *= 2;
  const bool tree = !is_int && op != B200SHM_MIN && op != B200SHM_MAX && algo != B200SHM_LINEAR;
  const int leaves = algo == B200SHM_BINOMIAL ? pe_size : p2s;
  if (tree && leaves > (1 << (kMaxLevels - 1)))
    return fail(B200SHM_ERR_UNSUPPORTED, "reduce: float combine trees are limited to %d members",
                1 << (kMaxLevels - 1));
  if (dtype == B200SHM_F80 && (op == B200SHM_MIN || op == B200SHM_MAX) &&
      pe_size > kFixMaxMembersF80)
    return fail(B200SHM_ERR_UNSUPPORTED, "reduce: long double MIN/MAX is limited to %d members",
                kFixMaxMembersF80);
  if (!is_int && (op == B200SHM_MIN || op == B200SHM_MAX) && pe_size > kFixMaxMembers)
    return fail(B200SHM_ERR_UNSUPPORTED, "reduce: float MIN/MAX is limited to %d members",
                kFixMaxMembers);
  return B200SHM_OK;
}

static RArgs reduce_args(const char *src, char *dst, uint64_t sstep, uint64_t dstep, int P,
                         uint64_t nelems, int algo) {
  RArgs a;
  int logp = 0, p2s = 1;
  while (p2s * 2 <= P) {
    p2s *= 2;
    logp++;
  }
  a.src = src;
  a.dst = dst;
  a.sstep = sstep;
  a.dstep = dstep;
  a.e_begin = 0;
  a.nvec = 0;
  a.N = nelems;
  a.g_off = 0;
  a.g_n = nelems;
  a.P = P;
  a.p2s = p2s;
  a.logp2s = logp;
  a.algo = algo;
  a.fix_list = a.fix_count = a.fix_done = nullptr;
  a.fix_cap = 0;
  a.status = nullptr;
  return a;
}

static int reduce_dispatch(int op, int dtype, const RArgs &a, bool aligned, cudaStream_t s);

int reduce_launch(int op, int dtype, int algo, int pe_start, int pe_stride, int pe_size,
                  uint64_t dest_off, uint64_t src_off, uint64_t nelems, cudaStream_t s) {
  int rc = check_team(pe_start, pe_stride, pe_size);
  if (rc) return rc;
  if ((rc = reduce_check(op, dtype, algo, pe_size))) return rc;
  const uint64_t es = (uint64_t)kDtypeSize[dtype];
  if (nelems > st().slice / es) return fail(B200SHM_ERR_ARG, "reduce: nelems too large");
  const uint64_t bytes = nelems * es;
  if ((rc = check_extent(src_off, bytes, "reduce source"))) return rc;
  if ((rc = check_extent(dest_off, bytes, "reduce dest"))) return rc;
  if (dest_off != src_off && overlaps(dest_off, bytes, src_off, bytes))
    return fail(B200SHM_ERR_ARG, "reduce: dest and source overlap without being identical");
  if (nelems == 0) return B200SHM_OK;
  Members m = members(pe_start, pe_stride, pe_size);
  RArgs a = reduce_args(m.first + src_off, m.first + dest_off, m.step, m.step, pe_size, nelems,
                        algo);
  a.fix_list = st().fix_list;
  a.fix_count = st().call_fix;
  a.fix_done = st().call_fix + 1;
  a.fix_cap = st().fix_cap;
  a.status = st().d_status;
  const bool aligned = ((src_off | dest_off | m.step) & 15u) == 0;
  return reduce_dispatch(op, dtype, a, aligned, s);
}

/* Elements [e0, e0 + count) of a reduction of nelems elements (validated by
 * the caller), as one more launch sequence on stream s: the per-element
 * result is that of the whole reduction. */
int reduce_range_launch(int op, int dtype, int algo, int pe_start, int pe_stride, int pe_size,
                        uint64_t dest_off, uint64_t src_off, uint64_t nelems, uint64_t e0,
                        uint64_t count, cudaStream_t s) {
  if (count == 0) return B200SHM_OK;
  const uint64_t es = (uint64_t)kDtypeSize[dtype];
  Members m = members(pe_start, pe_stride, pe_size);
  RArgs a = reduce_args(m.first + src_off + e0 * es, m.first + dest_off + e0 * es, m.step, m.step,
                        pe_size, count, algo);
  a.g_off = e0;
  a.g_n = nelems;
  a.fix_list = st().fix_list;
  a.fix_count = st().call_fix;
  a.fix_done = st().call_fix + 1;
  a.fix_cap = st().fix_cap;
  a.status = st().d_status;
  const bool aligned = (((src_off + e0 * es) | (dest_off + e0 * es) | m.step) & 15u) == 0;
  return reduce_dispatch(op, dtype, a, aligned, s);
}

static int reduce_dispatch(int op, int dtype, const RArgs &a, bool aligned, cudaStream_t s) {
  switch (dtype) {
  case B200SHM_F32: return reduce_dispatch_f32(op, a, aligned, s);
  case B200SHM_F64: return reduce_dispatch_f64(op, a, aligned, s);
  case B200SHM_F80:
    switch (op) {
    case B200SHM_MIN: return reduce_dispatch_f80_min(a, aligned, s);
    case B200SHM_MAX: return reduce_dispatch_f80_max(a, aligned, s);
    case B200SHM_SUM: return reduce_dispatch_f80_sum(a, aligned, s);
    default: return reduce_dispatch_f80_prod(a, aligned, s);
    }
  case B200SHM_C32: return reduce_dispatch_c32(op, a, aligned, s);
  case B200SHM_C64: return reduce_dispatch_c64(op, a, aligned, s);
  default: return reduce_dispatch_int(op, dtype, a, aligned, s);
  }
}

}  // namespace b200

extern "C" int b200shm_reduce(int op, int dtype, int algo, int pe_start, int pe_stride,
                              int pe_size, uint64_t dest_off, uint64_t src_off, uint64_t nelems,
                              void *stream) {
  int rc = b200::reduce_launch(op, dtype, algo, pe_start, pe_stride, pe_size, dest_off, src_off,
                               nelems, b200::pick_stream(stream));
  if (rc) return rc;
  return b200::finish(stream, "b200shm_reduce");
}

/* ---------------------------------------------------------------------------
 * b200shm_reduce_host: put_host + reduce + get_host of host rows, pipelined.
 * The elements are cut into chunks; chunk c's copy in (one 2-D copy for all
 * members), its reduction and its copy out run on three streams joined by
 * events, so the copy engines move chunk c+1 in and chunk c-1 out while
 * chunk c is reduced.  A chunk's results are those of the whole reduction
 * (the global element index is kept for the order-dependent elements).
 * ------------------------------------------------------------------------- */
namespace b200 {
namespace {
struct HostPipe {
  cudaStream_t in = nullptr, comp = nullptr, out = nullptr;
  std::vector<cudaEvent_t> ev;
  std::mutex mu;
};
HostPipe &host_pipe() {
  static HostPipe p;
  return p;
}
int pipe_events(HostPipe &p, size_t n) {
  while (p.ev.size() < n) {
    cudaEvent_t e;
    B200_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    p.ev.push_back(e);
  }
  return B200SHM_OK;
}
}  // namespace
}  // namespace b200

extern "C" int b200shm_reduce_host(int op, int dtype, int algo, int pe_start, int pe_stride,
                                   int pe_size, void *host_dest, uint64_t dest_pitch,
                                   const void *host_src, uint64_t src_pitch, uint64_t dest_off,
                                   uint64_t src_off, uint64_t nelems, void *stream) {
  using namespace b200;
  int rc = check_team(pe_start, pe_stride, pe_size);
  if (rc) return rc;
  if ((rc = reduce_check(op, dtype, algo, pe_size))) return rc;
  const uint64_t es = (uint64_t)kDtypeSize[dtype];
  if (nelems > st().slice / es) return fail(B200SHM_ERR_ARG, "reduce_host: nelems too large");
  const uint64_t bytes = nelems * es;
  if ((rc = check_extent(src_off, bytes, "reduce_host source")) ||
      (rc = check_extent(dest_off, bytes, "reduce_host dest")))
    return rc;
  if (dest_off != src_off && overlaps(dest_off, bytes, src_off, bytes))
    return fail(B200SHM_ERR_ARG, "reduce_host: dest and source overlap without being identical");
  if (nelems == 0) return B200SHM_OK;
  if (!host_dest || !host_src || dest_pitch < bytes || src_pitch < bytes)
    return fail(B200SHM_ERR_ARG, "reduce_host: null host row or pitch below the row size");
  /* chunks of about 32 MiB over all members (B200SHM_HOST_CHUNK_BYTES overrides),
   * a whole number of 4 KiB per member */
  uint64_t target = 32ull << 20;
  if (const char *e = getenv("B200SHM_HOST_CHUNK_BYTES")) target = strtoull(e, nullptr, 0);
  uint64_t chunk = target / ((uint64_t)pe_size * es);
  chunk = chunk / (4096 / es) * (4096 / es);
  if (chunk < 4096 / es) chunk = 4096 / es;
  const uint64_t nch = (nelems + chunk - 1) / chunk;
  HostPipe &p = host_pipe();
  std::lock_guard<std::mutex> lk(p.mu);
  if (!p.in) {
    B200_CK(cudaStreamCreateWithFlags(&p.in, cudaStreamNonBlocking));
    B200_CK(cudaStreamCreateWithFlags(&p.comp, cudaStreamNonBlocking));
    B200_CK(cudaStreamCreateWithFlags(&p.out, cudaStreamNonBlocking));
  }
  if ((rc = pipe_events(p, 2 * nch + 2))) return rc;
  cudaStream_t caller = pick_stream(stream);
  /* start after the caller's earlier work */
  B200_CK(cudaEventRecord(p.ev[2 * nch], caller));
  B200_CK(cudaStreamWaitEvent(p.in, p.ev[2 * nch], 0));
  B200_CK(cudaStreamWaitEvent(p.comp, p.ev[2 * nch], 0));
  const Members m = members(pe_start, pe_stride, pe_size);
  const uint64_t pitch = m.step ? m.step : st().slice;
  for (uint64_t c = 0; c < nch; c++) {
    const uint64_t e0 = c * chunk, cnt = nelems - e0 < chunk ? nelems - e0 : chunk;
    B200_CK(cudaMemcpy2DAsync(m.first + src_off + e0 * es, pitch,
                              (const char *)host_src + e0 * es, src_pitch, cnt * es, pe_size,
                              cudaMemcpyHostToDevice, p.in));
    B200_CK(cudaEventRecord(p.ev[2 * c], p.in));
    B200_CK(cudaStreamWaitEvent(p.comp, p.ev[2 * c], 0));
    if ((rc = reduce_range_launch(op, dtype, algo, pe_start, pe_stride, pe_size, dest_off,
                                  src_off, nelems, e0, cnt, p.comp)))
      return rc;
    B200_CK(cudaEventRecord(p.ev[2 * c + 1], p.comp));
    B200_CK(cudaStreamWaitEvent(p.out, p.ev[2 * c + 1], 0));
    B200_CK(cudaMemcpy2DAsync((char *)host_dest + e0 * es, dest_pitch,
                              m.first + dest_off + e0 * es, pitch, cnt * es, pe_size,
                              cudaMemcpyDeviceToHost, p.out));
  }
  /* the caller's stream continues after the last copy out */
  B200_CK(cudaEventRecord(p.ev[2 * nch + 1], p.out));
  B200_CK(cudaStreamWaitEvent(caller, p.ev[2 * nch + 1], 0));
  return finish(stream, "b200shm_reduce_host");
}

/* ---------------------------------------------------------------------------
 * b200shm_reduce_noalloc: the all-reduce for callers that cannot allocate
 * device memory.
 *
 * Some callers of this code cannot call cudaMalloc: a host runtime that
 * owns all device memory through its own pool and hands out only buffers it
 * has already placed, or an embedding that registers its buffers up front
 * and forbids the library any allocation of its own.  They cannot use
 * b200shm_reduce either, because that needs the arena and the
 * deferred-element list that b200shm_init allocates.  This entry point
 * takes caller-owned device buffers directly and allocates nothing: the one
 * piece of scratch the reduction needs -- the list of float MIN/MAX
 * elements whose result depends on operand order (NaN, or both +0 and -0,
 * among the inputs), plus its counter and a status word -- lives in the
 * file-scope array below, which every GPU that loads this library holds
 * until the process exits.  The first call on a device resolves the
 * array's device address (set-up, once per device); that first call should
 * come before any stream capture.  Every call blocks until its result is
 * in every dest.
 * ------------------------------------------------------------------------- */
namespace b200 {

/* at most this many elements per member for a float MIN/MAX reduction,
 * since in the worst case every element is deferred */
constexpr uint64_t kNoAllocMaxDeferred = 1ull << 18;
/* [0] deferred count, [1] status bits, [2] the replay's exit counter,
 * [32 ..] deferred element indices:
 * 2 MiB + 256 bytes */
static __device__ __align__(256) unsigned long long g_noalloc_scratch[32 + kNoAllocMaxDeferred];

/* Device address of g_noalloc_scratch, resolved once per device with that
 * device current (in host code the symbol names a host-side stand-in). */
static int noalloc_scratch(unsigned long long **out) {
  static std::mutex mu;
  static unsigned long long *addr[256] = {nullptr};
  int dev = 0;
  B200_CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 256) return fail(B200SHM_ERR_UNSUPPORTED, "device ordinal %d", dev);
  std::lock_guard<std::mutex> lk(mu);
  if (addr[dev] == nullptr) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    addr[dev] = (unsigned long long *)p;
  }
  *out = addr[dev];
  return B200SHM_OK;
}

}  // namespace b200

extern "C" int b200shm_reduce_noalloc(int op, int dtype, int algo, int npes, void *dest,
                                      uint64_t dest_stride, const void *source,
                                      uint64_t source_stride, uint64_t nelems, void *stream) {
  using namespace b200;
  int rc = reduce_check(op, dtype, algo, npes);
  if (rc) return rc;
  if (nelems == 0) return B200SHM_OK;
  if (dest == nullptr || source == nullptr)
    return fail(B200SHM_ERR_ARG, "reduce_noalloc: null buffer");
  const uint64_t es = (uint64_t)kDtypeSize[dtype];
  if (nelems > UINT64_MAX / es)
    return fail(B200SHM_ERR_ARG, "reduce_noalloc: nelems %llu overflows the row size",
                (unsigned long long)nelems);
  const uint64_t bytes = nelems * es;
  if (npes > 1 && (dest_stride < bytes || source_stride < bytes))
    return fail(B200SHM_ERR_ARG, "reduce_noalloc: member stride smaller than the %llu-byte row",
                (unsigned long long)bytes);
  /* the spans every member's rows cover: [buf, buf + (npes-1)*stride + bytes) */
  const uint64_t rows = (uint64_t)(npes - 1);
  if ((rows && (dest_stride > (UINT64_MAX - bytes) / rows ||
                source_stride > (UINT64_MAX - bytes) / rows)))
    return fail(B200SHM_ERR_ARG, "reduce_noalloc: member strides overflow the address space");
  const uint64_t dspan = rows * dest_stride + bytes, sspan = rows * source_stride + bytes;
  const uint64_t d0 = (uint64_t)(uintptr_t)dest, s0 = (uint64_t)(uintptr_t)source;
  if (d0 > UINT64_MAX - dspan || s0 > UINT64_MAX - sspan)
    return fail(B200SHM_ERR_ARG, "reduce_noalloc: buffer span wraps the address space");
  /* The kernels read every member's source row of a column while other
   * CTAs write dest rows, and the float MIN/MAX replay reads the sources
   * after the dests of other elements are written: so no dest row may
   * touch any source row, except that a dest row may be its own member's
   * source row (in place: same base, same stride).  Source rows are
   * disjoint and sorted (stride >= row size), so a dest row can only touch
   * the source row at or before its start and the one after: O(npes). */
  const bool in_place = d0 == s0 && (dest_stride == source_stride || npes == 1);
  for (uint64_t i = 0; i < (uint64_t)npes; i++) {
    const uint64_t di = d0 + i * dest_stride;
    uint64_t jc = 0;
    if (npes > 1 && di >= s0) jc = (di - s0) / source_stride;
    for (uint64_t j = jc; j <= jc + 1 && j < (uint64_t)npes; j++) {
      if (in_place && j == i) continue;
      if (overlaps(di, bytes, s0 + j * source_stride, bytes))
        return fail(B200SHM_ERR_ARG,
                    "reduce_noalloc: member %llu's dest row overlaps member %llu's source row",
                    (unsigned long long)i, (unsigned long long)j);
    }
  }
  const bool minmax_float = (op == B200SHM_MIN || op == B200SHM_MAX) &&
                            (dtype == B200SHM_F32 || dtype == B200SHM_F64 ||
                             dtype == B200SHM_F80);
  if (minmax_float && nelems > kNoAllocMaxDeferred)
    return fail(B200SHM_ERR_UNSUPPORTED,
                "reduce_noalloc: float MIN/MAX is limited to %llu elements per member (the "
                "static deferred list); use b200shm_reduce for more",
                (unsigned long long)kNoAllocMaxDeferred);
  unsigned long long *scratch = nullptr;
  if ((rc = noalloc_scratch(&scratch))) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  RArgs a = reduce_args((const char *)source, (char *)dest, source_stride, dest_stride, npes,
                        nelems, algo);
  a.fix_count = scratch;
  a.status = (int *)(scratch + 1);
  a.fix_done = scratch + 2;
  a.fix_list = scratch + 32;
  a.fix_cap = kNoAllocMaxDeferred;
  /* the scratch keeps the previous call's contents: clear the counter, the
   * status word and the replay's exit counter first */
  B200_CK(cudaMemsetAsync(scratch, 0, 3 * sizeof(unsigned long long), s));
  const bool aligned = (((uintptr_t)dest | (uintptr_t)source | dest_stride | source_stride) & 15u) == 0;
  if ((rc = reduce_dispatch(op, dtype, a, aligned, s))) return rc;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "b200shm_reduce_noalloc launch");
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "b200shm_reduce_noalloc");
  unsigned long long status = 0;
  e = cudaMemcpy(&status, scratch + 1, sizeof(status), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "b200shm_reduce_noalloc status");
  if (status)
    return fail(B200SHM_ERR_NOMEM, "reduce_noalloc: deferred-element list overflowed");
  return B200SHM_OK;
}
