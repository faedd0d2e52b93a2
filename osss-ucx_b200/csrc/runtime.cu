/*
 * runtime.cu -- arena, host<->heap copies and error handling of the B200
 * engine.
 *
 * The reference gives every PE (an OS process) its own heap registered
 * with UCX (src/shmemc/ucx/init.c:174-218) and a dlmalloc mspace on top
 * (src/api/allocator/memalloc.c).  Here all PEs share one HBM arena: PE p
 * owns slice p, and symmetric allocation is one allocator over slice
 * offsets, which is symmetric by construction (the reference gets symmetry
 * by having every PE allocate in the same order, with a barrier in
 * shmem_malloc, src/api/shmalloc.c:47-61).  The allocator runs on the
 * device (heap_core.cuh, heap.cu).
 */
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <atomic>
#include <mutex>

#include "internal.cuh"

namespace b200 {

static State g_state;
State &st() { return g_state; }

static thread_local char t_err[512] = "";
static std::atomic<unsigned long long> g_launches{0};
void count_launch(unsigned n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
void uncount_launches(unsigned long long n) { g_launches.fetch_sub(n, std::memory_order_relaxed); }

int fail(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(t_err, sizeof(t_err), fmt, ap);
  va_end(ap);
  return code;
}

int cuda_fail(cudaError_t e, const char *what) {
  return fail(B200SHM_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

int take_status(const char *what) {
  volatile int *h = st().h_status;
  if (h == nullptr) return B200SHM_OK;
  const int bits = *h;
  if (bits == 0) return B200SHM_OK;
  *h = 0;
  if (bits & B200SHM_STATUS_TIMEOUT)
    return fail(B200SHM_ERR_TIMEOUT, "%s: a device wait ran out of its spin budget", what);
  if (bits & B200SHM_STATUS_BADREQ)
    return fail(B200SHM_ERR_ARG, "%s: a request named a PE or offset outside the heap", what);
  return fail(B200SHM_ERR_NOMEM,
              "%s: more order-dependent MIN/MAX elements than the deferred list holds", what);
}

int finish(void *stream_arg, const char *what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, what);
  if (stream_arg == nullptr) {
    e = cudaStreamSynchronize(st().stream);
    if (e != cudaSuccess) return cuda_fail(e, what);
    return take_status(what);
  }
  return B200SHM_OK;
}

int grid_sms() {
  if (st().up) return st().sm_count;
  static std::atomic<int> sms[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    (void)cudaGetLastError();
    return st().sm_count;
  }
  int n = sms[dev].load(std::memory_order_relaxed);
  if (n == 0) {
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1) {
      (void)cudaGetLastError();
      return st().sm_count;
    }
    sms[dev].store(n, std::memory_order_relaxed);
  }
  return n;
}

int check_team(int pe_start, int pe_stride, int pe_size) {
  if (!st().up) return fail(B200SHM_ERR_STATE, "b200shm is not initialised");
  if (pe_size < 1) return fail(B200SHM_ERR_ARG, "team size %d < 1", pe_size);
  if (pe_start < 0) return fail(B200SHM_ERR_ARG, "team start %d < 0", pe_start);
  if (pe_stride < 1 && pe_size > 1)
    return fail(B200SHM_ERR_ARG, "team stride %d < 1", pe_stride);
  const int64_t last = (int64_t)pe_start + (int64_t)(pe_size - 1) * (pe_size > 1 ? pe_stride : 0);
  if (last >= st().npes)
    return fail(B200SHM_ERR_ARG, "team member PE %lld >= npes %d", (long long)last,
                st().npes);
  return B200SHM_OK;
}

int check_extent(uint64_t off, uint64_t bytes, const char *what) {
  if (off > st().slice || bytes > st().slice - off)
    return fail(B200SHM_ERR_ARG, "%s [%llu, +%llu) exceeds the %llu-byte heap slice",
                what, (unsigned long long)off, (unsigned long long)bytes,
                (unsigned long long)st().slice);
  return B200SHM_OK;
}

}  // namespace b200

using namespace b200;

extern "C" {

const char *b200shm_last_error(void) { return t_err; }
unsigned long long b200shm_launch_count(void) { return g_launches.load(); }
int b200shm_initialized(void) { return st().up ? 1 : 0; }
int b200shm_n_pes(void) { return st().npes; }
uint64_t b200shm_heap_slice(void) { return st().slice; }
void *b200shm_heap_base(void) { return st().base; }
void *b200shm_stream(void) { return (void *)st().stream; }

int b200shm_init(int npes, uint64_t heap_bytes_per_pe, int flags) {
  State &s = st();
  if (s.up) return fail(B200SHM_ERR_STATE, "b200shm_init called twice");
  if (npes < 1 || npes > (1 << 20)) return fail(B200SHM_ERR_ARG, "npes %d out of range", npes);
  const uint64_t two_mib = 2ull << 20;
  uint64_t slice = (heap_bytes_per_pe + two_mib - 1) / two_mib * two_mib;
  if (slice == 0) slice = two_mib;
  int dev = 0;
  B200_CK(cudaGetDevice(&dev));
  cudaDeviceProp prop;
  B200_CK(cudaGetDeviceProperties(&prop, dev));
  if (prop.major < 10)
    return fail(B200SHM_ERR_UNSUPPORTED, "device %d is sm_%d%d; this build targets sm_100a",
                dev, prop.major, prop.minor);
  s.device = dev;
  s.sm_count = prop.multiProcessorCount;
  s.managed = (flags & B200SHM_INIT_MANAGED) != 0;
  const uint64_t total = slice * (uint64_t)npes;
  cudaError_t e = s.managed ? cudaMallocManaged((void **)&s.base, total)
                            : cudaMalloc((void **)&s.base, total);
  if (e != cudaSuccess) {
    s.base = nullptr;
    return fail(B200SHM_ERR_NOMEM, "arena of %llu bytes: %s", (unsigned long long)total,
                cudaGetErrorString(e));
  }
  s.flag_rounds = 64;
  const uint64_t flag_words = (uint64_t)npes * (uint64_t)s.flag_rounds * 8ull;
  e = cudaMalloc((void **)&s.flags, flag_words * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(s.flags, 0, flag_words * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaHostAlloc((void **)&s.h_status, sizeof(int) * 16, cudaHostAllocMapped);
  if (e == cudaSuccess) {
    memset(s.h_status, 0, sizeof(int) * 16);
    e = cudaHostGetDevicePointer((void **)&s.d_status, s.h_status, 0);
  }
  s.fix_cap = 1ull << 22;
  if (e == cudaSuccess) e = cudaMalloc((void **)&s.fix_list, s.fix_cap * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc((void **)&s.fix_count, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc((void **)&s.call_fix, 2 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(s.call_fix, 0, 2 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    cudaFree(s.base);
    cudaFree(s.flags);
    cudaFreeHost(s.h_status);
    cudaFree(s.fix_list);
    cudaFree(s.fix_count);
    cudaFree(s.call_fix);
    s = State();
    return cuda_fail(e, "b200shm_init");
  }
  s.npes = npes;
  s.slice = slice;
  const int hrc = heap_setup(slice); /* the allocator's state, on the device */
  if (hrc != B200SHM_OK) {
    cudaStreamDestroy(s.stream);
    cudaFree(s.base);
    cudaFree(s.flags);
    cudaFreeHost(s.h_status);
    cudaFree(s.fix_list);
    cudaFree(s.fix_count);
    cudaFree(s.call_fix);
    s = State();
    return hrc;
  }
  s.up = true;
  return B200SHM_OK;
}

int b200shm_finalize(void) {
  State &s = st();
  if (!s.up) return fail(B200SHM_ERR_STATE, "b200shm is not initialised");
  cudaStreamSynchronize(s.stream);
  cudaStreamDestroy(s.stream);
  cudaFree(s.base);
  cudaFree(s.flags);
  cudaFreeHost(s.h_status);
  cudaFree(s.fix_list);
  cudaFree(s.fix_count);
  cudaFree(s.call_fix);
  heap_teardown();
  span_teardown();
  s = State();
  return B200SHM_OK;
}

void *b200shm_ptr(int pe, uint64_t off) {
  const State &s = st();
  if (!s.up || pe < 0 || pe >= s.npes || off >= s.slice) return nullptr;
  return s.base + (uint64_t)pe * s.slice + off;
}

int b200shm_quiet(void) {
  if (!st().up) return fail(B200SHM_ERR_STATE, "b200shm is not initialised");
  B200_CK(cudaStreamSynchronize(st().stream));
  return B200SHM_OK;
}

int b200shm_malloc(uint64_t bytes, uint64_t align, uint64_t *off) {
  if (!st().up) return fail(B200SHM_ERR_STATE, "b200shm is not initialised");
  if (off == nullptr) return fail(B200SHM_ERR_ARG, "null offset pointer");
  if (align < 256) align = 256; /* keeps every object 128-bit and TMA aligned */
  if (align & (align - 1)) return fail(B200SHM_ERR_ARG, "alignment %llu is not a power of two",
                                       (unsigned long long)align);
  if (bytes > st().slice) return fail(B200SHM_ERR_NOMEM, "symmetric heap exhausted (%llu bytes requested)",
                                      (unsigned long long)bytes);
  return heap_alloc(bytes, align, off);
}

int b200shm_free(uint64_t off) {
  if (!st().up) return fail(B200SHM_ERR_STATE, "b200shm is not initialised");
  return heap_release(off);
}

uint64_t b200shm_heap_free_bytes(void) { return st().up ? heap_free_bytes() : 0; }

/* One 2-D copy moves all members' rows when the member pitch fits the
 * copy engine's pitch limit; otherwise one copy per member. */
static int rows_copy(void *dst, size_t dpitch, const void *src, size_t spitch, size_t width,
                     size_t height, cudaMemcpyKind kind, cudaStream_t s) {
  if (width == 0 || height == 0) return B200SHM_OK;
  const size_t pitch_limit = (size_t)1 << 31;
  if (height == 1) {
    B200_CK(cudaMemcpyAsync(dst, src, width, kind, s));
  } else if (dpitch < pitch_limit && spitch < pitch_limit) {
    B200_CK(cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, height, kind, s));
  } else {
    for (size_t r = 0; r < height; r++)
      B200_CK(cudaMemcpyAsync((char *)dst + r * dpitch, (const char *)src + r * spitch, width,
                              kind, s));
  }
  return B200SHM_OK;
}

int b200shm_put_host(int pe_start, int pe_stride, int pe_count, uint64_t off,
                     const void *host_src, uint64_t bytes_per_pe, void *stream) {
  int rc = check_team(pe_start, pe_stride, pe_count);
  if (rc) return rc;
  if ((rc = check_extent(off, bytes_per_pe, "put_host"))) return rc;
  Members m = members(pe_start, pe_stride, pe_count);
  rc = rows_copy(m.first + off, m.step, host_src, bytes_per_pe, bytes_per_pe, pe_count,
                 cudaMemcpyHostToDevice, pick_stream(stream));
  if (rc) return rc;
  return finish(stream, "b200shm_put_host");
}

int b200shm_get_host(void *host_dst, int pe_start, int pe_stride, int pe_count, uint64_t off,
                     uint64_t bytes_per_pe, void *stream) {
  int rc = check_team(pe_start, pe_stride, pe_count);
  if (rc) return rc;
  if ((rc = check_extent(off, bytes_per_pe, "get_host"))) return rc;
  Members m = members(pe_start, pe_stride, pe_count);
  rc = rows_copy(host_dst, bytes_per_pe, m.first + off, m.step, bytes_per_pe, pe_count,
                 cudaMemcpyDeviceToHost, pick_stream(stream));
  if (rc) return rc;
  return finish(stream, "b200shm_get_host");
}

int b200shm_memcpy(void *dst, const void *src, uint64_t bytes, void *stream) {
  if (!st().up) return fail(B200SHM_ERR_STATE, "b200shm is not initialised");
  if (bytes == 0) return B200SHM_OK;
  if (!dst || !src) return fail(B200SHM_ERR_ARG, "memcpy: null pointer");
  B200_CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, pick_stream(stream)));
  return finish(stream, "b200shm_memcpy");
}

int b200shm_memcpy_strided(void *dst, int64_t dst_stride, const void *src, int64_t src_stride,
                           uint64_t elem_bytes, uint64_t nelems, void *stream) {
  if (!st().up) return fail(B200SHM_ERR_STATE, "b200shm is not initialised");
  if (nelems == 0 || elem_bytes == 0) return B200SHM_OK;
  if (!dst || !src) return fail(B200SHM_ERR_ARG, "memcpy_strided: null pointer");
  if (dst_stride < 1 || src_stride < 1)
    return fail(B200SHM_ERR_ARG, "memcpy_strided: strides must be positive");
  const uint64_t dp = (uint64_t)dst_stride * elem_bytes, sp = (uint64_t)src_stride * elem_bytes;
  if (dp / elem_bytes != (uint64_t)dst_stride || sp / elem_bytes != (uint64_t)src_stride)
    return fail(B200SHM_ERR_ARG, "memcpy_strided: stride overflows");
  cudaStream_t s = pick_stream(stream);
  if (dp == elem_bytes && sp == elem_bytes) {
    B200_CK(cudaMemcpyAsync(dst, src, elem_bytes * nelems, cudaMemcpyDefault, s));
  } else {
    /* one 2-D copy: a row per element, the strides as pitches */
    B200_CK(cudaMemcpy2DAsync(dst, dp, src, sp, elem_bytes, nelems, cudaMemcpyDefault, s));
  }
  return finish(stream, "b200shm_memcpy_strided");
}

int b200shm_memset(int pe_start, int pe_stride, int pe_count, uint64_t off, int byte,
                   uint64_t bytes_per_pe, void *stream) {
  int rc = check_team(pe_start, pe_stride, pe_count);
  if (rc) return rc;
  if ((rc = check_extent(off, bytes_per_pe, "memset"))) return rc;
  Members m = members(pe_start, pe_stride, pe_count);
  if (bytes_per_pe && pe_count)
    B200_CK(cudaMemset2DAsync(m.first + off, m.step, byte, bytes_per_pe, pe_count,
                              pick_stream(stream)));
  return finish(stream, "b200shm_memset");
}

}  // extern "C"
