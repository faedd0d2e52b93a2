/*
 * internal.cuh -- state and helpers shared by the CUDA translation units
 * of libb200shm.so.  Not part of the public ABI.
 */
#ifndef B200SHM_INTERNAL_CUH
#define B200SHM_INTERNAL_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/b200shm.h"

namespace b200 {

/* Process-wide engine state (one arena per process and device). */
struct State {
  bool up = false;
  int device = 0;
  int sm_count = 148;
  int npes = 0;
  uint64_t slice = 0;       /* bytes per PE slice (multiple of 2 MiB)      */
  char *base = nullptr;     /* arena: npes * slice bytes                   */
  bool managed = false;
  cudaStream_t stream = nullptr;
  /* library-owned flag words for device barriers: one cache line per
   * (PE, barrier round); cleared after use, so every barrier starts at 0 */
  unsigned long long *flags = nullptr;
  int flag_rounds = 0;
  /* sticky device status bits (B200SHM_STATUS_*), in mapped pinned host
   * memory so a blocking call reads them after its stream synchronises */
  int *h_status = nullptr;
  int *d_status = nullptr;
  /* deferred-element list of the float MIN/MAX reduce (reduce.cu): element
   * indices whose result depends on operand order; scratch owned by the
   * library, shared by all calls (calls that overlap on the GPU race) */
  unsigned long long *fix_list = nullptr;
  unsigned long long *fix_count = nullptr; /* the batch path's count (zeroed per run) */
  /* the per-call path's count and the replay kernel's exit counter: the
   * replay's last CTA sets both back to zero, so they start every call at 0 */
  unsigned long long *call_fix = nullptr;
  uint64_t fix_cap = 0;
};

/* status bits set on the device */
enum {
  B200SHM_STATUS_FIX_OVERFLOW = 1, /* too many order-dependent MIN/MAX elements */
  B200SHM_STATUS_TIMEOUT = 2,      /* a bounded wait gave up                     */
  B200SHM_STATUS_BADREQ = 4        /* an AMO / queued request named a bad target */
};
/* Read and clear the device status bits (after the stream synchronised) and
 * turn them into an error code. */
int take_status(const char *what);
State &st();

/* error reporting: set the calling thread's message, return `code` */
int fail(int code, const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what);
#define B200_CK(call)                                                          \
  do {                                                                         \
    cudaError_t _e = (call);                                                   \
    if (_e != cudaSuccess) return ::b200::cuda_fail(_e, #call);                \
  } while (0)

/* bytes per element of each b200shm_dtype (long double occupies 16) */
static constexpr int kDtypeSize[B200SHM_NDTYPE] = {1, 2, 4, 8, 1, 2, 4, 8, 4, 8, 16, 8, 16};

/* Kernels launched by this library since load (b200shm_launch_count). */
void count_launch(unsigned n = 1);
/* launches recorded into a CUDA graph run only when it is replayed */
void uncount_launches(unsigned long long n);

/* Resolve the stream argument of an entry point. */
inline cudaStream_t pick_stream(void *s) {
  return s ? (cudaStream_t)s : st().stream;
}
/* After enqueueing: check the launch, and block when the caller passed no
 * stream (OpenSHMEM blocking semantics). */
int finish(void *stream_arg, const char *what);

/* Validate a member list against the arena; returns B200SHM_OK or sets the
 * error.  bytes_per_member: the extent [off, off+bytes) every member uses. */
int check_team(int pe_start, int pe_stride, int pe_size);
int check_extent(uint64_t off, uint64_t bytes, const char *what);
/* True when [a, a+na) and [b, b+nb) intersect. */
inline bool overlaps(uint64_t a, uint64_t na, uint64_t b, uint64_t nb) {
  return na && nb && a < b + nb && b < a + na;
}

/* SMs that grids are sized for: the engine's device once b200shm_init has
 * run, else the current device (entry points that need no init). */
int grid_sms();

/* Grid size for a grid-stride kernel: enough CTAs to cover `items` work
 * items with `threads` per CTA, capped at `per_sm` resident CTAs per SM. */
inline unsigned grid_for(uint64_t items, int threads, int per_sm) {
  uint64_t need = (items + (uint64_t)threads - 1) / (uint64_t)threads;
  uint64_t cap = (uint64_t)grid_sms() * (uint64_t)per_sm;
  if (need < 1) need = 1;
  return (unsigned)(need < cap ? need : cap);
}

/* The per-call reduce (reduce.cu), validated and enqueued on stream s. */
int reduce_launch(int op, int dtype, int algo, int pe_start, int pe_stride, int pe_size,
                  uint64_t dest_off, uint64_t src_off, uint64_t nelems, cudaStream_t s);

/* The device allocator of the symmetric heap (heap.cu, heap_core.cuh). */
int heap_setup(uint64_t slice);
void heap_teardown();
void span_teardown(); /* closes the peer mappings still open */
int heap_alloc(uint64_t bytes, uint64_t align, uint64_t *off);
int heap_release(uint64_t off);
uint64_t heap_free_bytes();
unsigned heap_unit_shift();

/* One atomic with operands by value, stream-ordered (amo.cu). */
int amo_one_launch(int amo, int dtype, int pe, uint64_t off, uint64_t value, uint64_t cond,
                   void *fetched, cudaStream_t s);

/* Member addressing: member i of a team lives at
 * base + (pe_start + i*pe_stride) * slice + off. */
struct Members {
  char *first;    /* address of member 0 at offset 0 */
  uint64_t step;  /* pe_stride * slice                */
  int size;
};
inline Members members(int pe_start, int pe_stride, int pe_size) {
  Members m;
  m.first = st().base + (uint64_t)pe_start * st().slice;
  m.step = (uint64_t)pe_stride * st().slice;
  m.size = pe_size;
  return m;
}

}  // namespace b200
#endif
