/*
 * heap.cu -- host side of the device allocator (heap_core.cuh): its set-up
 * with the arena, and the one-thread kernels behind b200shm_malloc /
 * b200shm_free.  The serving loop calls the same device functions inline.
 */
#include <stdint.h>
#include <string.h>

#include <mutex>

#include "heap_core.cuh"
#include "internal.cuh"

namespace b200 {
namespace {

enum { kOpAlloc = 0, kOpFree = 1 };

__global__ void k_heap_init(HeapDev h, unsigned nunits, unsigned shift) {
  HeapCtl *c = h.ctl;
  c->lock = 0;
  c->fl_map = 0;
  for (int i = 0; i < kHeapFL; i++) {
    c->sl_map[i] = 0;
    for (int j = 0; j < kHeapSL; j++) c->head[i][j] = kHeapNil;
  }
  c->free_units = 0;
  c->blocks_used = 0;
  c->nunits = nunits;
  c->unit_shift = shift;
  c->err = 0;
  h.size[0] = nunits;
  h.prev_phys[0] = kHeapNil;
  heap_link(h, 0);
  if (h.free_bytes_host) *h.free_bytes_host = (unsigned long long)nunits << shift;
  __threadfence_system();
}

/* out[0] = status (kHeap*), out[1] = unit */
__global__ void k_heap_op(HeapDev h, int op, unsigned a, unsigned b, unsigned long long *out) {
  if (!heap_lock(h)) {
    out[0] = kHeapBusy;
    __threadfence_system();
    return;
  }
  if (op == kOpAlloc) {
    const unsigned u = heap_alloc_locked(h, a, b);
    out[0] = u == kHeapNil ? kHeapNoMem : kHeapOk;
    out[1] = u;
  } else {
    out[0] = (unsigned long long)heap_free_locked(h, a);
  }
  heap_unlock(h);
  __threadfence_system();
}

struct Heap {
  HeapDev dev{};
  char *mem = nullptr;                 /* device: control block and arrays */
  unsigned long long *h_map = nullptr; /* mapped host: [0] free bytes, [8..9] an op's result */
  unsigned long long *d_map = nullptr;
  cudaStream_t stream = nullptr;
  unsigned shift = 8;
  unsigned nunits = 0;
  std::mutex mu;
};
Heap g_heap;

/* One operation: launch, wait, read the result word pair.  Host calls are
 * serialised (allocation is not on any hot path, and one result slot then
 * serves every thread); the serving loop takes the device lock on its own. */
int heap_call(int op, unsigned a, unsigned b, unsigned long long *res) {
  std::lock_guard<std::mutex> lk(g_heap.mu);
  volatile unsigned long long *h = g_heap.h_map + 8;
  h[0] = ~0ull;
  k_heap_op<<<1, 1, 0, g_heap.stream>>>(g_heap.dev, op, a, b, g_heap.d_map + 8);
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(g_heap.stream);
  if (e != cudaSuccess) return cuda_fail(e, "symmetric heap");
  res[0] = h[0];
  res[1] = h[1];
  if (res[0] == kHeapBusy)
    return fail(B200SHM_ERR_TIMEOUT, "symmetric heap: the allocator lock was not obtained");
  return B200SHM_OK;
}

}  // namespace

HeapDev heap_dev() { return g_heap.dev; }

int heap_setup(uint64_t slice) {
  Heap &H = g_heap;
  unsigned shift = 8;
  while ((slice >> shift) > kHeapMaxUnits) shift++;
  const uint64_t n = slice >> shift;
  H.shift = shift;
  H.nunits = (unsigned)n;
  const size_t ctl = (sizeof(HeapCtl) + 255) & ~(size_t)255;
  const size_t words = ((size_t)n * 4 + 255) & ~(size_t)255;
  const size_t bytes = ctl + 4 * words + (((size_t)n + 255) & ~(size_t)255);
  B200_CK(cudaMalloc((void **)&H.mem, bytes));
  cudaError_t e = cudaMemset(H.mem, 0, bytes);
  if (e == cudaSuccess)
    e = cudaHostAlloc((void **)&H.h_map, 16 * sizeof(unsigned long long), cudaHostAllocMapped);
  if (e == cudaSuccess) e = cudaHostGetDevicePointer((void **)&H.d_map, H.h_map, 0);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&H.stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    heap_teardown();
    return cuda_fail(e, "symmetric heap set-up");
  }
  HeapDev &d = H.dev;
  d.ctl = (HeapCtl *)H.mem;
  d.size = (unsigned *)(H.mem + ctl);
  d.prev_phys = (unsigned *)(H.mem + ctl + words);
  d.next_free = (unsigned *)(H.mem + ctl + 2 * words);
  d.prev_free = (unsigned *)(H.mem + ctl + 3 * words);
  d.flags = (unsigned char *)(H.mem + ctl + 4 * words);
  d.free_bytes_host = H.d_map;
  k_heap_init<<<1, 1, 0, H.stream>>>(d, H.nunits, shift);
  count_launch();
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(H.stream);
  if (e != cudaSuccess) {
    heap_teardown();
    return cuda_fail(e, "symmetric heap set-up");
  }
  return B200SHM_OK;
}

void heap_teardown() {
  Heap &H = g_heap;
  if (H.stream) {
    cudaStreamSynchronize(H.stream);
    cudaStreamDestroy(H.stream);
  }
  if (H.mem) cudaFree(H.mem);
  if (H.h_map) cudaFreeHost(H.h_map);
  H.mem = nullptr;
  H.h_map = H.d_map = nullptr;
  H.stream = nullptr;
  H.dev = HeapDev{};
  H.nunits = 0;
}

unsigned heap_unit_shift() { return g_heap.shift; }

int heap_alloc(uint64_t bytes, uint64_t align, uint64_t *off) {
  Heap &H = g_heap;
  if (!H.mem) return fail(B200SHM_ERR_STATE, "b200shm is not initialised");
  const uint64_t units = heap_units(bytes ? bytes : 1, H.shift);
  uint64_t au = align >> H.shift;
  if (au < 1) au = 1;
  if (units > H.nunits || au > H.nunits)
    return fail(B200SHM_ERR_NOMEM, "symmetric heap exhausted (%llu bytes requested)",
                (unsigned long long)bytes);
  unsigned long long res[2];
  int rc = heap_call(kOpAlloc, (unsigned)units, (unsigned)au, res);
  if (rc) return rc;
  if (res[0] != kHeapOk)
    return fail(B200SHM_ERR_NOMEM, "symmetric heap exhausted (%llu bytes requested)",
                (unsigned long long)bytes);
  *off = res[1] << H.shift;
  return B200SHM_OK;
}

int heap_release(uint64_t off) {
  Heap &H = g_heap;
  if (!H.mem) return fail(B200SHM_ERR_STATE, "b200shm is not initialised");
  if (off & ((1ull << H.shift) - 1) || (off >> H.shift) >= H.nunits)
    return fail(B200SHM_ERR_ARG, "offset %llu is not an allocated symmetric object",
                (unsigned long long)off);
  unsigned long long res[2];
  int rc = heap_call(kOpFree, (unsigned)(off >> H.shift), 0, res);
  if (rc) return rc;
  if (res[0] != kHeapOk)
    return fail(B200SHM_ERR_ARG, "offset %llu is not an allocated symmetric object",
                (unsigned long long)off);
  return B200SHM_OK;
}

uint64_t heap_free_bytes() {
  return g_heap.h_map ? *(volatile unsigned long long *)g_heap.h_map : 0;
}

}  // namespace b200
