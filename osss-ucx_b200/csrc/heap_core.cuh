/*
 * heap_core.cuh -- the symmetric-heap allocator, run on the device.
 *
 * The reference gives each PE a heap registered with UCX and runs dlmalloc
 * over it (src/shmemc/ucx/init.c:174-218, src/api/allocator/memalloc.c:
 * 29-93); every PE allocates in the same order, so the same offset comes
 * back everywhere (src/api/shmalloc.c:47-77).  Here one allocator hands out
 * offsets that are valid in every PE's slice of the arena, and it lives on
 * the GPU: its state is in device memory and every operation is a device
 * function run by one thread under a spin lock taken with an atomic
 * compare-and-swap.  The host's b200shm_malloc / b200shm_free launch a
 * one-thread kernel that runs it; the serving loop runs it inline, to admit
 * a request whose dest it allocates only when the heap has room.
 *
 * Algorithm: two-level segregated fit over the slice in units of U bytes
 * (256, or more for slices above 1 GiB): free blocks sit in lists by size
 * class (a power of two, cut into 16 sub-ranges), two bitmaps say which
 * lists are non-empty, so finding a block is two find-first-set operations;
 * a freed block merges with free physical neighbours at once (boundary
 * links per block start), so no two free blocks are ever adjacent.  Every
 * metadata access is volatile (L2, never a stale L1 line) and the lock's
 * acquire and release are fenced.
 */
#ifndef B200SHM_HEAP_CORE_CUH
#define B200SHM_HEAP_CORE_CUH

#include <stdint.h>

namespace b200 {

constexpr unsigned kHeapNil = 0xFFFFFFFFu;
constexpr int kHeapSLog = 4, kHeapSL = 1 << kHeapSLog; /* sub-ranges per power of two */
constexpr int kHeapFL = 29;                             /* first-level classes          */
constexpr unsigned kHeapMaxUnits = 1u << 22;            /* units per slice, at most     */
constexpr unsigned char kBlkFree = 1, kBlkStart = 2;

/* allocator state (device memory) */
struct HeapCtl {
  unsigned lock;
  unsigned fl_map;
  unsigned sl_map[kHeapFL];
  unsigned head[kHeapFL][kHeapSL];
  unsigned long long free_units;
  unsigned long long blocks_used;
  unsigned nunits;
  unsigned unit_shift; /* log2 of bytes per unit */
  int err;             /* sticky: lock not obtained, or metadata found inconsistent */
};

/* arrays indexed by unit; entries are meaningful at block starts */
struct HeapDev {
  HeapCtl *ctl;
  unsigned *size;      /* units of the block that starts here */
  unsigned *prev_phys; /* start of the physically preceding block, or nil */
  unsigned *next_free, *prev_free;
  unsigned char *flags;
  unsigned long long *free_bytes_host; /* mapped host word: free bytes after each operation */
};

enum { kHeapOk = 0, kHeapNoMem = 1, kHeapBusy = 2, kHeapBadFree = 3 };

/* The allocator's bookkeeping is plain code (host and device): the device
 * runs it under the lock below; a host build of the same functions is how
 * the CPU tests check it. */
#define B200_HEAP_FN __host__ __device__ __forceinline__

template <class T>
B200_HEAP_FN T hv(const T *p) {
  return *(const volatile T *)p;
}
template <class T>
B200_HEAP_FN void hs(T *p, T v) {
  *(volatile T *)p = v;
}
B200_HEAP_FN int heap_clz(unsigned n) {
#ifdef __CUDA_ARCH__
  return __clz(n);
#else
  return n ? __builtin_clz(n) : 32;
#endif
}
B200_HEAP_FN int heap_ffs(unsigned n) {
#ifdef __CUDA_ARCH__
  return __ffs(n);
#else
  return __builtin_ffs((int)n);
#endif
}

/* class of a free block of n units (n >= 1) */
B200_HEAP_FN void heap_class(unsigned n, int &fl, int &sl) {
  if (n < (unsigned)kHeapSL) {
    fl = 0;
    sl = (int)n;
  } else {
    const int f = 31 - heap_clz(n);
    fl = f - kHeapSLog + 1;
    sl = (int)(n >> (f - kHeapSLog)) - kHeapSL;
  }
}

B200_HEAP_FN void heap_unlink(const HeapDev &h, unsigned b) {
  HeapCtl *c = h.ctl;
  int fl, sl;
  heap_class(hv(&h.size[b]), fl, sl);
  const unsigned p = hv(&h.prev_free[b]), n = hv(&h.next_free[b]);
  if (p != kHeapNil) hs(&h.next_free[p], n);
  else hs(&c->head[fl][sl], n);
  if (n != kHeapNil) hs(&h.prev_free[n], p);
  if (hv(&c->head[fl][sl]) == kHeapNil) {
    const unsigned m = hv(&c->sl_map[fl]) & ~(1u << sl);
    hs(&c->sl_map[fl], m);
    if (!m) hs(&c->fl_map, hv(&c->fl_map) & ~(1u << fl));
  }
  hs(&h.flags[b], (unsigned char)(hv(&h.flags[b]) & ~kBlkFree));
  hs(&c->free_units, hv(&c->free_units) - hv(&h.size[b]));
}

B200_HEAP_FN void heap_link(const HeapDev &h, unsigned b) {
  HeapCtl *c = h.ctl;
  int fl, sl;
  heap_class(hv(&h.size[b]), fl, sl);
  const unsigned n = hv(&c->head[fl][sl]);
  hs(&h.next_free[b], n);
  hs(&h.prev_free[b], kHeapNil);
  if (n != kHeapNil) hs(&h.prev_free[n], b);
  hs(&c->head[fl][sl], b);
  hs(&c->sl_map[fl], hv(&c->sl_map[fl]) | (1u << sl));
  hs(&c->fl_map, hv(&c->fl_map) | (1u << fl));
  hs(&h.flags[b], (unsigned char)(kBlkStart | kBlkFree));
  hs(&c->free_units, hv(&c->free_units) + hv(&h.size[b]));
}

/* a free block of at least n units, or nil: the first block of the first
 * non-empty class whose every block is large enough, else a bounded scan
 * of n's own class */
B200_HEAP_FN unsigned heap_find(const HeapDev &h, unsigned n) {
  HeapCtl *c = h.ctl;
  int fl, sl;
  unsigned r = n;
  if (n >= (unsigned)kHeapSL) {
    const int f = 31 - heap_clz(n);
    r = n + (1u << (f - kHeapSLog)) - 1u;
    if (r < n) r = 0xFFFFFFFFu;
  }
  heap_class(r, fl, sl);
  if (fl < kHeapFL) {
    unsigned sm = hv(&c->sl_map[fl]) & (~0u << sl);
    if (!sm) {
      const unsigned fm = fl + 1 < 32 ? hv(&c->fl_map) & (~0u << (fl + 1)) : 0u;
      if (fm) {
        fl = heap_ffs(fm) - 1;
        sm = hv(&c->sl_map[fl]);
      }
    }
    if (sm) return hv(&c->head[fl][heap_ffs(sm) - 1]);
  }
  heap_class(n, fl, sl);
  unsigned b = hv(&c->head[fl][sl]);
  for (int k = 0; k < 256 && b != kHeapNil; k++, b = hv(&h.next_free[b]))
    if (hv(&h.size[b]) >= n) return b;
  return kHeapNil;
}

/* cut block b (not in a list) to n units; the rest becomes a free block */
B200_HEAP_FN void heap_trim(const HeapDev &h, unsigned b, unsigned n) {
  const unsigned sz = hv(&h.size[b]);
  if (sz <= n) return;
  const unsigned c = b + n, rest = sz - n;
  hs(&h.size[b], n);
  hs(&h.size[c], rest);
  hs(&h.prev_phys[c], b);
  if (c + rest < hv(&h.ctl->nunits)) hs(&h.prev_phys[c + rest], c);
  heap_link(h, c);
}

__device__ __forceinline__ bool heap_lock(const HeapDev &h) {
  for (unsigned i = 0; i < (1u << 22); i++) { /* bounded: ~0.5 s */
    if (atomicCAS(&h.ctl->lock, 0u, 1u) == 0u) {
      __threadfence();
      return true;
    }
    __nanosleep(100);
  }
  atomicOr(&h.ctl->err, 1);
  return false;
}
__device__ __forceinline__ void heap_unlock(const HeapDev &h) {
  if (h.free_bytes_host)
    hs(h.free_bytes_host, hv(&h.ctl->free_units) << hv(&h.ctl->unit_shift));
  __threadfence();
  atomicExch(&h.ctl->lock, 0u);
}

/* Allocate `units` units aligned to `align` units (a power of two); the
 * caller holds the lock.  Returns the first unit or nil. */
B200_HEAP_FN unsigned heap_alloc_locked(const HeapDev &h, unsigned units,
                                                      unsigned align) {
  if (units == 0) units = 1;
  const unsigned long long want = (unsigned long long)units + (align > 1 ? align - 1 : 0);
  if (want > hv(&h.ctl->free_units)) return kHeapNil;
  unsigned b = heap_find(h, (unsigned)want);
  if (b == kHeapNil) return kHeapNil;
  heap_unlink(h, b);
  const unsigned s = (b + align - 1) & ~(align - 1);
  if (s > b) { /* the lead before the aligned start stays free */
    const unsigned sz = hv(&h.size[b]), lead = s - b;
    hs(&h.size[b], lead);
    hs(&h.size[s], sz - lead);
    hs(&h.prev_phys[s], b);
    if (s + sz - lead < hv(&h.ctl->nunits)) hs(&h.prev_phys[s + sz - lead], s);
    heap_link(h, b);
    b = s;
  }
  heap_trim(h, b, units);
  hs(&h.flags[b], kBlkStart);
  hs(&h.ctl->blocks_used, hv(&h.ctl->blocks_used) + 1ull);
  return b;
}

/* Free the block that starts at unit b; the caller holds the lock.
 * kHeapBadFree when b is not the start of an allocated block. */
B200_HEAP_FN int heap_free_locked(const HeapDev &h, unsigned b) {
  const unsigned N = hv(&h.ctl->nunits);
  if (b >= N || hv(&h.flags[b]) != kBlkStart) return kHeapBadFree;
  unsigned sz = hv(&h.size[b]);
  const unsigned nx = b + sz;
  if (nx < N && (hv(&h.flags[nx]) & kBlkFree)) { /* merge the next block */
    heap_unlink(h, nx);
    sz += hv(&h.size[nx]);
    hs(&h.flags[nx], (unsigned char)0);
    hs(&h.size[nx], 0u);
  }
  const unsigned p = hv(&h.prev_phys[b]);
  if (p != kHeapNil && (hv(&h.flags[p]) & kBlkFree)) { /* merge into the previous block */
    heap_unlink(h, p);
    hs(&h.flags[b], (unsigned char)0);
    hs(&h.size[b], 0u);
    sz += hv(&h.size[p]);
    b = p;
  }
  hs(&h.size[b], sz);
  if (b + sz < N) hs(&h.prev_phys[b + sz], b);
  heap_link(h, b);
  hs(&h.ctl->blocks_used, hv(&h.ctl->blocks_used) - 1ull);
  return kHeapOk;
}

/* bytes -> units, and an alignment in bytes -> units (a power of two) */
__host__ __device__ __forceinline__ unsigned long long heap_units(unsigned long long bytes,
                                                                   unsigned shift) {
  return (bytes + (1ull << shift) - 1) >> shift;
}

#ifdef __CUDACC__
/* the engine's allocator state, for kernels that allocate (heap.cu) */
HeapDev heap_dev();
#endif

}  // namespace b200
#endif
