/*
 * serve.cu -- the serving loop (b200shm_serve_*).
 *
 * In the reference every operation is a blocking call: a collective runs
 * its whole algorithm with flag handshakes (src/shcoll/src/*.c), an atomic
 * or a put is a UCX round trip plus a progress loop (src/shmemc/ucx/
 * comms.c:265-292, 677-762).  For a stream of many small requests that
 * per-call cost dominates.  Here one persistent kernel serves a ring of
 * requests that the host publishes in mapped host memory:
 *
 *  - the host writes a request into its ring slot (sequence word last) and
 *    then the ring's tail, both with release ordering;
 *  - one CTA at a time copies newly published requests into device memory
 *    (the mirror) and opens each to claims by setting its slot's claim
 *    word;
 *  - every request is cut into tiles on the host (a range of elements of a
 *    reduction, a chunk or a run of segments of a copy, one atomic) and
 *    its tiles into at most one share per CTA; a CTA claims a share with
 *    one fetch-and-add on the slot's claim word, only on requests already
 *    mirrored, so no CTA ever holds a claim it cannot serve and no CTA
 *    ever waits for another CTA;
 *  - the CTA that finishes a request's last tile writes its completion word
 *    (sequence, AMO old value, status) to host memory after a system-scope
 *    fence;
 *  - a CTA with no published work sleeps with a growing back-off (at most
 *    128 ns); once the loop has had no new request for the idle limit, or
 *    the host asked it to stop and every published request is mirrored, it
 *    exits, holding no claim; the last CTA out tells the host through a
 *    host word, and the host relaunches the kernel when work arrives again.
 *    Every wait in the kernel is bounded by that limit;
 *  - with a heap budget, the mirror opens requests to claims only while the
 *    heap bytes of the admitted, incomplete ones fit the budget.
 *
 * Results equal the per-call entry points': a reduction combines in the
 * reference algorithm's exact order (a left fold where any order is exact,
 * the algorithm's tree for float SUM/PROD, an exact replay for float
 * MIN/MAX elements whose result depends on operand order).
 */
#include <stddef.h>
#include <stdint.h>
#include <string.h>
#include <time.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <type_traits>
#include <vector>

#include "amo_core.cuh"
#include "heap_core.cuh"
#include "internal.cuh"
#include "reduce_core.cuh"

namespace b200 {
namespace {

constexpr int kServeThreads = 256;
constexpr unsigned long long kStopBit = 1ull << 63;
/* The claim word of a ring slot: [63:40] the request it serves (its low 24
 * bits), [39:24] the number of shares its tiles are cut into, [23:0] the
 * next share to hand out. */
constexpr int kTagShift = 40, kShareShift = 24;
constexpr unsigned long long kField24 = (1ull << 24) - 1;
constexpr unsigned long long kTileLimit = 1ull << 22;
__host__ __device__ __forceinline__ unsigned long long claim_word(unsigned long long r,
                                                                  unsigned long long nshares) {
  return ((r & kField24) << kTagShift) | (nshares << kShareShift);
}
/* The symmetric-heap bytes a request writes, over all the members it
 * writes to: what admission by heap bytes accounts for. */
__host__ __device__ __forceinline__ unsigned long long heap_bytes(const b200shm_request &r) {
  const unsigned long long P = r.pe_size > 0 ? (unsigned long long)r.pe_size : 1ull;
  switch (r.kind) {
  case B200SHM_REQ_REDUCE: {
    const bool w8 = r.dtype == B200SHM_I64 || r.dtype == B200SHM_U64 || r.dtype == B200SHM_F64;
    return r.n * (w8 ? 8ull : 4ull) * P;
  }
  case B200SHM_REQ_FCOLLECT:
  case B200SHM_REQ_ALLTOALL: return r.n * P * P;
  case B200SHM_REQ_PUT:
  case B200SHM_REQ_GET: return r.n;
  default: return 8;
  }
}
/* The bytes one member's dest spans: what the loop allocates for a request
 * whose dest_off is B200SHM_SERVE_ALLOC. */
__host__ __device__ __forceinline__ unsigned long long dest_bytes(const b200shm_request &r) {
  const unsigned long long P = r.pe_size > 0 ? (unsigned long long)r.pe_size : 1ull;
  switch (r.kind) {
  case B200SHM_REQ_REDUCE: {
    const bool w8 = r.dtype == B200SHM_I64 || r.dtype == B200SHM_U64 || r.dtype == B200SHM_F64;
    return r.n * (w8 ? 8ull : 4ull);
  }
  case B200SHM_REQ_FCOLLECT:
  case B200SHM_REQ_ALLTOALL: return r.n * P;
  default: return r.n;
  }
}
constexpr unsigned kMirrorMax = 1024; /* the largest mirror batch */

/* tiles per share: at most one share per CTA */
__host__ __device__ __forceinline__ unsigned long long share_tiles(unsigned long long ntiles,
                                                                   unsigned ctas) {
  return (ntiles + ctas - 1) / ctas;
}
/* Tile sizes.  A tile is one CTA's work, so a smaller tile finishes a large
 * request sooner (and frees its ring slot sooner) at the cost of more
 * claims.  Measured on the serving workload (200k requests/s offered, and
 * the same stream saturated), reduce tiles reading 256 / 128 / 64 KiB:
 * p99 67.5 / 48.5 / 40.7 us, saturated 1.17M / 1.15M / 1.10M requests/s;
 * copy chunks of 16 KiB lost on both counts against 32 KiB. */
constexpr uint64_t kCopyChunk = 32u << 10;       /* bytes per copy tile            */
constexpr uint64_t kReduceTileRead = 128u << 10; /* source bytes per reduce tile   */

/* The tile sizes in force: the defaults above, or B200SHM_SERVE_COPY_CHUNK /
 * B200SHM_SERVE_REDUCE_TILE (bytes, a multiple of 4 KiB from 4 KiB to
 * 16 MiB), read once. */
uint64_t tile_bytes(const char *var, uint64_t dflt) {
  const char *e = getenv(var);
  if (!e) return dflt;
  const unsigned long long v = strtoull(e, nullptr, 0);
  return v >= 4096 && v <= (16ull << 20) && v % 4096 == 0 ? v : dflt;
}
uint64_t copy_chunk() {
  static const uint64_t v = tile_bytes("B200SHM_SERVE_COPY_CHUNK", kCopyChunk);
  return v;
}
uint64_t reduce_tile_read() {
  static const uint64_t v = tile_bytes("B200SHM_SERVE_REDUCE_TILE", kReduceTileRead);
  return v;
}

/* A ring slot (mapped host memory, written by the host). */
struct alignas(16) SReq {
  b200shm_request r;        /* 72 bytes */
  unsigned long long ntiles; /* >= 1 */
  unsigned long long unit;   /* REDUCE: elements per tile; copies: bytes per chunk */
  unsigned long long nseg;   /* copies: segments of r.n bytes */
  unsigned long long spt;    /* copies with small segments: segments per tile, else 0 */
  unsigned long long cps;    /* copies with large segments: chunks per segment */
  unsigned long long seq;    /* ticket + 1 once the slot holds the request; written last */
  /* in the ring: the request's heap bytes (host-written, read by the
   * mirror for admission); in the device copy: when it was mirrored */
  unsigned long long pad;
};
static_assert(sizeof(SReq) == 128, "ring slot of 128 bytes");
static_assert(offsetof(SReq, ntiles) == 9 * 8 && offsetof(SReq, seq) == 14 * 8,
              "the mirror reads ntiles as word 9 and publishes seq as word 14");

/* A completion word (mapped host memory, written by the device), with the
 * device clock (globaltimer, ns) when the request was copied from the
 * ring, when its last tile was claimed and when it completed. */
struct alignas(64) SDone {
  unsigned long long seq; /* ticket + 1 once complete */
  unsigned long long fetched;
  unsigned long long t[3]; /* copied into device memory, last tiles claimed, complete */
  int status;
  int pad[5];
};
static_assert(sizeof(SDone) == 64, "completion record of 64 bytes");

/* Host-written control words (mapped host memory). */
struct SCtl {
  /* requests published, with kStopBit set once the host asked the loop to
   * stop: one word, so a poll is one read of host memory */
  unsigned long long tail;
  unsigned long long pad[7];
  /* written by the device: the launch (epoch) whose CTAs have all left the
   * loop; on a line of its own, away from the host-written words */
  unsigned long long down;
  unsigned long long pad2[7];
};
static_assert(offsetof(SCtl, down) == 64 && sizeof(SCtl) == 128, "host and device lines apart");

/* Device-side state. */
struct SDev {
  unsigned long long cursor;      /* the request whose tiles are handed out  */
  unsigned long long tail_mirror; /* last tail a CTA read from host memory   */
  unsigned int poll_lock;         /* one CTA at a time reads host memory     */
  int stop;                       /* the host's stop flag, as last read      */
  unsigned long long last_active; /* globaltimer of the last mirrored request */
  unsigned long long inflight;    /* heap bytes of admitted, incomplete requests */
  unsigned long long exited;      /* CTAs that left the loop, over all launches */
};

struct SArgs {
  const SReq *ring;
  SDone *done;
  SCtl *ctl;
  SDev *dev;
  unsigned int *tiles_done; /* per slot */
  unsigned long long *tctr; /* per slot: the claim word, set when the request is mirrored */
  SReq *mreq;               /* per slot: device copy of the request (seq = ticket + 1) */
  unsigned int Q;
  char *base;
  uint64_t slice;
  int npes;
  unsigned long long idle_ns;
  unsigned long long epoch; /* this launch's number, reported in ctl->down */
  unsigned mirror_batch;    /* requests one poll copies at most */
  unsigned long long budget; /* heap bytes admitted requests may hold, 0 = no limit */
  HeapDev heap;              /* the symmetric-heap allocator, for B200SHM_SERVE_ALLOC dests */
};

__device__ __forceinline__ unsigned long long ld_acquire_sys(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.sys.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_sys(unsigned long long *p, unsigned long long v) {
  asm volatile("st.release.sys.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
/* Release/acquire fences (lighter than the sequentially consistent
 * __threadfence, which stalls behind the atomics of the waiting CTAs). */
__device__ __forceinline__ void fence_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
__device__ __forceinline__ void fence_sys() { asm volatile("fence.acq_rel.sys;" ::: "memory"); }
__device__ __forceinline__ unsigned long long vld(const unsigned long long *p) {
  return *(const volatile unsigned long long *)p;
}
__device__ __forceinline__ unsigned long long now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void copy_words(SReq *dst, const SReq *src) {
  const volatile unsigned long long *s = (const volatile unsigned long long *)src;
  unsigned long long *d = (unsigned long long *)dst;
#pragma unroll
  for (int i = 0; i < 16; i++) d[i] = s[i];
}

/* The device mirror of the ring: the CTA that holds the poll lock copies
 * newly published requests from host memory into it (sequence word last)
 * before it opens them to claims, so the other CTAs read requests from L2
 * only.  Copy request r into *out, for a CTA that holds a share of r (the
 * caller has fenced after its claim): the slot keeps r until r completes,
 * which needs that share, so one copy is consistent; 1 when the copy is of
 * r (always, by that argument). */
__device__ int copy_req(const SArgs &a, unsigned long long r, SReq *out) {
  copy_words(out, &a.mreq[r % a.Q]);
  return out->seq == r + 1 ? 1 : 0;
}

/* Requests one poll copies at most (B200SHM_SERVE_MIRROR_BATCH overrides
 * it).  The copy costs about one round trip to host memory whatever its
 * size, so a saturated loop is bounded by batch / round trip: on the
 * serving workload, saturated, 16 per poll served 0.78 M requests/s (1.09 M
 * fetch-adds/s), 64 served 1.08 M (1.93 M), 256 served 1.16 M (2.29 M). */
constexpr unsigned kMirrorBatch = 256;

/* Claim the next tiles (thread 0).  Returns 1 with request *cr, tiles
 * [*ct, *ct + *count) and the request in *req; 2 when this CTA took the poll
 * lock and found requests [*mfrom, *mupto) published but not yet copied
 * into device memory (the CTA copies them, then publishes and releases the
 * lock); or 0 when the CTA should exit (stop requested or idle past the
 * limit, in both cases holding no claim).
 * A claim is one fetch-and-add of 1 on the slot's claim word, which says
 * by itself whether a share was left: no request descriptor is read before
 * the claim, and a CTA that finds nothing left walks on to the next
 * request at once (the cursor is only a hint of where unclaimed shares
 * start; whoever takes a request's last share moves it on).  An add that
 * lands after the slot moved on to a later request x (only possible once
 * the request it aimed at is complete) holds a share of x, which is served
 * as such, so no tile is ever lost or handed out twice.  *r_hint carries
 * the request this CTA looks at next from one claim to the next. */
__device__ int claim(const SArgs &a, SReq *req, unsigned long long *cr, unsigned long long *ct,
                     unsigned *count, unsigned long long *mfrom, unsigned long long *mupto,
                     unsigned long long idle_since, unsigned long long *r_hint) {
  unsigned backoff = 32;
  unsigned long long r = *r_hint;
  for (;;) {
    const unsigned long long cur = vld(&a.dev->cursor);
    const unsigned long long tl = vld(&a.dev->tail_mirror);
    if (cur > r) r = cur;
    if (r >= tl) {
      /* test, then test-and-set: waiting CTAs only read the lock word */
      if (*(const volatile unsigned *)&a.dev->poll_lock == 0u &&
          atomicCAS(&a.dev->poll_lock, 0u, 1u) == 0u) {
        const unsigned long long mt = vld(&a.dev->tail_mirror);
        const unsigned long long hv = ld_acquire_sys(&a.ctl->tail);
        const unsigned long long ht = hv & ~kStopBit;
        /* a stop takes effect once every published request is in the
         * mirror (with a heap budget some may still wait for room), so the
         * loop drains before it exits */
        if ((hv & kStopBit) && ht == mt) *(volatile int *)&a.dev->stop = 1;
        if (ht > mt) { /* the whole CTA copies them, still holding the lock */
          *mfrom = mt;
          *mupto = ht < mt + a.mirror_batch ? ht : mt + a.mirror_batch;
          *r_hint = r;
          return 2;
        }
        atomicExch(&a.dev->poll_lock, 0u);
      }
      if (vld(&a.dev->tail_mirror) <= r) {
        /* only the lock holder reads host memory: a read of host memory by
         * every waiting CTA on every turn floods the path to the host and
         * stalls every other memory access behind it */
        if (*(const volatile int *)&a.dev->stop) return 0;
        /* idle is the loop's idle time, not this CTA's: a CTA that wins no
         * claim for a while stays as long as requests keep arriving */
        const unsigned long long act = vld(&a.dev->last_active), now = now_ns();
        const unsigned long long since = act > idle_since ? act : idle_since;
        if (now > since && now - since > a.idle_ns) return 0;
        __nanosleep(backoff);
        backoff = backoff < 128 ? backoff * 2 : 128;
      }
      continue;
    }
    fence_gpu(); /* the claim words of requests below tail_mirror are set */
    for (; r < tl; r++) {
      const unsigned long long old = atomicAdd(&a.tctr[r % a.Q], 1ull);
      const unsigned long long x = r + (((old >> kTagShift) - r) & kField24);
      const unsigned long long nsh = (old >> kShareShift) & 0xFFFFull, sh = old & kField24;
      /* r is handed out: the cursor moves past it (a CTA that finds the
       * shares gone leaves that to the one that took the last) */
      if (x != r || sh + 1 == nsh) atomicMax(&a.dev->cursor, r + 1);
      if (sh >= nsh) continue;
      /* share sh of request x is ours; x stays in its slot until it completes */
      fence_gpu();
      if (req->seq != x + 1 && !copy_req(a, x, req)) continue; /* not reached */
      const unsigned long long k = share_tiles(req->ntiles, gridDim.x);
      *cr = x;
      *ct = sh * k;
      *count = (unsigned)(req->ntiles - sh * k < k ? req->ntiles - sh * k : k);
      *r_hint = x == r && sh + 1 < nsh ? r : r + 1;
      return 1;
    }
  }
}

/* ---- reductions ------------------------------------------------------------ */
template <class T>
__device__ __forceinline__ T ldv(const char *p) {
  T v;
  memcpy(&v, p, sizeof(T));
  return v;
}
template <class T>
__device__ __forceinline__ void stv(char *p, T v) {
  memcpy(p, &v, sizeof(T));
}

/* Where a float MIN/MAX result depends on operand order (a NaN, or both
 * zeros, among the inputs): replay the algorithm's order for element e
 * and write what each member receives (rec_dbl gives members different
 * bits; the other algorithms give every member the block owner's). */
template <class T, int OP>
__device__ void exact_element(int algo, const char *s, char *d, uint64_t step, int P, int p2s,
                              int lg, uint64_t e, uint64_t N) {
  auto get = [&](int j) { return ldv<T>(s + (uint64_t)j * step); };
  const bool lower = e < N / 2;
  if (algo == B200SHM_REC_DBL) {
    for (int qq = 0; qq < p2s; qq++) {
      const T x = exact_value<T, OP>(get, P, p2s, lg, algo, lower, qq);
      const int as = p2s_member(qq, P, p2s);
      stv<T>(d + (uint64_t)as * step, x);
      if (p2s_extra(qq, P, p2s)) stv<T>(d + (uint64_t)(as + 1) * step, x);
    }
    return;
  }
  int qq = 0;
  if (algo == B200SHM_RABENSEIFNER || algo == B200SHM_RABENSEIFNER2)
    qq = rev_bits(rab_block(e, N, p2s), lg);
  const T x = exact_value<T, OP>(get, P, p2s, lg, algo, lower, qq);
  for (int j = 0; j < P; j++) stv<T>(d + (uint64_t)j * step, x);
}

/* The tree the algorithm builds for float SUM/PROD, for one pack: the value
 * is the same in every member, the ops being exactly commutative.  Leaves
 * four at a time (own and extra members loaded together), a full batch
 * pushed as a subtree of 4 into a binary counter whose levels combine
 * earlier subtree first.  Binomial: op(upper block, lower block), then the
 * set bits of P from the lowest (reduce.c:137-154); butterfly: extra
 * members folded as op(extra, own), then log2(p2s) levels (reduce.c:
 * 206-272). */
template <class T, int V, int OP>
__device__ Pack<T, V> tree_pack(const char *s, uint64_t step, int P, int p2s, int lg,
                                bool binomial) {
  typedef Pack<T, V> PK;
  PK stk[kMaxLevels + 1];
  int c = 0;
  auto comb = [&](const PK &lo, const PK &hi) {
    return binomial ? papply<OP>(hi, lo) : papply<OP>(lo, hi);
  };
  auto push = [&](PK v, int lv) {
    const int t = __ffs(~(c >> lv)) - 1 + lv;
    for (int L = lv; L < t; L++) v = comb(stk[L], v);
    stk[t] = v;
    c += 1 << lv;
  };
  const int nl = binomial ? P : p2s;
  for (int qb = 0; qb < nl; qb += 4) {
    const int k = nl - qb < 4 ? nl - qb : 4;
    PK x[4], e[4];
    bool ex[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      ex[u] = false;
      if (u < k) {
        const int q = qb + u;
        const int own = binomial ? q : (int)(((long long)q * P + p2s - 1) >> lg);
        x[u] = ld_pack<T, V>(s + (uint64_t)own * step);
        if (!binomial) {
          ex[u] = (int)(((long long)(q + 1) * P + p2s - 1) >> lg) - own == 2;
          if (ex[u]) e[u] = ld_pack<T, V>(s + (uint64_t)(own + 1) * step);
        }
      }
    }
#pragma unroll
    for (int u = 0; u < 4; u++)
      if (ex[u]) x[u] = papply<OP>(e[u], x[u]);
    if (k == 4) {
      push(comb(comb(x[0], x[1]), comb(x[2], x[3])), 2);
    } else {
#pragma unroll
      for (int u = 0; u < 4; u++)
        if (u < k) push(x[u], 0);
    }
  }
  if (!binomial) return stk[lg];
  bool have = false;
  PK v = stk[0];
  for (int L = 0; L <= kMaxLevels; L++)
    if (P & (1 << L)) {
      v = have ? comb(stk[L], v) : stk[L];
      have = true;
    }
  return v;
}

/* Units [u0, u1) of V elements each, one per thread at a time, members
 * loaded eight at a time. */
template <class T, int V, int OP>
__device__ void reduce_units(const b200shm_request &r, const char *src0, char *dst0,
                             uint64_t step, uint64_t u0, uint64_t u1, int P, int p2s, int lg) {
  typedef Pack<T, V> PK;
  constexpr uint64_t UB = sizeof(T) * V;
  constexpr bool FL = std::is_floating_point<T>::value;
  constexpr bool MM = FL && (OP == B200SHM_MIN || OP == B200SHM_MAX);
  const bool chain = !FL || MM || r.algo == B200SHM_LINEAR;
  const bool bin = r.algo == B200SHM_BINOMIAL;
  for (uint64_t k = u0 + threadIdx.x; k < u1; k += kServeThreads) {
    const char *s = src0 + k * UB;
    PK v;
    unsigned cls[V];
#pragma unroll
    for (int i = 0; i < V; i++) cls[i] = 0;
    if (chain) {
      v = ld_pack<T, V>(s);
      if constexpr (MM) {
#pragma unroll
        for (int i = 0; i < V; i++) cls[i] = fclass(v.x[i]);
      }
      for (int j = 1; j < P; j += 8) {
        PK x[8];
#pragma unroll
        for (int m = 0; m < 8; m++)
          if (j + m < P) x[m] = ld_pack<T, V>(s + (uint64_t)(j + m) * step);
#pragma unroll
        for (int m = 0; m < 8; m++)
          if (j + m < P) {
            v = papply<OP>(v, x[m]);
            if constexpr (MM) {
#pragma unroll
              for (int i = 0; i < V; i++) cls[i] |= fclass(x[m].x[i]);
            }
          }
      }
    } else {
      v = tree_pack<T, V, OP>(s, step, P, p2s, lg, bin);
    }
    if constexpr (MM) {
      bool amb = false;
#pragma unroll
      for (int i = 0; i < V; i++) amb |= ambiguous(cls[i]);
      if (amb && r.algo != B200SHM_LINEAR) {
        for (int i = 0; i < V; i++) {
          const uint64_t e = k * V + i;
          exact_element<T, OP>(r.algo, src0 + e * sizeof(T), dst0 + e * sizeof(T), step, P, p2s,
                               lg, e, r.n);
        }
        continue;
      }
    }
    char *d = dst0 + k * UB;
    for (int j = 0; j < P; j++) st_pack<T, V>(d + (uint64_t)j * step, v);
  }
}

/* Elements [e0, e1) of a reduction: 16-byte packs where the source and
 * dest offsets allow (member strides are whole slices), then the rest. */
template <class T, int OP>
__device__ void reduce_range(const b200shm_request &r, uint64_t e0, uint64_t e1, char *base,
                             uint64_t slice) {
  constexpr int V = (int)(16 / sizeof(T));
  const int P = r.pe_size;
  int p2s = 1, lg = 0;
  while (p2s * 2 <= P) {
    p2s *= 2;
    lg++;
  }
  const uint64_t step = (uint64_t)(P > 1 ? r.pe_stride : 1) * slice;
  const char *src0 = base + (uint64_t)r.pe_start * slice + r.src_off;
  char *dst0 = base + (uint64_t)r.pe_start * slice + r.dest_off;
  uint64_t e = e0;
  if (((r.src_off | r.dest_off) & 15) == 0 && e0 % V == 0) {
    const uint64_t pend = e1 / V;
    reduce_units<T, V, OP>(r, src0, dst0, step, e0 / V, pend, P, p2s, lg);
    e = pend * V;
  }
  if (e < e1) reduce_units<T, 1, OP>(r, src0, dst0, step, e, e1, P, p2s, lg);
}

template <class T>
__device__ __noinline__ void serve_reduce(const SReq &q, uint64_t e0, uint64_t e1, char *base,
                                          uint64_t slice) {
  const b200shm_request &r = q.r;
  if constexpr (std::is_floating_point<T>::value) {
    switch (r.op) {
    case B200SHM_MIN: reduce_range<T, B200SHM_MIN>(r, e0, e1, base, slice); break;
    case B200SHM_MAX: reduce_range<T, B200SHM_MAX>(r, e0, e1, base, slice); break;
    case B200SHM_SUM: reduce_range<T, B200SHM_SUM>(r, e0, e1, base, slice); break;
    default: reduce_range<T, B200SHM_PROD>(r, e0, e1, base, slice); break;
    }
  } else {
    switch (r.op) {
    case B200SHM_AND: reduce_range<T, B200SHM_AND>(r, e0, e1, base, slice); break;
    case B200SHM_OR: reduce_range<T, B200SHM_OR>(r, e0, e1, base, slice); break;
    case B200SHM_XOR: reduce_range<T, B200SHM_XOR>(r, e0, e1, base, slice); break;
    case B200SHM_MIN: reduce_range<T, B200SHM_MIN>(r, e0, e1, base, slice); break;
    case B200SHM_MAX: reduce_range<T, B200SHM_MAX>(r, e0, e1, base, slice); break;
    case B200SHM_SUM: reduce_range<T, B200SHM_SUM>(r, e0, e1, base, slice); break;
    default: reduce_range<T, B200SHM_PROD>(r, e0, e1, base, slice); break;
    }
  }
}

/* ---- copies ------------------------------------------------------------------ */
template <class W>
__device__ __forceinline__ void words_copy(W *d, const W *s, uint64_t n, int tid, int nthr) {
  uint64_t i = tid;
  const uint64_t st = (uint64_t)nthr;
  for (; i + 7 * st < n; i += 8 * st) {
    W x[8];
#pragma unroll
    for (int u = 0; u < 8; u++) x[u] = s[i + u * st];
#pragma unroll
    for (int u = 0; u < 8; u++) d[i + u * st] = x[u];
  }
  for (; i < n; i += st) d[i] = s[i];
}

/* Copy n bytes with threads [tid, tid + nthr): bytes up to the dest's
 * alignment, then the widest word the two addresses share an alignment
 * for, four words in flight per thread, then the remaining bytes. */
__device__ void span_copy(char *dst, const char *src, uint64_t n, int tid, int nthr) {
  const uint64_t x = (uint64_t)dst ^ (uint64_t)src;
  const uint64_t w = (x & 15) == 0 ? 16 : (x & 7) == 0 ? 8 : (x & 3) == 0 ? 4 : 1;
  uint64_t head = (w - ((uint64_t)dst & (w - 1))) & (w - 1);
  if (head > n) head = n;
  for (uint64_t i = tid; i < head; i += nthr) dst[i] = src[i];
  dst += head;
  src += head;
  n -= head;
  const uint64_t nw = n / w;
  switch (w) {
  case 16: words_copy((uint4 *)dst, (const uint4 *)src, nw, tid, nthr); break;
  case 8:
    words_copy((unsigned long long *)dst, (const unsigned long long *)src, nw, tid, nthr);
    break;
  case 4: words_copy((unsigned *)dst, (const unsigned *)src, nw, tid, nthr); break;
  default: words_copy((unsigned char *)dst, (const unsigned char *)src, nw, tid, nthr); break;
  }
  for (uint64_t i = nw * w + tid; i < n; i += nthr) dst[i] = src[i];
}

/* Segment s of a copy request: fcollect dest block k of member j <- member
 * k's source (fcollect.c:32-484); alltoall dest block k of member j <-
 * block j of member k's source (alltoall.c:75-201); put / get one span. */
__device__ void segment(const SReq &q, uint64_t s, char *base, uint64_t slice, char **dst,
                        const char **src) {
  const b200shm_request &r = q.r;
  const uint64_t n = r.n;
  if (r.kind == B200SHM_REQ_FCOLLECT || r.kind == B200SHM_REQ_ALLTOALL) {
    const uint64_t P = (uint64_t)r.pe_size, j = s / P, k = s - j * P;
    const uint64_t stride = (uint64_t)(r.pe_size > 1 ? r.pe_stride : 1);
    char *mj = base + ((uint64_t)r.pe_start + j * stride) * slice;
    char *mk = base + ((uint64_t)r.pe_start + k * stride) * slice;
    *dst = mj + r.dest_off + k * n;
    *src = mk + r.src_off + (r.kind == B200SHM_REQ_ALLTOALL ? j * n : 0);
  } else if (r.kind == B200SHM_REQ_PUT) {
    *dst = base + (uint64_t)r.pe * slice + r.dest_off;
    *src = base + (uint64_t)r.pe_start * slice + r.src_off;
  } else {
    *dst = base + (uint64_t)r.pe_start * slice + r.dest_off;
    *src = base + (uint64_t)r.pe * slice + r.src_off;
  }
}

__device__ __noinline__ void serve_copy(const SReq &q, uint64_t t, char *base, uint64_t slice) {
  char *d;
  const char *s;
  if (q.spt == 0) { /* one chunk of one large segment: the whole CTA */
    const uint64_t seg = t / q.cps, off = (t - seg * q.cps) * q.unit;
    const uint64_t len = q.r.n - off < q.unit ? q.r.n - off : q.unit;
    segment(q, seg, base, slice, &d, &s);
    span_copy(d + off, s + off, len, threadIdx.x, kServeThreads);
  } else { /* a run of small segments: one warp per segment */
    const uint64_t s0 = t * q.spt, s1 = s0 + q.spt < q.nseg ? s0 + q.spt : q.nseg;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (uint64_t g = s0 + warp; g < s1; g += kServeThreads / 32) {
      segment(q, g, base, slice, &d, &s);
      span_copy(d, s, q.r.n, lane, 32);
    }
  }
}

/* Copy ring slots [from, upto) from host memory into the device mirror,
 * the whole CTA at once (one host word per thread, all reads in flight
 * together), then publish them: sequence words, tile counters tagged with
 * their request, tail_mirror; then release the poll lock (thread 0 holds
 * it).  The sequence word is cleared before the copy is written, so a late
 * reader of the slot's previous request sees the change. */
__device__ void mirror_ring(const SArgs &a, unsigned long long from, unsigned long long upto) {
  unsigned n = (unsigned)(upto - from);
  __shared__ unsigned long long s_bytes[kMirrorMax]; /* heap bytes per request (budget only) */
  __shared__ unsigned long long s_nt[kMirrorMax];    /* tiles per request, as copied */
  __shared__ unsigned char s_alloc[kMirrorMax];      /* the loop allocates the dest */
  __shared__ unsigned s_admit, s_nalloc;
  /* a snapshot taken early, overlapping the copy: completions only lower
   * the count meanwhile, so an early reading can only admit less */
  const unsigned long long used = a.budget && threadIdx.x == 0 ? vld(&a.dev->inflight) : 0;
  if (threadIdx.x == 0) s_nalloc = 0;
  for (unsigned i = threadIdx.x; i < n; i += kServeThreads)
    ((volatile unsigned long long *)&a.mreq[(from + i) % a.Q])[14] = 0;
  fence_gpu();
  __syncthreads();
  const unsigned long long now = now_ns();
  /* the words of host memory four at a time per thread, all loads issued
   * before the first store, so a batch costs about one round trip to the
   * host rather than one per pass */
  for (unsigned w0 = threadIdx.x; w0 < n * 16; w0 += 4 * kServeThreads) {
    unsigned long long v[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const unsigned w = w0 + j * kServeThreads, i = w >> 4, k = w & 15;
      v[j] = 0;
      if (w < n * 16 && k != 14 && (k != 15 || a.budget))
        v[j] = ((const volatile unsigned long long *)&a.ring[(from + i) % a.Q])[k];
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const unsigned w = w0 + j * kServeThreads, i = w >> 4, k = w & 15;
      if (w < n * 16 && k != 14)
        ((volatile unsigned long long *)&a.mreq[(from + i) % a.Q])[k] = k == 15 ? now : v[j];
      if (w < n * 16 && k == 15) s_bytes[i] = v[j];
      if (w < n * 16 && k == 9) s_nt[i] = v[j];
      if (w < n * 16 && k == 4) { /* the dest offset */
        s_alloc[i] = v[j] == B200SHM_SERVE_ALLOC;
        if (v[j] == B200SHM_SERVE_ALLOC) atomicAdd(&s_nalloc, 1u);
      }
    }
  }
  fence_gpu();
  __syncthreads();
  if (a.budget || s_nalloc) {
    /* admission: the longest run of the batch, in arrival order, whose
     * bytes fit beside those of the admitted requests not yet complete
     * (with a budget), and whose dests the heap can hold (for requests
     * that ask the loop to allocate theirs).  Only the poll-lock holder
     * adds to the count and completions only lower it, so the check cannot
     * overshoot.  The rest stay in the host ring for a later poll. */
    if (threadIdx.x == 0) {
      unsigned long long add = 0;
      unsigned k = 0;
      bool locked = false;
      const unsigned shift = s_nalloc ? hv(&a.heap.ctl->unit_shift) : 0u;
      const unsigned nunits = s_nalloc ? hv(&a.heap.ctl->nunits) : 0u;
      while (k < n) {
        if (a.budget && used + add + s_bytes[k] > a.budget) break;
        if (s_alloc[k]) {
          if (!locked && !(locked = heap_lock(a.heap))) break;
          b200shm_request *rq = &a.mreq[(from + k) % a.Q].r;
          const unsigned long long units = heap_units(dest_bytes(*(const b200shm_request *)rq), shift);
          const unsigned u = units <= nunits ? heap_alloc_locked(a.heap, (unsigned)(units ? units : 1), 1)
                                             : kHeapNil;
          if (u == kHeapNil) break; /* waits for room: frees or completions */
          *(volatile unsigned long long *)&rq->dest_off = (unsigned long long)u << shift;
        }
        add += s_bytes[k++];
      }
      if (locked) heap_unlock(a.heap);
      if (a.budget && add) atomicAdd(&a.dev->inflight, add);
      s_admit = k;
    }
    __syncthreads();
    n = s_admit;
    upto = from + n;
  }
  for (unsigned i = threadIdx.x; i < n; i += kServeThreads) {
    const unsigned long long x = from + i;
    ((volatile unsigned long long *)&a.mreq[x % a.Q])[14] = x + 1;
  }
  fence_gpu();
  __syncthreads();
  for (unsigned i = threadIdx.x; i < n; i += kServeThreads) {
    /* the claim word last: it opens the request to claims */
    const unsigned long long x = from + i;
    const unsigned long long nt = s_nt[i];
    const unsigned long long k = share_tiles(nt, gridDim.x);
    fence_gpu(); /* the whole request before its claim word, from this thread too */
    atomicExch(&a.tctr[x % a.Q], claim_word(x, (nt + k - 1) / k));
  }
  fence_gpu();
  __syncthreads();
  if (threadIdx.x == 0) {
    *(volatile unsigned long long *)&a.dev->last_active = now;
    *(volatile unsigned long long *)&a.dev->tail_mirror = upto;
    fence_gpu();
    atomicExch(&a.dev->poll_lock, 0u);
  }
  __syncthreads();
}

/* ---- the loop -------------------------------------------------------------------- */
__global__ void __launch_bounds__(kServeThreads) k_serve(const SArgs a) {
  __shared__ SReq s_req;
  __shared__ unsigned long long s_cr, s_ct, s_mfrom, s_mupto;
  __shared__ unsigned s_count;
  __shared__ int s_go;
  __shared__ unsigned long long s_fetched;
  __shared__ int s_status;
  __shared__ unsigned long long s_tclaim;
  unsigned long long idle_since = now_ns();
  unsigned long long r_hint = 0;
  if (threadIdx.x == 0) s_req.seq = 0;
  for (;;) {
    if (threadIdx.x == 0) {
      s_go = claim(a, &s_req, &s_cr, &s_ct, &s_count, &s_mfrom, &s_mupto, idle_since, &r_hint);
      s_tclaim = now_ns();
      s_fetched = 0;
      s_status = 0;
    }
    __syncthreads();
    if (!s_go) {
      if (threadIdx.x == 0) { /* the launch's last CTA out tells the host */
        const unsigned long long out = atomicAdd(&a.dev->exited, 1ull) + 1;
        if (out % gridDim.x == 0) {
          fence_sys();
          st_release_sys(&a.ctl->down, a.epoch);
        }
      }
      return;
    }
    if (s_go == 2) {
      mirror_ring(a, s_mfrom, s_mupto);
      idle_since = now_ns();
      continue;
    }
    const unsigned long long r = s_cr, t0 = s_ct;
    const SReq &q = s_req;
    for (unsigned long long t = t0; t < t0 + s_count; t++) {
      switch (q.r.kind) {
      case B200SHM_REQ_REDUCE: {
        const uint64_t e0 = t * q.unit;
        const uint64_t e1 = e0 + q.unit < q.r.n ? e0 + q.unit : q.r.n;
        switch (q.r.dtype) {
        case B200SHM_I32: serve_reduce<int32_t>(q, e0, e1, a.base, a.slice); break;
        case B200SHM_U32: serve_reduce<uint32_t>(q, e0, e1, a.base, a.slice); break;
        case B200SHM_I64: serve_reduce<int64_t>(q, e0, e1, a.base, a.slice); break;
        case B200SHM_U64: serve_reduce<uint64_t>(q, e0, e1, a.base, a.slice); break;
        case B200SHM_F32: serve_reduce<float>(q, e0, e1, a.base, a.slice); break;
        case B200SHM_F64: serve_reduce<double>(q, e0, e1, a.base, a.slice); break;
        default:
          if (threadIdx.x == 0) s_status = B200SHM_STATUS_BADREQ;
        }
        break;
      }
      case B200SHM_REQ_FCOLLECT:
      case B200SHM_REQ_ALLTOALL:
      case B200SHM_REQ_PUT:
      case B200SHM_REQ_GET: serve_copy(q, t, a.base, a.slice); break;
      case B200SHM_REQ_AMO:
        if (threadIdx.x == 0) {
          char *p = a.base + (uint64_t)q.r.pe * a.slice + q.r.dest_off;
          const bool w8 = q.r.dtype == B200SHM_I64 || q.r.dtype == B200SHM_U64 ||
                          q.r.dtype == B200SHM_F64;
          if (w8)
            s_fetched = amo_one<unsigned long long>(q.r.op, (unsigned long long *)p, q.r.value,
                                                    q.r.cond);
          else
            s_fetched = amo_one<unsigned int>(q.r.op, (unsigned int *)p,
                                              (unsigned int)q.r.value, (unsigned int)q.r.cond);
        }
        break;
      default:
        if (threadIdx.x == 0) s_status = B200SHM_STATUS_BADREQ;
      }
    }
    fence_gpu();
    __syncthreads();
    if (threadIdx.x == 0) {
      const unsigned slot = (unsigned)(r % a.Q);
      fence_gpu();
      /* a CTA that claimed every tile of the request is its only finisher
       * (most small requests): no count to keep */
      if (s_count == q.ntiles ||
          atomicAdd(&a.tiles_done[slot], s_count) + (unsigned long long)s_count == q.ntiles) {
        fence_sys();
        a.tiles_done[slot] = 0;
        SDone *dn = &a.done[slot];
        /* AMOs: the old value; other kinds: the dest offset they wrote to
         * (the one the loop allocated, for B200SHM_SERVE_ALLOC) */
        *(volatile unsigned long long *)&dn->fetched =
            q.r.kind == B200SHM_REQ_AMO ? s_fetched : q.r.dest_off;
        *(volatile unsigned long long *)&dn->t[0] = q.pad;
        *(volatile unsigned long long *)&dn->t[1] = s_tclaim;
        *(volatile unsigned long long *)&dn->t[2] = now_ns();
        *(volatile int *)&dn->status = s_status;
        st_release_sys(&dn->seq, r + 1);
        if (a.budget) /* its heap bytes free for the next admissions, once complete */
          atomicAdd(&a.dev->inflight, 0ull - heap_bytes(q.r));
      }
    }
    idle_since = now_ns();
    __syncthreads();
  }
}

double host_now() {
  timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

}  // namespace
}  // namespace b200

using namespace b200;

struct b200shm_server {
  SReq *h_ring = nullptr, *d_ring = nullptr;
  SDone *h_done = nullptr, *d_done = nullptr;
  SCtl *h_ctl = nullptr, *d_ctl = nullptr;
  char *d_mem = nullptr;
  SArgs args{};
  unsigned Q = 0;
  int ctas = 0;
  cudaStream_t stream = nullptr;
  unsigned long long tail = 0; /* next ticket */
  bool stopping = false;       /* stop asked: every tail written carries kStopBit */
  std::mutex mu;
};

namespace b200 {
namespace {

/* A fault of the loop's kernel, if it had one (the loop is otherwise
 * watched through host words only). */
int stream_error(b200shm_server *s) {
  const cudaError_t e = cudaStreamQuery(s->stream);
  return e == cudaSuccess || e == cudaErrorNotReady ? B200SHM_OK : cuda_fail(e, "serving loop");
}

/* Relaunch the loop when its last launch has left (all of its CTAs have,
 * or are about to: the new launch is ordered after them on the stream).
 * One read of a host word, no driver call, while the loop runs. */
int ensure_running(b200shm_server *s) {
  if (s->args.epoch && *(const volatile unsigned long long *)&s->h_ctl->down != s->args.epoch)
    return B200SHM_OK;
  const cudaError_t e = cudaStreamQuery(s->stream);
  if (e != cudaSuccess && e != cudaErrorNotReady) return cuda_fail(e, "serving loop");
  s->args.epoch++;
  k_serve<<<s->ctas, kServeThreads, 0, s->stream>>>(s->args);
  count_launch();
  const cudaError_t le = cudaGetLastError();
  return le == cudaSuccess ? B200SHM_OK : cuda_fail(le, "serving loop launch");
}

bool reduce_dtype_ok(int dt) {
  return dt == B200SHM_I32 || dt == B200SHM_U32 || dt == B200SHM_I64 || dt == B200SHM_U64 ||
         dt == B200SHM_F32 || dt == B200SHM_F64;
}

/* Validate a request and fill in its tiling. */
int plan_request(const b200shm_request &r0, SReq *q) {
  memset(q, 0, sizeof(*q));
  q->r = r0;
  b200shm_request &r = q->r;
  int rc = B200SHM_OK;
  const State &S = st();
  /* the loop allocates the dest at admission: no dest to check here */
  const bool alloc = r.dest_off == B200SHM_SERVE_ALLOC;
  switch (r.kind) {
  case B200SHM_REQ_REDUCE: {
    if ((rc = check_team(r.pe_start, r.pe_stride, r.pe_size))) return rc;
    if (!reduce_dtype_ok(r.dtype))
      return fail(B200SHM_ERR_UNSUPPORTED, "serve: reduce dtype %d (32/64-bit ints, float, double)",
                  r.dtype);
    const bool fl = r.dtype == B200SHM_F32 || r.dtype == B200SHM_F64;
    if (r.op < 0 || r.op >= B200SHM_NOP || (fl && r.op < B200SHM_MIN))
      return fail(B200SHM_ERR_UNSUPPORTED, "serve: reduce op %d on dtype %d", r.op, r.dtype);
    if (r.algo == B200SHM_ALGO_AUTO) r.algo = B200SHM_REC_DBL;
    if (r.algo < 0 || r.algo >= B200SHM_NALGO)
      return fail(B200SHM_ERR_ARG, "serve: reduce algorithm %d", r.algo);
    if (r.pe_size > kFixMaxMembers)
      return fail(B200SHM_ERR_UNSUPPORTED, "serve: teams above %d members", kFixMaxMembers);
    const uint64_t es = (uint64_t)kDtypeSize[r.dtype];
    if (r.n > S.slice / es) return fail(B200SHM_ERR_ARG, "serve: nelems too large");
    const uint64_t bytes = r.n * es;
    if ((rc = check_extent(r.src_off, bytes, "serve reduce source")) ||
        (!alloc && (rc = check_extent(r.dest_off, bytes, "serve reduce dest"))))
      return rc;
    if (!alloc && r.dest_off != r.src_off && overlaps(r.dest_off, bytes, r.src_off, bytes))
      return fail(B200SHM_ERR_ARG, "serve: reduce dest and source overlap");
    uint64_t unit = reduce_tile_read() / ((uint64_t)r.pe_size * es);
    unit = (unit + kServeThreads - 1) / kServeThreads * kServeThreads;
    if (unit < kServeThreads) unit = kServeThreads;
    q->unit = unit;
    q->ntiles = r.n ? (r.n + unit - 1) / unit : 1;
    break;
  }
  case B200SHM_REQ_FCOLLECT:
  case B200SHM_REQ_ALLTOALL: {
    if ((rc = check_team(r.pe_start, r.pe_stride, r.pe_size))) return rc;
    const uint64_t P = (uint64_t)r.pe_size;
    if (r.n > S.slice / P) return fail(B200SHM_ERR_ARG, "serve: block too large");
    const uint64_t sb = r.kind == B200SHM_REQ_FCOLLECT ? r.n : P * r.n;
    if ((rc = check_extent(r.src_off, sb, "serve source")) ||
        (rc = check_extent(alloc ? 0 : r.dest_off, P * r.n, "serve dest")))
      return rc;
    if (!alloc && overlaps(r.dest_off, P * r.n, r.src_off, sb))
      return fail(B200SHM_ERR_ARG, "serve: dest and source overlap");
    q->nseg = P * P;
    break;
  }
  case B200SHM_REQ_PUT:
  case B200SHM_REQ_GET: {
    if (r.pe_start < 0 || r.pe_start >= S.npes || r.pe < 0 || r.pe >= S.npes)
      return fail(B200SHM_ERR_ARG, "serve: PE out of range");
    if ((rc = check_extent(r.src_off, r.n, "serve source")) ||
        (rc = check_extent(alloc ? 0 : r.dest_off, r.n, "serve dest")))
      return rc;
    const int dpe = r.kind == B200SHM_REQ_PUT ? r.pe : r.pe_start;
    const int spe = r.kind == B200SHM_REQ_PUT ? r.pe_start : r.pe;
    if (!alloc && dpe == spe && overlaps(r.dest_off, r.n, r.src_off, r.n))
      return fail(B200SHM_ERR_ARG, "serve: dest and source overlap");
    q->nseg = 1;
    break;
  }
  case B200SHM_REQ_AMO: {
    if (alloc) return fail(B200SHM_ERR_ARG, "serve: an atomic needs an existing target");
    if (r.pe < 0 || r.pe >= S.npes) return fail(B200SHM_ERR_ARG, "serve: AMO PE out of range");
    if (r.op < 0 || r.op >= B200SHM_AMO_NOP) return fail(B200SHM_ERR_ARG, "serve: AMO op %d", r.op);
    const bool w4 = r.dtype == B200SHM_I32 || r.dtype == B200SHM_U32 || r.dtype == B200SHM_F32;
    const bool w8 = r.dtype == B200SHM_I64 || r.dtype == B200SHM_U64 || r.dtype == B200SHM_F64;
    if (!w4 && !w8) return fail(B200SHM_ERR_UNSUPPORTED, "serve: AMO dtype %d", r.dtype);
    const bool fl = r.dtype == B200SHM_F32 || r.dtype == B200SHM_F64;
    if (fl && r.op != B200SHM_AMO_SWAP && r.op != B200SHM_AMO_SET && r.op != B200SHM_AMO_FETCH)
      return fail(B200SHM_ERR_UNSUPPORTED, "serve: float AMOs are swap/set/fetch only");
    const uint64_t w = w8 ? 8 : 4;
    if (r.dest_off % w || (rc = check_extent(r.dest_off, w, "serve AMO target")))
      return rc ? rc : fail(B200SHM_ERR_ARG, "serve: AMO target not aligned");
    if (w4) {
      r.value &= 0xffffffffull;
      r.cond &= 0xffffffffull;
    }
    q->ntiles = 1;
    break;
  }
  default: return fail(B200SHM_ERR_ARG, "serve: request kind %d", r.kind);
  }
  if (q->nseg) { /* copy tiling */
    q->unit = copy_chunk();
    if (r.n >= copy_chunk()) {
      q->cps = (r.n + copy_chunk() - 1) / copy_chunk();
      q->spt = 0;
      q->ntiles = q->nseg * q->cps;
    } else {
      q->spt = r.n ? copy_chunk() / r.n : q->nseg;
      if (q->spt < 1) q->spt = 1;
      q->ntiles = (q->nseg + q->spt - 1) / q->spt;
    }
    if (q->ntiles == 0) q->ntiles = 1;
  }
  /* a request is cut into at most one share per CTA; the adds that land
   * on its claim word past the last share are at most a few per CTA, far
   * inside the word's 24-bit share field */
  if (q->ntiles > kTileLimit)
    return fail(B200SHM_ERR_ARG, "serve: request of more than 2^22 tiles");
  return B200SHM_OK;
}

}  // namespace
}  // namespace b200

extern "C" {

int b200shm_serve_start(uint32_t queue_slots, int ctas, double idle_seconds,
                        b200shm_server **out) {
  return b200shm_serve_start_budget(queue_slots, ctas, idle_seconds, 0, out);
}

int b200shm_serve_start_budget(uint32_t queue_slots, int ctas, double idle_seconds,
                               uint64_t heap_budget, b200shm_server **out) {
  if (!st().up) return fail(B200SHM_ERR_STATE, "b200shm is not initialised");
  if (!out) return fail(B200SHM_ERR_ARG, "serve_start: null argument");
  if (queue_slots < 1 || queue_slots > (1u << 20))
    return fail(B200SHM_ERR_ARG, "serve_start: queue_slots must be in [1, 2^20]");
  *out = nullptr;
  b200shm_server *s = new b200shm_server();
  s->Q = queue_slots;
  /* every CTA resident at once: a CTA that only starts when another exits
   * would add an idle period to some requests' latency */
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_serve, kServeThreads, 0) !=
          cudaSuccess ||
      occ < 1)
    occ = 1;
  const int cap = occ * st().sm_count;
  s->ctas = ctas > 0 ? std::min(ctas, cap) : std::min(2 * st().sm_count, cap);
  const double idle = idle_seconds > 0 ? idle_seconds : 0.25;
  auto bail = [&](int rc) {
    if (s->h_ring) cudaFreeHost(s->h_ring);
    if (s->h_done) cudaFreeHost(s->h_done);
    if (s->h_ctl) cudaFreeHost(s->h_ctl);
    if (s->d_mem) cudaFree(s->d_mem);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return rc;
  };
  cudaError_t e = cudaHostAlloc((void **)&s->h_ring, sizeof(SReq) * s->Q, cudaHostAllocMapped);
  if (e == cudaSuccess)
    e = cudaHostAlloc((void **)&s->h_done, sizeof(SDone) * s->Q, cudaHostAllocMapped);
  if (e == cudaSuccess) e = cudaHostAlloc((void **)&s->h_ctl, sizeof(SCtl), cudaHostAllocMapped);
  if (e != cudaSuccess) return bail(cuda_fail(e, "serve_start: host ring"));
  memset(s->h_ring, 0, sizeof(SReq) * s->Q);
  memset(s->h_done, 0, sizeof(SDone) * s->Q);
  memset(s->h_ctl, 0, sizeof(SCtl));
  e = cudaHostGetDevicePointer((void **)&s->d_ring, s->h_ring, 0);
  if (e == cudaSuccess) e = cudaHostGetDevicePointer((void **)&s->d_done, s->h_done, 0);
  if (e == cudaSuccess) e = cudaHostGetDevicePointer((void **)&s->d_ctl, s->h_ctl, 0);
  if (e != cudaSuccess) return bail(cuda_fail(e, "serve_start: mapping"));
  const size_t dev_bytes = 256 + (size_t)s->Q * (sizeof(unsigned) + sizeof(unsigned long long)) +
                           (size_t)s->Q * sizeof(SReq) + 256;
  e = cudaMalloc((void **)&s->d_mem, dev_bytes);
  if (e == cudaSuccess) e = cudaMemset(s->d_mem, 0, dev_bytes);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return bail(cuda_fail(e, "serve_start: device state"));
  SArgs &a = s->args;
  a.ring = s->d_ring;
  a.done = s->d_done;
  a.ctl = s->d_ctl;
  a.dev = (SDev *)s->d_mem;
  a.mreq = (SReq *)(s->d_mem + 256);
  a.tctr = (unsigned long long *)(s->d_mem + 256 + (size_t)s->Q * sizeof(SReq));
  a.tiles_done = (unsigned *)(a.tctr + s->Q);
  a.Q = s->Q;
  a.base = st().base;
  a.slice = st().slice;
  a.npes = st().npes;
  a.idle_ns = (unsigned long long)(idle * 1e9);
  a.budget = heap_budget;
  a.heap = heap_dev();
  a.mirror_batch = kMirrorBatch;
  if (const char *mb = getenv("B200SHM_SERVE_MIRROR_BATCH"))
    if (atoi(mb) > 0) a.mirror_batch = (unsigned)std::min(atoi(mb), (int)kMirrorMax);
  int rc = ensure_running(s);
  if (rc) return bail(rc);
  *out = s;
  return B200SHM_OK;
}

int b200shm_serve_enqueue(b200shm_server *s, const b200shm_request *req, uint64_t *ticket) {
  if (!s || !req) return fail(B200SHM_ERR_ARG, "serve_enqueue: null argument");
  SReq q;
  int rc = plan_request(*req, &q);
  if (rc) return rc;
  if (s->args.budget && heap_bytes(q.r) > s->args.budget)
    return fail(B200SHM_ERR_ARG, "serve: request of %llu heap bytes, above the server's budget of %llu",
                (unsigned long long)heap_bytes(q.r), (unsigned long long)s->args.budget);
  std::lock_guard<std::mutex> lk(s->mu);
  const unsigned long long tk = s->tail;
  const unsigned slot = (unsigned)(tk % s->Q);
  if (tk >= s->Q) { /* the slot's previous request must be complete */
    const unsigned long long prev = tk - s->Q;
    if (*(volatile unsigned long long *)&s->h_done[slot].seq < prev + 1)
      return fail(B200SHM_ERR_BUSY, "serve: all %u queue slots are in flight", s->Q);
  }
  SReq *dst = &s->h_ring[slot];
  *(volatile unsigned long long *)&dst->seq = 0;
  std::atomic_thread_fence(std::memory_order_release);
  q.seq = 0;
  q.pad = heap_bytes(q.r); /* for admission by heap bytes */
  memcpy(dst, &q, sizeof(SReq));
  std::atomic_thread_fence(std::memory_order_release);
  *(volatile unsigned long long *)&dst->seq = tk + 1;
  std::atomic_thread_fence(std::memory_order_release);
  *(volatile unsigned long long *)&s->h_ctl->tail = (tk + 1) | (s->stopping ? kStopBit : 0);
  std::atomic_thread_fence(std::memory_order_seq_cst);
  s->tail = tk + 1;
  if (ticket) *ticket = tk;
  return ensure_running(s);
}

int b200shm_serve_poll(b200shm_server *s, uint64_t ticket, uint64_t *fetched) {
  if (!s) return fail(B200SHM_ERR_ARG, "serve_poll: null server");
  const SDone *d = &s->h_done[ticket % s->Q];
  const unsigned long long seq = *(const volatile unsigned long long *)&d->seq;
  if (seq < ticket + 1) {
    /* a loop that idled out right after this request was published is
     * brought back here too (one read of a host word while it runs) */
    if (*(const volatile unsigned long long *)&s->h_ctl->down == s->args.epoch) {
      std::lock_guard<std::mutex> lk(s->mu);
      const int er = ensure_running(s);
      if (er) return er;
    }
    return 0;
  }
  std::atomic_thread_fence(std::memory_order_acquire);
  if (fetched) *fetched = *(const volatile unsigned long long *)&d->fetched;
  const int status = *(const volatile int *)&d->status;
  if (status) return fail(B200SHM_ERR_ARG, "serve: request %llu was refused on the device",
                          (unsigned long long)ticket);
  return 1;
}

int b200shm_serve_trace(b200shm_server *s, uint64_t ticket, uint64_t stamps[3]) {
  if (!s || !stamps) return fail(B200SHM_ERR_ARG, "serve_trace: null argument");
  const SDone *d = &s->h_done[ticket % s->Q];
  if (*(const volatile unsigned long long *)&d->seq != ticket + 1) return 0;
  std::atomic_thread_fence(std::memory_order_acquire);
  for (int i = 0; i < 3; i++) stamps[i] = ((const volatile unsigned long long *)d->t)[i];
  return 1;
}

int b200shm_serve_wait(b200shm_server *s, uint64_t ticket, double timeout_seconds,
                       uint64_t *fetched) {
  const double t0 = host_now();
  for (unsigned it = 0;; it++) {
    const int rc = b200shm_serve_poll(s, ticket, fetched);
    if (rc) return rc < 0 ? rc : B200SHM_OK;
    if ((it & 63) == 63) {
      std::lock_guard<std::mutex> lk(s->mu);
      const int er = ensure_running(s); /* the kernel may have idled out meanwhile */
      if (er) return er;
    }
    if (host_now() - t0 > timeout_seconds) {
      const int se = stream_error(s);
      if (se) return se;
      return fail(B200SHM_ERR_TIMEOUT, "serve_wait: request %llu not complete after %.3f s",
                  (unsigned long long)ticket, timeout_seconds);
    }
  }
}

int b200shm_serve_stop(b200shm_server *s) {
  if (!s) return B200SHM_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
    *(volatile unsigned long long *)&s->h_ctl->tail = s->tail | kStopBit;
  }
  std::atomic_thread_fence(std::memory_order_seq_cst);
  const double limit = (double)s->args.idle_ns * 1e-9 + 30.0, t0 = host_now();
  cudaError_t e;
  while ((e = cudaStreamQuery(s->stream)) == cudaErrorNotReady) {
    if (host_now() - t0 > limit)
      return fail(B200SHM_ERR_TIMEOUT, "serve_stop: the loop did not exit (server kept)");
    struct timespec ts = {0, 200000};
    nanosleep(&ts, nullptr);
  }
  cudaStreamDestroy(s->stream);
  cudaFreeHost(s->h_ring);
  cudaFreeHost(s->h_done);
  cudaFreeHost(s->h_ctl);
  cudaFree(s->d_mem);
  delete s;
  return e == cudaSuccess ? B200SHM_OK : cuda_fail(e, "serve_stop");
}

int b200shm_serve_replay(b200shm_server *s, const b200shm_request *reqs, uint64_t n,
                         const double *arrival_s, double *latency_s, uint64_t *fetched) {
  if (!st().up) return fail(B200SHM_ERR_STATE, "b200shm is not initialised");
  if (n && (!reqs || !arrival_s || !latency_s)) return fail(B200SHM_ERR_ARG, "serve_replay: null");
  const double t0 = host_now();
  if (!s) { /* per call: each request one blocking entry point, in arrival order */
    for (uint64_t k = 0; k < n; k++) {
      while (host_now() - t0 < arrival_s[k]) {
      }
      const b200shm_request &r = reqs[k];
      int rc;
      uint64_t f = 0;
      switch (r.kind) {
      case B200SHM_REQ_REDUCE:
        rc = b200shm_reduce(r.op, r.dtype, r.algo, r.pe_start, r.pe_stride, r.pe_size, r.dest_off,
                            r.src_off, r.n, nullptr);
        break;
      case B200SHM_REQ_FCOLLECT:
        rc = b200shm_fcollect(r.pe_start, r.pe_stride, r.pe_size, r.dest_off, r.src_off, r.n,
                              nullptr);
        break;
      case B200SHM_REQ_ALLTOALL:
        rc = b200shm_alltoall(r.pe_start, r.pe_stride, r.pe_size, r.dest_off, r.src_off, r.n,
                              nullptr);
        break;
      case B200SHM_REQ_PUT:
      case B200SHM_REQ_GET: {
        const int dpe = r.kind == B200SHM_REQ_PUT ? r.pe : r.pe_start;
        const int spe = r.kind == B200SHM_REQ_PUT ? r.pe_start : r.pe;
        void *d = b200shm_ptr(dpe, r.dest_off);
        const void *sp = b200shm_ptr(spe, r.src_off);
        rc = (d && sp) ? b200shm_memcpy(d, sp, r.n, nullptr)
                       : fail(B200SHM_ERR_ARG, "serve_replay: bad put/get");
        break;
      }
      case B200SHM_REQ_AMO:
        rc = b200shm_amo(r.op, r.dtype, r.pe, r.dest_off, &r.value, &r.cond, &f);
        break;
      default: rc = fail(B200SHM_ERR_ARG, "serve_replay: request kind %d", r.kind);
      }
      if (rc) return rc;
      latency_s[k] = host_now() - t0 - arrival_s[k];
      if (fetched) fetched[k] = f;
    }
    return B200SHM_OK;
  }
  std::vector<uint64_t> tickets(n);
  std::vector<uint64_t> pend;
  pend.reserve(s->Q);
  uint64_t k = 0, done = 0;
  double last_progress = host_now();
  for (unsigned it = 0; done < n; it++) {
    const double now = host_now();
    if (k < n && now - t0 >= arrival_s[k]) {
      uint64_t tk;
      const int rc = b200shm_serve_enqueue(s, &reqs[k], &tk);
      if (rc == B200SHM_OK) {
        tickets[k] = tk;
        pend.push_back(k);
        k++;
        last_progress = now;
        continue;
      }
      if (rc != B200SHM_ERR_BUSY) return rc;
    }
    for (size_t i = 0; i < pend.size();) {
      const uint64_t j = pend[i];
      uint64_t f = 0;
      const int rc = b200shm_serve_poll(s, tickets[j], &f);
      if (rc < 0) return rc;
      if (rc == 1) {
        latency_s[j] = host_now() - t0 - arrival_s[j];
        if (fetched) fetched[j] = f;
        pend[i] = pend.back();
        pend.pop_back();
        done++;
        last_progress = host_now();
      } else {
        i++;
      }
    }
    if ((it & 63) == 63 && !pend.empty()) {
      std::lock_guard<std::mutex> lk(s->mu);
      const int er = ensure_running(s);
      if (er) return er;
    }
    if (host_now() - last_progress > 30.0) {
      const int se = stream_error(s);
      if (se) return se;
      return fail(B200SHM_ERR_TIMEOUT, "serve_replay: no progress for 30 s (%llu of %llu done)",
                  (unsigned long long)done, (unsigned long long)n);
    }
  }
  return B200SHM_OK;
}

int b200shm_serve_replay_ordered(const b200shm_request *reqs, uint64_t n, void *stream,
                                 double *seconds, uint64_t *fetched) {
  if (!st().up) return fail(B200SHM_ERR_STATE, "b200shm is not initialised");
  if (n && !reqs) return fail(B200SHM_ERR_ARG, "serve_replay_ordered: null requests");
  cudaStream_t s = pick_stream(stream);
  unsigned long long *h_f = nullptr, *d_f = nullptr;
  if (n) {
    B200_CK(cudaHostAlloc((void **)&h_f, n * sizeof(unsigned long long), cudaHostAllocMapped));
    cudaError_t e = cudaHostGetDevicePointer((void **)&d_f, h_f, 0);
    if (e != cudaSuccess) {
      cudaFreeHost(h_f);
      return cuda_fail(e, "serve_replay_ordered");
    }
    memset(h_f, 0, n * sizeof(unsigned long long));
  }
  B200_CK(cudaStreamSynchronize(s));
  const double t0 = host_now();
  int rc = B200SHM_OK;
  for (uint64_t k = 0; k < n && rc == B200SHM_OK; k++) {
    const b200shm_request &r = reqs[k];
    switch (r.kind) {
    case B200SHM_REQ_REDUCE:
      rc = b200shm_reduce(r.op, r.dtype, r.algo, r.pe_start, r.pe_stride, r.pe_size, r.dest_off,
                          r.src_off, r.n, s);
      break;
    case B200SHM_REQ_FCOLLECT:
      rc = b200shm_fcollect(r.pe_start, r.pe_stride, r.pe_size, r.dest_off, r.src_off, r.n, s);
      break;
    case B200SHM_REQ_ALLTOALL:
      rc = b200shm_alltoall(r.pe_start, r.pe_stride, r.pe_size, r.dest_off, r.src_off, r.n, s);
      break;
    case B200SHM_REQ_PUT:
    case B200SHM_REQ_GET: {
      const int dpe = r.kind == B200SHM_REQ_PUT ? r.pe : r.pe_start;
      const int spe = r.kind == B200SHM_REQ_PUT ? r.pe_start : r.pe;
      void *d = b200shm_ptr(dpe, r.dest_off);
      const void *sp = b200shm_ptr(spe, r.src_off);
      rc = (d && sp) ? b200shm_memcpy(d, sp, r.n, s)
                     : fail(B200SHM_ERR_ARG, "serve_replay_ordered: bad put/get");
      break;
    }
    case B200SHM_REQ_AMO:
      rc = amo_one_launch(r.op, r.dtype, r.pe, r.dest_off, r.value, r.cond, d_f + k, s);
      break;
    default: rc = fail(B200SHM_ERR_ARG, "serve_replay_ordered: request kind %d", r.kind);
    }
  }
  cudaError_t e = cudaStreamSynchronize(s);
  const double t1 = host_now();
  if (rc == B200SHM_OK && e != cudaSuccess) rc = cuda_fail(e, "serve_replay_ordered");
  if (rc == B200SHM_OK) rc = take_status("serve_replay_ordered");
  if (rc == B200SHM_OK) {
    if (seconds) *seconds = t1 - t0;
    if (fetched)
      for (uint64_t k = 0; k < n; k++) fetched[k] = h_f[k];
  }
  if (h_f) cudaFreeHost(h_f);
  return rc;
}

}  // extern "C"
