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
 *  - every request is cut into tiles on the host (a range of elements of a
 *    reduction, a chunk or a run of segments of a copy, one atomic), and a
 *    single device cursor (request << 24 | tile) hands tiles out: a CTA
 *    claims (r, t) only when request r is published, with a compare-and-
 *    swap, so no CTA ever holds a claim it cannot serve and no CTA ever
 *    waits for another CTA;
 *  - the CTA that finishes a request's last tile writes its completion word
 *    (sequence, AMO old value, status) to host memory after a system-scope
 *    fence;
 *  - a CTA with no published work sleeps with a growing back-off; after the
 *    idle limit (or when the host asks it to stop) it exits, holding no
 *    claim, and the host relaunches the kernel when work arrives again.
 *    Every wait in the kernel is bounded by that limit.
 *
 * Results equal the per-call entry points': a reduction combines in the
 * reference algorithm's exact order (a left fold where any order is exact,
 * the algorithm's tree for float SUM/PROD, an exact replay for float
 * MIN/MAX elements whose result depends on operand order).
 */
#include <stdint.h>
#include <string.h>
#include <time.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <type_traits>
#include <vector>

#include "amo_core.cuh"
#include "internal.cuh"
#include "reduce_core.cuh"

namespace b200 {
namespace {

constexpr int kServeThreads = 256;
constexpr int kTileBits = 24;
constexpr unsigned long long kTileMask = (1ull << kTileBits) - 1;
constexpr uint64_t kCopyChunk = 64u << 10;       /* bytes per copy tile            */
constexpr uint64_t kReduceTileRead = 256u << 10; /* source bytes per reduce tile   */

/* A ring slot (mapped host memory, written by the host). */
struct alignas(16) SReq {
  b200shm_request r;        /* 72 bytes */
  unsigned long long ntiles; /* >= 1 */
  unsigned long long unit;   /* REDUCE: elements per tile; copies: bytes per chunk */
  unsigned long long nseg;   /* copies: segments of r.n bytes */
  unsigned long long spt;    /* copies with small segments: segments per tile, else 0 */
  unsigned long long cps;    /* copies with large segments: chunks per segment */
  unsigned long long seq;    /* ticket + 1 once the slot holds the request; written last */
  unsigned long long pad;
};
static_assert(sizeof(SReq) == 128, "ring slot of 128 bytes");

/* A completion word (mapped host memory, written by the device). */
struct alignas(32) SDone {
  unsigned long long seq; /* ticket + 1 once complete */
  unsigned long long fetched;
  int status;
  int pad[3];
};

/* Host-written control words (mapped host memory). */
struct SCtl {
  unsigned long long tail; /* requests published */
  int stop;
  int pad[13];
};

/* Device-side state. */
struct SDev {
  unsigned long long cursor;      /* next (request, tile) to hand out        */
  unsigned long long tail_mirror; /* last tail a CTA read from host memory   */
  unsigned int poll_lock;         /* one CTA at a time reads the host tail   */
  unsigned int pad;
};

struct SArgs {
  const SReq *ring;
  SDone *done;
  const SCtl *ctl;
  SDev *dev;
  unsigned int *tiles_done; /* per slot */
  unsigned long long *mtag; /* per slot: ticket + 1 of the mirrored request, 0 while written */
  SReq *mreq;               /* per slot: device copy of the request */
  unsigned int Q;
  char *base;
  uint64_t slice;
  int npes;
  unsigned long long idle_ns;
};

__device__ __forceinline__ unsigned long long ld_acquire_sys(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.sys.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_sys(unsigned long long *p, unsigned long long v) {
  asm volatile("st.release.sys.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
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

/* Read request r into *out (thread 0): 1 = consistent copy, 0 = the slot
 * was already recycled for a later request (so r is complete and all its
 * tiles were handed out), -1 = not visible yet.  The device mirror is a
 * seqlock: the tag is cleared, the copy written, the tag set. */
__device__ int read_req(const SArgs &a, unsigned long long r, SReq *out) {
  const unsigned slot = (unsigned)(r % a.Q);
  if (vld(&a.mtag[slot]) == r + 1) {
    __threadfence();
    copy_words(out, &a.mreq[slot]);
    __threadfence();
    if (vld(&a.mtag[slot]) == r + 1) return 1;
  }
  const unsigned long long s1 = ld_acquire_sys(&a.ring[slot].seq);
  if (s1 > r + 1) return 0;
  if (s1 < r + 1) return -1;
  copy_words(out, &a.ring[slot]);
  __threadfence_system();
  const unsigned long long s2 = ld_acquire_sys(&a.ring[slot].seq);
  if (s2 != r + 1) return s2 > r + 1 ? 0 : -1;
  *(volatile unsigned long long *)&a.mtag[slot] = 0;
  __threadfence();
  unsigned long long *d = (unsigned long long *)&a.mreq[slot];
  const unsigned long long *w = (const unsigned long long *)out;
  for (int i = 0; i < 16; i++) ((volatile unsigned long long *)d)[i] = w[i];
  __threadfence();
  *(volatile unsigned long long *)&a.mtag[slot] = r + 1;
  return 1;
}

/* Claim the next tile (thread 0).  Returns 1 with *claimed = (r << 24 | t)
 * and the request in *req, or 0 when the CTA should exit (stop requested or
 * idle past the limit, in both cases with no published work unclaimed). */
__device__ int claim(const SArgs &a, SReq *req, unsigned long long *claimed,
                     unsigned long long idle_since) {
  unsigned backoff = 32;
  for (;;) {
    const unsigned long long v = vld(&a.dev->cursor);
    const unsigned long long r = v >> kTileBits, t = v & kTileMask;
    unsigned long long tl = vld(&a.dev->tail_mirror);
    if (r >= tl) {
      if (atomicCAS(&a.dev->poll_lock, 0u, 1u) == 0u) {
        tl = ld_acquire_sys(&a.ctl->tail);
        atomicMax(&a.dev->tail_mirror, tl);
        atomicExch(&a.dev->poll_lock, 0u);
      }
      if (r >= tl) {
        if (*(const volatile int *)&a.ctl->stop) return 0;
        if (now_ns() - idle_since > a.idle_ns) return 0;
        __nanosleep(backoff);
        backoff = backoff < 1024 ? backoff * 2 : 1024;
        continue;
      }
    }
    const int rc = read_req(a, r, req);
    if (rc < 0) {
      if (now_ns() - idle_since > a.idle_ns) return 0;
      __nanosleep(64);
      continue;
    }
    const unsigned long long nt = rc ? req->ntiles : 0;
    if (t >= nt) {
      atomicCAS(&a.dev->cursor, v, (r + 1) << kTileBits);
      continue;
    }
    if (atomicCAS(&a.dev->cursor, v, v + 1) == v) {
      *claimed = v;
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

/* The tree the algorithm builds for float SUM/PROD (the value is the same
 * in every member, the ops being exactly commutative), leaves loaded four
 * at a time.  Binomial: op(upper block, lower block), then the set bits of
 * P from the lowest (reduce.c:137-154); butterfly: extra members folded as
 * op(extra, own), then log2(p2s) levels (reduce.c:206-272). */
template <class T, int OP>
__device__ T tree_value(const char *s, uint64_t step, int P, int p2s, int logp2s, bool binomial) {
  T stk[kMaxLevels + 1];
  if (binomial) {
    for (int j0 = 0; j0 < P; j0 += 4) {
      T x[4];
#pragma unroll
      for (int u = 0; u < 4; u++)
        if (j0 + u < P) x[u] = ldv<T>(s + (uint64_t)(j0 + u) * step);
#pragma unroll
      for (int u = 0; u < 4; u++)
        if (j0 + u < P) {
          const int j = j0 + u;
          T y = x[u];
          for (int L = 0; L <= kMaxLevels; L++) {
            if (j & (1 << L)) {
              y = apply<OP>(y, stk[L]);
            } else {
              stk[L] = y;
              break;
            }
          }
        }
    }
    bool have = false;
    T v = stk[0];
    for (int L = 0; L <= kMaxLevels; L++)
      if (P & (1 << L)) {
        v = have ? apply<OP>(v, stk[L]) : stk[L];
        have = true;
      }
    return v;
  }
  for (int q0 = 0; q0 < p2s; q0 += 4) {
    T x[4], e[4];
    bool ex[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      ex[u] = false;
      if (q0 + u < p2s) {
        const int own = (int)(((long long)(q0 + u) * P + p2s - 1) >> logp2s);
        const int nxt = (int)(((long long)(q0 + u + 1) * P + p2s - 1) >> logp2s);
        x[u] = ldv<T>(s + (uint64_t)own * step);
        ex[u] = nxt - own == 2;
        if (ex[u]) e[u] = ldv<T>(s + (uint64_t)(own + 1) * step);
      }
    }
#pragma unroll
    for (int u = 0; u < 4; u++)
      if (q0 + u < p2s) {
        const int leaf = q0 + u;
        T y = ex[u] ? apply<OP>(e[u], x[u]) : x[u];
        for (int L = 0; L <= kMaxLevels; L++) {
          if (leaf & (1 << L)) {
            y = apply<OP>(stk[L], y);
          } else {
            stk[L] = y;
            break;
          }
        }
      }
  }
  return stk[logp2s];
}

template <class T, int OP>
__device__ void serve_reduce(const SReq &q, uint64_t e0, uint64_t e1, char *base,
                             uint64_t slice) {
  const b200shm_request &r = q.r;
  const int P = r.pe_size;
  int p2s = 1, lg = 0;
  while (p2s * 2 <= P) {
    p2s *= 2;
    lg++;
  }
  const uint64_t step = (uint64_t)(P > 1 ? r.pe_stride : 1) * slice;
  const char *src0 = base + (uint64_t)r.pe_start * slice + r.src_off;
  char *dst0 = base + (uint64_t)r.pe_start * slice + r.dest_off;
  constexpr bool FL = std::is_floating_point<T>::value;
  constexpr bool MM = OP == B200SHM_MIN || OP == B200SHM_MAX;
  const bool chain = !FL || MM || r.algo == B200SHM_LINEAR;
  for (uint64_t e = e0 + threadIdx.x; e < e1; e += kServeThreads) {
    const char *s = src0 + e * sizeof(T);
    T v;
    if (chain) {
      v = ldv<T>(s);
      unsigned cls = 0;
      if constexpr (FL && MM) cls = fclass(v);
      for (int j = 1; j < P; j += 8) {
        T x[8];
#pragma unroll
        for (int u = 0; u < 8; u++)
          if (j + u < P) x[u] = ldv<T>(s + (uint64_t)(j + u) * step);
#pragma unroll
        for (int u = 0; u < 8; u++)
          if (j + u < P) {
            v = apply<OP>(v, x[u]);
            if constexpr (FL && MM) cls |= fclass(x[u]);
          }
      }
      if constexpr (FL && MM) {
        /* order-dependent element: replay the algorithm's operand order
         * (the left fold above already is the linear algorithm's) */
        if (ambiguous(cls) && r.algo != B200SHM_LINEAR) {
          auto get = [&](int j) { return ldv<T>(s + (uint64_t)j * step); };
          const bool lower = e < r.n / 2;
          if (r.algo == B200SHM_REC_DBL) {
            for (int qq = 0; qq < p2s; qq++) {
              const T x = exact_value<T, OP>(get, P, p2s, lg, r.algo, lower, qq);
              const int as = p2s_member(qq, P, p2s);
              stv<T>(dst0 + (uint64_t)as * step + e * sizeof(T), x);
              if (p2s_extra(qq, P, p2s)) stv<T>(dst0 + (uint64_t)(as + 1) * step + e * sizeof(T), x);
            }
            continue;
          }
          int qq = 0;
          if (r.algo == B200SHM_RABENSEIFNER || r.algo == B200SHM_RABENSEIFNER2)
            qq = rev_bits(rab_block(e, r.n, p2s), lg);
          v = exact_value<T, OP>(get, P, p2s, lg, r.algo, lower, qq);
        }
      }
    } else {
      v = tree_value<T, OP>(s, step, P, p2s, lg, r.algo == B200SHM_BINOMIAL);
    }
    char *d = dst0 + e * sizeof(T);
    for (int j = 0; j < P; j++) stv<T>(d + (uint64_t)j * step, v);
  }
}

template <class T>
__device__ void serve_reduce_int(const SReq &q, uint64_t e0, uint64_t e1, char *base,
                                 uint64_t slice) {
  switch (q.r.op) {
  case B200SHM_AND: serve_reduce<T, B200SHM_AND>(q, e0, e1, base, slice); break;
  case B200SHM_OR: serve_reduce<T, B200SHM_OR>(q, e0, e1, base, slice); break;
  case B200SHM_XOR: serve_reduce<T, B200SHM_XOR>(q, e0, e1, base, slice); break;
  case B200SHM_MIN: serve_reduce<T, B200SHM_MIN>(q, e0, e1, base, slice); break;
  case B200SHM_MAX: serve_reduce<T, B200SHM_MAX>(q, e0, e1, base, slice); break;
  case B200SHM_SUM: serve_reduce<T, B200SHM_SUM>(q, e0, e1, base, slice); break;
  default: serve_reduce<T, B200SHM_PROD>(q, e0, e1, base, slice); break;
  }
}
template <class T>
__device__ void serve_reduce_flt(const SReq &q, uint64_t e0, uint64_t e1, char *base,
                                 uint64_t slice) {
  switch (q.r.op) {
  case B200SHM_MIN: serve_reduce<T, B200SHM_MIN>(q, e0, e1, base, slice); break;
  case B200SHM_MAX: serve_reduce<T, B200SHM_MAX>(q, e0, e1, base, slice); break;
  case B200SHM_SUM: serve_reduce<T, B200SHM_SUM>(q, e0, e1, base, slice); break;
  default: serve_reduce<T, B200SHM_PROD>(q, e0, e1, base, slice); break;
  }
}

/* ---- copies ------------------------------------------------------------------ */
/* Copy n bytes with threads [tid, tid + nthr) at the widest width that the
 * two addresses and the length allow. */
__device__ void span_copy(char *dst, const char *src, uint64_t n, int tid, int nthr) {
  const uint64_t al = (uint64_t)dst | (uint64_t)src | n;
  if ((al & 15) == 0) {
    for (uint64_t i = tid; i < n / 16; i += nthr) ((uint4 *)dst)[i] = ((const uint4 *)src)[i];
  } else if ((al & 7) == 0) {
    for (uint64_t i = tid; i < n / 8; i += nthr)
      ((unsigned long long *)dst)[i] = ((const unsigned long long *)src)[i];
  } else if ((al & 3) == 0) {
    for (uint64_t i = tid; i < n / 4; i += nthr) ((unsigned *)dst)[i] = ((const unsigned *)src)[i];
  } else {
    for (uint64_t i = tid; i < n; i += nthr) dst[i] = src[i];
  }
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

__device__ void serve_copy(const SReq &q, uint64_t t, char *base, uint64_t slice) {
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

/* ---- the loop -------------------------------------------------------------------- */
__global__ void __launch_bounds__(kServeThreads) k_serve(const SArgs a) {
  __shared__ SReq s_req;
  __shared__ unsigned long long s_claim;
  __shared__ int s_go;
  __shared__ unsigned long long s_fetched;
  __shared__ int s_status;
  unsigned long long idle_since = now_ns();
  for (;;) {
    if (threadIdx.x == 0) {
      s_go = claim(a, &s_req, &s_claim, idle_since);
      s_fetched = 0;
      s_status = 0;
    }
    __syncthreads();
    if (!s_go) return;
    const unsigned long long r = s_claim >> kTileBits, t = s_claim & kTileMask;
    const SReq &q = s_req;
    switch (q.r.kind) {
    case B200SHM_REQ_REDUCE: {
      const uint64_t e0 = t * q.unit;
      const uint64_t e1 = e0 + q.unit < q.r.n ? e0 + q.unit : q.r.n;
      switch (q.r.dtype) {
      case B200SHM_I32: serve_reduce_int<int32_t>(q, e0, e1, a.base, a.slice); break;
      case B200SHM_U32: serve_reduce_int<uint32_t>(q, e0, e1, a.base, a.slice); break;
      case B200SHM_I64: serve_reduce_int<int64_t>(q, e0, e1, a.base, a.slice); break;
      case B200SHM_U64: serve_reduce_int<uint64_t>(q, e0, e1, a.base, a.slice); break;
      case B200SHM_F32: serve_reduce_flt<float>(q, e0, e1, a.base, a.slice); break;
      case B200SHM_F64: serve_reduce_flt<double>(q, e0, e1, a.base, a.slice); break;
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
          s_fetched = amo_one<unsigned int>(q.r.op, (unsigned int *)p, (unsigned int)q.r.value,
                                            (unsigned int)q.r.cond);
      }
      break;
    default:
      if (threadIdx.x == 0) s_status = B200SHM_STATUS_BADREQ;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
      const unsigned slot = (unsigned)(r % a.Q);
      __threadfence_system();
      if (atomicAdd(&a.tiles_done[slot], 1u) + 1ull == q.ntiles) {
        a.tiles_done[slot] = 0;
        SDone *dn = &a.done[slot];
        *(volatile unsigned long long *)&dn->fetched = s_fetched;
        *(volatile int *)&dn->status = s_status;
        __threadfence_system();
        st_release_sys(&dn->seq, r + 1);
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
  std::mutex mu;
};

namespace b200 {
namespace {

int ensure_running(b200shm_server *s) {
  const cudaError_t e = cudaStreamQuery(s->stream);
  if (e == cudaErrorNotReady) return B200SHM_OK;
  if (e != cudaSuccess) return cuda_fail(e, "serving loop");
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
        (rc = check_extent(r.dest_off, bytes, "serve reduce dest")))
      return rc;
    if (r.dest_off != r.src_off && overlaps(r.dest_off, bytes, r.src_off, bytes))
      return fail(B200SHM_ERR_ARG, "serve: reduce dest and source overlap");
    uint64_t unit = kReduceTileRead / ((uint64_t)r.pe_size * es);
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
        (rc = check_extent(r.dest_off, P * r.n, "serve dest")))
      return rc;
    if (overlaps(r.dest_off, P * r.n, r.src_off, sb))
      return fail(B200SHM_ERR_ARG, "serve: dest and source overlap");
    q->nseg = P * P;
    break;
  }
  case B200SHM_REQ_PUT:
  case B200SHM_REQ_GET: {
    if (r.pe_start < 0 || r.pe_start >= S.npes || r.pe < 0 || r.pe >= S.npes)
      return fail(B200SHM_ERR_ARG, "serve: PE out of range");
    if ((rc = check_extent(r.src_off, r.n, "serve source")) ||
        (rc = check_extent(r.dest_off, r.n, "serve dest")))
      return rc;
    const int dpe = r.kind == B200SHM_REQ_PUT ? r.pe : r.pe_start;
    const int spe = r.kind == B200SHM_REQ_PUT ? r.pe_start : r.pe;
    if (dpe == spe && overlaps(r.dest_off, r.n, r.src_off, r.n))
      return fail(B200SHM_ERR_ARG, "serve: dest and source overlap");
    q->nseg = 1;
    break;
  }
  case B200SHM_REQ_AMO: {
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
    q->unit = kCopyChunk;
    if (r.n >= kCopyChunk) {
      q->cps = (r.n + kCopyChunk - 1) / kCopyChunk;
      q->spt = 0;
      q->ntiles = q->nseg * q->cps;
    } else {
      q->spt = r.n ? kCopyChunk / r.n : q->nseg;
      if (q->spt < 1) q->spt = 1;
      q->ntiles = (q->nseg + q->spt - 1) / q->spt;
    }
    if (q->ntiles == 0) q->ntiles = 1;
  }
  if (q->ntiles > kTileMask) return fail(B200SHM_ERR_ARG, "serve: request of more than 2^24 tiles");
  return B200SHM_OK;
}

}  // namespace
}  // namespace b200

extern "C" {

int b200shm_serve_start(uint32_t queue_slots, int ctas, double idle_seconds,
                        b200shm_server **out) {
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
  const double idle = idle_seconds > 0 ? idle_seconds : 1.0;
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
  a.mtag = (unsigned long long *)(s->d_mem + 256 + (size_t)s->Q * sizeof(SReq));
  a.tiles_done = (unsigned *)(a.mtag + s->Q);
  a.Q = s->Q;
  a.base = st().base;
  a.slice = st().slice;
  a.npes = st().npes;
  a.idle_ns = (unsigned long long)(idle * 1e9);
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
  memcpy(dst, &q, sizeof(SReq));
  std::atomic_thread_fence(std::memory_order_release);
  *(volatile unsigned long long *)&dst->seq = tk + 1;
  std::atomic_thread_fence(std::memory_order_release);
  *(volatile unsigned long long *)&s->h_ctl->tail = tk + 1;
  std::atomic_thread_fence(std::memory_order_seq_cst);
  s->tail = tk + 1;
  if (ticket) *ticket = tk;
  return ensure_running(s);
}

int b200shm_serve_poll(b200shm_server *s, uint64_t ticket, uint64_t *fetched) {
  if (!s) return fail(B200SHM_ERR_ARG, "serve_poll: null server");
  const SDone *d = &s->h_done[ticket % s->Q];
  const unsigned long long seq = *(const volatile unsigned long long *)&d->seq;
  if (seq < ticket + 1) return 0;
  std::atomic_thread_fence(std::memory_order_acquire);
  if (fetched) *fetched = *(const volatile unsigned long long *)&d->fetched;
  const int status = *(const volatile int *)&d->status;
  if (status) return fail(B200SHM_ERR_ARG, "serve: request %llu was refused on the device",
                          (unsigned long long)ticket);
  return 1;
}

int b200shm_serve_wait(b200shm_server *s, uint64_t ticket, double timeout_seconds,
                       uint64_t *fetched) {
  const double t0 = host_now();
  for (unsigned it = 0;; it++) {
    const int rc = b200shm_serve_poll(s, ticket, fetched);
    if (rc) return rc < 0 ? rc : B200SHM_OK;
    if ((it & 1023) == 1023) {
      std::lock_guard<std::mutex> lk(s->mu);
      const int er = ensure_running(s); /* the kernel may have idled out meanwhile */
      if (er) return er;
    }
    if (host_now() - t0 > timeout_seconds)
      return fail(B200SHM_ERR_TIMEOUT, "serve_wait: request %llu not complete after %.3f s",
                  (unsigned long long)ticket, timeout_seconds);
  }
}

int b200shm_serve_stop(b200shm_server *s) {
  if (!s) return B200SHM_OK;
  *(volatile int *)&s->h_ctl->stop = 1;
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
    if ((it & 4095) == 4095 && !pend.empty()) {
      std::lock_guard<std::mutex> lk(s->mu);
      const int er = ensure_running(s);
      if (er) return er;
    }
    if (host_now() - last_progress > 30.0)
      return fail(B200SHM_ERR_TIMEOUT, "serve_replay: no progress for 30 s (%llu of %llu done)",
                  (unsigned long long)done, (unsigned long long)n);
  }
  return B200SHM_OK;
}

}  // extern "C"
