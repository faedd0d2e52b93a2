/*
 * span.cu -- teams that span GPUs: the cross-GPU halves of the collectives
 * as kernels that read the other GPUs' arenas directly.
 *
 * Every GPU runs its own engine (its own arena of npes slices, the same
 * npes and slice size on every GPU); a team of G x L members puts L
 * members on each of G GPUs.  The arenas are shared with CUDA IPC
 * (b200shm_ipc_handle / b200shm_peer_open), so a kernel on one GPU loads
 * another GPU's symmetric objects over NVLink with ordinary loads -- no
 * multicast of any kind -- and writes only its own GPU's members.  The
 * caller keeps the phases apart with a host barrier across the processes
 * (every rank's inputs ready before any rank reads them; every rank done
 * reading before any input is overwritten), so no kernel ever waits on
 * another GPU's kernel.
 *
 *  - b200shm_span_combine: the butterfly levels of a reduction across the
 *    G ranks' partial vectors (round j pairs rank r with r ^ 2^j and keeps
 *    op(own, partner), as the reference's rec_dbl does member by member,
 *    src/shcoll/src/reduce.c:250-272), fused with the write of the result
 *    to every local member's dest;
 *  - b200shm_span_fcollect: every member's block, read once from the GPU
 *    that holds it, written to every local member's dest
 *    (src/shcoll/src/fcollect.c:32-484);
 *  - b200shm_span_alltoall: each local member's dest blocks, read from the
 *    members that hold them on whichever GPU (src/shcoll/src/alltoall.c:
 *    75-201);
 *  - b200shm_span_amo: one-sided atomics on any member's words, run by the
 *    calling GPU as system-scope atomics on the owner's arena (the
 *    reference's shmemc_ctx_{fadd,...} over UCX, src/shmemc/ucx/comms.c:
 *    409-671): no other rank takes part.
 */
#include <stdint.h>
#include <string.h>

#include <map>
#include <mutex>
#include <string>
#include <type_traits>

#include "internal.cuh"
#include "reduce_core.cuh"

namespace b200 {
namespace {

constexpr int kSpanMax = 16; /* GPUs a team spans, at most */

struct SpanPtrs {
  const char *p[kSpanMax];
};

__device__ __forceinline__ uint4 ld16(const char *p) {
  uint4 u;
  asm volatile("ld.global.v4.u32 {%0,%1,%2,%3}, [%4];"
               : "=r"(u.x), "=r"(u.y), "=r"(u.z), "=r"(u.w)
               : "l"(p));
  return u;
}
/* Stores are streaming (evict-first): every byte written here is written
 * once and not read again by the kernel.  The fcollect span kernel (one
 * read, L writes of each byte) ran 5.99 TB/s with them against 5.21 with
 * write-back stores on 8 ranks x 8 members x 256 KiB; alltoall moved the
 * same either way. */
#ifndef B200_SPAN_ST
#define B200_SPAN_ST "st.global.cs"
#endif
__device__ __forceinline__ void st16(char *p, uint4 u) {
  asm volatile(B200_SPAN_ST ".v4.u32 [%0], {%1,%2,%3,%4};" ::"l"(p), "r"(u.x), "r"(u.y), "r"(u.z),
               "r"(u.w)
               : "memory");
}

/* V consecutive elements: one 16-byte access when VEC, else one element */
template <class T, bool VEC>
struct SpanUnit {
  static constexpr int V = VEC ? 16 / (int)sizeof(T) : 1;
  union {
    uint4 raw;
    T x[V];
  };
};

template <class T, bool VEC>
__device__ __forceinline__ SpanUnit<T, VEC> ld_unit(const char *p) {
  SpanUnit<T, VEC> u;
  if constexpr (VEC) u.raw = ld16(p);
  else u.x[0] = *(const T *)p;
  return u;
}

template <class T, bool VEC>
__device__ __forceinline__ void st_unit(char *p, const SpanUnit<T, VEC> &u) {
  if constexpr (VEC) st16(p, u.raw);
  else *(T *)p = u.x[0];
}

/* The butterfly across G ranks, as rank `rank` finishes it.  After level l
 * the rank x holds the reduction over its block of 2^(l+1) ranks, formed as
 * op(own block value, partner block value) with partner x ^ 2^l.  Only the
 * G-1 combines on this rank's own path are needed: indexing the partials
 * relative to the rank (slot y holds rank y ^ rank's partial; the host
 * orders the pointers so), level l updates the slots y with y's low l+1
 * bits zero, slot[y] = op(slot[y], slot[y ^ 2^l]), and slot 0 ends with
 * the rank's result.  Every slot and level index is static. */
template <class T, int OP, bool VEC>
__device__ __forceinline__ SpanUnit<T, VEC> span_unit(const SpanPtrs &src, int G, uint64_t byte) {
  constexpr int V = SpanUnit<T, VEC>::V;
  SpanUnit<T, VEC> w[kSpanMax];
#pragma unroll
  for (int g = 0; g < kSpanMax; g++)
    if (g < G) w[g] = ld_unit<T, VEC>(src.p[g] + byte);
#pragma unroll
  for (int lvl = 0; lvl < 4; lvl++) {
    const int b = 1 << lvl;
    if (b < G) {
#pragma unroll
      for (int y = 0; y < kSpanMax; y += 2 * b)
        if (y < G) {
#pragma unroll
          for (int i = 0; i < V; i++) w[y].x[i] = apply<OP>(w[y].x[i], w[y + b].x[i]);
        }
    }
  }
  return w[0];
}

/* the combine over n elements, fused with the write of the result to the
 * L local members (dst0 + j*dstep); 16-byte units first, then the tail */
template <class T, int OP, bool VEC>
__global__ void __launch_bounds__(256) k_span_combine(const SpanPtrs src, int G, char *dst0,
                                                      uint64_t dstep, int L, uint64_t n) {
  constexpr uint64_t U = sizeof(SpanUnit<T, VEC>::x);
  const uint64_t units = n * sizeof(T) / U;
  const uint64_t t0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t nt = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t u = t0; u < units; u += nt) {
    const SpanUnit<T, VEC> r = span_unit<T, OP, VEC>(src, G, u * U);
    for (int j = 0; j < L; j++) st_unit<T, VEC>(dst0 + (uint64_t)j * dstep + u * U, r);
  }
  if constexpr (VEC) {
    for (uint64_t e = units * (U / sizeof(T)) + t0; e < n; e += nt) {
      const SpanUnit<T, false> r = span_unit<T, OP, false>(src, G, e * sizeof(T));
      for (int j = 0; j < L; j++) st_unit<T, false>(dst0 + (uint64_t)j * dstep + e * sizeof(T), r);
    }
  }
}

/* fcollect: source member m = q*L + k lives on GPU q; blockIdx.y walks the
 * members, each vector read once and written to the L local members */
template <bool VEC>
__global__ void __launch_bounds__(256) k_span_fcollect(const __grid_constant__ SpanPtrs base, uint64_t first,
                                                       uint64_t step, int L, int M, char *own,
                                                       uint64_t dest_off, uint64_t src_off,
                                                       uint64_t nbytes) {
  const uint64_t n = VEC ? nbytes / 16 : nbytes;
  for (int m = blockIdx.y; m < M; m += gridDim.y) {
    const char *src = base.p[m / L] + first + (uint64_t)(m % L) * step + src_off;
    char *dst = own + first + dest_off + (uint64_t)m * nbytes;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
         v += (uint64_t)gridDim.x * blockDim.x) {
      if constexpr (VEC) {
        const uint4 u = ld16(src + v * 16);
        for (int j = 0; j < L; j++) st16(dst + (uint64_t)j * step + v * 16, u);
      } else {
        const char c = src[v];
        for (int j = 0; j < L; j++) dst[(uint64_t)j * step + v] = c;
      }
    }
  }
}

/* alltoall: local member j's dest block m (m = q*L + k, on GPU q) = member
 * m's source block rank*L + j; pairs (m, j) over blockIdx.y */
template <bool VEC>
__global__ void __launch_bounds__(256) k_span_alltoall(const __grid_constant__ SpanPtrs base, uint64_t first,
                                                       uint64_t step, int L, int M, int rank,
                                                       char *own, uint64_t dest_off,
                                                       uint64_t src_off, uint64_t B) {
  const uint64_t n = VEC ? B / 16 : B;
  const uint64_t pairs = (uint64_t)M * (uint64_t)L;
  for (uint64_t pr = blockIdx.y; pr < pairs; pr += gridDim.y) {
    const int m = (int)(pr / (uint64_t)L), j = (int)(pr % (uint64_t)L);
    const char *src = base.p[m / L] + first + (uint64_t)(m % L) * step + src_off +
                      ((uint64_t)rank * L + j) * B;
    char *dst = own + first + (uint64_t)j * step + dest_off + (uint64_t)m * B;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
         v += (uint64_t)gridDim.x * blockDim.x) {
      if constexpr (VEC) st16(dst + v * 16, ld16(src + v * 16));
      else dst[v] = src[v];
    }
  }
}

/* one AMO as a system-scope atomic: the word may be updated at the same
 * time by kernels of other GPUs through their mappings of this arena, and
 * only system scope makes those updates atomic with each other */
template <class W>
__device__ __forceinline__ W amo_sys(int amo, W *p, W v, W c) {
  switch (amo) {
  case B200SHM_AMO_FETCH_ADD:
  case B200SHM_AMO_ADD: return atomicAdd_system(p, v);
  case B200SHM_AMO_FETCH_INC:
  case B200SHM_AMO_INC: return atomicAdd_system(p, (W)1);
  case B200SHM_AMO_SWAP:
  case B200SHM_AMO_SET: return atomicExch_system(p, v);
  case B200SHM_AMO_CSWAP: return atomicCAS_system(p, c, v);
  case B200SHM_AMO_FETCH: return atomicAdd_system(p, (W)0);
  case B200SHM_AMO_FETCH_AND:
  case B200SHM_AMO_AND: return atomicAnd_system(p, v);
  case B200SHM_AMO_FETCH_OR:
  case B200SHM_AMO_OR: return atomicOr_system(p, v);
  default: return atomicXor_system(p, v);
  }
}

/* atomics on (member, offset) targets of a spanning team: member m = q*L +
 * k is PE first/slice + k*step/slice of GPU q's arena */
template <class W>
__global__ void __launch_bounds__(256) k_span_amo(const __grid_constant__ SpanPtrs base, int M,
                                                  int L, uint64_t first, uint64_t step,
                                                  uint64_t slice, int amo, uint64_t nops,
                                                  const int32_t *member, const uint64_t *off,
                                                  const W *value, const W *cond, W *fetched,
                                                  int *status) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nops;
       k += (uint64_t)gridDim.x * blockDim.x) {
    const int m = member[k];
    const uint64_t o = off[k];
    if (m < 0 || m >= M || o > slice - sizeof(W) || (o % sizeof(W)) != 0) {
      atomicOr(status, (int)B200SHM_STATUS_BADREQ);
      continue;
    }
    W *t = (W *)(base.p[m / L] + first + (uint64_t)(m % L) * step + o);
    const W old = amo_sys<W>(amo, t, value ? value[k] : (W)0, cond ? cond[k] : (W)0);
    if (fetched) fetched[k] = old;
  }
}

template <class T, int OP>
void combine_launch(bool vec, dim3 g, cudaStream_t s, const SpanPtrs &p, int G, char *d,
                    uint64_t step, int L, uint64_t n) {
  if (vec && sizeof(T) < 16) k_span_combine<T, OP, true><<<g, 256, 0, s>>>(p, G, d, step, L, n);
  else k_span_combine<T, OP, false><<<g, 256, 0, s>>>(p, G, d, step, L, n);
}

template <class T>
int combine_for(int op, bool vec, dim3 g, cudaStream_t s, const SpanPtrs &p, int G, char *d,
                uint64_t step, int L, uint64_t n) {
  constexpr bool kInt = std::is_integral<T>::value;
  constexpr bool kCplx = std::is_same<T, cf32>::value || std::is_same<T, cf64>::value;
  switch (op) {
  case B200SHM_AND: if constexpr (kInt) { combine_launch<T, B200SHM_AND>(vec, g, s, p, G, d, step, L, n); return B200SHM_OK; } break;
  case B200SHM_OR: if constexpr (kInt) { combine_launch<T, B200SHM_OR>(vec, g, s, p, G, d, step, L, n); return B200SHM_OK; } break;
  case B200SHM_XOR: if constexpr (kInt) { combine_launch<T, B200SHM_XOR>(vec, g, s, p, G, d, step, L, n); return B200SHM_OK; } break;
  case B200SHM_MIN: if constexpr (!kCplx) { combine_launch<T, B200SHM_MIN>(vec, g, s, p, G, d, step, L, n); return B200SHM_OK; } break;
  case B200SHM_MAX: if constexpr (!kCplx) { combine_launch<T, B200SHM_MAX>(vec, g, s, p, G, d, step, L, n); return B200SHM_OK; } break;
  case B200SHM_SUM: combine_launch<T, B200SHM_SUM>(vec, g, s, p, G, d, step, L, n); return B200SHM_OK;
  case B200SHM_PROD: combine_launch<T, B200SHM_PROD>(vec, g, s, p, G, d, step, L, n); return B200SHM_OK;
  default: break;
  }
  return fail(B200SHM_ERR_UNSUPPORTED, "span_combine: op %d on this dtype", op);
}

/* the peers' arenas mapped in this process, by IPC handle: a handle opened
 * twice shares one mapping (counted), and finalize closes what is left */
struct PeerMap {
  void *base;
  int refs;
};
struct Peers {
  std::mutex mu;
  std::map<std::string, PeerMap> by_handle;
};
Peers &peers() {
  static Peers p;
  return p;
}

/* validation shared by the span entry points */
int span_check(int G, int rank, const uint64_t *addrs, int pe_start, int pe_stride, int L) {
  if (G < 1 || G > kSpanMax || (G & (G - 1)))
    return fail(B200SHM_ERR_ARG, "span: %d GPUs (a power of two up to %d)", G, kSpanMax);
  if (rank < 0 || rank >= G) return fail(B200SHM_ERR_ARG, "span: rank %d of %d", rank, G);
  if (!addrs) return fail(B200SHM_ERR_ARG, "span: null address table");
  for (int g = 0; g < G; g++)
    if (!addrs[g]) return fail(B200SHM_ERR_ARG, "span: no address for rank %d", g);
  return check_team(pe_start, pe_stride, L);
}

/* [a, a + bytes) lies wholly inside this process's arena or inside an open
 * peer mapping.  A peer's arena has this one's geometry (npes slices of
 * `slice` bytes): every rank of a spanning team initialises the engine with
 * the same PE count and heap size.  Checked before any launch, so an
 * address from nowhere is refused instead of faulting the kernel. */
bool known_range(uint64_t a, uint64_t bytes) {
  const uint64_t len = (uint64_t)st().npes * st().slice;
  auto inside = [&](uint64_t b) { return a >= b && bytes <= len && a - b <= len - bytes; };
  if (inside((uint64_t)(uintptr_t)st().base)) return true;
  std::lock_guard<std::mutex> lk(peers().mu);
  for (const auto &kv : peers().by_handle)
    if (inside((uint64_t)(uintptr_t)kv.second.base)) return true;
  return false;
}

/* Each rank's base, as the span kernels read it: its members' slices
 * [base + first, base + first + (L-1)*step + slice) are all they touch
 * there (offsets within a slice are checked separately). */
int check_bases(const char *what, int G, const uint64_t *bases, uint64_t first, uint64_t step,
                int L) {
  const uint64_t span = (uint64_t)(L - 1) * step + st().slice;
  for (int g = 0; g < G; g++)
    if (bases[g] > UINT64_MAX - first || !known_range(bases[g] + first, span))
      return fail(B200SHM_ERR_ARG,
                  "%s: rank %d's base %#llx is not in this arena or an open peer mapping", what,
                  g, (unsigned long long)bases[g]);
  return B200SHM_OK;
}

}  // namespace

/* at finalize: every peer mapping still open is closed */
void span_teardown() {
  std::lock_guard<std::mutex> lk(peers().mu);
  for (auto &kv : peers().by_handle) (void)cudaIpcCloseMemHandle(kv.second.base);
  peers().by_handle.clear();
  (void)cudaGetLastError();
}

}  // namespace b200

using namespace b200;

extern "C" {

int b200shm_ipc_handle(void *handle) {
  if (!st().up) return fail(B200SHM_ERR_STATE, "b200shm is not initialised");
  if (!handle) return fail(B200SHM_ERR_ARG, "ipc_handle: null handle");
  if (st().managed)
    return fail(B200SHM_ERR_UNSUPPORTED, "ipc_handle: a managed-memory arena cannot be shared");
  cudaIpcMemHandle_t h;
  B200_CK(cudaIpcGetMemHandle(&h, st().base));
  memcpy(handle, &h, sizeof(h));
  return B200SHM_OK;
}

int b200shm_peer_open(const void *handle, void **peer_base) {
  if (!st().up) return fail(B200SHM_ERR_STATE, "b200shm is not initialised");
  if (!handle || !peer_base) return fail(B200SHM_ERR_ARG, "peer_open: null argument");
  std::lock_guard<std::mutex> lk(peers().mu);
  std::string key((const char *)handle, sizeof(cudaIpcMemHandle_t));
  auto it = peers().by_handle.find(key);
  if (it != peers().by_handle.end()) { /* mapped already: share the mapping */
    it->second.refs++;
    *peer_base = it->second.base;
    return B200SHM_OK;
  }
  cudaIpcMemHandle_t h;
  memcpy(&h, handle, sizeof(h));
  void *b = nullptr;
  B200_CK(cudaIpcOpenMemHandle(&b, h, cudaIpcMemLazyEnablePeerAccess));
  peers().by_handle[key] = PeerMap{b, 1};
  *peer_base = b;
  return B200SHM_OK;
}

int b200shm_peer_close(void *peer_base) {
  if (!peer_base) return B200SHM_OK;
  std::lock_guard<std::mutex> lk(peers().mu);
  for (auto it = peers().by_handle.begin(); it != peers().by_handle.end(); ++it) {
    if (it->second.base != peer_base) continue;
    if (--it->second.refs > 0) return B200SHM_OK;
    peers().by_handle.erase(it);
    B200_CK(cudaIpcCloseMemHandle(peer_base));
    return B200SHM_OK;
  }
  return fail(B200SHM_ERR_ARG, "peer_close: %p is not an open peer mapping", peer_base);
}

int b200shm_span_combine(int op, int dtype, int G, int rank, const uint64_t *partials,
                         int pe_start, int pe_stride, int pe_count, uint64_t dest_off,
                         uint64_t nelems, void *stream) {
  int rc = span_check(G, rank, partials, pe_start, pe_stride, pe_count);
  if (rc) return rc;
  if (dtype < 0 || dtype >= B200SHM_NDTYPE || dtype == B200SHM_F80)
    return fail(B200SHM_ERR_UNSUPPORTED, "span_combine: dtype %d", dtype);
  const uint64_t es = (uint64_t)kDtypeSize[dtype];
  if (nelems > st().slice / es) return fail(B200SHM_ERR_ARG, "span_combine: nelems too large");
  if ((rc = check_extent(dest_off, nelems * es, "span_combine dest"))) return rc;
  const uint64_t al = es > 8 ? 8 : es; /* the element's own alignment */
  if (dest_off % al) return fail(B200SHM_ERR_ARG, "span_combine: dest misaligned");
  for (int g = 0; g < G; g++)
    if (partials[g] % al) return fail(B200SHM_ERR_ARG, "span_combine: partial %d misaligned", g);
  for (int g = 0; g < G; g++)
    if (!known_range(partials[g], nelems * es))
      return fail(B200SHM_ERR_ARG,
                  "span_combine: rank %d's partial %#llx is not in this arena or an open peer "
                  "mapping", g, (unsigned long long)partials[g]);
  if (nelems == 0) return B200SHM_OK;
  /* slot y holds rank (y ^ rank)'s partial: the kernel's static indexing */
  SpanPtrs p{};
  for (int y = 0; y < G; y++) p.p[y] = (const char *)(uintptr_t)partials[y ^ rank];
  Members m = members(pe_start, pe_stride, pe_count);
  cudaStream_t s = pick_stream(stream);
  char *d = m.first + dest_off;
  bool vec = (((uintptr_t)d | (uintptr_t)m.step) & 15u) == 0;
  for (int g = 0; g < G; g++) vec = vec && (partials[g] & 15u) == 0;
  const uint64_t per = vec ? 16 / es : 1;
  const dim3 grid(grid_for((nelems + per - 1) / per, 256, 8));
  switch (dtype) {
  case B200SHM_I8: rc = combine_for<int8_t>(op, vec, grid, s, p, G, d, m.step, pe_count, nelems); break;
  case B200SHM_I16: rc = combine_for<int16_t>(op, vec, grid, s, p, G, d, m.step, pe_count, nelems); break;
  case B200SHM_I32: rc = combine_for<int32_t>(op, vec, grid, s, p, G, d, m.step, pe_count, nelems); break;
  case B200SHM_I64: rc = combine_for<int64_t>(op, vec, grid, s, p, G, d, m.step, pe_count, nelems); break;
  case B200SHM_U8: rc = combine_for<uint8_t>(op, vec, grid, s, p, G, d, m.step, pe_count, nelems); break;
  case B200SHM_U16: rc = combine_for<uint16_t>(op, vec, grid, s, p, G, d, m.step, pe_count, nelems); break;
  case B200SHM_U32: rc = combine_for<uint32_t>(op, vec, grid, s, p, G, d, m.step, pe_count, nelems); break;
  case B200SHM_U64: rc = combine_for<uint64_t>(op, vec, grid, s, p, G, d, m.step, pe_count, nelems); break;
  case B200SHM_F32: rc = combine_for<float>(op, vec, grid, s, p, G, d, m.step, pe_count, nelems); break;
  case B200SHM_F64: rc = combine_for<double>(op, vec, grid, s, p, G, d, m.step, pe_count, nelems); break;
  case B200SHM_C32: rc = combine_for<cf32>(op, vec, grid, s, p, G, d, m.step, pe_count, nelems); break;
  default: rc = combine_for<cf64>(op, vec, grid, s, p, G, d, m.step, pe_count, nelems); break;
  }
  if (rc) return rc;
  count_launch();
  return finish(stream, "b200shm_span_combine");
}

int b200shm_span_fcollect(int G, int rank, const uint64_t *bases, int pe_start, int pe_stride,
                          int pe_count, uint64_t dest_off, uint64_t src_off, uint64_t nbytes,
                          void *stream) {
  int rc = span_check(G, rank, bases, pe_start, pe_stride, pe_count);
  if (rc) return rc;
  const uint64_t M = (uint64_t)G * (uint64_t)pe_count;
  if (nbytes > st().slice / M) return fail(B200SHM_ERR_ARG, "span_fcollect: too large");
  if ((rc = check_extent(src_off, nbytes, "span_fcollect source")) ||
      (rc = check_extent(dest_off, nbytes * M, "span_fcollect dest")))
    return rc;
  if (overlaps(dest_off, nbytes * M, src_off, nbytes))
    return fail(B200SHM_ERR_ARG, "span_fcollect: dest and source overlap");
  const uint64_t first = (uint64_t)pe_start * st().slice;
  const uint64_t step = (uint64_t)(pe_count > 1 ? pe_stride : 1) * st().slice;
  if ((rc = check_bases("span_fcollect", G, bases, first, step, pe_count))) return rc;
  if (nbytes == 0) return B200SHM_OK;
  SpanPtrs p{};
  for (int g = 0; g < G; g++) p.p[g] = (const char *)(uintptr_t)bases[g];
  bool vec = ((src_off | dest_off | nbytes | step | first) & 15u) == 0;
  for (int g = 0; g < G; g++) vec = vec && (bases[g] & 15u) == 0;
  const uint64_t n = vec ? nbytes / 16 : nbytes;
  const unsigned gy = (unsigned)(M < 65535 ? M : 65535);
  uint64_t gx = (n + 255) / 256, cap = (8ull * st().sm_count * 4 + gy - 1) / gy;
  if (gx > cap) gx = cap;
  if (gx < 1) gx = 1;
  const dim3 grid((unsigned)gx, gy);
  cudaStream_t s = pick_stream(stream);
  if (vec)
    k_span_fcollect<true><<<grid, 256, 0, s>>>(p, first, step, pe_count, (int)M, st().base,
                                               dest_off, src_off, nbytes);
  else
    k_span_fcollect<false><<<grid, 256, 0, s>>>(p, first, step, pe_count, (int)M, st().base,
                                                dest_off, src_off, nbytes);
  count_launch();
  return finish(stream, "b200shm_span_fcollect");
}

int b200shm_span_alltoall(int G, int rank, const uint64_t *bases, int pe_start, int pe_stride,
                          int pe_count, uint64_t dest_off, uint64_t src_off, uint64_t nbytes,
                          void *stream) {
  int rc = span_check(G, rank, bases, pe_start, pe_stride, pe_count);
  if (rc) return rc;
  const uint64_t M = (uint64_t)G * (uint64_t)pe_count;
  if (nbytes > st().slice / M) return fail(B200SHM_ERR_ARG, "span_alltoall: too large");
  if ((rc = check_extent(src_off, nbytes * M, "span_alltoall source")) ||
      (rc = check_extent(dest_off, nbytes * M, "span_alltoall dest")))
    return rc;
  if (overlaps(dest_off, nbytes * M, src_off, nbytes * M))
    return fail(B200SHM_ERR_ARG, "span_alltoall: dest and source overlap");
  const uint64_t first = (uint64_t)pe_start * st().slice;
  const uint64_t step = (uint64_t)(pe_count > 1 ? pe_stride : 1) * st().slice;
  if ((rc = check_bases("span_alltoall", G, bases, first, step, pe_count))) return rc;
  if (nbytes == 0) return B200SHM_OK;
  SpanPtrs p{};
  for (int g = 0; g < G; g++) p.p[g] = (const char *)(uintptr_t)bases[g];
  bool vec = ((src_off | dest_off | nbytes | step | first) & 15u) == 0;
  for (int g = 0; g < G; g++) vec = vec && (bases[g] & 15u) == 0;
  const uint64_t n = vec ? nbytes / 16 : nbytes;
  const uint64_t pairs = M * (uint64_t)pe_count;
  const unsigned gy = (unsigned)(pairs < 65535 ? pairs : 65535);
  uint64_t gx = (n + 255) / 256, cap = (8ull * st().sm_count * 4 + gy - 1) / gy;
  if (gx > cap) gx = cap;
  if (gx < 1) gx = 1;
  const dim3 grid((unsigned)gx, gy);
  cudaStream_t s = pick_stream(stream);
  if (vec)
    k_span_alltoall<true><<<grid, 256, 0, s>>>(p, first, step, pe_count, (int)M, rank, st().base,
                                               dest_off, src_off, nbytes);
  else
    k_span_alltoall<false><<<grid, 256, 0, s>>>(p, first, step, pe_count, (int)M, rank, st().base,
                                                dest_off, src_off, nbytes);
  count_launch();
  return finish(stream, "b200shm_span_alltoall");
}

int b200shm_span_amo(int amo, int dtype, int G, const uint64_t *bases, int pe_start,
                     int pe_stride, int pe_count, uint64_t nops, const int32_t *member,
                     const uint64_t *off, const void *value, const void *cond, void *fetched,
                     void *stream) {
  int rc = span_check(G, 0, bases, pe_start, pe_stride, pe_count);
  if (rc) return rc;
  if (amo < 0 || amo >= B200SHM_AMO_NOP) return fail(B200SHM_ERR_ARG, "span_amo: unknown op %d", amo);
  const bool w4 = dtype == B200SHM_I32 || dtype == B200SHM_U32 || dtype == B200SHM_F32;
  const bool w8 = dtype == B200SHM_I64 || dtype == B200SHM_U64 || dtype == B200SHM_F64;
  if (!w4 && !w8) return fail(B200SHM_ERR_UNSUPPORTED, "span_amo: dtype %d is not 4 or 8 bytes", dtype);
  const bool is_float = dtype == B200SHM_F32 || dtype == B200SHM_F64;
  if (is_float && amo != B200SHM_AMO_SWAP && amo != B200SHM_AMO_SET && amo != B200SHM_AMO_FETCH)
    return fail(B200SHM_ERR_UNSUPPORTED, "span_amo: floating types support only swap/set/fetch");
  const bool needs_value = !(amo == B200SHM_AMO_FETCH || amo == B200SHM_AMO_INC ||
                             amo == B200SHM_AMO_FETCH_INC);
  const uint64_t first = (uint64_t)pe_start * st().slice;
  const uint64_t step = (uint64_t)(pe_count > 1 ? pe_stride : 1) * st().slice;
  if ((rc = check_bases("span_amo", G, bases, first, step, pe_count))) return rc;
  if (nops == 0) return B200SHM_OK;
  if (!member || !off || (needs_value && !value) || (amo == B200SHM_AMO_CSWAP && !cond))
    return fail(B200SHM_ERR_ARG, "span_amo: missing operand array");
  SpanPtrs p{};
  for (int g = 0; g < G; g++) p.p[g] = (const char *)(uintptr_t)bases[g];
  const int M = G * pe_count;
  const unsigned grid = grid_for(nops, 256, 8);
  cudaStream_t s = pick_stream(stream);
  if (w8)
    k_span_amo<unsigned long long><<<grid, 256, 0, s>>>(
        p, M, pe_count, first, step, st().slice, amo, nops, member, off,
        (const unsigned long long *)value, (const unsigned long long *)cond,
        (unsigned long long *)fetched, st().d_status);
  else
    k_span_amo<unsigned int><<<grid, 256, 0, s>>>(
        p, M, pe_count, first, step, st().slice, amo, nops, member, off,
        (const unsigned int *)value, (const unsigned int *)cond, (unsigned int *)fetched,
        st().d_status);
  count_launch();
  return finish(stream, "b200shm_span_amo");
}

}  // extern "C"
