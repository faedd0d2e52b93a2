/*
 * sync.cu -- device barriers among the members of a team.
 *
 * Each member is one PE context (a thread); the contexts of a team of more
 * than 256 members are the CTAs of a cooperative launch, so all of them
 * are resident together (a team of up to 256 is one CTA, which always is,
 * and keeps its flag words in shared memory).  They synchronise through flag words
 * with the message pattern of the reference algorithm chosen
 * (src/shcoll/src/barrier.c): poke = atomic add with release semantics
 * (shmem_long_atomic_inc), wait = acquire load loop (shmem_long_wait_until,
 * which spins without bound in the reference, src/shmemc/ucx/waituntil.c).
 * Here every wait has a time budget; a context that runs out sets the
 * TIMEOUT status bit and returns, so a missing member yields an error code
 * instead of a hung GPU.
 *
 * Flags: one 64-byte line per (global PE, round) in a library-owned area;
 * every algorithm returns its flags to zero, as the reference returns
 * pSync to SHMEM_SYNC_VALUE.
 */
#include <stdint.h>
#include <string.h>

#include <atomic>
#include <vector>

#include "internal.cuh"

namespace b200 {

/* default budget of a barrier wait: 2 s */
constexpr long long kDefaultWaitBudgetNs = 2000000000ll;

namespace {

struct BArgs {
  unsigned long long *flags;
  int rounds;      /* flag lines per PE */
  int pe_start, pe_stride, P, algo;
  int *status;
  long long budget_ns;
  int absent;      /* member that never arrives (failure injection), or -1 */
};

/* Flag words: for a team over several CTAs, one 64-byte line per (global
 * PE, round) in the library's global area, used with gpu-scope
 * release/acquire; for a team that is one CTA (up to 256 members), the
 * same pattern on words in that CTA's shared memory with cta scope, which
 * costs tens of nanoseconds a hop instead of a round trip to L2. */
constexpr int kCtaRounds = 8; /* dissemination rounds of a 256-member team */
template <bool CTA>
__device__ __forceinline__ unsigned long long *flag(const BArgs &a, unsigned long long *sfl,
                                                   int member, int round) {
  if constexpr (CTA) return sfl + member * kCtaRounds + round;
  const uint64_t pe = (uint64_t)a.pe_start + (uint64_t)member * (uint64_t)a.pe_stride;
  return a.flags + (pe * (uint64_t)a.rounds + (uint64_t)round) * 8ull;
}
__device__ __forceinline__ long long now_ns() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
template <bool CTA>
__device__ __forceinline__ unsigned long long ld_acq(const unsigned long long *p) {
  unsigned long long v;
  if constexpr (CTA) asm volatile("ld.acquire.cta.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  else asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
template <bool CTA>
__device__ __forceinline__ void poke(unsigned long long *p, unsigned long long v = 1) {
  if constexpr (CTA) asm volatile("red.release.cta.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
  else asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
template <bool CTA>
__device__ __forceinline__ void st_rel(unsigned long long *p, unsigned long long v) {
  if constexpr (CTA) asm volatile("st.release.cta.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
  else asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

enum { W_EQ, W_NE, W_GE };
/* Bounded wait; false (and the TIMEOUT bit) when the budget runs out. */
template <bool CTA>
__device__ bool wait_flag(const BArgs &a, unsigned long long *p, int cmp, unsigned long long v,
                          long long deadline) {
  for (;;) {
    const unsigned long long x = ld_acq<CTA>(p);
    if (cmp == W_EQ ? x == v : cmp == W_NE ? x != v : x >= v) return true;
    if (now_ns() > deadline) {
      atomicOr(a.status, (int)B200SHM_STATUS_TIMEOUT);
      return false;
    }
    __nanosleep(CTA ? 32 : 64);
  }
}

/* tree shapes (src/shcoll/src/util/trees.c) restated: parent and children
 * of node i in a tree of n nodes rooted at 0 */
__device__ int binomial_children(int i, int n, int *ch) {
  int mask = (i == 0) ? (1 << 30) : ((i & -i) >> 1);
  int c = 0;
  for (; mask; mask >>= 1)
    if ((i | mask) < n) ch[c++] = i | mask;
  return c;
}
__device__ int complete_children(int i, int n, int deg, int *ch) {
  int c = 0;
  for (int x = i * deg + 1; x < n && x <= i * deg + deg; x++) ch[c++] = x;
  return c;
}
/* k-nomial: descend into the group containing i; the last `left` seen on
 * the way is the parent; then the children are the group leaders of the
 * remaining levels, largest distance first */
__device__ int knomial_node(int i, int n, int k, int *parent, int *ch) {
  int left = 0, right = n, par = -1, dist = -1;
  while (i != left) {
    par = left;
    dist = (right - left + k - 1) / k;
    const int group = (i - left) / dist;
    const int nr = left + (group + 1) * dist;
    right = nr > right ? right : nr;
    left = left + group * dist;
  }
  *parent = par;
  int c = 0;
  while (dist != 0) {
    dist = (right - left + k - 1) / k;
    int child = left + dist * ((right - left - 1) / dist);
    if (child == left) break;
    do {
      ch[c++] = child;
      child -= dist;
    } while (child > left);
    right = left + dist;
  }
  return c;
}

/* gather-to-root then release, barrier.c:96-228 */
template <bool CTA>
__device__ void tree_barrier(const BArgs &a, unsigned long long *sfl, int me, int parent,
                             const int *ch, int nch, long long deadline) {
  unsigned long long *mine = flag<CTA>(a, sfl, me, 0);
  if (nch && !wait_flag<CTA>(a, mine, W_EQ, (unsigned long long)nch, deadline)) return;
  if (parent >= 0) {
    poke<CTA>(flag<CTA>(a, sfl, parent, 0));
    if (!wait_flag<CTA>(a, mine, W_EQ, (unsigned long long)nch + 1, deadline)) return;
  }
  st_rel<CTA>(mine, 0);
  for (int c = 0; c < nch; c++) poke<CTA>(flag<CTA>(a, sfl, ch[c], 0));
}

/* One PE context's part of barrier a.algo (member `me`). */
template <bool CTA>
__device__ void barrier_body(const BArgs &a, unsigned long long *sfl, int me) {
  const long long deadline = now_ns() + a.budget_ns;
  const int P = a.P;
  int ch[32];
  switch (a.algo) {
  case B200SHM_BAR_LINEAR: { /* barrier.c:56-84 */
    unsigned long long *mine = flag<CTA>(a, sfl, me, 0);
    if (me == 0) {
      if (!wait_flag<CTA>(a, mine, W_EQ, (unsigned long long)(P - 1), deadline)) return;
      st_rel<CTA>(mine, 0);
      for (int i = 1; i < P; i++) st_rel<CTA>(flag<CTA>(a, sfl, i, 0), 1);
    } else {
      poke<CTA>(flag<CTA>(a, sfl, 0, 0));
      if (!wait_flag<CTA>(a, mine, W_NE, 0, deadline)) return;
      st_rel<CTA>(mine, 0);
    }
    break;
  }
  case B200SHM_BAR_COMPLETE_TREE: { /* barrier.c:96-132, degree 2 */
    const int n = complete_children(me, P, 2, ch);
    tree_barrier<CTA>(a, sfl, me, me ? (me - 1) / 2 : -1, ch, n, deadline);
    break;
  }
  case B200SHM_BAR_BINOMIAL_TREE: { /* barrier.c:144-180 */
    const int n = binomial_children(me, P, ch);
    tree_barrier<CTA>(a, sfl, me, me ? (me & (me - 1)) : -1, ch, n, deadline);
    break;
  }
  case B200SHM_BAR_KNOMIAL_TREE: { /* barrier.c:192-228, radix 2 */
    int parent;
    const int n = knomial_node(me, P, 2, &parent, ch);
    tree_barrier<CTA>(a, sfl, me, parent, ch, n, deadline);
    break;
  }
  default: { /* dissemination, barrier.c:241-266 */
    for (int r = 0, d = 1; d < P; r++, d <<= 1) {
      poke<CTA>(flag<CTA>(a, sfl, (me + d) % P, r));
      unsigned long long *mine = flag<CTA>(a, sfl, me, r);
      if (!wait_flag<CTA>(a, mine, W_NE, 0, deadline)) return;
      atomicAdd(mine, (unsigned long long)-1ll);
    }
    break;
  }
  }
}

/* a team over several CTAs (cooperative launch), flags in global memory */
__global__ void k_barrier(const BArgs a) {
  const int me = blockIdx.x * blockDim.x + threadIdx.x;
  if (me >= a.P || me == a.absent) return;
  barrier_body<false>(a, nullptr, me);
}

/* a team of up to 256 members as one CTA, flags in its shared memory
 * (the P members' lines zeroed before any context pokes one -- no member
 * touches another line; the contexts that do not take part leave only
 * after that) */
__global__ void __launch_bounds__(256) k_barrier_cta(const BArgs a) {
  __shared__ unsigned long long sfl[256 * kCtaRounds];
  for (int i = threadIdx.x; i < a.P * kCtaRounds; i += blockDim.x) sfl[i] = 0;
  __syncthreads();
  const int me = threadIdx.x;
  if (me >= a.P || me == a.absent) return;
  barrier_body<true>(a, sfl, me);
}

}  // namespace

/* budget of every barrier wait, ns (b200shm_set_wait_budget) */
static std::atomic<long long> g_wait_budget_ns{kDefaultWaitBudgetNs};

int barrier_launch(int algo, int pe_start, int pe_stride, int P, cudaStream_t s, int absent) {
  int rc = check_team(pe_start, pe_stride, P);
  if (rc) return rc;
  if (algo < 0 || algo >= B200SHM_BAR_NALGO)
    return fail(B200SHM_ERR_ARG, "barrier: unknown algorithm %d", algo);
  if (algo == B200SHM_BAR_DISSEMINATION) {
    int r = 0;
    while ((1 << r) < P) r++;
    if (r > st().flag_rounds) return fail(B200SHM_ERR_UNSUPPORTED, "barrier: team too large");
  }
  BArgs a;
  a.flags = st().flags;
  a.rounds = st().flag_rounds;
  a.pe_start = pe_start;
  a.pe_stride = P > 1 ? pe_stride : 1;
  a.P = P;
  a.algo = algo;
  a.status = st().d_status;
  a.budget_ns = g_wait_budget_ns.load(std::memory_order_relaxed);
  a.absent = absent;
  const int threads = P < 256 ? P : 256;
  const int blocks = (P + threads - 1) / threads;
  if (blocks == 1) { /* one CTA, flags in its shared memory: a plain launch */
    k_barrier_cta<<<1, threads, 0, s>>>(a);
    count_launch();
    return B200SHM_OK;
  }
  /* CTAs of 256 contexts one SM holds at once (queried once) */
  static std::atomic<int> per_sm_cache{0};
  int per_sm = per_sm_cache.load(std::memory_order_relaxed);
  if (per_sm == 0) {
    B200_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_barrier, 256, 0));
    per_sm_cache.store(per_sm, std::memory_order_relaxed);
  }
  if ((long long)per_sm * st().sm_count < blocks)
    return fail(B200SHM_ERR_UNSUPPORTED, "barrier: %d PE contexts cannot be co-resident", P);
  void *args[] = {(void *)&a};
  B200_CK(cudaLaunchCooperativeKernel((const void *)k_barrier, dim3(blocks), dim3(threads), args,
                                      0, s));
  count_launch();
  return B200SHM_OK;
}

/* After a timed-out barrier some flags may be left non-zero: clear them. */
int barrier_reset_flags(cudaStream_t s) {
  const uint64_t words = (uint64_t)st().npes * (uint64_t)st().flag_rounds * 8ull;
  B200_CK(cudaMemsetAsync(st().flags, 0, words * sizeof(unsigned long long), s));
  return B200SHM_OK;
}

/* One barrier, blocking or stream-ordered; a timed-out barrier leaves its
 * flag lines cleared before it returns. */
static int barrier_call(int algo, int pe_start, int pe_stride, int pe_size, int absent,
                        void *stream, const char *what) {
  cudaStream_t s = pick_stream(stream);
  int rc = barrier_launch(algo, pe_start, pe_stride, pe_size, s, absent);
  if (rc) return rc;
  rc = finish(stream, what);
  if (rc == B200SHM_ERR_TIMEOUT) {
    barrier_reset_flags(s);
    cudaStreamSynchronize(s);
  }
  return rc;
}

}  // namespace b200

extern "C" {

int b200shm_barrier(int algo, int pe_start, int pe_stride, int pe_size, void *stream) {
  return b200::barrier_call(algo, pe_start, pe_stride, pe_size, -1, stream, "b200shm_barrier");
}

uint64_t b200shm_set_wait_budget(uint64_t ns) {
  const long long v = ns == 0 ? b200::kDefaultWaitBudgetNs
                              : (long long)(ns > (uint64_t)INT64_MAX / 2 ? (uint64_t)INT64_MAX / 2 : ns);
  return (uint64_t)b200::g_wait_budget_ns.exchange(v);
}

int b200shm_barrier_absent(int algo, int pe_start, int pe_stride, int pe_size, int absent,
                           void *stream) {
  if (absent < 0 || absent >= pe_size)
    return b200::fail(B200SHM_ERR_ARG, "barrier_absent: member %d is not in the team", absent);
  return b200::barrier_call(algo, pe_start, pe_stride, pe_size, absent, stream,
                            "b200shm_barrier_absent");
}

int64_t b200shm_barrier_flags_nonzero(void) {
  using namespace b200;
  if (!st().up) return fail(B200SHM_ERR_STATE, "b200shm is not initialised");
  const uint64_t words = (uint64_t)st().npes * (uint64_t)st().flag_rounds * 8ull;
  std::vector<unsigned long long> h(words);
  B200_CK(cudaStreamSynchronize(st().stream));
  B200_CK(cudaMemcpy(h.data(), st().flags, words * sizeof(unsigned long long),
                     cudaMemcpyDeviceToHost));
  int64_t n = 0;
  for (unsigned long long w : h) n += w != 0;
  return n;
}

}  // extern "C"

/* ---------------------------------------------------------------------------
 * Point-to-point synchronisation: the comparisons behind shmem_<T>_test,
 * test_all/any/some[_vector] and (polled) wait_until* (src/shmemc/ucx/
 * test.c:10-170, waituntil.c:18-320).  One launch compares a whole vector of
 * symmetric words with acquire loads, so words written by the engine's
 * puts, atomics and serving loop are seen.
 * ------------------------------------------------------------------------- */
namespace b200 {
namespace {

template <class T>
__device__ __forceinline__ T ld_acquire_word(const T *p) {
  if constexpr (sizeof(T) == 8) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return (T)v;
  } else if constexpr (sizeof(T) == 4) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return (T)v;
  } else {
    unsigned short v;
    asm volatile("ld.acquire.gpu.global.u16 %0, [%1];" : "=h"(v) : "l"(p) : "memory");
    return (T)v;
  }
}

/* out[i] = 1 when vars[i] cmp value (values[i] for the vector forms),
 * 0 when not, 2 when status[i] excludes it; loaded[i] = the bits read */
template <class T>
__global__ void __launch_bounds__(256) k_test_words(const T *vars, uint64_t n, int cmp, T value,
                                                    const T *values, const int *status,
                                                    unsigned char *out,
                                                    unsigned long long *loaded) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    if (status && status[i] != 0) {
      out[i] = 2;
      continue;
    }
    const T x = ld_acquire_word(vars + i);
    const T v = values ? values[i] : value;
    bool r;
    switch (cmp) {
    case 0: r = x == v; break; /* SHMEM_CMP_EQ */
    case 1: r = x != v; break; /* NE */
    case 2: r = x > v; break;  /* GT */
    case 3: r = x <= v; break; /* LE */
    case 4: r = x < v; break;  /* LT */
    default: r = x >= v; break; /* GE */
    }
    out[i] = r ? 1 : 0;
    if (loaded) {
      unsigned long long bits = 0;
      memcpy(&bits, &x, sizeof(T));
      loaded[i] = bits;
    }
  }
}

/* per-thread mapped staging for the host arrays of b200shm_test_words */
struct TestStage {
  char *h = nullptr, *d = nullptr;
  size_t cap = 0;
  ~TestStage() {
    if (h) cudaFreeHost(h);
  }
};

}  // namespace
}  // namespace b200

extern "C" int b200shm_test_words(int cmp, int dtype, int pe, uint64_t off, uint64_t nelems,
                                  const int *status, const void *cmp_value,
                                  const void *cmp_values, uint8_t *out, uint64_t *loaded) {
  using namespace b200;
  if (!st().up) return fail(B200SHM_ERR_STATE, "b200shm is not initialised");
  if (cmp < 0 || cmp > 5) return fail(B200SHM_ERR_ARG, "test: unknown comparison %d", cmp);
  uint64_t w;
  switch (dtype) {
  case B200SHM_I16: case B200SHM_U16: w = 2; break;
  case B200SHM_I32: case B200SHM_U32: w = 4; break;
  case B200SHM_I64: case B200SHM_U64: w = 8; break;
  default: return fail(B200SHM_ERR_UNSUPPORTED, "test: dtype %d is not a 2/4/8-byte integer", dtype);
  }
  if (nelems == 0) return B200SHM_OK;
  if (!out || (!cmp_value && !cmp_values))
    return fail(B200SHM_ERR_ARG, "test: missing result or comparison value");
  if (pe < 0 || pe >= st().npes || off % w || nelems > st().slice / w ||
      off > st().slice - nelems * w)
    return fail(B200SHM_ERR_ARG, "test: %llu words at (PE %d, offset %llu) are not in the heap",
                (unsigned long long)nelems, pe, (unsigned long long)off);
  static thread_local TestStage stg;
  /* layout: out bytes | status ints | values | loaded words, 16-byte aligned parts */
  auto up16 = [](size_t x) { return (x + 15) & ~(size_t)15; };
  const size_t o_st = up16(nelems), o_val = o_st + up16(status ? nelems * 4 : 0);
  const size_t o_ld = o_val + up16(cmp_values ? nelems * w : 0);
  const size_t need = o_ld + (loaded ? nelems * 8 : 0) + 16;
  if (need > stg.cap) {
    if (stg.h) cudaFreeHost(stg.h);
    stg.h = stg.d = nullptr;
    stg.cap = 0;
    size_t cap = need < 4096 ? 4096 : need;
    B200_CK(cudaHostAlloc((void **)&stg.h, cap, cudaHostAllocMapped));
    cudaError_t e = cudaHostGetDevicePointer((void **)&stg.d, stg.h, 0);
    if (e != cudaSuccess) return cuda_fail(e, "test staging");
    stg.cap = cap;
  }
  if (status) memcpy(stg.h + o_st, status, nelems * 4);
  if (cmp_values) memcpy(stg.h + o_val, cmp_values, nelems * w);
  const char *vars = st().base + (uint64_t)pe * st().slice + off;
  const int *d_st = status ? (const int *)(stg.d + o_st) : nullptr;
  unsigned char *d_out = (unsigned char *)stg.d;
  unsigned long long *d_ld = loaded ? (unsigned long long *)(stg.d + o_ld) : nullptr;
  cudaStream_t s = st().stream;
  const unsigned grid = grid_for(nelems, 256, 4);
  uint64_t v = 0;
  if (cmp_value) memcpy(&v, cmp_value, w);
  switch (dtype) {
  case B200SHM_I16:
    k_test_words<int16_t><<<grid, 256, 0, s>>>((const int16_t *)vars, nelems, cmp, (int16_t)v,
        cmp_values ? (const int16_t *)(stg.d + o_val) : nullptr, d_st, d_out, d_ld);
    break;
  case B200SHM_U16:
    k_test_words<uint16_t><<<grid, 256, 0, s>>>((const uint16_t *)vars, nelems, cmp, (uint16_t)v,
        cmp_values ? (const uint16_t *)(stg.d + o_val) : nullptr, d_st, d_out, d_ld);
    break;
  case B200SHM_I32:
    k_test_words<int32_t><<<grid, 256, 0, s>>>((const int32_t *)vars, nelems, cmp, (int32_t)v,
        cmp_values ? (const int32_t *)(stg.d + o_val) : nullptr, d_st, d_out, d_ld);
    break;
  case B200SHM_U32:
    k_test_words<uint32_t><<<grid, 256, 0, s>>>((const uint32_t *)vars, nelems, cmp, (uint32_t)v,
        cmp_values ? (const uint32_t *)(stg.d + o_val) : nullptr, d_st, d_out, d_ld);
    break;
  case B200SHM_I64:
    k_test_words<int64_t><<<grid, 256, 0, s>>>((const int64_t *)vars, nelems, cmp, (int64_t)v,
        cmp_values ? (const int64_t *)(stg.d + o_val) : nullptr, d_st, d_out, d_ld);
    break;
  default:
    k_test_words<uint64_t><<<grid, 256, 0, s>>>((const uint64_t *)vars, nelems, cmp, (uint64_t)v,
        cmp_values ? (const uint64_t *)(stg.d + o_val) : nullptr, d_st, d_out, d_ld);
    break;
  }
  count_launch();
  const int rc = finish(nullptr, "b200shm_test_words");
  if (rc) return rc;
  memcpy(out, stg.h, nelems);
  if (loaded) memcpy(loaded, stg.h + o_ld, nelems * 8);
  return B200SHM_OK;
}
