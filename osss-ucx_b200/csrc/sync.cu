/*
 * sync.cu -- device barriers among the members of a team.
 *
 * Each member is one PE context (a thread) of a cooperative launch, so all
 * contexts are resident together.  They synchronise through flag words
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

__device__ __forceinline__ unsigned long long *flag(const BArgs &a, int member, int round) {
  const uint64_t pe = (uint64_t)a.pe_start + (uint64_t)member * (uint64_t)a.pe_stride;
  return a.flags + (pe * (uint64_t)a.rounds + (uint64_t)round) * 8ull;
}
__device__ __forceinline__ long long now_ns() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ unsigned long long ld_acq(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void poke(unsigned long long *p, unsigned long long v = 1) {
  asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void st_rel(unsigned long long *p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

enum { W_EQ, W_NE, W_GE };
/* Bounded wait; false (and the TIMEOUT bit) when the budget runs out. */
__device__ bool wait_flag(const BArgs &a, unsigned long long *p, int cmp, unsigned long long v,
                          long long deadline) {
  for (;;) {
    const unsigned long long x = ld_acq(p);
    if (cmp == W_EQ ? x == v : cmp == W_NE ? x != v : x >= v) return true;
    if (now_ns() > deadline) {
      atomicOr(a.status, (int)B200SHM_STATUS_TIMEOUT);
      return false;
    }
    __nanosleep(64);
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
__device__ void tree_barrier(const BArgs &a, int me, int parent, const int *ch, int nch,
                             long long deadline) {
  unsigned long long *mine = flag(a, me, 0);
  if (nch && !wait_flag(a, mine, W_EQ, (unsigned long long)nch, deadline)) return;
  if (parent >= 0) {
    poke(flag(a, parent, 0));
    if (!wait_flag(a, mine, W_EQ, (unsigned long long)nch + 1, deadline)) return;
  }
  st_rel(mine, 0);
  for (int c = 0; c < nch; c++) poke(flag(a, ch[c], 0));
}

__global__ void k_barrier(const BArgs a) {
  const int me = blockIdx.x * blockDim.x + threadIdx.x;
  if (me >= a.P || me == a.absent) return;
  const long long deadline = now_ns() + a.budget_ns;
  const int P = a.P;
  int ch[32];
  switch (a.algo) {
  case B200SHM_BAR_LINEAR: { /* barrier.c:56-84 */
    unsigned long long *mine = flag(a, me, 0);
    if (me == 0) {
      if (!wait_flag(a, mine, W_EQ, (unsigned long long)(P - 1), deadline)) return;
      st_rel(mine, 0);
      for (int i = 1; i < P; i++) st_rel(flag(a, i, 0), 1);
    } else {
      poke(flag(a, 0, 0));
      if (!wait_flag(a, mine, W_NE, 0, deadline)) return;
      st_rel(mine, 0);
    }
    break;
  }
  case B200SHM_BAR_COMPLETE_TREE: { /* barrier.c:96-132, degree 2 */
    const int n = complete_children(me, P, 2, ch);
    tree_barrier(a, me, me ? (me - 1) / 2 : -1, ch, n, deadline);
    break;
  }
  case B200SHM_BAR_BINOMIAL_TREE: { /* barrier.c:144-180 */
    const int n = binomial_children(me, P, ch);
    tree_barrier(a, me, me ? (me & (me - 1)) : -1, ch, n, deadline);
    break;
  }
  case B200SHM_BAR_KNOMIAL_TREE: { /* barrier.c:192-228, radix 2 */
    int parent;
    const int n = knomial_node(me, P, 2, &parent, ch);
    tree_barrier(a, me, parent, ch, n, deadline);
    break;
  }
  default: { /* dissemination, barrier.c:241-266 */
    for (int r = 0, d = 1; d < P; r++, d <<= 1) {
      poke(flag(a, (me + d) % P, r));
      unsigned long long *mine = flag(a, me, r);
      if (!wait_flag(a, mine, W_NE, 0, deadline)) return;
      atomicAdd(mine, (unsigned long long)-1ll);
    }
    break;
  }
  }
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
  int per_sm = 0;
  B200_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_barrier, threads, 0));
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
