/*
 * reduce.cu -- one-pass all-reduce over the members of a team.
 *
 * The reference moves O(N log P) bytes per PE through log2(P) rounds of
 * put + flag handshake (rec_dbl, src/shcoll/src/reduce.c:182-293) or
 * reduce-scatter + allgather (Rabenseifner, 306-724).  On one GPU every
 * member's slice is directly addressable, so each thread owns a 16-byte
 * column of elements, streams that column in from all P members' sources
 * with 128-bit loads, combines it in registers and streams the result out
 * to all P members' dests: 2*P*N*sizeof(T) bytes, the algorithmic minimum.
 *
 * Exactness.  The algorithm fixes the combine order and so the exact
 * floating-point result.  Three facts keep the kernel cheap:
 *  - integer AND/OR/XOR/SUM/PROD (wrapping) and MIN/MAX are associative
 *    and commutative bit for bit, so any order is exact: a running chain;
 *  - float and complex SUM/PROD are exactly commutative (a+b == b+a, and
 *    the naive complex product is symmetric), so only the tree SHAPE
 *    matters: linear = left fold (reduce.c:78-81); binomial = balanced
 *    binary tree over members combining op(upper block, lower block)
 *    (reduce.c:137-154, children in increasing mask order); rec_dbl and
 *    both Rabenseifner variants = butterfly over the power-of-two subset
 *    after folding the extra members (reduce.c:206-272, 338-454) -- the
 *    same tree for all three;
 *  - float MIN/MAX written a<b?a:b (reduce.c:731-732) is order dependent
 *    only when the operands include a NaN or both +0 and -0; elements with
 *    such operands take an exact per-member path that replays the
 *    algorithm's operand order (rec_dbl then gives different members
 *    different bits, exactly as the reference does).
 * Trees are evaluated as a binary counter over the leaves, with one
 * register slot per tree level, so leaves stream in member order.
 * No fused multiply-add is ever formed: float ops use the _rn intrinsics.
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
namespace {

/* Second pass over the elements the streaming kernel deferred (it left
 * their dests untouched, so in-place sources are still intact): one CTA
 * per element stages the P inputs in shared memory, then replays the
 * algorithm's operand order from there.  Launched as a programmatic
 * dependent of the streaming kernel: its CTAs may become resident during
 * that kernel's last wave and wait here until its results are visible.
 * The last CTA to leave sets the counter back to zero for the next call
 * (every CTA reads it before it counts itself out), so no memset precedes
 * the streaming kernel. */
template <class T, int OP>
__global__ void __launch_bounds__(256) k_minmax_fix(const RArgs a,
                                                    const unsigned long long *list,
                                                    unsigned long long *count,
                                                    unsigned long long *done,
                                                    unsigned long long cap) {
  __shared__ T vals[fix_max_members<T>()];
  __shared__ T common;
  asm volatile("griddepcontrol.wait;" ::: "memory");
  const unsigned long long cnt = *(volatile unsigned long long *)count;
  const unsigned long long n = cnt < cap ? cnt : cap;
  for (unsigned long long k = blockIdx.x; k < n; k += gridDim.x) {
    const uint64_t e = list[k];
    for (int j = threadIdx.x; j < a.P; j += blockDim.x)
      memcpy(&vals[j], a.src + (uint64_t)j * a.sstep + e * sizeof(T), sizeof(T));
    __syncthreads();
    const uint64_t eg = a.g_off + e; /* the order depends on the position in the whole */
    const bool lower = eg < a.g_n / 2;
    if (a.algo == B200SHM_REC_DBL) {
      /* every p2s member (and the extra folded into it) keeps its own value */
      for (int q = threadIdx.x; q < a.p2s; q += blockDim.x) {
        const T v = exact_value<T, OP>([&](int j) { return vals[j]; }, a.P, a.p2s, a.logp2s,
                                       a.algo, lower, q);
        const int as = p2s_member(q, a.P, a.p2s);
        memcpy(a.dst + (uint64_t)as * a.dstep + e * sizeof(T), &v, sizeof(T));
        if (p2s_extra(q, a.P, a.p2s))
          memcpy(a.dst + (uint64_t)(as + 1) * a.dstep + e * sizeof(T), &v, sizeof(T));
      }
    } else {
      if (threadIdx.x == 0) {
        int q = 0;
        if (a.algo != B200SHM_LINEAR && a.algo != B200SHM_BINOMIAL)
          q = rev_bits(rab_block(eg, a.g_n, a.p2s), a.logp2s); /* owner of e's block */
        common = exact_value<T, OP>([&](int j) { return vals[j]; }, a.P, a.p2s, a.logp2s, a.algo,
                                    lower, q);
      }
      __syncthreads();
      for (int j = threadIdx.x; j < a.P; j += blockDim.x)
        memcpy(a.dst + (uint64_t)j * a.dstep + e * sizeof(T), &common, sizeof(T));
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(done, 1ull) == (unsigned long long)gridDim.x - 1) {
      *(volatile unsigned long long *)count = 0;
      *(volatile unsigned long long *)done = 0;
      __threadfence();
    }
  }
}

/* Let the replay kernel that follows a MIN/MAX-checking launch be
 * scheduled once every CTA of this grid has started (it waits for this
 * grid's results before it reads anything). */
__device__ __forceinline__ void allow_dependents() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

/* ---- the streaming kernels -------------------------------------------- */
template <class T, int OP, int ORDER, int V, int U, bool MINMAX_CHECK, int LV>
__global__ void __launch_bounds__(256) k_reduce(const RArgs a) {
  typedef Pack<T, V> PK;
  if constexpr (MINMAX_CHECK) allow_dependents();
  /* grid-stride: all CTAs sweep one contiguous front of every member's
   * slice together, which keeps DRAM row locality (contiguous per-CTA
   * ranges measured ~20% slower) */
  const uint64_t gstride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < a.nvec; v += gstride) {
    const uint64_t e0 = a.e_begin + v * V;
    const char *src = a.src + e0 * sizeof(T);
    PK r;
    unsigned cls[V];
    if constexpr (ORDER == ORD_CHAIN) {
      r = ld_pack<T, V>(src);
      if constexpr (MINMAX_CHECK) {
#pragma unroll
        for (int i = 0; i < V; i++) cls[i] = fclass(r.x[i]);
      }
      for (int j = 1; j < a.P; j += U) {
        PK x[U];
#pragma unroll
        for (int u = 0; u < U; u++)
          if (j + u < a.P) x[u] = ld_pack<T, V>(src + (uint64_t)(j + u) * a.sstep);
#pragma unroll
        for (int u = 0; u < U; u++)
          if (j + u < a.P) {
            r = papply<OP>(r, x[u]);
            if constexpr (MINMAX_CHECK) {
#pragma unroll
              for (int i = 0; i < V; i++) cls[i] |= fclass(x[u].x[i]);
            }
          }
      }
    } else {
      PK stk[LV]; /* LV levels hold trees of up to 2^LV - 1 leaves */
      const int nleaves = ORDER == ORD_BUTTERFLY ? a.p2s : a.P;
      /* comb(lower block, upper block) in the algorithm's operand order */
      auto comb = [](const PK &lo, const PK &hi) {
        return ORDER == ORD_BUTTERFLY ? papply<OP>(lo, hi) : papply<OP>(hi, lo);
      };
      /* binary counter: pushing block number q at level `base` closes
       * t = trailing_ones(q) blocks and parks the result at level base+t
       * (all register indices static) */
      auto push = [&](PK y, int q, int base) {
        const int t = base + __ffs(~q) - 1;
#pragma unroll
        for (int L = 0; L < LV - 1; L++)
          if (L >= base && L < t) y = comb(stk[L], y);
#pragma unroll
        for (int L = 0; L < LV; L++)
          if (L == t) stk[L] = y;
      };
      /* p2s member q is member ceil(q*P/p2s) (p2s is a power of two, so the
       * division is a shift); it has an extra member folded into it exactly
       * when the next p2s member is two members further on */
      auto member_of = [&](int q) -> int {
        return ORDER == ORD_BUTTERFLY
                   ? (int)(((long long)q * a.P + a.p2s - 1) >> a.logp2s)
                   : q;
      };
      auto leaf_addr = [&](int q) { return src + (uint64_t)member_of(q) * a.sstep; };
      auto fold_extra = [&](PK &x, int q) {
        /* rec_dbl / Rabenseifner fold the extra member in first as
         * op(extra, own) (reduce.c:232-241) */
        if (ORDER == ORD_BUTTERFLY && a.P != a.p2s && member_of(q + 1) - member_of(q) == 2)
          x = papply<OP>(ld_pack<T, V>(leaf_addr(q) + a.sstep), x);
      };
      int q0 = 0;
      /* full chunks of 8 leaves: 8 loads in flight, a fixed 8-leaf subtree */
      for (; q0 + 8 <= nleaves; q0 += 8) {
        PK x[8];
#pragma unroll
        for (int u = 0; u < 8; u++) x[u] = ld_pack<T, V>(leaf_addr(q0 + u));
#pragma unroll
        for (int u = 0; u < 8; u++) fold_extra(x[u], q0 + u);
        const PK c = comb(comb(comb(x[0], x[1]), comb(x[2], x[3])),
                          comb(comb(x[4], x[5]), comb(x[6], x[7])));
        push(c, q0 >> 3, 3);
      }
      /* the last < 8 leaves (trees of < 8 leaves, binomial with P % 8 != 0) */
#pragma unroll 1
      for (; q0 < nleaves; q0++) {
        PK x = ld_pack<T, V>(leaf_addr(q0));
        fold_extra(x, q0);
        push(x, q0, 0);
      }
      if constexpr (ORDER == ORD_BUTTERFLY) {
#pragma unroll
        for (int L = 0; L < LV; L++)
          if (L == a.logp2s) r = stk[L];
      } else {
        bool have = false;
#pragma unroll
        for (int L = 0; L < LV; L++)
          if (a.P & (1 << L)) {
            r = have ? papply<OP>(r, stk[L]) : stk[L];
            have = true;
          }
      }
    }
    if constexpr (MINMAX_CHECK) {
      bool amb = false;
#pragma unroll
      for (int i = 0; i < V; i++) amb |= ambiguous(cls[i]);
      if (amb) {
        /* defer the whole pack; its dests stay untouched until k_minmax_fix */
        const unsigned long long slot = atomicAdd(a.fix_count, (unsigned long long)V);
        for (int i = 0; i < V; i++) {
          if (slot + i < a.fix_cap) a.fix_list[slot + i] = e0 + i;
          else atomicOr(a.status, (int)B200SHM_STATUS_FIX_OVERFLOW);
        }
        continue;
      }
    }
    char *dst = a.dst + e0 * sizeof(T);
    for (int j = 0; j < a.P; j++) st_pack<T, V>(dst + (uint64_t)j * a.dstep, r);
  }
}

/* Launch the packed body over [0, N - N%V) and a scalar tail, or scalar
 * throughout when the buffers are not 16-byte aligned. */
/* ---- warp-cooperative variant ----------------------------------------
 * G lanes (a power of two) share one 16-byte column.  Lane group g owns a
 * contiguous share of the leaves -- for the butterfly and for binomial
 * trees over a power-of-two team that share is a complete subtree -- and
 * reduces it from loads it keeps 8 deep; the G partial results are then
 * combined across lanes with __shfl_xor over masks 1, 2, ..., G/2, which
 * is exactly the butterfly's remaining levels (mask m pairs group g with
 * g^m, lower group first: reduce.c:250-272).  Every lane then stores the
 * result to its own share of the members.  Registers per lane no longer
 * grow with the tree depth, and a pack's 2*P memory operations are spread
 * over G lanes. */

/* The MIN/MAX-checking instances take 78 registers (3 CTAs per SM), the
 * others 48 (5).  Holding the MIN/MAX ones to 64 (4 CTAs per SM, no spills)
 * measured slower on the 64-PE headline (f64 MAX 5908-5912 against
 * 5938-5950 GB/s), so they are left unbounded. */
template <class T, int OP, int ORDER, int V, int G, bool MM, int LVL, bool POW2>
__global__ void __launch_bounds__(256) k_reduce_coop(const RArgs a) {
  typedef Pack<T, V> PK;
  if constexpr (MM) allow_dependents();
  constexpr int COLS = 32 / G; /* packs per warp per iteration */
  const int lane = threadIdx.x & 31;
  const int g = lane & (G - 1), c = lane / G;
  const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const int P = a.P;
  const int nleaves = ORDER == ORD_BUTTERFLY ? a.p2s : P;
  /* this lane's leaves [l0, l1) */
  const int l0 = (int)((long long)g * nleaves / G), l1 = (int)((long long)(g + 1) * nleaves / G);
  /* members this lane stores to: [m0, m1) */
  int m0, m1;
  if (ORDER == ORD_BUTTERFLY) {
    m0 = (int)(((long long)l0 * P + a.p2s - 1) >> a.logp2s);
    m1 = (int)(((long long)l1 * P + a.p2s - 1) >> a.logp2s);
  } else {
    m0 = l0;
    m1 = l1;
  }
  auto member_of = [&](int q) -> int {
    return ORDER == ORD_BUTTERFLY ? (int)(((long long)q * P + a.p2s - 1) >> a.logp2s) : q;
  };
  auto comb = [](const PK &lo, const PK &hi) {
    if constexpr (ORDER == ORD_BINOMIAL) return papply<OP>(hi, lo);
    else return papply<OP>(lo, hi);
  };
  for (uint64_t base = warp * COLS; base < a.nvec; base += nwarps * COLS) {
    const uint64_t v = base + c;
    const bool live = v < a.nvec; /* uniform per column group */
    const uint64_t e0 = a.e_begin + (live ? v : 0) * V;
    const char *src = a.src + e0 * sizeof(T);
    PK r;
    unsigned cls[V];
#pragma unroll
    for (int i = 0; i < V; i++) cls[i] = 0;
    if (live) {
      if constexpr (ORDER == ORD_CHAIN) {
        r = ld_pack<T, V>(src + (uint64_t)l0 * a.sstep);
        if constexpr (MM) {
#pragma unroll
          for (int i = 0; i < V; i++) cls[i] = fclass(r.x[i]);
        }
        for (int j = l0 + 1; j < l1; j += 8) {
          PK x[8];
#pragma unroll
          for (int u = 0; u < 8; u++)
            if (j + u < l1) x[u] = ld_pack<T, V>(src + (uint64_t)(j + u) * a.sstep);
#pragma unroll
          for (int u = 0; u < 8; u++)
            if (j + u < l1) {
              r = papply<OP>(r, x[u]);
              if constexpr (MM) {
#pragma unroll
                for (int i = 0; i < V; i++) cls[i] |= fclass(x[u].x[i]);
              }
            }
        }
      } else {
        /* complete subtree of l1-l0 (a power of two) leaves: chunks of 8
         * as fixed subtrees; LVL == 1: one chunk, LVL == 2: two chunks, LVL == 4: four,
         * else a counter over the chunks (LVL levels hold 2^(LVL-1)) */
        const int n = l1 - l0;
        auto chunk = [&](int q0) {
          PK x[8];
          if constexpr (POW2) { /* member == leaf */
            const char *p = src + (uint64_t)q0 * a.sstep;
#pragma unroll
            for (int u = 0; u < 8; u++) x[u] = ld_pack<T, V>(p + (uint64_t)u * a.sstep);
          } else {
#pragma unroll
            for (int u = 0; u < 8; u++) x[u] = ld_pack<T, V>(src + (uint64_t)member_of(q0 + u) * a.sstep);
#pragma unroll
            for (int u = 0; u < 8; u++) /* op(extra, own), reduce.c:232-241 */
              if (member_of(q0 + u + 1) - member_of(q0 + u) == 2)
                x[u] = papply<OP>(ld_pack<T, V>(src + (uint64_t)(member_of(q0 + u) + 1) * a.sstep), x[u]);
          }
          return comb(comb(comb(x[0], x[1]), comb(x[2], x[3])), comb(comb(x[4], x[5]), comb(x[6], x[7])));
        };
        if constexpr (LVL == 1) {
          r = chunk(l0);
        } else if constexpr (LVL == 2) {
          /* two chunks, one at a time (keeps 8 loads in flight, not 16) */
#pragma unroll 1
          for (int c2 = 0; c2 < 2; c2++) {
            const PK y = chunk(l0 + 8 * c2);
            r = c2 ? comb(r, y) : y;
          }
        } else if constexpr (LVL == 4) {
          /* four chunks, one at a time: ((c0 c1)(c2 c3)) with two slots */
          PK h, s2;
#pragma unroll 1
          for (int c4 = 0; c4 < 4; c4++) {
            PK y = chunk(l0 + 8 * c4);
            if (c4 & 1) {
              y = comb(h, y);
              if (c4 == 1) s2 = y;
              else r = comb(s2, y);
            } else {
              h = y;
            }
          }
        } else {
          PK stk[LVL];
          for (int q0 = 0; q0 < n; q0 += 8) {
            PK y = chunk(l0 + q0);
            const int sidx = q0 >> 3, t = __ffs(~sidx) - 1;
#pragma unroll
            for (int L = 0; L < LVL - 1; L++)
              if (L < t) y = comb(stk[L], y);
#pragma unroll
            for (int L = 0; L < LVL; L++)
              if (L == t) stk[L] = y;
          }
          const int top = __ffs(n >> 3) - 1; /* log2(n/8) */
#pragma unroll
          for (int L = 0; L < LVL; L++)
            if (L == top) r = stk[L];
        }
      }
    }
    /* butterfly levels across the G lanes of this column */
#pragma unroll
    for (int m = 1; m < G; m <<= 1) {
      const PK o = shfl_xor_pack<T, V>(r, m);
      r = (g & m) ? comb(o, r) : comb(r, o);
      if constexpr (MM) {
#pragma unroll
        for (int i = 0; i < V; i++) cls[i] |= __shfl_xor_sync(0xffffffffu, cls[i], m);
      }
    }
    if (!live) continue;
    if constexpr (MM) {
      bool amb = false;
#pragma unroll
      for (int i = 0; i < V; i++) amb |= ambiguous(cls[i]);
      if (amb) { /* defer the pack; its dests stay untouched */
        if (g == 0) {
          const unsigned long long slot = atomicAdd(a.fix_count, (unsigned long long)V);
          for (int i = 0; i < V; i++) {
            if (slot + i < a.fix_cap) a.fix_list[slot + i] = e0 + i;
            else atomicOr(a.status, (int)B200SHM_STATUS_FIX_OVERFLOW);
          }
        }
        continue;
      }
    }
    char *dst = a.dst + e0 * sizeof(T);
    for (int j = m0; j < m1; j++) st_pack<T, V>(dst + (uint64_t)j * a.dstep, r);
  }
}

/* Grid for one register-path launch: at most `occ` CTAs per SM (8 unless
 * B200SHM_REDUCE_CTAS_PER_SM overrides it for tuning sweeps); CTAs
 * grid-stride over the packs. */
template <class K>
unsigned reduce_grid(K kernel, int &occ, uint64_t nvec, int threads) {
  (void)kernel;
  if (occ < 0) { /* cached per kernel instantiation by the caller */
    int o = 8; /* oversubscribed grid-stride grid: measured best */
    const char *env = getenv("B200SHM_REDUCE_CTAS_PER_SM");
    if (env && atoi(env) > 0) o = atoi(env);
    occ = o;
  }
  const uint64_t need = (nvec + threads - 1) / threads;
  const uint64_t cap = (uint64_t)grid_sms() * (uint64_t)occ;
  return (unsigned)(need < cap ? (need ? need : 1) : cap);
}

/* CTAs of 256 threads of `kernel` that one SM holds at once (cached per
 * kernel). */
int resident_ctas(const void *kernel) {
  static std::mutex mu;
  static std::unordered_map<const void *, int> cache;
  std::lock_guard<std::mutex> g(mu);
  auto it = cache.find(kernel);
  if (it != cache.end()) return it->second;
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, 256, 0) != cudaSuccess || n < 1) {
    (void)cudaGetLastError();
    n = 1;
  }
  cache[kernel] = n;
  return n;
}

/* Grid of the warp-cooperative kernel, in waves of the CTAs one SM holds
 * at once: 8 waves by default (B200SHM_REDUCE_WAVES overrides it, or
 * B200SHM_REDUCE_CTAS_PER_SM gives a fixed count).  On the 64-PE x 2^20
 * workload one exact wave was slowest (5.27 TB/s over the six
 * reductions): CTAs of a grid-stride loop finish unevenly and leave their
 * SM's slots idle, while the CTAs of later waves backfill them.  4 waves
 * gave 5.73, 6-16 waves 5.78-5.80, one pack per lane 5.76. */
unsigned coop_grid(const void *kernel, uint64_t lanes) {
  static int per_sm_env = -1, waves = 8;
  if (per_sm_env < 0) {
    const char *e = getenv("B200SHM_REDUCE_CTAS_PER_SM");
    per_sm_env = e && atoi(e) > 0 ? atoi(e) : 0;
    const char *w = getenv("B200SHM_REDUCE_WAVES");
    if (w && atoi(w) > 0) waves = atoi(w);
  }
  const int per_sm = per_sm_env ? per_sm_env : waves * resident_ctas(kernel);
  return grid_for(lanes, 256, per_sm);
}

template <class K>
void launch_one(K kernel, uint64_t lanes, cudaStream_t s, const RArgs &a) {
  kernel<<<coop_grid((const void *)kernel, lanes), 256, 0, s>>>(a);
}

template <class T, int OP, int ORDER, int V, bool MM, int G>
void launch_coop_g(int lvl, bool pow2, uint64_t lanes, cudaStream_t s, const RArgs &a) {
  if constexpr (ORDER == ORD_CHAIN) {
    launch_one(k_reduce_coop<T, OP, ORDER, V, G, MM, 1, true>, lanes, s, a);
  } else if constexpr (ORDER == ORD_BINOMIAL) { /* only power-of-two teams get here */
    if (lvl == 1) launch_one(k_reduce_coop<T, OP, ORDER, V, G, MM, 1, true>, lanes, s, a);
    else if (lvl == 2) launch_one(k_reduce_coop<T, OP, ORDER, V, G, MM, 2, true>, lanes, s, a);
    else if (lvl == 4) launch_one(k_reduce_coop<T, OP, ORDER, V, G, MM, 4, true>, lanes, s, a);
    else launch_one(k_reduce_coop<T, OP, ORDER, V, G, MM, 7, true>, lanes, s, a);
  } else {
    if (pow2) {
      if (lvl == 1) launch_one(k_reduce_coop<T, OP, ORDER, V, G, MM, 1, true>, lanes, s, a);
      else if (lvl == 2) launch_one(k_reduce_coop<T, OP, ORDER, V, G, MM, 2, true>, lanes, s, a);
      else if (lvl == 4) launch_one(k_reduce_coop<T, OP, ORDER, V, G, MM, 4, true>, lanes, s, a);
      else launch_one(k_reduce_coop<T, OP, ORDER, V, G, MM, 7, true>, lanes, s, a);
    } else {
      if (lvl == 1) launch_one(k_reduce_coop<T, OP, ORDER, V, G, MM, 1, false>, lanes, s, a);
      else if (lvl == 2) launch_one(k_reduce_coop<T, OP, ORDER, V, G, MM, 2, false>, lanes, s, a);
      else if (lvl == 4) launch_one(k_reduce_coop<T, OP, ORDER, V, G, MM, 4, false>, lanes, s, a);
      else launch_one(k_reduce_coop<T, OP, ORDER, V, G, MM, 7, false>, lanes, s, a);
    }
  }
}

template <class T, int OP, int ORDER, int V, bool MM>
void launch_coop(int G, int lvl, bool pow2, uint64_t lanes, cudaStream_t s, const RArgs &a) {
  switch (G) {
  case 2: launch_coop_g<T, OP, ORDER, V, MM, 2>(lvl, pow2, lanes, s, a); break;
  case 4: launch_coop_g<T, OP, ORDER, V, MM, 4>(lvl, pow2, lanes, s, a); break;
  default: launch_coop_g<T, OP, ORDER, V, MM, 8>(lvl, pow2, lanes, s, a); break;
  }
}

template <class T, int OP, int ORDER, bool MM, int LV>
int run_lv(const RArgs &base, bool aligned, cudaStream_t s) {
  constexpr int V = sizeof(T) >= 16 ? 1 : (int)(16 / sizeof(T));
  constexpr int U = ORDER == ORD_CHAIN ? 8 : 4;
  static int occ_pack = -1, occ_tail = -1;
  RArgs a = base;
  uint64_t done = 0;
  /* packs of several elements need 16-byte-aligned rows; a pack of one
   * 16-byte element (complex double, long double) moves at any alignment,
   * and its trees split over lanes too (long double SUM 1.52 -> 2.11 TB/s,
   * PROD 2.20 -> 3.16 on 64 members x 2^18), while its chains stay one
   * lane per element (long double MAX split over lanes: 2.56 -> 2.11) */
  if ((V > 1 ? aligned : ORDER != ORD_CHAIN) && done < base.N) {
    a.e_begin = done;
    a.nvec = (base.N - done) / V;
    if (a.nvec) {
      /* warp-cooperative split of the leaves is exact for any-order ops,
       * for butterflies, and for binomial trees over power-of-two teams.
       * G lanes per column: 2 for chains; for float trees as many as give
       * each lane 32 leaves (2 to 8).  On the 64-PE workload G = 2 with
       * 32 leaves per lane ran the f32 tree at 5.6-5.9 TB/s, G = 4 with 16
       * at 5.2-5.4 (a warp then reads 128 rather than 256 consecutive bytes
       * of each member per load).  B200SHM_REDUCE_COOP overrides (0 or 1 =
       * one lane per column). */
      constexpr bool any_order = ORDER == ORD_CHAIN && (std::is_integral<T>::value || MM);
      const int nleaves = ORDER == ORD_BUTTERFLY ? base.p2s : base.P;
      const bool splittable = any_order || ORDER == ORD_BUTTERFLY ||
                              (ORDER == ORD_BINOMIAL && (base.P & (base.P - 1)) == 0);
      /* float trees: 32 leaves per lane (four 8-leaf chunks, two slots),
       * so G = 2 at 64 leaves; chains: G = 2 */
      int G = 2;
      if constexpr (ORDER != ORD_CHAIN) G = std::max(2, std::min(8, nleaves / 32));
      static const char *ec = getenv("B200SHM_REDUCE_COOP"); /* read once */
      if (ec) G = atoi(ec);
      if (G < 1) G = 1;
      if (G > 32) G = 32;
      if (G > 8) G = 8;
      G = 1 << (31 - __builtin_clz((unsigned)G)); /* power of two */
      while (G > 1 && G * 8 > nleaves) G >>= 1;
      if constexpr (ORDER != ORD_CHAIN || any_order) {
        if (splittable && G >= 2) {
          const uint64_t lanes = a.nvec * (uint64_t)G;
          const int chunks = nleaves / G / 8; /* tree chunks per lane */
          const bool pow2 = ORDER != ORD_BUTTERFLY || base.P == base.p2s;
          launch_coop<T, OP, ORDER, V, MM>(G, ORDER == ORD_CHAIN ? 1 : chunks <= 1 ? 1 : chunks == 2 ? 2
                                                 : chunks == 4 ? 4 : 7,
                                           pow2, lanes, s, a);
          count_launch();
          done += a.nvec * V;
        }
      }
      if (done < base.N && a.e_begin == done) {
        auto k = k_reduce<T, OP, ORDER, V, U, MM, LV>;
        k<<<reduce_grid(k, occ_pack, a.nvec, 256), 256, 0, s>>>(a);
        count_launch();
        done += a.nvec * V;
      }
    }
  }
  if (done < base.N) {
    a.e_begin = done;
    a.nvec = base.N - done;
    auto k = k_reduce<T, OP, ORDER, 1, U, MM, LV>;
    k<<<reduce_grid(k, occ_tail, a.nvec, 256), 256, 0, s>>>(a);
    count_launch();
  }
  if constexpr (MM) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2 * grid_sms());
    cfg.blockDim = dim3(256);
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    B200_CK(cudaLaunchKernelEx(&cfg, k_minmax_fix<T, OP>, base,
                               (const unsigned long long *)base.fix_list, base.fix_count,
                               base.fix_done, base.fix_cap));
    count_launch();
  }
  return B200SHM_OK;
}

template <class T, int OP, int ORDER, bool MM>
int run(const RArgs &base, bool aligned, cudaStream_t s) {
  if constexpr (ORDER == ORD_CHAIN) {
    return run_lv<T, OP, ORDER, MM, 1>(base, aligned, s);
  } else {
    const int leaves = ORDER == ORD_BUTTERFLY ? base.p2s : base.P;
    if (leaves < (1 << 8)) return run_lv<T, OP, ORDER, MM, 8>(base, aligned, s);
    return run_lv<T, OP, ORDER, MM, kMaxLevels>(base, aligned, s);
  }
}

template <class T, int OP>
int run_float(const RArgs &a, bool aligned, cudaStream_t s) {
  if constexpr (OP == B200SHM_MIN || OP == B200SHM_MAX) {
    /* the deferred count is zero here: the previous replay cleared it */
    return run<T, OP, ORD_CHAIN, true>(a, aligned, s);
  } else {
    switch (a.algo) {
    case B200SHM_LINEAR: return run<T, OP, ORD_CHAIN, false>(a, aligned, s);
    case B200SHM_BINOMIAL: return run<T, OP, ORD_BINOMIAL, false>(a, aligned, s);
    default: return run<T, OP, ORD_BUTTERFLY, false>(a, aligned, s);
    }
  }
}

template <class T, int OP>
int run_cplx(const RArgs &a, bool aligned, cudaStream_t s) {
  switch (a.algo) {
  case B200SHM_LINEAR: return run<T, OP, ORD_CHAIN, false>(a, aligned, s);
  case B200SHM_BINOMIAL: return run<T, OP, ORD_BINOMIAL, false>(a, aligned, s);
  default: return run<T, OP, ORD_BUTTERFLY, false>(a, aligned, s);
  }
}

/* Integer ops other than MIN/MAX give the same bits on signed and unsigned
 * views, so they run on the unsigned type of the same width. */
template <class S, class U>
int run_int(int op, const RArgs &a, bool aligned, cudaStream_t s) {
  switch (op) {
  case B200SHM_AND: return run<U, B200SHM_AND, ORD_CHAIN, false>(a, aligned, s);
  case B200SHM_OR: return run<U, B200SHM_OR, ORD_CHAIN, false>(a, aligned, s);
  case B200SHM_XOR: return run<U, B200SHM_XOR, ORD_CHAIN, false>(a, aligned, s);
  case B200SHM_MIN: return run<S, B200SHM_MIN, ORD_CHAIN, false>(a, aligned, s);
  case B200SHM_MAX: return run<S, B200SHM_MAX, ORD_CHAIN, false>(a, aligned, s);
  case B200SHM_SUM: return run<U, B200SHM_SUM, ORD_CHAIN, false>(a, aligned, s);
  default: return run<U, B200SHM_PROD, ORD_CHAIN, false>(a, aligned, s);
  }
}

}  // namespace


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
  case B200SHM_I8: return run_int<int8_t, uint8_t>(op, a, aligned, s);
  case B200SHM_I16: return run_int<int16_t, uint16_t>(op, a, aligned, s);
  case B200SHM_I32: return run_int<int32_t, uint32_t>(op, a, aligned, s);
  case B200SHM_I64: return run_int<int64_t, uint64_t>(op, a, aligned, s);
  case B200SHM_U8: return run_int<uint8_t, uint8_t>(op, a, aligned, s);
  case B200SHM_U16: return run_int<uint16_t, uint16_t>(op, a, aligned, s);
  case B200SHM_U32: return run_int<uint32_t, uint32_t>(op, a, aligned, s);
  case B200SHM_U64: return run_int<uint64_t, uint64_t>(op, a, aligned, s);
  case B200SHM_F32:
    switch (op) {
    case B200SHM_MIN: return run_float<float, B200SHM_MIN>(a, aligned, s);
    case B200SHM_MAX: return run_float<float, B200SHM_MAX>(a, aligned, s);
    case B200SHM_SUM: return run_float<float, B200SHM_SUM>(a, aligned, s);
    default: return run_float<float, B200SHM_PROD>(a, aligned, s);
    }
  case B200SHM_F64:
    switch (op) {
    case B200SHM_MIN: return run_float<double, B200SHM_MIN>(a, aligned, s);
    case B200SHM_MAX: return run_float<double, B200SHM_MAX>(a, aligned, s);
    case B200SHM_SUM: return run_float<double, B200SHM_SUM>(a, aligned, s);
    default: return run_float<double, B200SHM_PROD>(a, aligned, s);
    }
  case B200SHM_F80:
    switch (op) {
    case B200SHM_MIN: return run_float<f80, B200SHM_MIN>(a, aligned, s);
    case B200SHM_MAX: return run_float<f80, B200SHM_MAX>(a, aligned, s);
    case B200SHM_SUM: return run_float<f80, B200SHM_SUM>(a, aligned, s);
    default: return run_float<f80, B200SHM_PROD>(a, aligned, s);
    }
  case B200SHM_C32:
    return op == B200SHM_SUM ? run_cplx<cf32, B200SHM_SUM>(a, aligned, s)
                             : run_cplx<cf32, B200SHM_PROD>(a, aligned, s);
  default:
    return op == B200SHM_SUM ? run_cplx<cf64, B200SHM_SUM>(a, aligned, s)
                             : run_cplx<cf64, B200SHM_PROD>(a, aligned, s);
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
