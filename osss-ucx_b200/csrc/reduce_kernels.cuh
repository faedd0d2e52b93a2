/*
 * reduce_kernels.cuh -- the one-pass all-reduce kernels and their launch
 * sequences, included by the translation units that instantiate them for
 * one family of element types each (reduce_int.cu, reduce_f32.cu,
 * reduce_f64.cu, reduce_c32.cu, reduce_c64.cu, and reduce_f80_<op>.cu for
 * long double, one op each), so the families compile in parallel.
 * Everything here has internal linkage.
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
#pragma once
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <mutex>
#include <type_traits>
#include <unordered_map>
#include <vector>

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
}  // namespace b200
