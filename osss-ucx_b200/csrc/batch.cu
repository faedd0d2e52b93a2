/*
 * batch.cu -- many independent reductions submitted together
 * (b200shm_batch_create / run / destroy, b200shm_reduce_batch).
 *
 * The reference can only issue shcoll_<T>_<op>_reduce_<algo> calls one
 * after the other (src/shcoll/src/reduce.c:1078-1102), each a full
 * algorithm with its own synchronisation.  Here a batch is planned once:
 * every descriptor is cut into tiles of 16-byte columns, descriptors are
 * sorted into groups of one (type slot, op, combine order), and each group
 * runs as ONE persistent kernel specialised for it that takes tiles from a
 * counter.  Groups are spread over a few side streams so that one group's
 * tail overlaps the next group's start; with B200SHM_BATCH_GRAPH the whole
 * run is captured once into a CUDA graph.
 *
 * Every result is bit-identical to b200shm_reduce on the same descriptor:
 * a lane combines its members in the same order as the per-call kernels
 * (a chain for order-free ops, the reference's tree shape for float
 * SUM/PROD, deferral plus exact replay for order-dependent float MIN/MAX
 * elements).  Per descriptor the plan picks the lanes per 16-byte column
 * G, the columns per lane U (small teams serve 2 or 4 columns at once so a
 * lane keeps ~8 loads in flight) and the tile size, by a measured
 * heuristic, and then (by default) an autotuner that times candidate
 * (G, tile) plans per shape class inside the whole batch as it runs.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include <type_traits>
#include <vector>

#include "internal.cuh"
/* The batch kernels keep write-back stores and L1-bypassing loads: with
 * the streaming (evict-first) policy of the per-call kernels the batching
 * workload ran 2.63-2.66 ms against 2.615-2.620. */
#define B200_LD_OP "ld.global.nc.L1::no_allocate"
#define B200_ST_OP "st.global"
#include "reduce_core.cuh"

namespace b200 {
namespace {

/* type slots of the batch kernels */
enum { DS_I32 = 0, DS_U32, DS_I64, DS_U64, DS_F32, DS_F64, DS_N };
/* group id: type slot, op, combine order, and the column class (0, 1, 2:
 * each lane serves 1, 2 or 4 columns at once) */
constexpr int kbase(int ds, int op, int order) { return (ds * 7 + op) * 3 + order; }
constexpr int kid_of(int ds, int op, int order, int uc = 0) {
  return kbase(ds, op, order) * 3 + uc;
}
constexpr int kBatchThreads = 256;
constexpr int kBatchStackLevels = 9;     /* subtree levels a lane keeps */
constexpr int kBatchMaxLaneLeaves = 256; /* leaves per lane: 2^(levels - 1) */

struct BDesc {
  const char *src;
  char *dst;
  uint64_t step;    /* bytes between consecutive members             */
  uint64_t N;       /* elements                                      */
  uint64_t npacks;  /* 16-byte packs of the vector part (0 if !vec)  */
  int P, p2s, logp2s, algo;
  int kid, vec, G, TP; /* TP: packs (vec) or elements (!vec) per tile */
  int U;               /* columns each lane serves at once (small teams) */
  int id;              /* index of the caller's descriptor */
};

struct BPlan {
  const BDesc *d;
  const uint32_t *prefix; /* ndesc + 1 tile prefix sums */
  const uint2 *tile_map;  /* per tile of the plan: (descriptor, tile within it) */
  uint32_t ndesc, total;
  unsigned long long *fix_list, *fix_count;
  unsigned long long fix_cap;
  int *status;
};

/* A lane's stack of complete subtrees lives in shared memory, one 32-bit
 * word per thread per row ([level][word][thread]), so that a warp's
 * accesses fall in 32 distinct banks. */
template <class PK>
__device__ __forceinline__ void stk_put(uint32_t *stk, int L, const PK &v) {
  constexpr int W = sizeof(PK) / 4;
  uint32_t w[W];
  memcpy(w, &v, sizeof(PK));
#pragma unroll
  for (int k = 0; k < W; k++) stk[(L * W + k) * kBatchThreads + threadIdx.x] = w[k];
}
template <class PK>
__device__ __forceinline__ PK stk_get(const uint32_t *stk, int L) {
  constexpr int W = sizeof(PK) / 4;
  uint32_t w[W];
#pragma unroll
  for (int k = 0; k < W; k++) w[k] = stk[(L * W + k) * kBatchThreads + threadIdx.x];
  PK v;
  memcpy(&v, w, sizeof(PK));
  return v;
}

/* One tile: units [u0, u0+cnt) of descriptor d, a unit being a V-element
 * pack.  G lanes share a column; lane g reduces leaves [l0, l1) (members
 * [m0, m1), a butterfly leaf's extra member included), the G partials are
 * combined with shuffles over masks 1, 2, ..., G/2 (the tree's top
 * levels), and each lane stores the result to its own members. */
template <class T, int OP, int ORDER, bool MM, int V>
__device__ void run_tile(const BDesc &d, uint32_t di, uint64_t u0, uint64_t cnt, const BPlan &p,
                         uint32_t *stk) {
  typedef Pack<T, V> PK;
  const int G = d.G;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = kBatchThreads >> 5;
  const int g = lane & (G - 1), cw = lane / G, cpw = 32 / G;
  const int P = d.P;
  const int nleaves = ORDER == ORD_BUTTERFLY ? d.p2s : P;
  const int l0 = (int)((long long)g * nleaves / G), l1 = (int)((long long)(g + 1) * nleaves / G);
  /* the member holding leaf q: ceil(q * P / p2s) for the butterfly */
  auto member_of = [&](int q) -> int {
    return ORDER == ORD_BUTTERFLY ? (int)(((long long)q * P + d.p2s - 1) >> d.logp2s) : q;
  };
  const int m0 = member_of(l0), m1 = member_of(l1);
  auto comb = [](const PK &lo, const PK &hi) {
    if constexpr (ORDER == ORD_BINOMIAL) return papply<OP>(hi, lo);
    else return papply<OP>(lo, hi);
  };
  for (uint64_t base = (uint64_t)warp * cpw; base < cnt; base += (uint64_t)nw * cpw) {
    const uint64_t col = base + cw;
    const bool live = col < cnt;
    const uint64_t e0 = (u0 + (live ? col : 0)) * V;
    const char *src = d.src + e0 * sizeof(T);
    PK r;
    unsigned cls[V];
#pragma unroll
    for (int i = 0; i < V; i++) cls[i] = 0;
    if (live) {
      if constexpr (ORDER == ORD_CHAIN) {
        r = ld_pack<T, V>(src + (uint64_t)m0 * d.step);
        if constexpr (MM) {
#pragma unroll
          for (int i = 0; i < V; i++) cls[i] = fclass(r.x[i]);
        }
        for (int j = m0 + 1; j < m1; j += 8) {
          PK x[8];
#pragma unroll
          for (int u = 0; u < 8; u++)
            if (j + u < m1) x[u] = ld_pack<T, V>(src + (uint64_t)(j + u) * d.step);
#pragma unroll
          for (int u = 0; u < 8; u++)
            if (j + u < m1) {
              r = papply<OP>(r, x[u]);
              if constexpr (MM) {
#pragma unroll
                for (int i = 0; i < V; i++) cls[i] |= fclass(x[u].x[i]);
              }
            }
        }
      } else {
        /* The lane's leaves are taken KB at a time: their own members and
         * (for a butterfly over a non-power-of-two team) extra members
         * are all loaded before any is used, the extras are folded on
         * (op(extra, own)), a full batch is reduced as a register subtree
         * of KB leaves, and subtrees enter a binary counter kept in shared
         * memory: pushing a subtree of 2^lv leaves when c leaves are in
         * combines it with the stacked subtrees of levels lv .. lv +
         * (trailing ones of c >> lv) - 1, earlier subtree first -- the
         * reference tree's shape.  8 leaves without extras, 4 with: either
         * way at most 8 loads, and registers for 8 packs, in flight. */
        int c = 0;
        auto push_lv = [&](PK v, int lv) {
          const int t = __ffs(~(c >> lv)) - 1 + lv;
          for (int L = lv; L < t; L++) v = comb(stk_get<PK>(stk, L), v);
          stk_put(stk, t, v);
          c += 1 << lv;
        };
        auto leaves = [&](auto kb_c, auto ex_c) {
          constexpr int KB = decltype(kb_c)::value;
          constexpr bool EX = decltype(ex_c)::value;
          constexpr int LB = KB == 8 ? 3 : 2;
          for (int qb = l0; qb < l1; qb += KB) {
            const int k = l1 - qb < KB ? l1 - qb : KB;
            PK x[KB], e[EX ? KB : 1];
            bool ex[KB];
#pragma unroll
            for (int u = 0; u < KB; u++) {
              ex[u] = false;
              if (u < k) {
                const int mo = member_of(qb + u);
                x[u] = ld_pack<T, V>(src + (uint64_t)mo * d.step);
                if constexpr (EX) {
                  ex[u] = member_of(qb + u + 1) - mo == 2;
                  if (ex[u]) e[u] = ld_pack<T, V>(src + (uint64_t)(mo + 1) * d.step);
                }
              }
            }
            if constexpr (EX) {
#pragma unroll
              for (int u = 0; u < KB; u++)
                if (ex[u]) x[u] = papply<OP>(e[u], x[u]);
            }
            if (k == KB) {
#pragma unroll
              for (int w = KB; w > 1; w >>= 1) {
#pragma unroll
                for (int i = 0; i < w / 2; i++) x[i] = comb(x[2 * i], x[2 * i + 1]);
              }
              push_lv(x[0], LB);
            } else {
#pragma unroll
              for (int u = 0; u < KB; u++)
                if (u < k) push_lv(x[u], 0);
            }
          }
        };
        if (ORDER == ORD_BUTTERFLY && P != d.p2s)
          leaves(std::integral_constant<int, 4>{}, std::true_type{});
        else
          leaves(std::integral_constant<int, 8>{}, std::false_type{});
        const int n = l1 - l0;
        if ((n & (n - 1)) == 0) {
          r = stk_get<PK>(stk, __ffs(n) - 1);
        } else { /* binomial over a whole non-power-of-two team (G == 1) */
          bool have = false;
          for (int L = 0; L < kBatchStackLevels; L++)
            if (n & (1 << L)) {
              const PK sub = stk_get<PK>(stk, L);
              r = have ? comb(sub, r) : sub;
              have = true;
            }
        }
      }
    }
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
      if (amb) { /* deferred: (descriptor, element) pairs, dests untouched */
        if (g == 0) {
          const unsigned long long slot = atomicAdd(p.fix_count, (unsigned long long)V);
          for (int i = 0; i < V; i++) {
            if (slot + i < p.fix_cap)
              p.fix_list[slot + i] = ((unsigned long long)di << 40) | (e0 + i);
            else
              atomicOr(p.status, (int)B200SHM_STATUS_FIX_OVERFLOW);
          }
        }
        continue;
      }
    }
    char *dst = d.dst + e0 * sizeof(T);
    for (int j = m0; j < m1; j++) st_pack<T, V>(dst + (uint64_t)j * d.step, r);
  }
}

/* The small-team form of a tile: each lane serves U columns at once, so a
 * lane of a 2-member team still has 8 loads in flight.  Chains (members in
 * batches of 8/U per column), and butterflies whose lanes hold at most 2
 * leaves (combined in registers per column, extras loaded alongside). */
template <class T, int OP, int ORDER, bool MM, int V, int U>
__device__ void run_tile_multi(const BDesc &d, uint32_t di, uint64_t u0, uint64_t cnt,
                               const BPlan &p) {
  typedef Pack<T, V> PK;
  const int G = d.G;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = kBatchThreads >> 5;
  const int g = lane & (G - 1), cw = lane / G, cpw = 32 / G;
  const int P = d.P;
  const int nleaves = ORDER == ORD_BUTTERFLY ? d.p2s : P;
  const int l0 = (int)((long long)g * nleaves / G), l1 = (int)((long long)(g + 1) * nleaves / G);
  auto member_of = [&](int q) -> int {
    return ORDER == ORD_BUTTERFLY ? (int)(((long long)q * P + d.p2s - 1) >> d.logp2s) : q;
  };
  const int m0 = member_of(l0), m1 = member_of(l1);
  auto comb = [](const PK &lo, const PK &hi) { return papply<OP>(lo, hi); };
  for (uint64_t base = (uint64_t)warp * cpw * U; base < cnt; base += (uint64_t)nw * cpw * U) {
    PK r[U];
    unsigned cls[U][V];
    bool live[U];
    const char *src[U];
#pragma unroll
    for (int k = 0; k < U; k++) {
      const uint64_t col = base + cw + (uint64_t)k * cpw;
      live[k] = col < cnt;
      src[k] = d.src + (u0 + (live[k] ? col : 0)) * V * sizeof(T);
#pragma unroll
      for (int i = 0; i < V; i++) cls[k][i] = 0;
    }
    if constexpr (ORDER == ORD_CHAIN) {
      constexpr int MB = 8 / U; /* members per batch, per column */
#pragma unroll
      for (int k = 0; k < U; k++)
        if (live[k]) {
          r[k] = ld_pack<T, V>(src[k] + (uint64_t)m0 * d.step);
          if constexpr (MM) {
#pragma unroll
            for (int i = 0; i < V; i++) cls[k][i] = fclass(r[k].x[i]);
          }
        }
      for (int j = m0 + 1; j < m1; j += MB) {
        PK x[U][MB];
#pragma unroll
        for (int k = 0; k < U; k++)
#pragma unroll
          for (int u = 0; u < MB; u++)
            if (live[k] && j + u < m1) x[k][u] = ld_pack<T, V>(src[k] + (uint64_t)(j + u) * d.step);
#pragma unroll
        for (int k = 0; k < U; k++)
#pragma unroll
          for (int u = 0; u < MB; u++)
            if (live[k] && j + u < m1) {
              r[k] = papply<OP>(r[k], x[k][u]);
              if constexpr (MM) {
#pragma unroll
                for (int i = 0; i < V; i++) cls[k][i] |= fclass(x[k][u].x[i]);
              }
            }
      }
    } else { /* butterfly, l1 - l0 in {1, 2} leaves per lane */
      const int n = l1 - l0;
      PK x[U][2], e[U][2];
      bool ex[U][2];
#pragma unroll
      for (int k = 0; k < U; k++)
#pragma unroll
        for (int u = 0; u < 2; u++) {
          ex[k][u] = false;
          if (live[k] && u < n) {
            const int own = member_of(l0 + u);
            x[k][u] = ld_pack<T, V>(src[k] + (uint64_t)own * d.step);
            ex[k][u] = member_of(l0 + u + 1) - own == 2;
            if (ex[k][u]) e[k][u] = ld_pack<T, V>(src[k] + (uint64_t)(own + 1) * d.step);
          }
        }
#pragma unroll
      for (int k = 0; k < U; k++) {
#pragma unroll
        for (int u = 0; u < 2; u++)
          if (ex[k][u]) x[k][u] = papply<OP>(e[k][u], x[k][u]); /* op(extra, own) */
        r[k] = n == 1 ? x[k][0] : comb(x[k][0], x[k][1]);
      }
    }
    for (int m = 1; m < G; m <<= 1) {
#pragma unroll
      for (int k = 0; k < U; k++) {
        const PK o = shfl_xor_pack<T, V>(r[k], m);
        r[k] = (g & m) ? comb(o, r[k]) : comb(r[k], o);
        if constexpr (MM) {
#pragma unroll
          for (int i = 0; i < V; i++) cls[k][i] |= __shfl_xor_sync(0xffffffffu, cls[k][i], m);
        }
      }
    }
#pragma unroll
    for (int k = 0; k < U; k++) {
      if (!live[k]) continue;
      const uint64_t e0 = (uint64_t)(src[k] - d.src) / sizeof(T);
      if constexpr (MM) {
        bool amb = false;
#pragma unroll
        for (int i = 0; i < V; i++) amb |= ambiguous(cls[k][i]);
        if (amb) { /* deferred: (descriptor, element) pairs, dests untouched */
          if (g == 0) {
            const unsigned long long slot = atomicAdd(p.fix_count, (unsigned long long)V);
            for (int i = 0; i < V; i++) {
              if (slot + i < p.fix_cap)
                p.fix_list[slot + i] = ((unsigned long long)di << 40) | (e0 + i);
              else
                atomicOr(p.status, (int)B200SHM_STATUS_FIX_OVERFLOW);
            }
          }
          continue;
        }
      }
      char *dst = d.dst + e0 * sizeof(T);
      for (int j = m0; j < m1; j++) st_pack<T, V>(dst + (uint64_t)j * d.step, r[k]);
    }
  }
}

template <class T, int OP, int ORDER, bool MM, int U>
__device__ __forceinline__ void run_desc_tile(const BDesc &d, uint32_t di, uint32_t lt,
                                              const BPlan &p, uint32_t *stk) {
  constexpr int V = sizeof(T) >= 16 ? 1 : (int)(16 / sizeof(T));
  const uint64_t nvt = d.vec ? (d.npacks + d.TP - 1) / d.TP : 0;
  if (d.vec && lt < nvt) {
    const uint64_t pb = (uint64_t)lt * d.TP;
    const uint64_t c = d.npacks - pb < (uint64_t)d.TP ? d.npacks - pb : (uint64_t)d.TP;
    if constexpr (U > 1) run_tile_multi<T, OP, ORDER, MM, V, U>(d, di, pb, c, p);
    else run_tile<T, OP, ORDER, MM, V>(d, di, pb, c, p, stk);
  } else {
    uint64_t eb, ec;
    if (d.vec) { /* the < V elements after the packs */
      eb = d.npacks * V;
      ec = d.N - eb;
    } else {
      eb = (uint64_t)lt * d.TP;
      ec = d.N - eb < (uint64_t)d.TP ? d.N - eb : (uint64_t)d.TP;
    }
    run_tile<T, OP, ORDER, MM, 1>(d, di, eb, ec, p, stk);
  }
}

/* One (type, op, order) group of a batch: descriptors [d0, d0+nd) of the
 * plan (sorted by group), tiles taken from the group's counter. */
template <class T, int OP, int ORDER, bool MM, int U>
__global__ void __launch_bounds__(kBatchThreads, 2) k_batch_group(const BPlan p, uint32_t d0,
                                                               uint32_t nd, unsigned *counter) {
  __shared__ unsigned s_tile;
  /* 16-byte packs: 4 words per level per thread (chains keep no stack) */
  __shared__ uint32_t s_stk[ORDER == ORD_CHAIN ? 1 : kBatchStackLevels * 4 * kBatchThreads];
  const uint32_t base = p.prefix[d0], total = p.prefix[d0 + nd] - base;
  /* A tile's descriptor comes from the plan's tile map in one load, not
   * from a binary search over the group's descriptors. */
  for (;;) {
    if (threadIdx.x == 0) s_tile = atomicAdd(counter, 1u);
    __syncthreads();
    const unsigned t = s_tile;
    __syncthreads();
    if (t >= total) return;
    const uint2 m = p.tile_map[base + t];
    const BDesc d = p.d[m.x];
    run_desc_tile<T, OP, ORDER, MM, U>(d, m.x, m.y, p, s_stk);
  }
}

/* exact replay of the deferred float MIN/MAX elements of a batch */
template <class T, int OP>
__device__ void batch_fix_one(const BDesc &d, uint64_t e, T *vals, T &common) {
  for (int j = threadIdx.x; j < d.P; j += blockDim.x)
    memcpy(&vals[j], d.src + (uint64_t)j * d.step + e * sizeof(T), sizeof(T));
  __syncthreads();
  const bool lower = e < d.N / 2;
  auto get = [&](int j) { return vals[j]; };
  if (d.algo == B200SHM_REC_DBL) {
    for (int q = threadIdx.x; q < d.p2s; q += blockDim.x) {
      const T v = exact_value<T, OP>(get, d.P, d.p2s, d.logp2s, d.algo, lower, q);
      const int as = p2s_member(q, d.P, d.p2s);
      memcpy(d.dst + (uint64_t)as * d.step + e * sizeof(T), &v, sizeof(T));
      if (p2s_extra(q, d.P, d.p2s))
        memcpy(d.dst + (uint64_t)(as + 1) * d.step + e * sizeof(T), &v, sizeof(T));
    }
  } else {
    if (threadIdx.x == 0) {
      int q = 0;
      if (d.algo == B200SHM_RABENSEIFNER || d.algo == B200SHM_RABENSEIFNER2)
        q = rev_bits(rab_block(e, d.N, d.p2s), d.logp2s);
      common = exact_value<T, OP>(get, d.P, d.p2s, d.logp2s, d.algo, lower, q);
    }
    __syncthreads();
    for (int j = threadIdx.x; j < d.P; j += blockDim.x)
      memcpy(d.dst + (uint64_t)j * d.step + e * sizeof(T), &common, sizeof(T));
  }
  __syncthreads();
}

__global__ void __launch_bounds__(256) k_batch_fix(const BPlan p) {
  __shared__ double vals[kFixMaxMembers];
  __shared__ double common;
  const unsigned long long n = *p.fix_count < p.fix_cap ? *p.fix_count : p.fix_cap;
  for (unsigned long long k = blockIdx.x; k < n; k += gridDim.x) {
    const unsigned long long ent = p.fix_list[k];
    const BDesc d = p.d[ent >> 40];
    const uint64_t e = ent & ((1ull << 40) - 1);
    float *vf = (float *)vals;
    float &cf = *(float *)&common;
    switch (d.kid / 3) {
    case kbase(DS_F32, B200SHM_MIN, ORD_CHAIN): batch_fix_one<float, B200SHM_MIN>(d, e, vf, cf); break;
    case kbase(DS_F32, B200SHM_MAX, ORD_CHAIN): batch_fix_one<float, B200SHM_MAX>(d, e, vf, cf); break;
    case kbase(DS_F64, B200SHM_MIN, ORD_CHAIN): batch_fix_one<double, B200SHM_MIN>(d, e, vals, common); break;
    default: batch_fix_one<double, B200SHM_MAX>(d, e, vals, common); break;
    }
  }
}

/* ---- host-side planning -------------------------------------------------- */
int dslot_of(int dtype) {
  switch (dtype) {
  case B200SHM_I32: return DS_I32;
  case B200SHM_U32: return DS_U32;
  case B200SHM_I64: return DS_I64;
  case B200SHM_U64: return DS_U64;
  case B200SHM_F32: return DS_F32;
  case B200SHM_F64: return DS_F64;
  default: return -1;
  }
}

struct Shape {
  int order, esize, pb, nb, vec;
  bool operator<(const Shape &o) const {
    return std::tie(order, esize, pb, nb, vec) < std::tie(o.order, o.esize, o.pb, o.nb, o.vec);
  }
};
std::mutex g_tune_mu;
std::map<Shape, std::pair<int, int>> g_tune; /* shape -> (G, TP), chosen by the autotuner */

int log2_floor(uint64_t x) {
  int l = 0;
  while (x > 1) {
    x >>= 1;
    l++;
  }
  return l;
}

inline int ds_of(const BDesc &d) { return d.kid / 3 / 21; }
inline int op_of(const BDesc &d) { return (d.kid / 3 / 3) % 7; }
inline int order_of(const BDesc &d) { return (d.kid / 3) % 3; }
inline int esize_of(const BDesc &d) {
  const int ds = ds_of(d);
  return (ds == DS_I32 || ds == DS_U32 || ds == DS_F32) ? 4 : 8;
}
inline bool is_mm_float(const BDesc &d) {
  return ds_of(d) >= DS_F32 && (op_of(d) == B200SHM_MIN || op_of(d) == B200SHM_MAX);
}
/* the shape class a plan is chosen (and cached) for */
inline Shape shape_of(const BDesc &d) {
  return Shape{order_of(d) * 2 + (is_mm_float(d) ? 1 : 0), esize_of(d),
               log2_floor((uint64_t)d.P), log2_floor(d.N) / 2, d.vec};
}
/* shape classes the autotuner tries, the heaviest (by bytes) first */
constexpr size_t kTuneClasses = 8;

/* Columns per lane for small teams: enough that a lane keeps about 8
 * loads in flight (chains: members per lane <= 2 -> 4 columns, <= 4 -> 2;
 * butterflies with at most 2 leaves per lane: 2 columns). */
void set_columns(BDesc &d) {
  const int order = order_of(d);
  const int mpl = (d.P + d.G - 1) / d.G;
  d.U = 1;
  if (d.vec) {
    if (order == ORD_CHAIN) d.U = mpl <= 2 ? 4 : mpl <= 4 ? 2 : 1;
    else if (order == ORD_BUTTERFLY && d.p2s / d.G <= 2) d.U = 2;
  }
  d.kid = d.kid / 3 * 3 + (d.U == 4 ? 2 : d.U == 2 ? 1 : 0);
}

/* lanes per column that keep the batch kernel exact and within its stack */
bool lanes_ok(const BDesc &d, int G) {
  const int order = order_of(d);
  if (order == ORD_CHAIN) {
    const bool any_order = ds_of(d) < DS_F32 || is_mm_float(d);
    if (!any_order) return G == 1; /* float linear left fold is sequential */
    return G <= d.P;
  }
  const int nleaves = order == ORD_BUTTERFLY ? d.p2s : d.P;
  if (order == ORD_BINOMIAL && (d.P & (d.P - 1)) && G > 1) return false;
  if (G > nleaves) return false;
  return nleaves / G <= kBatchMaxLaneLeaves;
}

uint32_t tiles_of(const BDesc &d) {
  if (d.vec) {
    const uint64_t V = 16 / (uint64_t)esize_of(d);
    const uint64_t t = (d.npacks + d.TP - 1) / d.TP;
    return (uint32_t)(t + (d.N > d.npacks * V ? 1 : 0));
  }
  return (uint32_t)((d.N + d.TP - 1) / d.TP);
}

/* An uploaded plan: descriptors sorted by (type, op, order) group, tile
 * prefix sums, one tile counter per group. */
struct Group {
  int kid;
  uint32_t d0, nd, tiles;
  int grid;
};
struct Batch {
  std::vector<BDesc> hd;
  std::vector<uint32_t> hp;
  std::vector<Group> groups;
  std::vector<b200shm_reduce_desc> fallback; /* run as separate launches */
  BDesc *dd = nullptr;
  uint32_t *dp = nullptr;
  uint2 *dmap = nullptr; /* tile map (BPlan::tile_map) */
  unsigned *dcount = nullptr;
  bool any_mm = false;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  unsigned graph_launches = 0; /* kernels one replay of `exec` runs */
  /* side streams the groups are spread over, so that one group's tail
   * overlaps the next group's start (forked from and joined back into the
   * caller's stream with events; inside a capture they become branches) */
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> ev; /* ev[0] = fork, ev[1 + k] = join of side[k] */
  cudaEvent_t done = nullptr;  /* recorded after each run on the caller's stream */
};

constexpr int kBatchSideStreams = 4;

/* Free a plan whose runs have completed (ordered on the library stream). */
void release(Batch &b) {
  for (cudaStream_t x : b.side) cudaStreamDestroy(x);
  for (cudaEvent_t e : b.ev) cudaEventDestroy(e);
  if (b.done) cudaEventDestroy(b.done);
  b.done = nullptr;
  b.side.clear();
  b.ev.clear();
  if (b.dd) cudaFreeAsync(b.dd, st().stream);
  if (b.dp) cudaFreeAsync(b.dp, st().stream);
  if (b.dmap) cudaFreeAsync(b.dmap, st().stream);
  if (b.dcount) cudaFreeAsync(b.dcount, st().stream);
  b.dd = nullptr;
  b.dp = nullptr;
  b.dmap = nullptr;
  b.dcount = nullptr;
}

int make_side(Batch &b) {
  const int k = (int)std::min<size_t>(b.groups.size(), kBatchSideStreams);
  if (k < 2) return B200SHM_OK;
  for (int i = 0; i < k; i++) {
    cudaStream_t x;
    B200_CK(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking));
    b.side.push_back(x);
  }
  for (int i = 0; i <= k; i++) {
    cudaEvent_t e;
    B200_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b.ev.push_back(e);
  }
  return B200SHM_OK;
}

BPlan plan_of(const Batch &b) {
  BPlan p;
  p.d = b.dd;
  p.prefix = b.dp;
  p.tile_map = b.dmap;
  p.ndesc = (uint32_t)b.hd.size();
  p.total = b.hp.empty() ? 0 : b.hp.back();
  p.fix_list = st().fix_list;
  p.fix_count = st().fix_count;
  p.fix_cap = st().fix_cap;
  p.status = st().d_status;
  return p;
}

/* the group kernel of a kid, and its resident CTAs per SM */
typedef void (*GroupKernel)(const BPlan, uint32_t, uint32_t, unsigned *);
template <class T, int OP, int ORDER, bool MM, int U>
GroupKernel gk() {
  return k_batch_group<T, OP, ORDER, MM, U>;
}
#define B200_CHAIN_KIDS(DS, T_, OP_, MM_)                                               \
  case kid_of(DS, OP_, ORD_CHAIN, 0): return gk<T_, OP_, ORD_CHAIN, MM_, 1>();          \
  case kid_of(DS, OP_, ORD_CHAIN, 1): return gk<T_, OP_, ORD_CHAIN, MM_, 2>();          \
  case kid_of(DS, OP_, ORD_CHAIN, 2): return gk<T_, OP_, ORD_CHAIN, MM_, 4>();
#define B200_INT_KIDS(DS, S_, U_)                                                       \
  B200_CHAIN_KIDS(DS, U_, B200SHM_AND, false)                                           \
  B200_CHAIN_KIDS(DS, U_, B200SHM_OR, false)                                            \
  B200_CHAIN_KIDS(DS, U_, B200SHM_XOR, false)                                           \
  B200_CHAIN_KIDS(DS, S_, B200SHM_MIN, false)                                           \
  B200_CHAIN_KIDS(DS, S_, B200SHM_MAX, false)                                           \
  B200_CHAIN_KIDS(DS, U_, B200SHM_SUM, false)                                           \
  B200_CHAIN_KIDS(DS, U_, B200SHM_PROD, false)
#define B200_TREE_KIDS(DS, F_, OP_)                                                     \
  case kid_of(DS, OP_, ORD_BINOMIAL, 0): return gk<F_, OP_, ORD_BINOMIAL, false, 1>();  \
  case kid_of(DS, OP_, ORD_BUTTERFLY, 0): return gk<F_, OP_, ORD_BUTTERFLY, false, 1>();\
  case kid_of(DS, OP_, ORD_BUTTERFLY, 1): return gk<F_, OP_, ORD_BUTTERFLY, false, 2>();
#define B200_FLT_KIDS(DS, F_)                                                           \
  B200_CHAIN_KIDS(DS, F_, B200SHM_MIN, true)                                            \
  B200_CHAIN_KIDS(DS, F_, B200SHM_MAX, true)                                            \
  B200_CHAIN_KIDS(DS, F_, B200SHM_SUM, false)                                           \
  B200_CHAIN_KIDS(DS, F_, B200SHM_PROD, false)                                          \
  B200_TREE_KIDS(DS, F_, B200SHM_SUM)                                                   \
  B200_TREE_KIDS(DS, F_, B200SHM_PROD)
GroupKernel group_kernel(int kid) {
  switch (kid) {
    B200_INT_KIDS(DS_I32, int32_t, uint32_t)
    B200_INT_KIDS(DS_U32, uint32_t, uint32_t)
    B200_INT_KIDS(DS_I64, int64_t, uint64_t)
    B200_INT_KIDS(DS_U64, uint64_t, uint64_t)
    B200_FLT_KIDS(DS_F32, float)
    B200_FLT_KIDS(DS_F64, double)
  default: return nullptr;
  }
}
int resident_ctas(int kid) {
  static std::mutex mu;
  static std::map<int, int> occ;
  std::lock_guard<std::mutex> lk(mu);
  auto it = occ.find(kid);
  if (it != occ.end()) return it->second;
  int o = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, group_kernel(kid), kBatchThreads, 0) !=
          cudaSuccess ||
      o < 1)
    o = 1;
  occ[kid] = o;
  return o;
}

int enqueue(const Batch &b, cudaStream_t s) {
  if (!b.hd.empty()) {
    B200_CK(cudaMemsetAsync(b.dcount, 0, b.groups.size() * sizeof(unsigned), s));
    if (b.any_mm) B200_CK(cudaMemsetAsync(st().fix_count, 0, sizeof(unsigned long long), s));
    const BPlan p = plan_of(b);
    const size_t ns = b.side.size();
    if (ns) {
      B200_CK(cudaEventRecord(b.ev[0], s));
      for (size_t k = 0; k < ns; k++) B200_CK(cudaStreamWaitEvent(b.side[k], b.ev[0], 0));
    }
    for (size_t gi = 0; gi < b.groups.size(); gi++) {
      const Group &g = b.groups[gi];
      cudaStream_t gs = ns ? b.side[gi % ns] : s;
      group_kernel(g.kid)<<<g.grid, kBatchThreads, 0, gs>>>(p, g.d0, g.nd, b.dcount + gi);
      count_launch();
    }
    if (ns) {
      for (size_t k = 0; k < ns; k++) {
        B200_CK(cudaEventRecord(b.ev[1 + k], b.side[k]));
        B200_CK(cudaStreamWaitEvent(s, b.ev[1 + k], 0));
      }
    }
    if (b.any_mm) {
      k_batch_fix<<<2 * st().sm_count, 256, 0, s>>>(p);
      count_launch();
    }
  }
  for (const b200shm_reduce_desc &d : b.fallback) {
    int rc = reduce_launch(d.op, d.dtype, d.algo, d.pe_start, d.pe_stride, d.pe_size, d.dest_off,
                           d.src_off, d.nelems, s);
    if (rc) return rc;
  }
  return B200SHM_OK;
}

/* Sort by group (stable), build prefix sums and groups, upload. */
int upload(Batch &b) {
  const size_t nd = b.hd.size();
  if (nd == 0) return B200SHM_OK;
  std::stable_sort(b.hd.begin(), b.hd.end(),
                   [](const BDesc &x, const BDesc &y) { return x.kid < y.kid; });
  b.hp.assign(nd + 1, 0);
  for (size_t i = 0; i < nd; i++) b.hp[i + 1] = b.hp[i] + tiles_of(b.hd[i]);
  b.groups.clear();
  for (size_t i = 0; i < nd;) {
    size_t j = i;
    while (j < nd && b.hd[j].kid == b.hd[i].kid) j++;
    Group g;
    g.kid = b.hd[i].kid;
    g.d0 = (uint32_t)i;
    g.nd = (uint32_t)(j - i);
    g.tiles = b.hp[j] - b.hp[i];
    const uint64_t cap = (uint64_t)st().sm_count * (uint64_t)resident_ctas(g.kid);
    g.grid = (int)(g.tiles < cap ? (g.tiles ? g.tiles : 1) : cap);
    b.groups.push_back(g);
    i = j;
  }
  /* stream-ordered allocations: no device-wide synchronisation, so a
   * running serving loop does not hold them up */
  cudaStream_t ls = st().stream;
  B200_CK(cudaMallocAsync((void **)&b.dd, nd * sizeof(BDesc), ls));
  B200_CK(cudaMallocAsync((void **)&b.dp, (nd + 1) * sizeof(uint32_t), ls));
  const uint32_t ntiles = b.hp[nd];
  std::vector<uint2> map(ntiles ? ntiles : 1);
  for (size_t i = 0; i < nd; i++)
    for (uint32_t t = b.hp[i]; t < b.hp[i + 1]; t++) map[t] = make_uint2((unsigned)i, t - b.hp[i]);
  B200_CK(cudaMallocAsync((void **)&b.dmap, map.size() * sizeof(uint2), ls));
  B200_CK(cudaMemcpyAsync(b.dmap, map.data(), map.size() * sizeof(uint2), cudaMemcpyHostToDevice,
                          ls));
  B200_CK(cudaMallocAsync((void **)&b.dcount, b.groups.size() * sizeof(unsigned), ls));
  B200_CK(cudaMemcpyAsync(b.dd, b.hd.data(), nd * sizeof(BDesc), cudaMemcpyHostToDevice, ls));
  B200_CK(cudaMemcpyAsync(b.dp, b.hp.data(), (nd + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice,
                          ls));
  B200_CK(cudaStreamSynchronize(ls)); /* the plan is then usable on any stream */
  return B200SHM_OK;
}

/* The plan of d: the autotuner's choice for its shape class when one is
 * cached, else the measured heuristic. */
void choose_plan(BDesc &d) {
  const int order = order_of(d);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(shape_of(d));
    if (it != g_tune.end() && lanes_ok(d, it->second.first)) {
      d.G = it->second.first;
      d.TP = it->second.second;
      return;
    }
  }
  /* heuristic default: 2 lanes per column, tiles of 1024 packs.  Trees
   * over more than 8 members at 2 lanes ran the batching workload in
   * 2.62 ms, at 4 lanes 2.72 ms, at 8 lanes 3.09 ms (fewer, longer runs
   * of each member per warp load). */
  /* small teams: columns per lane rather than lanes per column (a
   * butterfly over <= 8 members: lanes of 2 leaves each) */
  int G = order == ORD_CHAIN ? (d.P <= 8 ? 1 : 2)
                             : (order == ORD_BUTTERFLY && d.P <= 8 ? (d.p2s > 2 ? d.p2s / 2 : 1) : 2);
  while (G > 1 && !lanes_ok(d, G)) G >>= 1;
  while (!lanes_ok(d, G) && G < 8) G <<= 1;
  d.G = G;
  d.TP = 1024;
}

/* One timing of the whole batch as planned in `base` (plan applied, then
 * uploaded as a run uploads it): the best of three runs on stream s, ms. */
float time_batch(Batch &b, const std::vector<BDesc> &base, cudaStream_t s) {
  release(b);
  b.hd = base;
  for (BDesc &d : b.hd) set_columns(d);
  if (upload(b) != B200SHM_OK || make_side(b) != B200SHM_OK) return 1e30f;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return 1e30f;
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return 1e30f;
  }
  float best = 1e30f;
  if (enqueue(b, s) == B200SHM_OK) {
    for (int r = 0; r < 3; r++) {
      cudaEventRecord(e0, s);
      enqueue(b, s);
      cudaEventRecord(e1, s);
      cudaEventSynchronize(e1);
      float ms = 0;
      if (cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess && ms < best) best = ms;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return best;
}

/* The autotuner, inside the batch as it runs.  Start from the current plan
 * (cached choices, else the heuristic); then, for the shape classes that
 * carry the most bytes and have no cached choice yet, one class at a time,
 * give every descriptor of the class each other (lanes per column, tile)
 * and time the WHOLE batch -- its groups overlapping on the side streams,
 * as a run does -- keeping a change only when the batch got more than 1 %
 * faster.  The choices go to the per-process cache, which later batches
 * start from.  (Timing a shape class alone, where launch overhead
 * dominates, chose plans that lost inside the mixed batch.)  Tuning runs
 * the batch, so its dests are written, with the values a run writes; a
 * batch with an in-place descriptor is not tuned.  Results do not depend
 * on the plan: every plan keeps the algorithm's combine order. */
void tune_batch(Batch &b, cudaStream_t s) {
  std::vector<BDesc> base = b.hd;
  std::map<Shape, std::pair<double, std::vector<size_t>>> cls;
  for (size_t i = 0; i < base.size(); i++) {
    const BDesc &d = base[i];
    auto &c = cls[shape_of(d)];
    c.first += 2.0 * d.P * (double)d.N * esize_of(d);
    c.second.push_back(i);
  }
  std::vector<std::pair<double, Shape>> order;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (auto &kv : cls)
      if (!g_tune.count(kv.first)) order.push_back({kv.second.first, kv.first});
  }
  std::sort(order.begin(), order.end(),
            [](const std::pair<double, Shape> &x, const std::pair<double, Shape> &y) {
              return x.first > y.first;
            });
  if (order.size() > kTuneClasses) order.resize(kTuneClasses);
  float best = time_batch(b, base, s);
  for (auto &oc : order) {
    const std::vector<size_t> &idx = cls[oc.second].second;
    int bestG = base[idx[0]].G, bestTP = base[idx[0]].TP;
    for (int g = 1; g <= 8; g <<= 1) {
      for (int tp : {256, 1024, 4096}) {
        if (g == bestG && tp == bestTP) continue;
        std::vector<BDesc> cand = base;
        bool ok = true;
        for (size_t i : idx) {
          if (!lanes_ok(cand[i], g)) {
            ok = false;
            break;
          }
          cand[i].G = g;
          cand[i].TP = tp;
        }
        if (!ok) continue;
        const float ms = time_batch(b, cand, s);
        if (ms < best * 0.99f) {
          best = ms;
          base = cand;
          bestG = g;
          bestTP = tp;
        }
      }
    }
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[oc.second] = {bestG, bestTP};
  }
  release(b);
  b.hd = base;
  for (BDesc &d : b.hd) set_columns(d);
}

/* The reductions of a batch run concurrently, so no descriptor's dest may
 * touch another descriptor's dest or source in any member (two descriptors
 * may read the same source; one descriptor may run in place).  Every member
 * row is an interval of the arena; one sort and one sweep find a conflict. */
int check_independent(const b200shm_reduce_desc *descs, uint64_t n) {
  struct Span {
    uint64_t lo, hi;
    uint32_t desc;
    bool dest;
  };
  std::vector<Span> v;
  for (uint64_t i = 0; i < n; i++) {
    const b200shm_reduce_desc &x = descs[i];
    /* a descriptor that fails validation is reported when it runs */
    if (x.dtype < 0 || x.dtype >= B200SHM_NDTYPE) continue;
    const uint64_t es = (uint64_t)kDtypeSize[x.dtype];
    if (x.nelems == 0 || x.nelems > st().slice / es) continue;
    const uint64_t bytes = x.nelems * es;
    for (int m = 0; m < x.pe_size; m++) {
      const uint64_t row = (uint64_t)(x.pe_start + m * x.pe_stride) * st().slice;
      Span sp{row + x.src_off, row + x.src_off + bytes, (uint32_t)i, x.dest_off == x.src_off};
      v.push_back(sp);
      if (x.dest_off != x.src_off) {
        Span dp{row + x.dest_off, row + x.dest_off + bytes, (uint32_t)i, true};
        v.push_back(dp);
      }
    }
  }
  std::sort(v.begin(), v.end(), [](const Span &a, const Span &b) { return a.lo < b.lo; });
  /* the two farthest-reaching earlier spans of distinct descriptors */
  struct Top {
    uint64_t hi[2] = {0, 0};
    uint32_t d[2] = {~0u, ~0u};
    void add(const Span &s) {
      if (s.desc == d[0]) {
        if (s.hi > hi[0]) hi[0] = s.hi;
      } else if (s.hi > hi[0]) {
        hi[1] = hi[0];
        d[1] = d[0];
        hi[0] = s.hi;
        d[0] = s.desc;
      } else if (s.hi > hi[1]) {
        hi[1] = s.hi;
        d[1] = s.desc;
      }
    }
    /* an earlier span of another descriptor that reaches past s.lo */
    bool hits(const Span &s, uint32_t *other) const {
      for (int k = 0; k < 2; k++)
        if (d[k] != ~0u && d[k] != s.desc && hi[k] > s.lo) {
          *other = d[k];
          return true;
        }
      return false;
    }
  } any, dst;
  for (const Span &s : v) {
    uint32_t other = 0;
    if ((s.dest && any.hits(s, &other)) || dst.hits(s, &other))
      return fail(B200SHM_ERR_ARG,
                  "batch descriptors %u and %u overlap (one writes what the other reads or "
                  "writes, and the reductions of a batch run concurrently)",
                  std::min(other, s.desc), std::max(other, s.desc));
    any.add(s);
    if (s.dest) dst.add(s);
  }
  return B200SHM_OK;
}

}  // namespace
}  // namespace b200

using namespace b200;

struct b200shm_batch {
  Batch b;
};

extern "C" {

int b200shm_batch_create(b200shm_reduce_desc *descs, uint64_t n, int flags,
                         b200shm_batch **out) {
  if (!st().up) return fail(B200SHM_ERR_STATE, "b200shm is not initialised");
  if (!out || (n && !descs)) return fail(B200SHM_ERR_ARG, "batch_create: null argument");
  if (n >= (1ull << 24)) return fail(B200SHM_ERR_ARG, "batch_create: more than 2^24 reductions");
  *out = nullptr;
  b200shm_batch *bh = new b200shm_batch();
  Batch &b = bh->b;
  auto bail = [&](int rc) {
    release(b);
    delete bh;
    return rc;
  };
  bool tune = !(flags & B200SHM_BATCH_NO_TUNE);
  for (uint64_t i = 0; i < n; i++) {
    b200shm_reduce_desc &x = descs[i];
    if (x.algo == B200SHM_ALGO_AUTO) x.algo = B200SHM_REC_DBL;
    x.lanes = 0;
    x.tile = 0;
    /* the same validation as b200shm_reduce, without launching */
    int rc = check_team(x.pe_start, x.pe_stride, x.pe_size);
    if (rc)
      return bail(fail(rc, "batch descriptor %llu: %s", (unsigned long long)i,
                       b200shm_last_error()));
    const int ds = dslot_of(x.dtype);
    const bool is_int = x.dtype <= B200SHM_U64;
    const bool mm = x.op == B200SHM_MIN || x.op == B200SHM_MAX;
    int order = ORD_CHAIN;
    if (!is_int && !mm) {
      order = x.algo == B200SHM_LINEAR     ? ORD_CHAIN
              : x.algo == B200SHM_BINOMIAL ? ORD_BINOMIAL
                                           : ORD_BUTTERFLY;
    }
    const bool fusable = ds >= 0 && x.op >= 0 && x.op < B200SHM_NOP && x.algo >= 0 &&
                         x.algo < B200SHM_NALGO && (is_int || x.op >= B200SHM_MIN) &&
                         x.nelems > 0 && x.pe_size <= kFixMaxMembers;
    if (!fusable) {
      b.fallback.push_back(x); /* validated when it runs, by b200shm_reduce's path */
      continue;
    }
    const uint64_t es = (uint64_t)kDtypeSize[x.dtype];
    if (x.nelems > st().slice / es)
      return bail(fail(B200SHM_ERR_ARG, "batch descriptor %llu: nelems too large",
                       (unsigned long long)i));
    const uint64_t bytes = x.nelems * es;
    if ((rc = check_extent(x.src_off, bytes, "batch source")) ||
        (rc = check_extent(x.dest_off, bytes, "batch dest")))
      return bail(rc);
    if (x.dest_off != x.src_off && overlaps(x.dest_off, bytes, x.src_off, bytes))
      return bail(fail(B200SHM_ERR_ARG, "batch descriptor %llu: dest and source overlap",
                       (unsigned long long)i));
    Members m = members(x.pe_start, x.pe_stride, x.pe_size);
    BDesc d;
    d.src = m.first + x.src_off;
    d.dst = m.first + x.dest_off;
    d.step = m.step;
    d.N = x.nelems;
    d.P = x.pe_size;
    int p2s = 1, lg = 0;
    while (p2s * 2 <= d.P) {
      p2s *= 2;
      lg++;
    }
    d.p2s = p2s;
    d.logp2s = lg;
    d.algo = x.algo;
    d.kid = kid_of(ds, x.op, order);
    d.vec = ((x.src_off | x.dest_off | m.step) & 15u) == 0;
    d.npacks = d.vec ? x.nelems / (16 / es) : 0;
    d.G = 1;
    d.TP = 1024;
    d.U = 1;
    d.id = (int)i;
    if (!lanes_ok(d, 1) && !lanes_ok(d, 2) && !lanes_ok(d, 4) && !lanes_ok(d, 8)) {
      b.fallback.push_back(x); /* trees deeper than one lane's stack */
      continue;
    }
    if (x.dest_off == x.src_off) tune = false; /* tuning runs the batch: not in place */
    choose_plan(d);
    set_columns(d);
    x.lanes = d.G;
    x.tile = d.TP;
    if (!is_int && mm) b.any_mm = true;
    b.hd.push_back(d);
  }
  int rc = check_independent(descs, n);
  if (!rc && tune && !b.hd.empty()) {
    tune_batch(b, st().stream);
    for (const BDesc &d : b.hd) { /* report the tuned plan */
      descs[d.id].lanes = d.G;
      descs[d.id].tile = d.TP;
    }
  }
  if (!rc) rc = upload(b);
  if (!rc) rc = make_side(b);
  if (!rc && cudaEventCreateWithFlags(&b.done, cudaEventDisableTiming) != cudaSuccess)
    rc = fail(B200SHM_ERR_CUDA, "batch_create: event");
  if (rc) return bail(rc);
  if (flags & B200SHM_BATCH_GRAPH) {
    cudaStream_t cs;
    cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e != cudaSuccess) return bail(cuda_fail(e, "batch graph stream"));
    const unsigned long long l0 = b200shm_launch_count();
    e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      rc = enqueue(b, cs);
      const cudaError_t e2 = cudaStreamEndCapture(cs, &b.graph);
      if (e == cudaSuccess) e = e2;
    }
    b.graph_launches = (unsigned)(b200shm_launch_count() - l0);
    uncount_launches(b.graph_launches);
    if (e == cudaSuccess && rc == B200SHM_OK) e = cudaGraphInstantiate(&b.exec, b.graph, 0);
    cudaStreamDestroy(cs);
    if (e != cudaSuccess || rc) {
      if (b.graph) cudaGraphDestroy(b.graph);
      return bail(rc ? rc : cuda_fail(e, "batch graph capture"));
    }
  }
  *out = bh;
  return B200SHM_OK;
}

int b200shm_batch_run(b200shm_batch *bh, void *stream) {
  if (!bh) return fail(B200SHM_ERR_ARG, "batch_run: null batch");
  cudaStream_t s = pick_stream(stream);
  if (bh->b.exec) {
    B200_CK(cudaGraphLaunch(bh->b.exec, s));
    count_launch(bh->b.graph_launches);
  } else {
    int rc = enqueue(bh->b, s);
    if (rc) return rc;
  }
  B200_CK(cudaEventRecord(bh->b.done, s));
  return finish(stream, "b200shm_batch_run");
}

int b200shm_batch_destroy(b200shm_batch *bh) {
  if (!bh) return B200SHM_OK;
  if (bh->b.done) cudaEventSynchronize(bh->b.done); /* the last run, wherever it ran */
  if (bh->b.exec) cudaGraphExecDestroy(bh->b.exec);
  if (bh->b.graph) cudaGraphDestroy(bh->b.graph);
  release(bh->b);
  delete bh;
  return B200SHM_OK;
}

int b200shm_reduce_batch(b200shm_reduce_desc *descs, uint64_t n, void *stream) {
  b200shm_batch *b = nullptr;
  /* one run: tuning would cost more than it could save */
  int rc = b200shm_batch_create(descs, n, B200SHM_BATCH_NO_TUNE, &b);
  if (rc) return rc;
  rc = b200shm_batch_run(b, stream);
  if (stream) cudaStreamSynchronize((cudaStream_t)stream);
  b200shm_batch_destroy(b);
  return rc;
}

}  // extern "C"

/* ---- seeded device fill for the inputs of tests and benchmarks ------------ */
namespace b200 {
namespace {
__device__ __forceinline__ uint64_t mix64(uint64_t z) { /* splitmix64 finaliser */
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

template <class T>
__global__ void __launch_bounds__(256) k_fill(char *first, uint64_t step, int first_pe, int ps,
                                              int count, uint64_t n, uint64_t seed, double lo,
                                              double hi) {
  const uint64_t total = (uint64_t)count * n;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < total;
       k += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t m = k / n, i = k - m * n;
    const uint64_t pe = (uint64_t)first_pe + m * (uint64_t)ps;
    const uint64_t z = mix64(seed ^ mix64((pe << 40) ^ i));
    T v;
    if constexpr (std::is_floating_point<T>::value) {
      const double u = (double)(z >> 11) * (1.0 / 9007199254740992.0); /* [0, 1) */
      v = (T)(lo + (hi - lo) * u);
      if (v >= (T)hi || v < (T)lo) v = (T)lo; /* rounding to T may leave [lo, hi) */
    } else {
      const int64_t a = (int64_t)lo, b = (int64_t)hi;
      const uint64_t span = (uint64_t)(b - a) + 1;
      v = (T)(a + (int64_t)(span ? z % span : z));
    }
    memcpy(first + m * step + i * sizeof(T), &v, sizeof(T));
  }
}
}  // namespace
}  // namespace b200

extern "C" int b200shm_fill_uniform(int pe_start, int pe_stride, int pe_count, uint64_t off,
                                    int dtype, uint64_t nelems, uint64_t seed, double lo,
                                    double hi, void *stream) {
  using namespace b200;
  if (!st().up) return fail(B200SHM_ERR_STATE, "b200shm is not initialised");
  int rc = check_team(pe_start, pe_stride, pe_count);
  if (rc) return rc;
  if (dtype < 0 || dtype >= B200SHM_NDTYPE || dtype == B200SHM_F80 || dtype >= B200SHM_C32)
    return fail(B200SHM_ERR_UNSUPPORTED, "fill_uniform: dtype %d", dtype);
  if (!(lo <= hi)) return fail(B200SHM_ERR_ARG, "fill_uniform: lo > hi");
  if (nelems > st().slice / (uint64_t)kDtypeSize[dtype])
    return fail(B200SHM_ERR_ARG, "fill_uniform: nelems too large");
  if ((rc = check_extent(off, nelems * (uint64_t)kDtypeSize[dtype], "fill_uniform"))) return rc;
  if (nelems == 0) return B200SHM_OK;
  Members m = members(pe_start, pe_stride, pe_count);
  cudaStream_t s = pick_stream(stream);
  const unsigned grid = grid_for((uint64_t)pe_count * nelems, 256, 8);
  char *first = m.first + off;
  const int ps = pe_count > 1 ? pe_stride : 1;
#define B200_FILL(T)                                                                        \
  k_fill<T><<<grid, 256, 0, s>>>(first, m.step, pe_start, ps, pe_count, nelems, seed, lo, hi)
  switch (dtype) {
  case B200SHM_I8: B200_FILL(int8_t); break;
  case B200SHM_I16: B200_FILL(int16_t); break;
  case B200SHM_I32: B200_FILL(int32_t); break;
  case B200SHM_I64: B200_FILL(int64_t); break;
  case B200SHM_U8: B200_FILL(uint8_t); break;
  case B200SHM_U16: B200_FILL(uint16_t); break;
  case B200SHM_U32: B200_FILL(uint32_t); break;
  case B200SHM_U64: B200_FILL(uint64_t); break;
  case B200SHM_F32: B200_FILL(float); break;
  default: B200_FILL(double); break;
  }
#undef B200_FILL
  count_launch();
  return finish(stream, "b200shm_fill_uniform");
}
