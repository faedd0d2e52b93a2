/*
 * reduce_core.cuh -- the element operators, 16-byte packs and exact-order
 * helpers shared by the per-call reduce kernels (reduce_kernels.cuh) and the
 * batched reduce kernels (batch.cu).  The combine operators follow
 * src/shcoll/src/reduce.c:730-736; the tree-order helpers follow the
 * rec_dbl / Rabenseifner extra-PE fold (reduce.c:206-272, 338-454).
 */
#pragma once
#include <stdint.h>
#include <string.h>

#include <type_traits>

#include "f80.cuh"
#include "internal.cuh"

namespace b200 {
namespace {
struct cf32 {
  float re, im;
};
struct cf64 {
  double re, im;
};

enum { ORD_CHAIN = 0, ORD_BINOMIAL = 1, ORD_BUTTERFLY = 2 };

/* ---- element operators (reduce.c:730-736) ------------------------------ */
template <int OP, class T>
__device__ __forceinline__ T op_int(T a, T b) {
  typedef typename std::make_unsigned<T>::type U;
  if constexpr (OP == B200SHM_AND) return (T)(a & b);
  else if constexpr (OP == B200SHM_OR) return (T)(a | b);
  else if constexpr (OP == B200SHM_XOR) return (T)(a ^ b);
  else if constexpr (OP == B200SHM_MIN) return a < b ? a : b;
  else if constexpr (OP == B200SHM_MAX) return a > b ? a : b;
  else if constexpr (OP == B200SHM_SUM) return (T)(U)((uint64_t)(U)a + (uint64_t)(U)b);
  else return (T)(U)((uint64_t)(U)a * (uint64_t)(U)b);
}

__device__ __forceinline__ float f_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float f_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float f_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double f_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double f_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double f_sub(double a, double b) { return __dsub_rn(a, b); }

template <int OP, class F>
__device__ __forceinline__ F op_flt(F a, F b) {
  if constexpr (OP == B200SHM_MIN) return a < b ? a : b;
  else if constexpr (OP == B200SHM_MAX) return a > b ? a : b;
  else if constexpr (OP == B200SHM_SUM) return f_add(a, b);
  else return f_mul(a, b);
}

/* Complex product as C99 evaluates x*y: the naive formula, and only when
 * both parts come out NaN, the infinity recovery of ISO C Annex G.5.1
 * (what the reference's gcc build reaches through __muldc3/__mulsc3). */
template <class F>
__device__ __forceinline__ F cpy_sign(F mag, F sgn) { return copysign(mag, sgn); }
template <class F>
__device__ void cmul(F a, F b, F c, F d, F &re, F &im) {
  F ac = f_mul(a, c), bd = f_mul(b, d), ad = f_mul(a, d), bc = f_mul(b, c);
  re = f_sub(ac, bd);
  im = f_add(ad, bc);
  if (isnan(re) && isnan(im)) {
    bool recalc = false;
    if (isinf(a) || isinf(b)) {
      a = cpy_sign((F)(isinf(a) ? 1 : 0), a);
      b = cpy_sign((F)(isinf(b) ? 1 : 0), b);
      if (isnan(c)) c = cpy_sign((F)0, c);
      if (isnan(d)) d = cpy_sign((F)0, d);
      recalc = true;
    }
    if (isinf(c) || isinf(d)) {
      c = cpy_sign((F)(isinf(c) ? 1 : 0), c);
      d = cpy_sign((F)(isinf(d) ? 1 : 0), d);
      if (isnan(a)) a = cpy_sign((F)0, a);
      if (isnan(b)) b = cpy_sign((F)0, b);
      recalc = true;
    }
    if (!recalc && (isinf(ac) || isinf(bd) || isinf(ad) || isinf(bc))) {
      if (isnan(a)) a = cpy_sign((F)0, a);
      if (isnan(b)) b = cpy_sign((F)0, b);
      if (isnan(c)) c = cpy_sign((F)0, c);
      if (isnan(d)) d = cpy_sign((F)0, d);
      recalc = true;
    }
    if (recalc) {
      const F inf = (F)INFINITY;
      re = f_mul(inf, f_sub(f_mul(a, c), f_mul(b, d)));
      im = f_mul(inf, f_add(f_mul(a, d), f_mul(b, c)));
    }
  }
}

template <int OP, class T>
__device__ __forceinline__ T apply(T a, T b) {
  if constexpr (std::is_same<T, float>::value || std::is_same<T, double>::value) {
    return op_flt<OP>(a, b);
  } else if constexpr (std::is_same<T, f80>::value) {
    /* x87 long double, as reduce.c:730-736 evaluate it on the host */
    if constexpr (OP == B200SHM_MIN) return f80_lt(a, b) ? a : b;
    else if constexpr (OP == B200SHM_MAX) return f80_gt(a, b) ? a : b;
    else if constexpr (OP == B200SHM_SUM) return f80_add(a, b);
    else return f80_mul(a, b);
  } else if constexpr (std::is_same<T, cf32>::value || std::is_same<T, cf64>::value) {
    T r;
    if constexpr (OP == B200SHM_SUM) {
      r.re = f_add(a.re, b.re);
      r.im = f_add(a.im, b.im);
    } else {
      cmul(a.re, a.im, b.re, b.im, r.re, r.im);
    }
    return r;
  } else {
    return op_int<OP>(a, b);
  }
}

/* ---- packs: V consecutive elements moved as one 16-byte access -------- */
template <class T, int V>
struct alignas(V * sizeof(T) >= 16 ? 16 : alignof(T)) Pack {
  T x[V];
};

/* Cache policy of the pack accesses: every source and dest byte of a
 * reduction is touched once, so loads and stores are streaming (.cs:
 * evict-first in L1 and L2), which keeps fewer of a launch's dirty dest
 * lines in L2 for the next launch to write back.  On the 64-member x 2^20
 * headline step (six back-to-back reductions) streaming stores took the
 * step from 5928 to 6028 GB/s and streaming loads added ~0.1 %. */
#ifndef B200_LD_OP
#define B200_LD_OP "ld.global.cs.nc"
#endif
#ifndef B200_ST_OP
#define B200_ST_OP "st.global.cs"
#endif
/* One 16-byte element (complex double, long double) at any alignment: one
 * 16-byte access where the address allows it, else 8-, 4- or 1-byte
 * pieces.  A complex double array needs only 8-byte alignment, and the
 * C ABI takes byte offsets, so a single element may sit anywhere; the
 * branch is uniform across a warp whenever the member rows share their
 * alignment. */
__device__ __forceinline__ void ld16_any(const char *p, uint32_t w[4]) {
  const uintptr_t a = (uintptr_t)p;
  if ((a & 15) == 0) {
    asm(B200_LD_OP ".v4.u32 {%0,%1,%2,%3}, [%4];"
        : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3])
        : "l"(p));
  } else if ((a & 7) == 0) {
    asm(B200_LD_OP ".v2.u32 {%0,%1}, [%2];" : "=r"(w[0]), "=r"(w[1]) : "l"(p));
    asm(B200_LD_OP ".v2.u32 {%0,%1}, [%2];" : "=r"(w[2]), "=r"(w[3]) : "l"(p + 8));
  } else if ((a & 3) == 0) {
#pragma unroll
    for (int i = 0; i < 4; i++) asm(B200_LD_OP ".u32 %0, [%1];" : "=r"(w[i]) : "l"(p + 4 * i));
  } else {
    unsigned char b[16];
#pragma unroll
    for (int i = 0; i < 16; i++) b[i] = (unsigned char)p[i];
    memcpy(w, b, 16);
  }
}
__device__ __forceinline__ void st16_any(char *p, const uint32_t w[4]) {
  const uintptr_t a = (uintptr_t)p;
  if ((a & 15) == 0) {
    asm volatile(B200_ST_OP ".v4.u32 [%0], {%1,%2,%3,%4};" ::"l"(p), "r"(w[0]), "r"(w[1]),
                 "r"(w[2]), "r"(w[3])
                 : "memory");
  } else if ((a & 7) == 0) {
    asm volatile(B200_ST_OP ".v2.u32 [%0], {%1,%2};" ::"l"(p), "r"(w[0]), "r"(w[1]) : "memory");
    asm volatile(B200_ST_OP ".v2.u32 [%0], {%1,%2};" ::"l"(p + 8), "r"(w[2]), "r"(w[3])
                 : "memory");
  } else if ((a & 3) == 0) {
#pragma unroll
    for (int i = 0; i < 4; i++)
      asm volatile(B200_ST_OP ".u32 [%0], %1;" ::"l"(p + 4 * i), "r"(w[i]) : "memory");
  } else {
    unsigned char b[16];
    memcpy(b, w, 16);
#pragma unroll
    for (int i = 0; i < 16; i++) p[i] = (char)b[i];
  }
}

/* 16-byte packs move with one vector access whose registers have the
 * element's own class (f64 pairs, u64, f32, u32), so no moves are needed
 * between the load and the arithmetic.  Packs of several elements are
 * used only on 16-byte-aligned rows; a pack of one 16-byte element may be
 * at any alignment. */
template <class T, int V>
__device__ __forceinline__ Pack<T, V> ld_pack(const char *p) {
  Pack<T, V> r;
  if constexpr (sizeof(Pack<T, V>) == 16 && V == 1) {
    uint32_t w[4];
    ld16_any(p, w);
    memcpy(&r, w, 16);
  } else if constexpr (sizeof(Pack<T, V>) == 16 && std::is_same<T, double>::value) {
    asm(B200_LD_OP ".v2.f64 {%0,%1}, [%2];"
        : "=d"(r.x[0]), "=d"(r.x[1])
        : "l"(p));
  } else if constexpr (sizeof(Pack<T, V>) == 16 && std::is_integral<T>::value &&
                       sizeof(T) == 8) {
    unsigned long long a, b;
    asm(B200_LD_OP ".v2.u64 {%0,%1}, [%2];" : "=l"(a), "=l"(b) : "l"(p));
    r.x[0] = (T)a;
    r.x[1] = (T)b;
  } else if constexpr (sizeof(Pack<T, V>) == 16 && std::is_same<T, float>::value) {
    asm(B200_LD_OP ".v4.f32 {%0,%1,%2,%3}, [%4];"
        : "=f"(r.x[0]), "=f"(r.x[1]), "=f"(r.x[2]), "=f"(r.x[3])
        : "l"(p));
  } else if constexpr (sizeof(Pack<T, V>) == 16) {
    uint4 u;
    asm(B200_LD_OP ".v4.u32 {%0,%1,%2,%3}, [%4];"
        : "=r"(u.x), "=r"(u.y), "=r"(u.z), "=r"(u.w)
        : "l"(p));
    memcpy(&r, &u, 16);
  } else {
    memcpy(&r, p, sizeof(r));
  }
  return r;
}
template <class T, int V>
__device__ __forceinline__ void st_pack(char *p, const Pack<T, V> &v) {
  if constexpr (sizeof(Pack<T, V>) == 16 && V == 1) {
    uint32_t w[4];
    memcpy(w, &v, 16);
    st16_any(p, w);
  } else if constexpr (sizeof(Pack<T, V>) == 16 && std::is_same<T, double>::value) {
    asm volatile(B200_ST_OP ".v2.f64 [%0], {%1,%2};" ::"l"(p), "d"(v.x[0]), "d"(v.x[1])
                 : "memory");
  } else if constexpr (sizeof(Pack<T, V>) == 16 && std::is_integral<T>::value &&
                       sizeof(T) == 8) {
    asm volatile(B200_ST_OP ".v2.u64 [%0], {%1,%2};" ::"l"(p),
                 "l"((unsigned long long)v.x[0]), "l"((unsigned long long)v.x[1])
                 : "memory");
  } else if constexpr (sizeof(Pack<T, V>) == 16 && std::is_same<T, float>::value) {
    asm volatile(B200_ST_OP ".v4.f32 [%0], {%1,%2,%3,%4};" ::"l"(p), "f"(v.x[0]), "f"(v.x[1]),
                 "f"(v.x[2]), "f"(v.x[3])
                 : "memory");
  } else if constexpr (sizeof(Pack<T, V>) == 16) {
    uint4 u;
    memcpy(&u, &v, 16);
    asm volatile(B200_ST_OP ".v4.u32 [%0], {%1,%2,%3,%4};" ::"l"(p), "r"(u.x), "r"(u.y),
                 "r"(u.z), "r"(u.w)
                 : "memory");
  } else {
    memcpy(p, &v, sizeof(v));
  }
}
template <int OP, class T, int V>
__device__ __forceinline__ Pack<T, V> papply(const Pack<T, V> &a, const Pack<T, V> &b) {
  Pack<T, V> r;
#pragma unroll
  for (int i = 0; i < V; i++) r.x[i] = apply<OP>(a.x[i], b.x[i]);
  return r;
}

/* MIN/MAX on floats: flag bit 0 = NaN seen, bit 1 = +0 seen, bit 2 = -0. */
__device__ __forceinline__ unsigned fclass(float f) {
  const uint32_t u = __float_as_uint(f);
  return ((u & 0x7fffffffu) > 0x7f800000u ? 1u : 0u) | (u == 0u ? 2u : 0u) |
         (u == 0x80000000u ? 4u : 0u);
}
__device__ __forceinline__ unsigned fclass(double f) {
  const uint64_t u = (uint64_t)__double_as_longlong(f);
  return ((u & 0x7fffffffffffffffull) > 0x7ff0000000000000ull ? 1u : 0u) |
         (u == 0ull ? 2u : 0u) | (u == 0x8000000000000000ull ? 4u : 0u);
}
/* long double: bit 0 also for the operands whose comparisons are
 * unordered (unsupported encodings) and for pseudo-denormals, which compare
 * equal to the normal of the same value with other bits */
__device__ __forceinline__ unsigned fclass(const f80 &f) {
  if (f80_is_nan(f) || f80_is_unsupported(f) || f80_is_pseudo_denormal(f)) return 1u;
  if (f80_is_zero(f)) return (f.se & 0x8000) ? 4u : 2u;
  return 0u;
}
__device__ __forceinline__ bool ambiguous(unsigned f) { return (f & 1u) || (f & 6u) == 6u; }

}  // namespace

/* One reduction's launch arguments (outside the unnamed namespace: the
 * per-family launch sequences below take it across translation units). */
struct RArgs {
  const char *src;  /* member 0's source at element 0          */
  char *dst;        /* member 0's dest at element 0            */
  uint64_t sstep;   /* bytes from member i to member i+1 (src) */
  uint64_t dstep;   /* same for dest (equal; kept separate)    */
  uint64_t e_begin; /* first element of this launch            */
  uint64_t nvec;    /* packs in this launch                    */
  uint64_t N;       /* elements of this view                   */
  uint64_t g_off;   /* the view's element 0 in the whole reduction */
  uint64_t g_n;     /* elements of the whole reduction         */
  int P, p2s, logp2s, algo;
  unsigned long long *fix_list, *fix_count; /* deferred elements */
  unsigned long long *fix_done;  /* k_minmax_fix's exit counter (clears fix_count) */
  unsigned long long fix_cap;
  int *status;
};

/* The launch sequence of one validated reduction on stream s, one function
 * per element-type family, each in its own translation unit
 * (reduce_<family>.cu) so the families' kernels compile in parallel.
 * `aligned`: every row starts on a 16-byte boundary. */
int reduce_dispatch_int(int op, int dtype, const RArgs &a, bool aligned, cudaStream_t s);
int reduce_dispatch_f32(int op, const RArgs &a, bool aligned, cudaStream_t s);
int reduce_dispatch_f64(int op, const RArgs &a, bool aligned, cudaStream_t s);
/* long double: one function (and translation unit) per op */
int reduce_dispatch_f80_min(const RArgs &a, bool aligned, cudaStream_t s);
int reduce_dispatch_f80_max(const RArgs &a, bool aligned, cudaStream_t s);
int reduce_dispatch_f80_sum(const RArgs &a, bool aligned, cudaStream_t s);
int reduce_dispatch_f80_prod(const RArgs &a, bool aligned, cudaStream_t s);
int reduce_dispatch_c32(int op, const RArgs &a, bool aligned, cudaStream_t s);
int reduce_dispatch_c64(int op, const RArgs &a, bool aligned, cudaStream_t s);

namespace {

/* p2s membership, reduce.c:206-214 and 232 */
__device__ __forceinline__ int p2s_member(int q, int P, int p2s) {
  return (int)(((long long)q * P + p2s - 1) / p2s);
}
__device__ __forceinline__ bool p2s_extra(int q, int P, int p2s) {
  const int as = p2s_member(q, P, p2s);
  return (long long)(as + 1) * p2s / P == q;
}

constexpr int kMaxLevels = 13; /* trees of up to 4096 leaves */

/* ---- exact replay for order-dependent MIN/MAX elements ----------------- */
/* Value the algorithm leaves in p2s member q's dest (rec_dbl), or in every
 * member's dest (the other algorithms, q = block owner or 0), for one
 * element whose P inputs are vals[0..P). */
template <class T, int OP, class Get>
__device__ T exact_value(Get vals, int P, int p2s, int logp2s, int algo, bool lower_half, int q) {
  if (algo == B200SHM_LINEAR) {
    T acc = vals(0);
    for (int j = 1; j < P; j++) acc = apply<OP>(acc, vals(j));
    return acc;
  }
  T stk[kMaxLevels + 1];
  if (algo == B200SHM_BINOMIAL) {
    for (int j = 0; j < P; j++) {
      T x = vals(j);
      for (int L = 0; L <= kMaxLevels; L++) {
        if (j & (1 << L)) {
          x = apply<OP>(x, stk[L]); /* op(upper block, lower block) */
        } else {
          stk[L] = x;
          break;
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
  /* butterfly: rec_dbl / rabenseifner / rabenseifner2 */
  const bool rab = algo != B200SHM_REC_DBL;
  for (int leaf = 0; leaf < p2s; leaf++) {
    const int as = p2s_member(leaf, P, p2s);
    T x = vals(as);
    if (p2s_extra(leaf, P, p2s)) {
      const T ext = vals(as + 1);
      /* rec_dbl: op(extra, own) (reduce.c:241); Rabenseifner: op(extra,
       * own) on the lower half (397), op(own, extra) on the upper (375) */
      x = (!rab || lower_half) ? apply<OP>(ext, x) : apply<OP>(x, ext);
    }
    for (int L = 0; L <= kMaxLevels; L++) {
      if (leaf & (1 << L)) {
        /* member q computes op(own, partner's) (reduce.c:268, 448) */
        x = (q & (1 << L)) ? apply<OP>(x, stk[L]) : apply<OP>(stk[L], x);
      } else {
        stk[L] = x;
        break;
      }
    }
  }
  return stk[logp2s];
}

/* Block of element e in Rabenseifner's split: [b*N/p2s, (b+1)*N/p2s). */
__device__ int rab_block(uint64_t e, uint64_t N, int p2s) {
  int b = (int)((e * (uint64_t)p2s) / (N ? N : 1));
  if (b >= p2s) b = p2s - 1;
  while (b + 1 < p2s && (uint64_t)(b + 1) * N / (uint64_t)p2s <= e) b++;
  while (b > 0 && (uint64_t)b * N / (uint64_t)p2s > e) b--;
  return b;
}
__device__ __forceinline__ int rev_bits(int x, int n) {
  return n ? (int)(__brev((unsigned)x) >> (32 - n)) : 0;
}

constexpr int kFixMaxMembers = 4096;
/* members of a long double MIN/MAX team (the replay stages the P inputs of
 * 16 bytes each in shared memory) */
constexpr int kFixMaxMembersF80 = 2048;
template <class T>
constexpr int fix_max_members() {
  return sizeof(T) > 8 ? kFixMaxMembersF80 : kFixMaxMembers;
}

template <class T, int V>
__device__ __forceinline__ Pack<T, V> shfl_xor_pack(const Pack<T, V> &v, int m) {
  static_assert(sizeof(Pack<T, V>) % 4 == 0, "pack of 32-bit words");
  constexpr int W = (int)(sizeof(Pack<T, V>) / 4);
  uint32_t w[W];
  memcpy(w, &v, sizeof(w));
#pragma unroll
  for (int i = 0; i < W; i++) w[i] = __shfl_xor_sync(0xffffffffu, w[i], m);
  Pack<T, V> r;
  memcpy(&r, w, sizeof(w));
  return r;
}

}  // namespace
}  // namespace b200
