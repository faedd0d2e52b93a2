/*
 * f80.cuh -- x87 80-bit extended arithmetic in software, for the long
 * double reductions (host and device).
 *
 * The reference computes shmem_longdouble_<op>_reduce with the C operators
 * of reduce.c:730-736 on long double, which gcc on x86-64 evaluates on the
 * x87 unit: 64-bit significand with an explicit integer bit, 15-bit
 * exponent, round to nearest even (the Linux control word), every
 * exception masked.  These functions give the same bits:
 *  - finite results are the exact result rounded once to nearest even on
 *    the extended grid, with gradual underflow (a tiny result is rounded on
 *    the denormal grid) and overflow to infinity;
 *  - an operand the x87 does not support (an unnormal, a pseudo-NaN or a
 *    pseudo-infinity) and the invalid operations (inf - inf, 0 * inf) give
 *    the QNaN "indefinite" (sign 1, significand 0xC000000000000000);
 *  - NaN operands propagate as the x87 does: a NaN with a non-NaN gives
 *    that NaN; two NaNs give the QNaN if only one is quiet, else the one
 *    with the larger significand (the positive one on a tie); the result is
 *    always quiet;
 *  - pseudo-denormals (exponent 0, integer bit set) are valid operands with
 *    the value of their significand on the denormal grid;
 *  - comparisons (<, >) are false when either operand is a NaN or
 *    unsupported, as x87 compare-and-branch code reads them.
 * The storage is the x86-64 long double layout: 16 bytes, significand in
 * bytes 0-7, sign and exponent in bytes 8-9, six bytes of padding.
 */
#ifndef B200SHM_F80_CUH
#define B200SHM_F80_CUH

#include <stdint.h>

#ifdef __CUDACC__
#define B200_F80_FN __host__ __device__ __forceinline__
#else
#define B200_F80_FN static inline
#endif

namespace b200 {

struct alignas(16) f80 {
  uint64_t sig;
  uint16_t se;      /* sign (bit 15) and biased exponent */
  uint16_t pad[3];
};

typedef unsigned __int128 f80_u128;

constexpr int kF80Bias = 16383;
constexpr uint16_t kF80ExpMax = 0x7FFF;
constexpr uint64_t kF80J = 1ull << 63;    /* the explicit integer bit */
constexpr uint64_t kF80Quiet = 1ull << 62;

B200_F80_FN f80 f80_make(uint16_t se, uint64_t sig) {
  f80 r;
  r.sig = sig;
  r.se = se;
  r.pad[0] = r.pad[1] = r.pad[2] = 0;
  return r;
}
B200_F80_FN f80 f80_indefinite() { return f80_make(0xFFFF, 0xC000000000000000ull); }

B200_F80_FN int f80_clz64(uint64_t x) {
#ifdef __CUDA_ARCH__
  return __clzll((long long)x);
#else
  return x ? __builtin_clzll(x) : 64;
#endif
}

/* classes */
B200_F80_FN bool f80_is_nan(const f80 &a) {
  return (a.se & kF80ExpMax) == kF80ExpMax && (a.sig & kF80J) && (a.sig << 1) != 0;
}
B200_F80_FN bool f80_is_inf(const f80 &a) {
  return (a.se & kF80ExpMax) == kF80ExpMax && a.sig == kF80J;
}
/* encodings the x87 rejects as operands: unnormals, pseudo-NaNs and
 * pseudo-infinities (integer bit clear with a non-zero exponent) */
B200_F80_FN bool f80_is_unsupported(const f80 &a) {
  const unsigned e = a.se & kF80ExpMax;
  return e != 0 && !(a.sig & kF80J);
}
B200_F80_FN bool f80_is_zero(const f80 &a) { return (a.se & kF80ExpMax) == 0 && a.sig == 0; }
B200_F80_FN bool f80_is_pseudo_denormal(const f80 &a) {
  return (a.se & kF80ExpMax) == 0 && (a.sig & kF80J);
}

/* A finite non-zero operand as m * 2^(e - bias - 63) with m's top bit set
 * (e may drop below 1 for a denormal). */
B200_F80_FN void f80_unpack(const f80 &a, uint64_t &m, int &e) {
  const int ef = a.se & kF80ExpMax;
  m = a.sig;
  e = ef ? ef : 1;
  const int s = f80_clz64(m);
  m <<= s;
  e -= s;
}

/* Round the non-zero value M * 2^(e - bias - 125) once to nearest even on
 * the extended grid and encode it. */
B200_F80_FN f80 f80_round_pack(unsigned sign, int e, f80_u128 M) {
  if (M == 0) return f80_make((uint16_t)(sign << 15), 0); /* not reached by the callers */
  /* the most significant bit of M to bit 125 */
  const uint64_t hi = (uint64_t)(M >> 64), lo = (uint64_t)M;
  const int msb = hi ? 127 - f80_clz64(hi) : 63 - f80_clz64(lo);
  if (msb > 125) {
    const int sh = msb - 125;
    const bool sticky = (M & ((((f80_u128)1) << sh) - 1)) != 0;
    M = (M >> sh) | (f80_u128)(sticky ? 1 : 0);
    e += sh;
  } else if (msb < 125) {
    M <<= (125 - msb);
    e -= 125 - msb;
  }
  if (e < 1) { /* below the normal range: onto the denormal grid */
    const int sh = 1 - e;
    if (sh > 126) {
      M = 1; /* only a sticky bit is left: rounds to zero */
    } else {
      const bool sticky = (M & ((((f80_u128)1) << sh) - 1)) != 0;
      M = (M >> sh) | (f80_u128)(sticky ? 1 : 0);
    }
    e = 1;
  }
  /* keep bits 125..62, round at bit 61, sticky below */
  uint64_t keep = (uint64_t)(M >> 62);
  const uint64_t rem = (uint64_t)M & ((1ull << 62) - 1);
  const uint64_t half = 1ull << 61;
  if (rem > half || (rem == half && (keep & 1))) {
    keep++;
    if (keep == 0) { /* carried out of 64 bits */
      keep = kF80J;
      e++;
    }
  }
  const uint16_t s = (uint16_t)(sign << 15);
  if (e >= (int)kF80ExpMax) return f80_make(s | kF80ExpMax, kF80J); /* overflow */
  if (keep == 0) return f80_make(s, 0);
  return f80_make(s | (uint16_t)((keep & kF80J) ? e : 0), keep);
}

/* The NaN an operation with at least one NaN operand (and no unsupported
 * one) returns, quiet. */
B200_F80_FN f80 f80_nan_result(const f80 &a, const f80 &b) {
  const bool na = f80_is_nan(a), nb = f80_is_nan(b);
  f80 r;
  if (na && nb) {
    const bool qa = (a.sig & kF80Quiet) != 0, qb = (b.sig & kF80Quiet) != 0;
    if (qa != qb) r = qa ? a : b;
    else if (a.sig != b.sig) r = a.sig > b.sig ? a : b;
    else r = (a.se & 0x8000) ? b : a;
  } else {
    r = na ? a : b;
  }
  return f80_make(r.se, r.sig | kF80Quiet);
}

B200_F80_FN f80 f80_add(const f80 &a, const f80 &b) {
  if (f80_is_unsupported(a) || f80_is_unsupported(b)) return f80_indefinite();
  if (f80_is_nan(a) || f80_is_nan(b)) return f80_nan_result(a, b);
  const unsigned sa = a.se >> 15, sb = b.se >> 15;
  const bool ia = f80_is_inf(a), ib = f80_is_inf(b);
  if (ia || ib) {
    if (ia && ib && sa != sb) return f80_indefinite();
    return f80_make((uint16_t)((ia ? sa : sb) << 15) | kF80ExpMax, kF80J);
  }
  const bool za = f80_is_zero(a), zb = f80_is_zero(b);
  if (za && zb) return f80_make((uint16_t)((sa & sb) << 15), 0);
  uint64_t ma = 0, mb = 0;
  int ea = 0, eb = 0;
  if (!za) f80_unpack(a, ma, ea);
  if (!zb) f80_unpack(b, mb, eb);
  if (za) return f80_round_pack(sb, eb, (f80_u128)mb << 62);
  if (zb) return f80_round_pack(sa, ea, (f80_u128)ma << 62);
  /* |x| >= |y| */
  const bool swap = eb > ea || (eb == ea && mb > ma);
  const uint64_t mx = swap ? mb : ma, my = swap ? ma : mb;
  const int ex = swap ? eb : ea, ey = swap ? ea : eb;
  const unsigned sx = swap ? sb : sa, sy = swap ? sa : sb;
  const f80_u128 X = (f80_u128)mx << 62;
  f80_u128 Y = (f80_u128)my << 62;
  const int d = ex - ey;
  if (d > 0) {
    if (d > 126) {
      Y = 1; /* sticky only */
    } else {
      const bool sticky = (Y & ((((f80_u128)1) << d) - 1)) != 0;
      Y = (Y >> d) | (f80_u128)(sticky ? 1 : 0);
    }
  }
  if (sx == sy) return f80_round_pack(sx, ex, X + Y);
  const f80_u128 D = X - Y;
  if (D == 0) return f80_make(0, 0); /* exact cancellation: +0 */
  return f80_round_pack(sx, ex, D);
}

B200_F80_FN f80 f80_mul(const f80 &a, const f80 &b) {
  if (f80_is_unsupported(a) || f80_is_unsupported(b)) return f80_indefinite();
  if (f80_is_nan(a) || f80_is_nan(b)) return f80_nan_result(a, b);
  const unsigned s = (a.se >> 15) ^ (b.se >> 15);
  const bool ia = f80_is_inf(a), ib = f80_is_inf(b);
  const bool za = f80_is_zero(a), zb = f80_is_zero(b);
  if (ia || ib) {
    if (za || zb) return f80_indefinite();
    return f80_make((uint16_t)(s << 15) | kF80ExpMax, kF80J);
  }
  if (za || zb) return f80_make((uint16_t)(s << 15), 0);
  uint64_t ma, mb;
  int ea, eb;
  f80_unpack(a, ma, ea);
  f80_unpack(b, mb, eb);
  /* ma*mb * 2^(ea+eb-2*bias-126) = M * 2^(e-bias-125) with e = ea+eb-bias-1 */
  return f80_round_pack(s, ea + eb - kF80Bias - 1, (f80_u128)ma * (f80_u128)mb);
}

/* a < b as x87 compare code reads it: false when unordered */
B200_F80_FN bool f80_lt(const f80 &a, const f80 &b) {
  if (f80_is_unsupported(a) || f80_is_unsupported(b) || f80_is_nan(a) || f80_is_nan(b))
    return false;
  const bool za = f80_is_zero(a), zb = f80_is_zero(b);
  if (za && zb) return false;
  const unsigned sa = a.se >> 15, sb = b.se >> 15;
  if (f80_is_inf(a) || f80_is_inf(b)) {
    if (f80_is_inf(a) && f80_is_inf(b)) return sa && !sb;
    if (f80_is_inf(a)) return sa;  /* -inf < anything finite */
    return !sb;                    /* finite < +inf */
  }
  if (za) return !sb;  /* 0 < positive */
  if (zb) return sa;   /* negative < 0 */
  if (sa != sb) return sa;
  uint64_t ma, mb;
  int ea, eb;
  f80_unpack(a, ma, ea);
  f80_unpack(b, mb, eb);
  const bool mag_lt = ea < eb || (ea == eb && ma < mb);
  const bool mag_gt = ea > eb || (ea == eb && ma > mb);
  return sa ? mag_gt : mag_lt;
}
B200_F80_FN bool f80_gt(const f80 &a, const f80 &b) { return f80_lt(b, a); }

}  // namespace b200
#endif
