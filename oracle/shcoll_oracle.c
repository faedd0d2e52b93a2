/*
 * shcoll_oracle.c -- plain-C restatement of the reference's collective
 * results.  TEST INFRASTRUCTURE ONLY (checker for the parity tests and the
 * benchmark's CPU baseline); never linked into the product.
 *
 * Instead of emulating PEs and messages, each routine computes directly the
 * value every member ends up with, following the combine order of the
 * reference algorithm it names (BTMichalowicz/osss-ucx src/shcoll/src).
 * Build with -ffp-contract=off so that a*b+c is never fused, as in the
 * reference's own x86-64 build.
 */
#include "shcoll_oracle.h"

#include <complex.h>
#include <stdlib.h>
#include <string.h>

size_t or_dtype_size(int dtype) {
  static const size_t sz[OR_NDTYPE] = {1, 2, 4, 8, 1, 2, 4, 8,
                                       4, 8, sizeof(long double),
                                       sizeof(float _Complex),
                                       sizeof(double _Complex)};
  return (dtype >= 0 && dtype < OR_NDTYPE) ? sz[dtype] : 0;
}

/* util/bithacks.c:11-20: reverse the low nbits bits of number. */
int or_reverse_bits(int number, int nbits) {
  unsigned r = 0, a = (unsigned)number;
  for (int i = 0; i < nbits; i++) {
    r = (r << 1) | (a & 1u);
    a >>= 1;
  }
  return (int)r;
}

/* ------------------------------------------------------------------------ */
/* element operators, reduce.c:730-736.  Integer SUM/PROD wrap modulo 2^bits */
/* (what the reference's build does; done in unsigned arithmetic here so     */
/* the restatement itself has no undefined behaviour).                       */
/* ------------------------------------------------------------------------ */
#define INT_OPS(T, UT, WT)                                                     \
  static inline T op_##T(int op, T a, T b) {                                   \
    switch (op) {                                                              \
    case OR_AND: return (T)(a & b);                                            \
    case OR_OR: return (T)(a | b);                                             \
    case OR_XOR: return (T)(a ^ b);                                            \
    case OR_MIN: return a < b ? a : b;                                         \
    case OR_MAX: return a > b ? a : b;                                         \
    case OR_SUM: return (T)(UT)((WT)(UT)a + (WT)(UT)b);                        \
    default: return (T)(UT)((WT)(UT)a * (WT)(UT)b);                            \
    }                                                                          \
  }
#define FLT_OPS(T)                                                             \
  static inline T op_##T(int op, T a, T b) {                                   \
    switch (op) {                                                              \
    case OR_MIN: return a < b ? a : b;                                         \
    case OR_MAX: return a > b ? a : b;                                         \
    case OR_SUM: return a + b;                                                 \
    default: return a * b;                                                     \
    }                                                                          \
  }
#define CPX_OPS(T)                                                             \
  static inline T op_##T(int op, T a, T b) {                                   \
    return op == OR_SUM ? a + b : a * b;                                       \
  }

typedef long double ldouble;
typedef float _Complex cfloat;
typedef double _Complex cdouble;

INT_OPS(int8_t, uint8_t, uint32_t)
INT_OPS(int16_t, uint16_t, uint32_t)
INT_OPS(int32_t, uint32_t, uint32_t)
INT_OPS(int64_t, uint64_t, uint64_t)
INT_OPS(uint8_t, uint8_t, uint32_t)
INT_OPS(uint16_t, uint16_t, uint32_t)
INT_OPS(uint32_t, uint32_t, uint32_t)
INT_OPS(uint64_t, uint64_t, uint64_t)
FLT_OPS(float)
FLT_OPS(double)
FLT_OPS(ldouble)
CPX_OPS(cfloat)
CPX_OPS(cdouble)

/* ------------------------------------------------------------------------ */
/* The power-of-two subset used by rec_dbl and both Rabenseifner variants    */
/* (reduce.c:206-214, 337-346): p2s = largest power of two <= P; member      */
/* as = ceil(q*P/p2s) is p2s index q, and the member after it is folded into */
/* q when floor((as+1)*p2s/P) == q (reduce.c:232, 383).                      */
/* ------------------------------------------------------------------------ */
static int p2s_of(int P, int *logp) {
  int p = 1, l = 0;
  while (p * 2 <= P) {
    p *= 2;
    l++;
  }
  if (logp) *logp = l;
  return p;
}
static inline int p2s_member(int q, int P, int p2s) {
  return (int)(((long)q * P + p2s - 1) / p2s);
}
static inline int p2s_has_extra(int q, int P, int p2s) {
  const int as = p2s_member(q, P, p2s);
  return (long)(as + 1) * p2s / P == q;
}

#define REDUCE_ALGOS(T)                                                        \
  /* reduce.c:55-91: member 0 folds members 1..P-1 left to right, then the  \
   * result is broadcast from member 0. */                                     \
  static void linear_##T(int op, int P, size_t N, const T *in, T *out) {      \
    for (size_t i = 0; i < N; i++) {                                           \
      T acc = in[i];                                                           \
      for (int p = 1; p < P; p++) acc = op_##T(op, acc, in[(size_t)p * N + i]); \
      for (int p = 0; p < P; p++) out[(size_t)p * N + i] = acc;                \
    }                                                                          \
  }                                                                            \
  /* reduce.c:102-171: binomial tree towards member 0.  Member x combines   \
   * its children x|m (m = 1, 2, 4, ... below x's lowest set bit) in        \
   * increasing m, each as op(child, own) (reduce.c:143-149); then member   \
   * 0's value is broadcast. */                                                \
  static void binomial_node_##T(int op, int P, size_t N, const T *in, int x,   \
                                T *acc) {                                      \
    memcpy(acc, in + (size_t)x * N, N * sizeof(T));                            \
    T *child = (T *)malloc((N ? N : 1) * sizeof(T));                           \
    for (unsigned m = 1; !(x & (int)m) && (x | (int)m) < P; m <<= 1) {         \
      binomial_node_##T(op, P, N, in, x | (int)m, child);                      \
      for (size_t i = 0; i < N; i++) acc[i] = op_##T(op, child[i], acc[i]);   \
    }                                                                          \
    free(child);                                                               \
  }                                                                            \
  static void binomial_##T(int op, int P, size_t N, const T *in, T *out) {    \
    binomial_node_##T(op, P, N, in, 0, out);                                   \
    for (int p = 1; p < P; p++)                                                \
      memcpy(out + (size_t)p * N, out, N * sizeof(T));                         \
  }                                                                            \
  /* reduce.c:182-293: fold the extra member into its p2s partner as        \
   * op(extra, own) (reduce.c:240-241), then log2(p2s) butterfly rounds     \
   * with mask 1, 2, 4, ...; member q computes op(own, partner's)           \
   * (reduce.c:268).  Each p2s member (and the extra folded into it) ends   \
   * with its own value, so results may differ between members where op    \
   * is order dependent (float MIN/MAX with NaN or mixed-sign zeros). */     \
  static void rec_dbl_##T(int op, int P, size_t N, const T *in, T *out) {     \
    const int p2s = p2s_of(P, NULL);                                           \
    T *R = (T *)malloc(((size_t)p2s * N + 1) * sizeof(T));                     \
    for (int q = 0; q < p2s; q++) {                                            \
      const int as = p2s_member(q, P, p2s);                                    \
      T *r = R + (size_t)q * N;                                                \
      const T *mine = in + (size_t)as * N;                                     \
      if (p2s_has_extra(q, P, p2s)) {                                          \
        const T *ext = in + (size_t)(as + 1) * N;                              \
        for (size_t i = 0; i < N; i++) r[i] = op_##T(op, ext[i], mine[i]);     \
      } else {                                                                 \
        memcpy(r, mine, N * sizeof(T));                                        \
      }                                                                        \
    }                                                                          \
    for (int mask = 1; mask < p2s; mask <<= 1) {                               \
      for (int q = 0; q < p2s; q++) {                                          \
        const int o = q ^ mask;                                                \
        if (o < q) continue;                                                   \
        T *a = R + (size_t)q * N, *b = R + (size_t)o * N;                      \
        for (size_t i = 0; i < N; i++) {                                       \
          const T va = a[i], vb = b[i];                                        \
          a[i] = op_##T(op, va, vb);                                           \
          b[i] = op_##T(op, vb, va);                                           \
        }                                                                      \
      }                                                                        \
    }                                                                          \
    for (int q = 0; q < p2s; q++) {                                            \
      const int as = p2s_member(q, P, p2s);                                    \
      memcpy(out + (size_t)as * N, R + (size_t)q * N, N * sizeof(T));          \
      if (p2s_has_extra(q, P, p2s))                                            \
        memcpy(out + (size_t)(as + 1) * N, R + (size_t)q * N, N * sizeof(T));  \
    }                                                                          \
    free(R);                                                                   \
  }                                                                            \
  /* reduce.c:306-511 (and 521-724, whose ring allgather moves the same     \
   * blocks): the extra member's fold is op(extra, own) on the lower half   \
   * [0, N/2) and op(own, extra) on the upper half (reduce.c:375, 397);     \
   * recursive halving with distance 1, 2, 4, ... where member q keeps the  \
   * lower half of its block range when (q & d) == 0 and computes           \
   * op(own, partner's) over it (reduce.c:425-449).  Block b, elements      \
   * [b*N/p2s, (b+1)*N/p2s), ends on member reverse_bits(b); the allgather  \
   * copies it to everyone. */                                                 \
  static void rabenseifner_##T(int op, int P, size_t N, const T *in, T *out) { \
    int logp;                                                                  \
    const int p2s = p2s_of(P, &logp);                                          \
    T *R = (T *)malloc(((size_t)p2s * N + 1) * sizeof(T));                     \
    int *bb = (int *)malloc(sizeof(int) * (size_t)p2s);                        \
    int *be = (int *)malloc(sizeof(int) * (size_t)p2s);                        \
    const size_t half = N / 2;                                                 \
    for (int q = 0; q < p2s; q++) {                                            \
      const int as = p2s_member(q, P, p2s);                                    \
      T *r = R + (size_t)q * N;                                                \
      const T *mine = in + (size_t)as * N;                                     \
      if (p2s_has_extra(q, P, p2s)) {                                          \
        const T *ext = in + (size_t)(as + 1) * N;                              \
        for (size_t i = 0; i < half; i++) r[i] = op_##T(op, ext[i], mine[i]);  \
        for (size_t i = half; i < N; i++) r[i] = op_##T(op, mine[i], ext[i]);  \
      } else {                                                                 \
        memcpy(r, mine, N * sizeof(T));                                        \
      }                                                                        \
      bb[q] = 0;                                                               \
      be[q] = p2s;                                                             \
    }                                                                          \
    for (int d = 1; d < p2s; d <<= 1) {                                        \
      for (int q = 0; q < p2s; q++) {                                          \
        const int o = q ^ d;                                                   \
        if (o < q) continue;                                                   \
        /* q has bit d clear: keeps the lower half, o the upper half */        \
        const int mid = (bb[q] + be[q]) / 2;                                   \
        const size_t lo0 = (size_t)bb[q] * N / p2s;                            \
        const size_t lo1 = (size_t)mid * N / p2s;                              \
        const size_t hi1 = (size_t)be[q] * N / p2s;                            \
        T *a = R + (size_t)q * N, *b = R + (size_t)o * N;                      \
        for (size_t i = lo0; i < lo1; i++) a[i] = op_##T(op, a[i], b[i]);      \
        for (size_t i = lo1; i < hi1; i++) b[i] = op_##T(op, b[i], a[i]);      \
        be[q] = mid;                                                           \
        bb[o] = mid;                                                           \
      }                                                                        \
    }                                                                          \
    for (int b = 0; b < p2s; b++) {                                            \
      const int q = or_reverse_bits(b, logp);                                  \
      const size_t i0 = (size_t)b * N / p2s, i1 = (size_t)(b + 1) * N / p2s;   \
      for (int p = 0; p < P; p++)                                              \
        memcpy(out + (size_t)p * N + i0, R + (size_t)q * N + i0,               \
               (i1 - i0) * sizeof(T));                                         \
    }                                                                          \
    free(R);                                                                   \
    free(bb);                                                                  \
    free(be);                                                                  \
  }                                                                            \
  static int reduce_##T(int algo, int op, int P, size_t N, const void *in,     \
                        void *out) {                                           \
    switch (algo) {                                                            \
    case OR_LINEAR: linear_##T(op, P, N, (const T *)in, (T *)out); return 0;   \
    case OR_BINOMIAL: binomial_##T(op, P, N, (const T *)in, (T *)out); return 0; \
    case OR_REC_DBL: rec_dbl_##T(op, P, N, (const T *)in, (T *)out); return 0; \
    case OR_RABENSEIFNER:                                                      \
    case OR_RABENSEIFNER2:                                                     \
      rabenseifner_##T(op, P, N, (const T *)in, (T *)out);                     \
      return 0;                                                                \
    default: return -1;                                                        \
    }                                                                          \
  }

REDUCE_ALGOS(int8_t)
REDUCE_ALGOS(int16_t)
REDUCE_ALGOS(int32_t)
REDUCE_ALGOS(int64_t)
REDUCE_ALGOS(uint8_t)
REDUCE_ALGOS(uint16_t)
REDUCE_ALGOS(uint32_t)
REDUCE_ALGOS(uint64_t)
REDUCE_ALGOS(float)
REDUCE_ALGOS(double)
REDUCE_ALGOS(ldouble)
REDUCE_ALGOS(cfloat)
REDUCE_ALGOS(cdouble)

/* Which (op, dtype) pairs the reference instantiates (api_types.h type
 * tables): bitwise ops on integers, MIN/MAX on integers and reals, SUM/PROD
 * on everything including complex. */
static int op_supported(int op, int dtype) {
  const int is_int = dtype <= OR_U64;
  const int is_cpx = dtype == OR_C32 || dtype == OR_C64;
  if (op <= OR_XOR) return is_int;
  if (op == OR_MIN || op == OR_MAX) return !is_cpx;
  return op == OR_SUM || op == OR_PROD;
}

int or_reduce(int algo, int op, int dtype, int npes, size_t nelems,
              const void *in, void *out) {
  if (npes < 1 || algo < 0 || algo >= OR_NALGO || op < 0 || op >= OR_NOP ||
      dtype < 0 || dtype >= OR_NDTYPE || !op_supported(op, dtype))
    return -1;
  switch (dtype) {
  case OR_I8: return reduce_int8_t(algo, op, npes, nelems, in, out);
  case OR_I16: return reduce_int16_t(algo, op, npes, nelems, in, out);
  case OR_I32: return reduce_int32_t(algo, op, npes, nelems, in, out);
  case OR_I64: return reduce_int64_t(algo, op, npes, nelems, in, out);
  case OR_U8: return reduce_uint8_t(algo, op, npes, nelems, in, out);
  case OR_U16: return reduce_uint16_t(algo, op, npes, nelems, in, out);
  case OR_U32: return reduce_uint32_t(algo, op, npes, nelems, in, out);
  case OR_U64: return reduce_uint64_t(algo, op, npes, nelems, in, out);
  case OR_F32: return reduce_float(algo, op, npes, nelems, in, out);
  case OR_F64: return reduce_double(algo, op, npes, nelems, in, out);
  case OR_F80: return reduce_ldouble(algo, op, npes, nelems, in, out);
  case OR_C32: return reduce_cfloat(algo, op, npes, nelems, in, out);
  case OR_C64: return reduce_cdouble(algo, op, npes, nelems, in, out);
  default: return -1;
  }
}

/* ------------------------------------------------------------------------ */
/* data movement: the result does not depend on the algorithm chosen          */
/* ------------------------------------------------------------------------ */

/* fcollect.c:32-484: member p's dest is the members' sources concatenated
 * in member order (Bruck's final rotate_inplace, util/rotate.c:22-54,
 * restores this order). */
int or_fcollect(int npes, size_t nbytes, const void *in, void *out) {
  if (npes < 1) return -1;
  const char *src = (const char *)in;
  char *dst = (char *)out;
  const size_t total = (size_t)npes * nbytes;
  for (int p = 0; p < npes; p++) memcpy(dst + (size_t)p * total, src, total);
  return 0;
}

/* collect.c:35-591: every member contributes its own nbytes[k]; member p's
 * dest is the contributions concatenated in member order (each member's
 * block offset is the exclusive prefix sum of the sizes, collect.c:43,
 * util/scan.c:10).  in: member k's source starts at in + k*src_pitch;
 * out: member p's dest starts at out + p*dst_pitch. */
int or_collect(int npes, const uint64_t *nbytes, const void *in, size_t src_pitch, void *out,
               size_t dst_pitch) {
  if (npes < 1) return -1;
  const char *src = (const char *)in;
  char *dst = (char *)out;
  size_t total = 0;
  for (int k = 0; k < npes; k++) {
    if (nbytes[k] > src_pitch) return -1;
    total += nbytes[k];
  }
  if (total > dst_pitch) return -1;
  for (int p = 0; p < npes; p++) {
    size_t off = 0;
    for (int k = 0; k < npes; k++) {
      memcpy(dst + (size_t)p * dst_pitch + off, src + (size_t)k * src_pitch, nbytes[k]);
      off += nbytes[k];
    }
  }
  return 0;
}

/* alltoall.c:75-201: block k of member j's dest is block j of member k's
 * source. */
int or_alltoall(int npes, size_t nbytes, const void *in, void *out) {
  if (npes < 1) return -1;
  const char *src = (const char *)in;
  char *dst = (char *)out;
  const size_t row = (size_t)npes * nbytes;
  for (int j = 0; j < npes; j++)
    for (int k = 0; k < npes; k++)
      memcpy(dst + (size_t)j * row + (size_t)k * nbytes,
             src + (size_t)k * row + (size_t)j * nbytes, nbytes);
  return 0;
}

/* alltoalls.c:54-90 (index rule 39-50): element t from member k to member
 * l moves src_k[(l*n + t)*sst] -> dest_l[(k*n + t)*dst]; every other dest
 * element keeps its previous contents.  Rows are npes*n*max(stride) long:
 * in has npes*n*sst elements per member, out npes*n*dst. */
int or_alltoalls(int npes, size_t nelems, long dst, long sst, size_t esize,
                 const void *in, void *out) {
  if (npes < 1 || dst < 1 || sst < 1) return -1;
  const char *src = (const char *)in;
  char *d = (char *)out;
  const size_t srow = (size_t)npes * nelems * (size_t)sst * esize;
  const size_t drow = (size_t)npes * nelems * (size_t)dst * esize;
  for (int k = 0; k < npes; k++)
    for (int l = 0; l < npes; l++)
      for (size_t t = 0; t < nelems; t++) {
        const size_t so = ((size_t)l * nelems + t) * (size_t)sst * esize;
        const size_t doff = ((size_t)k * nelems + t) * (size_t)dst * esize;
        memcpy(d + (size_t)l * drow + doff, src + (size_t)k * srow + so, esize);
      }
  return 0;
}

/* broadcast.c:58-189: every member other than the root receives the root's
 * source; the root's dest is left as it was. */
int or_broadcast(int npes, int root, size_t nbytes, const void *in, void *out) {
  if (npes < 1 || root < 0 || root >= npes) return -1;
  const char *src = (const char *)in + (size_t)root * nbytes;
  for (int p = 0; p < npes; p++)
    if (p != root) memcpy((char *)out + (size_t)p * nbytes, src, nbytes);
  return 0;
}

/* comms.c:423-428 (shmemc_ctx_fadd): fetch the old value, add.  Applied in
 * operation order; concurrent issuers can only permute the fetched values
 * of operations that hit the same counter. */
int or_amo_fetch_add_i64(int npes, size_t ncounters, size_t nops, const int *pe,
                         const int64_t *off, const int64_t *val,
                         int64_t *fetched, int64_t *counters) {
  for (size_t k = 0; k < nops; k++) {
    if (pe[k] < 0 || pe[k] >= npes || off[k] < 0 || (size_t)off[k] >= ncounters)
      return -1;
    int64_t *c = counters + (size_t)pe[k] * ncounters + (size_t)off[k];
    fetched[k] = *c;
    *c = (int64_t)((uint64_t)*c + (uint64_t)val[k]);
  }
  return 0;
}
