/*
 * shcoll_oracle.h -- CPU restatement of the shcoll collective algorithms of
 * BTMichalowicz/osss-ucx (src/shcoll/src).  TEST INFRASTRUCTURE ONLY: the
 * parity tests and the benchmark's CPU baseline use it as the checker; the
 * product never links or calls it.
 *
 * Every function takes member-ordered arrays: member i of the team / active
 * set is row i, whatever its global PE number.  Results are the values the
 * reference leaves in each member's dest buffer.
 *
 * Parity is pinned: tests/test_oracle.py checks every function here against
 * the reference's own code compiled unmodified (oracle/_ref, built by
 * oracle/Makefile) and against the committed golden fixtures.
 */
#ifndef SHCOLL_ORACLE_H
#define SHCOLL_ORACLE_H
#include <stddef.h>
#include <stdint.h>

enum or_dtype {
  OR_I8 = 0, OR_I16, OR_I32, OR_I64,
  OR_U8, OR_U16, OR_U32, OR_U64,
  OR_F32, OR_F64, OR_F80, /* long double, 16-byte storage on x86-64 */
  OR_C32, OR_C64,         /* float _Complex, double _Complex */
  OR_NDTYPE
};
enum or_op { OR_AND = 0, OR_OR, OR_XOR, OR_MIN, OR_MAX, OR_SUM, OR_PROD, OR_NOP };
enum or_algo {
  OR_LINEAR = 0, OR_BINOMIAL, OR_REC_DBL, OR_RABENSEIFNER, OR_RABENSEIFNER2,
  OR_NALGO
};

/* Returns 0, or -1 for an unsupported (op, dtype) pair or bad sizes. */
int or_reduce(int algo, int op, int dtype, int npes, size_t nelems,
              const void *in, void *out);
size_t or_dtype_size(int dtype);

int or_fcollect(int npes, size_t nbytes, const void *in, void *out);
int or_collect(int npes, const uint64_t *nbytes, const void *in, size_t src_pitch, void *out,
               size_t dst_pitch);
int or_alltoall(int npes, size_t nbytes, const void *in, void *out);
int or_alltoalls(int npes, size_t nelems, long dst, long sst, size_t esize,
                 const void *in, void *out);
int or_broadcast(int npes, int root, size_t nbytes, const void *in, void *out);

/* Sequential fetch-and-add over int64 counters laid out [npes][ncounters]. */
int or_amo_fetch_add_i64(int npes, size_t ncounters, size_t nops, const int *pe,
                         const int64_t *off, const int64_t *val,
                         int64_t *fetched, int64_t *counters);

/* The bit-reversal used to order Rabenseifner blocks (util/bithacks.c). */
int or_reverse_bits(int number, int nbits);
#endif
