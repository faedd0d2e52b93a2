/*
 * shmem_generics.h -- the C11 generic names of the OpenSHMEM interface
 * (shmem_put, shmem_atomic_fetch_add, shmem_sum_reduce, shmem_wait_until,
 * ...), each a _Generic selection that calls the typed function of
 * include/shmem.h, as the reference's include/shmem/generics.h does for its
 * own library.  Included by shmem.h for C11 and later (define
 * SHMEM_B200_NO_GENERICS to leave them out).
 *
 * Selection is on the pointer type of the data argument.  The tables below
 * list each distinct C type once: the sized typedefs (int32_t, uint64_t,
 * size_t, ptrdiff_t, ...) are the same types as these on the platforms the
 * library builds for, and _Generic refuses two associations of one type.
 * The RMA and atomic names also take a context first (shmem_put(ctx, dest,
 * ...)): a first argument of type shmem_ctx_t selects the shmem_ctx_ form on
 * the next argument's type.  A data type outside an operation's table
 * selects b200_shmem_generic_type_error, a function of no parameters, so the
 * call fails to compile.
 */
#ifndef SHMEM_B200_GENERICS_H
#define SHMEM_B200_GENERICS_H

/* declared, never defined: a call through an unmatched selection does not
 * compile (it passes arguments to a function of none) */
void b200_shmem_generic_type_error(void);

/* ---- argument picking (padded, so short calls still expand) ------------ */
#define SHMEM_B200_ARG1(a, ...) a
#define SHMEM_B200_ARG2(a, b, ...) b
#define SHMEM_B200_FIRST(...) SHMEM_B200_ARG1(__VA_ARGS__, 0)
#define SHMEM_B200_SECOND(...) SHMEM_B200_ARG2(__VA_ARGS__, 0, 0)

/* ---- tables: CASE(F, type, name) per distinct C type -------------------- */
#define SHMEM_B200_GT_RMA(CASE, F)                                             \
  CASE(F, float, float) CASE(F, double, double) CASE(F, long double, longdouble) \
  CASE(F, char, char) CASE(F, signed char, schar) CASE(F, short, short)        \
  CASE(F, int, int) CASE(F, long, long) CASE(F, long long, longlong)           \
  CASE(F, unsigned char, uchar) CASE(F, unsigned short, ushort)                \
  CASE(F, unsigned int, uint) CASE(F, unsigned long, ulong)                    \
  CASE(F, unsigned long long, ulonglong)
#define SHMEM_B200_GT_AMO_STD(CASE, F)                                         \
  CASE(F, int, int) CASE(F, long, long) CASE(F, long long, longlong)           \
  CASE(F, unsigned int, uint) CASE(F, unsigned long, ulong)                    \
  CASE(F, unsigned long long, ulonglong)
#define SHMEM_B200_GT_AMO_EXT(CASE, F)                                         \
  CASE(F, float, float) CASE(F, double, double) SHMEM_B200_GT_AMO_STD(CASE, F)
/* the bitwise atomics' signed types are int32_t and int64_t (int, long) */
#define SHMEM_B200_GT_AMO_BIT(CASE, F)                                         \
  CASE(F, unsigned int, uint) CASE(F, unsigned long, ulong)                    \
  CASE(F, unsigned long long, ulonglong) CASE(F, int, int32) CASE(F, long, int64)
/* team reductions: AND/OR/XOR on unsigned and fixed-width types (the
 * signed ones are int8_t..int64_t), MIN/MAX and SUM/PROD on the rest */
#define SHMEM_B200_GT_RED_BIT(CASE, F)                                         \
  CASE(F, unsigned char, uchar) CASE(F, unsigned short, ushort)                \
  CASE(F, unsigned int, uint) CASE(F, unsigned long, ulong)                    \
  CASE(F, unsigned long long, ulonglong) CASE(F, signed char, int8)            \
  CASE(F, short, int16) CASE(F, int, int32) CASE(F, long, int64)
#define SHMEM_B200_GT_RED_MINMAX(CASE, F)                                      \
  CASE(F, char, char) CASE(F, signed char, schar) CASE(F, short, short)        \
  CASE(F, int, int) CASE(F, long, long) CASE(F, long long, longlong)           \
  CASE(F, unsigned char, uchar) CASE(F, unsigned short, ushort)                \
  CASE(F, unsigned int, uint) CASE(F, unsigned long, ulong)                    \
  CASE(F, unsigned long long, ulonglong) CASE(F, float, float)                 \
  CASE(F, double, double) CASE(F, long double, longdouble)
#define SHMEM_B200_GT_RED_ARITH(CASE, F)                                       \
  SHMEM_B200_GT_RED_MINMAX(CASE, F) CASE(F, double _Complex, complexd)         \
  CASE(F, float _Complex, complexf)
#define SHMEM_B200_GT_TOALL_BIT(CASE, F)                                       \
  CASE(F, short, short) CASE(F, int, int) CASE(F, long, long)                  \
  CASE(F, long long, longlong)
#define SHMEM_B200_GT_TOALL_MINMAX(CASE, F)                                    \
  SHMEM_B200_GT_TOALL_BIT(CASE, F) CASE(F, float, float) CASE(F, double, double) \
  CASE(F, long double, longdouble)
#define SHMEM_B200_GT_TOALL_ARITH(CASE, F)                                     \
  SHMEM_B200_GT_TOALL_MINMAX(CASE, F) CASE(F, double _Complex, complexd)       \
  CASE(F, float _Complex, complexf)
#define SHMEM_B200_GT_SYNC_VEC(CASE, F)                                        \
  CASE(F, int, int) CASE(F, long, long) CASE(F, long long, longlong)           \
  CASE(F, unsigned int, uint) CASE(F, unsigned long, ulong)                    \
  CASE(F, unsigned long long, ulonglong)
#define SHMEM_B200_GT_SYNC(CASE, F)                                            \
  CASE(F, short, short) CASE(F, unsigned short, ushort) SHMEM_B200_GT_SYNC_VEC(CASE, F)

/* association makers: shmem_<name>_<F> (or shmem_ctx_<name>_<F>) for T *,
 * and for const T * as well where the argument is a source */
#define SHMEM_B200_GC(F, T, N) T *: shmem_##N##_##F,
#define SHMEM_B200_GC_CTX(F, T, N) T *: shmem_ctx_##N##_##F,
#define SHMEM_B200_GC_SRC(F, T, N) T *: shmem_##N##_##F, const T *: shmem_##N##_##F,
#define SHMEM_B200_GC_SRC_CTX(F, T, N)                                         \
  T *: shmem_ctx_##N##_##F, const T *: shmem_ctx_##N##_##F,
/* reductions are named shmem_<name>_<op>_reduce / _to_all */
#define SHMEM_B200_GC_RED(F, T, N) T *: shmem_##N##_##F##_reduce,
#define SHMEM_B200_GC_TOALL(F, T, N) T *: shmem_##N##_##F##_to_all,

#define SHMEM_B200_SELECT(TABLE, CASE, F, x)                                   \
  _Generic((x), TABLE(CASE, F) default: b200_shmem_generic_type_error)

/* a routine with a context form: dispatch on the first argument, or on the
 * second when the first is a context */
#define SHMEM_B200_WITH_CTX(TABLE, CASE, CASE_CTX, F, ...)                     \
  _Generic((SHMEM_B200_FIRST(__VA_ARGS__)),                                    \
      shmem_ctx_t: SHMEM_B200_SELECT(TABLE, CASE_CTX, F, SHMEM_B200_SECOND(__VA_ARGS__)), \
      default: SHMEM_B200_SELECT(TABLE, CASE, F, SHMEM_B200_FIRST(__VA_ARGS__)))(__VA_ARGS__)
#define SHMEM_B200_RMA(F, ...)                                                 \
  SHMEM_B200_WITH_CTX(SHMEM_B200_GT_RMA, SHMEM_B200_GC, SHMEM_B200_GC_CTX, F, __VA_ARGS__)
#define SHMEM_B200_RMA_SRC(F, ...)                                             \
  SHMEM_B200_WITH_CTX(SHMEM_B200_GT_RMA, SHMEM_B200_GC_SRC, SHMEM_B200_GC_SRC_CTX, F, \
                      __VA_ARGS__)

/* ---- RMA (api.h: put/get/p/g, iput/iget, _nbi, put_signal) -------------- */
#define shmem_put(...) SHMEM_B200_RMA(put, __VA_ARGS__)
#define shmem_get(...) SHMEM_B200_RMA(get, __VA_ARGS__)
#define shmem_put_nbi(...) SHMEM_B200_RMA(put_nbi, __VA_ARGS__)
#define shmem_get_nbi(...) SHMEM_B200_RMA(get_nbi, __VA_ARGS__)
#define shmem_iput(...) SHMEM_B200_RMA(iput, __VA_ARGS__)
#define shmem_iget(...) SHMEM_B200_RMA(iget, __VA_ARGS__)
#define shmem_p(...) SHMEM_B200_RMA(p, __VA_ARGS__)
#define shmem_g(...) SHMEM_B200_RMA_SRC(g, __VA_ARGS__)
#define shmem_put_signal(...) SHMEM_B200_RMA(put_signal, __VA_ARGS__)
#define shmem_put_signal_nbi(...) SHMEM_B200_RMA(put_signal_nbi, __VA_ARGS__)

/* ---- atomics (src/api/atomics) ------------------------------------------ */
#define SHMEM_B200_AMO(TABLE, F, ...)                                          \
  SHMEM_B200_WITH_CTX(TABLE, SHMEM_B200_GC, SHMEM_B200_GC_CTX, F, __VA_ARGS__)
#define shmem_atomic_fetch_add(...) SHMEM_B200_AMO(SHMEM_B200_GT_AMO_STD, atomic_fetch_add, __VA_ARGS__)
#define shmem_atomic_add(...) SHMEM_B200_AMO(SHMEM_B200_GT_AMO_STD, atomic_add, __VA_ARGS__)
#define shmem_atomic_fetch_inc(...) SHMEM_B200_AMO(SHMEM_B200_GT_AMO_STD, atomic_fetch_inc, __VA_ARGS__)
#define shmem_atomic_inc(...) SHMEM_B200_AMO(SHMEM_B200_GT_AMO_STD, atomic_inc, __VA_ARGS__)
#define shmem_atomic_compare_swap(...)                                         \
  SHMEM_B200_AMO(SHMEM_B200_GT_AMO_STD, atomic_compare_swap, __VA_ARGS__)
#define shmem_atomic_swap(...) SHMEM_B200_AMO(SHMEM_B200_GT_AMO_EXT, atomic_swap, __VA_ARGS__)
#define shmem_atomic_set(...) SHMEM_B200_AMO(SHMEM_B200_GT_AMO_EXT, atomic_set, __VA_ARGS__)
#define shmem_atomic_fetch(...)                                                \
  SHMEM_B200_WITH_CTX(SHMEM_B200_GT_AMO_EXT, SHMEM_B200_GC_SRC, SHMEM_B200_GC_SRC_CTX, \
                      atomic_fetch, __VA_ARGS__)
#define shmem_atomic_fetch_and(...) SHMEM_B200_AMO(SHMEM_B200_GT_AMO_BIT, atomic_fetch_and, __VA_ARGS__)
#define shmem_atomic_fetch_or(...) SHMEM_B200_AMO(SHMEM_B200_GT_AMO_BIT, atomic_fetch_or, __VA_ARGS__)
#define shmem_atomic_fetch_xor(...) SHMEM_B200_AMO(SHMEM_B200_GT_AMO_BIT, atomic_fetch_xor, __VA_ARGS__)
#define shmem_atomic_and(...) SHMEM_B200_AMO(SHMEM_B200_GT_AMO_BIT, atomic_and, __VA_ARGS__)
#define shmem_atomic_or(...) SHMEM_B200_AMO(SHMEM_B200_GT_AMO_BIT, atomic_or, __VA_ARGS__)
#define shmem_atomic_xor(...) SHMEM_B200_AMO(SHMEM_B200_GT_AMO_BIT, atomic_xor, __VA_ARGS__)
/* the non-blocking fetching forms select on the fetch buffer's type */
#define shmem_atomic_fetch_add_nbi(...)                                        \
  SHMEM_B200_AMO(SHMEM_B200_GT_AMO_STD, atomic_fetch_add_nbi, __VA_ARGS__)
#define shmem_atomic_fetch_inc_nbi(...)                                        \
  SHMEM_B200_AMO(SHMEM_B200_GT_AMO_STD, atomic_fetch_inc_nbi, __VA_ARGS__)
#define shmem_atomic_compare_swap_nbi(...)                                     \
  SHMEM_B200_AMO(SHMEM_B200_GT_AMO_STD, atomic_compare_swap_nbi, __VA_ARGS__)
#define shmem_atomic_swap_nbi(...) SHMEM_B200_AMO(SHMEM_B200_GT_AMO_EXT, atomic_swap_nbi, __VA_ARGS__)
#define shmem_atomic_fetch_nbi(...) SHMEM_B200_AMO(SHMEM_B200_GT_AMO_EXT, atomic_fetch_nbi, __VA_ARGS__)
#define shmem_atomic_fetch_and_nbi(...)                                        \
  SHMEM_B200_AMO(SHMEM_B200_GT_AMO_BIT, atomic_fetch_and_nbi, __VA_ARGS__)
#define shmem_atomic_fetch_or_nbi(...)                                         \
  SHMEM_B200_AMO(SHMEM_B200_GT_AMO_BIT, atomic_fetch_or_nbi, __VA_ARGS__)
#define shmem_atomic_fetch_xor_nbi(...)                                        \
  SHMEM_B200_AMO(SHMEM_B200_GT_AMO_BIT, atomic_fetch_xor_nbi, __VA_ARGS__)

/* ---- team collectives: (team, dest, ...) select on dest ------------------ */
#define SHMEM_B200_TEAM(TABLE, CASE, F, ...)                                   \
  SHMEM_B200_SELECT(TABLE, CASE, F, SHMEM_B200_SECOND(__VA_ARGS__))(__VA_ARGS__)
#define shmem_fcollect(...) SHMEM_B200_TEAM(SHMEM_B200_GT_RMA, SHMEM_B200_GC, fcollect, __VA_ARGS__)
#define shmem_collect(...) SHMEM_B200_TEAM(SHMEM_B200_GT_RMA, SHMEM_B200_GC, collect, __VA_ARGS__)
#define shmem_alltoall(...) SHMEM_B200_TEAM(SHMEM_B200_GT_RMA, SHMEM_B200_GC, alltoall, __VA_ARGS__)
#define shmem_alltoalls(...) SHMEM_B200_TEAM(SHMEM_B200_GT_RMA, SHMEM_B200_GC, alltoalls, __VA_ARGS__)
#define shmem_broadcast(...) SHMEM_B200_TEAM(SHMEM_B200_GT_RMA, SHMEM_B200_GC, broadcast, __VA_ARGS__)

#define shmem_and_reduce(...) SHMEM_B200_TEAM(SHMEM_B200_GT_RED_BIT, SHMEM_B200_GC_RED, and, __VA_ARGS__)
#define shmem_or_reduce(...) SHMEM_B200_TEAM(SHMEM_B200_GT_RED_BIT, SHMEM_B200_GC_RED, or, __VA_ARGS__)
#define shmem_xor_reduce(...) SHMEM_B200_TEAM(SHMEM_B200_GT_RED_BIT, SHMEM_B200_GC_RED, xor, __VA_ARGS__)
#define shmem_min_reduce(...) SHMEM_B200_TEAM(SHMEM_B200_GT_RED_MINMAX, SHMEM_B200_GC_RED, min, __VA_ARGS__)
#define shmem_max_reduce(...) SHMEM_B200_TEAM(SHMEM_B200_GT_RED_MINMAX, SHMEM_B200_GC_RED, max, __VA_ARGS__)
#define shmem_sum_reduce(...) SHMEM_B200_TEAM(SHMEM_B200_GT_RED_ARITH, SHMEM_B200_GC_RED, sum, __VA_ARGS__)
#define shmem_prod_reduce(...) SHMEM_B200_TEAM(SHMEM_B200_GT_RED_ARITH, SHMEM_B200_GC_RED, prod, __VA_ARGS__)

/* active-set reductions (dest, source, nreduce, PE_start, ...): select on dest */
#define SHMEM_B200_TOALL(TABLE, F, ...)                                        \
  SHMEM_B200_SELECT(TABLE, SHMEM_B200_GC_TOALL, F, SHMEM_B200_FIRST(__VA_ARGS__))(__VA_ARGS__)
#define shmem_and_to_all(...) SHMEM_B200_TOALL(SHMEM_B200_GT_TOALL_BIT, and, __VA_ARGS__)
#define shmem_or_to_all(...) SHMEM_B200_TOALL(SHMEM_B200_GT_TOALL_BIT, or, __VA_ARGS__)
#define shmem_xor_to_all(...) SHMEM_B200_TOALL(SHMEM_B200_GT_TOALL_BIT, xor, __VA_ARGS__)
#define shmem_min_to_all(...) SHMEM_B200_TOALL(SHMEM_B200_GT_TOALL_MINMAX, min, __VA_ARGS__)
#define shmem_max_to_all(...) SHMEM_B200_TOALL(SHMEM_B200_GT_TOALL_MINMAX, max, __VA_ARGS__)
#define shmem_sum_to_all(...) SHMEM_B200_TOALL(SHMEM_B200_GT_TOALL_ARITH, sum, __VA_ARGS__)
#define shmem_prod_to_all(...) SHMEM_B200_TOALL(SHMEM_B200_GT_TOALL_ARITH, prod, __VA_ARGS__)

/* ---- point-to-point synchronisation (src/api/pt2pt_synch) --------------- */
#define SHMEM_B200_SYNC(TABLE, F, ...)                                         \
  SHMEM_B200_SELECT(TABLE, SHMEM_B200_GC, F, SHMEM_B200_FIRST(__VA_ARGS__))(__VA_ARGS__)
/* on one word: every integer type from short up; on arrays: int and up */
#define shmem_wait_until(...) SHMEM_B200_SYNC(SHMEM_B200_GT_SYNC, wait_until, __VA_ARGS__)
#define shmem_test(...) SHMEM_B200_SYNC(SHMEM_B200_GT_SYNC, test, __VA_ARGS__)
#define shmem_wait_until_all(...) SHMEM_B200_SYNC(SHMEM_B200_GT_SYNC_VEC, wait_until_all, __VA_ARGS__)
#define shmem_wait_until_any(...) SHMEM_B200_SYNC(SHMEM_B200_GT_SYNC_VEC, wait_until_any, __VA_ARGS__)
#define shmem_wait_until_some(...) SHMEM_B200_SYNC(SHMEM_B200_GT_SYNC_VEC, wait_until_some, __VA_ARGS__)
#define shmem_wait_until_all_vector(...)                                       \
  SHMEM_B200_SYNC(SHMEM_B200_GT_SYNC_VEC, wait_until_all_vector, __VA_ARGS__)
#define shmem_wait_until_any_vector(...)                                       \
  SHMEM_B200_SYNC(SHMEM_B200_GT_SYNC_VEC, wait_until_any_vector, __VA_ARGS__)
#define shmem_wait_until_some_vector(...)                                      \
  SHMEM_B200_SYNC(SHMEM_B200_GT_SYNC_VEC, wait_until_some_vector, __VA_ARGS__)
#define shmem_test_all(...) SHMEM_B200_SYNC(SHMEM_B200_GT_SYNC_VEC, test_all, __VA_ARGS__)
#define shmem_test_any(...) SHMEM_B200_SYNC(SHMEM_B200_GT_SYNC_VEC, test_any, __VA_ARGS__)
#define shmem_test_some(...) SHMEM_B200_SYNC(SHMEM_B200_GT_SYNC_VEC, test_some, __VA_ARGS__)
#define shmem_test_all_vector(...) SHMEM_B200_SYNC(SHMEM_B200_GT_SYNC_VEC, test_all_vector, __VA_ARGS__)
#define shmem_test_any_vector(...) SHMEM_B200_SYNC(SHMEM_B200_GT_SYNC_VEC, test_any_vector, __VA_ARGS__)
#define shmem_test_some_vector(...)                                            \
  SHMEM_B200_SYNC(SHMEM_B200_GT_SYNC_VEC, test_some_vector, __VA_ARGS__)

#endif /* SHMEM_B200_GENERICS_H */
