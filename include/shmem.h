/*
 * shmem.h -- the OpenSHMEM calls of the collective and atomic hot path,
 * with the names, argument lists and meanings of BTMichalowicz/osss-ucx
 * (include/shmem/api.h, include/shmem/teams.h, include/shmem/defs.h), backed
 * by the B200 engine (libshmem_b200.so over libb200shm.so).
 *
 * What is here: init/finalize/my_pe/n_pes, the symmetric heap
 * (shmem_malloc/free/calloc/align, shmem_ptr), put/get/p/g, fence/quiet,
 * barrier_all/sync_all/barrier/sync/team_sync, the reductions
 * (shmem_<T>_<op>_reduce and shmem_<T>_<op>_to_all over the reference's type
 * tables), fcollect / collect / broadcast / alltoall / alltoalls in their typed, mem
 * and 32/64 forms, the atomics (shmem_[ctx_]<T>_atomic_*), teams
 * (world, split_strided, split_2d, my_pe, n_pes, translate, destroy), the
 * strided and signalled puts and gets (iput/iget, put_signal[_nbi], the
 * sized put/get forms) and the point-to-point waits and tests
 * (wait_until / test and their _all/_any/_some[_vector] forms,
 * signal_fetch / signal_wait_until).
 *
 * How PEs run: every PE is a host thread of one process, started by
 * shmemx_b200_run (include/shmemx.h); its symmetric heap is a slice of one
 * GPU arena (CUDA managed memory by default, so host code may read and write
 * it directly).  A collective returns when it is complete for every member,
 * as in the reference.  Global and static variables are NOT symmetric here
 * (threads share them): symmetric data must come from shmem_malloc.
 */
#ifndef B200_SHMEM_H
#define B200_SHMEM_H

#include <stddef.h>
#include <stdint.h>
#include <sys/types.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- constants (values as in include/shmem/defs.h) -------------------- */
enum { SHMEM_CMP_EQ = 0, SHMEM_CMP_NE, SHMEM_CMP_GT, SHMEM_CMP_LE, SHMEM_CMP_LT, SHMEM_CMP_GE };
#define SHMEM_BCAST_SYNC_SIZE 64
#define SHMEM_BARRIER_SYNC_SIZE 2
#define SHMEM_REDUCE_SYNC_SIZE 128
#define SHMEM_REDUCE_MIN_WRKDATA_SIZE 64
#define SHMEM_COLLECT_SYNC_SIZE 128
#define SHMEM_ALLTOALL_SYNC_SIZE 64
#define SHMEM_ALLTOALLS_SYNC_SIZE 64
#define SHMEM_SYNC_SIZE SHMEM_REDUCE_SYNC_SIZE
#define SHMEM_SYNC_VALUE 0L
#define SHMEM_THREAD_SINGLE 0
#define SHMEM_THREAD_FUNNELED 1
#define SHMEM_THREAD_SERIALIZED 2
#define SHMEM_THREAD_MULTIPLE 3
/* the specification this surface follows, and this library's own name */
#define SHMEM_MAJOR_VERSION 1
#define SHMEM_MINOR_VERSION 5
#define SHMEM_MAX_NAME_LEN 64
#define SHMEM_VENDOR_STRING "b200-shmem"
#define SHMEM_VENDOR_MAJOR_VERSION 1
#define SHMEM_VENDOR_MINOR_VERSION 0
#define SHMEM_VENDOR_PATCH_VERSION 0
#define SHMEM_MALLOC_ATOMICS_REMOTE 0
#define SHMEM_MALLOC_SIGNAL_REMOTE 1

typedef void *shmem_team_t;
typedef void *shmem_ctx_t;
typedef struct {
  int num_contexts;
} shmem_team_config_t;
extern shmem_team_t SHMEM_TEAM_WORLD;
extern shmem_team_t SHMEM_TEAM_SHARED;
extern shmem_team_t SHMEM_TEAM_INVALID;
extern shmem_ctx_t SHMEM_CTX_DEFAULT;
extern shmem_ctx_t SHMEM_CTX_INVALID;

/* context options (api.h: SHMEM_CTX_SERIALIZED / PRIVATE / NOSTORE); they
 * are accepted and recorded: every context here is thread-safe */
#define SHMEM_CTX_SERIALIZED (1L << 0)
#define SHMEM_CTX_PRIVATE (1L << 1)
#define SHMEM_CTX_NOSTORE (1L << 2)

/* ---- setup / query ----------------------------------------------------- */
void shmem_init(void);
int shmem_init_thread(int requested, int *provided);
void shmem_finalize(void);
int shmem_my_pe(void);
int shmem_n_pes(void);
int shmem_pe_accessible(int pe);
void shmem_global_exit(int status);

/* ---- symmetric heap ---------------------------------------------------- */
void *shmem_malloc(size_t size);
void *shmem_calloc(size_t count, size_t size);
void *shmem_align(size_t alignment, size_t size);
void shmem_free(void *ptr);
void *shmem_ptr(const void *dest, int pe);

/* ---- RMA and ordering -------------------------------------------------- */
void shmem_putmem(void *dest, const void *source, size_t nelems, int pe);
void shmem_getmem(void *dest, const void *source, size_t nelems, int pe);
void shmem_putmem_nbi(void *dest, const void *source, size_t nelems, int pe);
void shmem_getmem_nbi(void *dest, const void *source, size_t nelems, int pe);
void shmem_fence(void);
void shmem_quiet(void);

/* ---- communication contexts (api.h:3619-3673, 1179-1202) ----------------
 * A context keeps its own non-blocking operations: shmem_ctx_quiet(ctx)
 * completes those of ctx and not those of other contexts.  A team's
 * context takes PE numbers relative to that team. */
int shmem_ctx_create(long options, shmem_ctx_t *ctx);
int shmem_team_create_ctx(shmem_team_t team, long options, shmem_ctx_t *ctx);
void shmem_ctx_destroy(shmem_ctx_t ctx);
int shmem_ctx_get_team(shmem_ctx_t ctx, shmem_team_t *team);
void shmem_ctx_quiet(shmem_ctx_t ctx);
void shmem_ctx_fence(shmem_ctx_t ctx);
void shmem_ctx_putmem(shmem_ctx_t ctx, void *dest, const void *source, size_t nelems, int pe);
void shmem_ctx_getmem(shmem_ctx_t ctx, void *dest, const void *source, size_t nelems, int pe);
void shmem_ctx_putmem_nbi(shmem_ctx_t ctx, void *dest, const void *source, size_t nelems,
                          int pe);
void shmem_ctx_getmem_nbi(shmem_ctx_t ctx, void *dest, const void *source, size_t nelems,
                          int pe);

/* ---- synchronisation --------------------------------------------------- */
void shmem_barrier_all(void);
void shmem_sync_all(void);
void shmem_barrier(int PE_start, int logPE_stride, int PE_size, long *pSync);
void shmem_sync(int PE_start, int logPE_stride, int PE_size, long *pSync);
/* the active-set form under the name the reference exports for it */
void shmem_sync_deprecated(int PE_start, int logPE_stride, int PE_size, long *pSync);
int shmem_team_sync(shmem_team_t team);
#if !defined(SHMEM_B200_NO_GENERICS)
/* shmem_sync(team) and shmem_sync(PE_start, logPE_stride, PE_size, pSync),
 * told apart by their number of arguments */
#define SHMEM_B200_SYNC_PICK(a, b, c, d, f, ...) f
#define SHMEM_B200_SYNC_4(s, l, n, p) shmem_sync_deprecated(s, l, n, p)
#define SHMEM_B200_SYNC_1(team) shmem_team_sync(team)
#define shmem_sync(...)                                                        \
  SHMEM_B200_SYNC_PICK(__VA_ARGS__, SHMEM_B200_SYNC_4, SHMEM_B200_SYNC_4,      \
                       SHMEM_B200_SYNC_4, SHMEM_B200_SYNC_1, 0)(__VA_ARGS__)
#endif

/* ---- locks (src/api/lock.c): a symmetric long, 0 when free -------------- */
void shmem_set_lock(long *lock);
int shmem_test_lock(long *lock);
void shmem_clear_lock(long *lock);

/* ---- library state and information (src/api/{init,info,tl_query}.c) ---- */
int shmem_initialized(void);
int shmem_finalized(void);
void shmem_query_thread(int *provided);
void shmem_info_get_version(int *major, int *minor);
void shmem_info_get_name(char *name);
void shmem_info_get_version_number(int *version);
void shmem_info_get_vendor_version(int *major, int *minor, int *patch);
void shmem_info_get_vendor_version_number(int *version);
void shmem_pcontrol(const int level, ...);
int shmem_addr_accessible(const void *addr, int pe);
void *shmem_realloc(void *ptr, size_t size);
void *shmem_malloc_with_hints(size_t size, long hints);
/* the address of `dest` on team member `pe`, NULL when not reachable */
void *shmem_team_ptr(shmem_team_t team, const void *dest, int pe);

/* ---- names before OpenSHMEM 1.2 and the cache routines (api.h, cache.h) -- */
void start_pes(int npes);
int _my_pe(void);
int _num_pes(void);
void *shmalloc(size_t size);
void shfree(void *ptr);
void *shrealloc(void *ptr, size_t size);
void *shmemalign(size_t alignment, size_t size);
/* no cache to manage: these do nothing */
void shmem_set_cache_inv(void);
void shmem_set_cache_line_inv(void *dest);
void shmem_clear_cache_inv(void);
void shmem_clear_cache_line_inv(void *dest);
void shmem_udcflush(void);
void shmem_udcflush_line(void *dest);

/* ---- teams (include/shmem/teams.h) -------------------------------------- */
int shmem_team_my_pe(shmem_team_t team);
int shmem_team_n_pes(shmem_team_t team);
int shmem_team_translate_pe(shmem_team_t src_team, int src_pe, shmem_team_t dest_team);
int shmem_team_split_strided(shmem_team_t parent_team, int start, int stride, int size,
                             const shmem_team_config_t *config, long config_mask,
                             shmem_team_t *new_team);
int shmem_team_split_2d(shmem_team_t parent_team, int xrange,
                        const shmem_team_config_t *xaxis_config, long xaxis_mask,
                        shmem_team_t *xaxis_team, const shmem_team_config_t *yaxis_config,
                        long yaxis_mask, shmem_team_t *yaxis_team);
void shmem_team_destroy(shmem_team_t team);
int shmem_team_get_config(shmem_team_t team, long config_mask, shmem_team_config_t *config);

/* ---- type tables (the names of include/shmem/api_types.h) -------------- */
#define SHMEM_B200_REDUCE_BITWISE_TYPES(X)                                      \
  X(unsigned char, uchar) X(unsigned short, ushort) X(unsigned int, uint)       \
  X(unsigned long, ulong) X(unsigned long long, ulonglong) X(int8_t, int8)      \
  X(int16_t, int16) X(int32_t, int32) X(int64_t, int64) X(uint8_t, uint8)       \
  X(uint16_t, uint16) X(uint32_t, uint32) X(uint64_t, uint64) X(size_t, size)
#define SHMEM_B200_REDUCE_MINMAX_TYPES(X)                                       \
  X(char, char) X(signed char, schar) X(short, short) X(int, int) X(long, long) \
  X(long long, longlong) X(ptrdiff_t, ptrdiff) X(unsigned char, uchar)          \
  X(unsigned short, ushort) X(unsigned int, uint) X(unsigned long, ulong)       \
  X(unsigned long long, ulonglong) X(int8_t, int8) X(int16_t, int16)            \
  X(int32_t, int32) X(int64_t, int64) X(uint8_t, uint8) X(uint16_t, uint16)     \
  X(uint32_t, uint32) X(uint64_t, uint64) X(size_t, size) X(float, float)       \
  X(double, double) X(long double, longdouble)
#define SHMEM_B200_REDUCE_ARITH_TYPES(X)                                        \
  SHMEM_B200_REDUCE_MINMAX_TYPES(X)                                             \
  X(double _Complex, complexd) X(float _Complex, complexf)
#define SHMEM_B200_TO_ALL_BITWISE_TYPES(X)                                      \
  X(short, short) X(int, int) X(long, long) X(long long, longlong)
#define SHMEM_B200_TO_ALL_MINMAX_TYPES(X)                                       \
  SHMEM_B200_TO_ALL_BITWISE_TYPES(X) X(float, float) X(double, double)          \
  X(long double, longdouble)
#define SHMEM_B200_TO_ALL_ARITH_TYPES(X)                                        \
  SHMEM_B200_TO_ALL_MINMAX_TYPES(X) X(double _Complex, complexd)                \
  X(float _Complex, complexf)
#define SHMEM_B200_RMA_TYPES(X)                                                 \
  X(float, float) X(double, double) X(long double, longdouble) X(char, char)    \
  X(signed char, schar) X(short, short) X(int, int) X(long, long)               \
  X(long long, longlong) X(unsigned char, uchar) X(unsigned short, ushort)      \
  X(unsigned int, uint) X(unsigned long, ulong) X(unsigned long long, ulonglong) \
  X(int8_t, int8) X(int16_t, int16) X(int32_t, int32) X(int64_t, int64)         \
  X(uint8_t, uint8) X(uint16_t, uint16) X(uint32_t, uint32) X(uint64_t, uint64) \
  X(size_t, size) X(ptrdiff_t, ptrdiff)
#define SHMEM_B200_AMO_STANDARD_TYPES(X)                                        \
  X(int, int) X(long, long) X(long long, longlong) X(unsigned int, uint)        \
  X(unsigned long, ulong) X(unsigned long long, ulonglong) X(int32_t, int32)    \
  X(int64_t, int64) X(uint32_t, uint32) X(uint64_t, uint64) X(size_t, size)     \
  X(ptrdiff_t, ptrdiff)
#define SHMEM_B200_AMO_EXTENDED_TYPES(X)                                        \
  X(float, float) X(double, double) SHMEM_B200_AMO_STANDARD_TYPES(X)
#define SHMEM_B200_AMO_BITWISE_TYPES(X)                                         \
  X(unsigned int, uint) X(unsigned long, ulong) X(unsigned long long, ulonglong) \
  X(int32_t, int32) X(int64_t, int64) X(uint32_t, uint32) X(uint64_t, uint64)

/* ---- reductions: team form (reduce.c:1078-1102) and active-set form ---- */
#define SHMEM_B200_DECL_REDUCE(_op)                                             \
  SHMEM_B200_DECL_REDUCE_##_op
#define SHMEM_B200_DECL_TEAM_REDUCE(_type, _tn, _op)                            \
  int shmem_##_tn##_##_op##_reduce(shmem_team_t team, _type *dest,             \
                                   const _type *source, size_t nreduce);
#define SHMEM_B200_DECL_TO_ALL(_type, _tn, _op)                                 \
  void shmem_##_tn##_##_op##_to_all(_type *dest, const _type *source,          \
                                    int nreduce, int PE_start,                  \
                                    int logPE_stride, int PE_size,              \
                                    _type *pWrk, long *pSync);
#define SHMEM_B200_D_AND(_t, _n) SHMEM_B200_DECL_TEAM_REDUCE(_t, _n, and)
#define SHMEM_B200_D_OR(_t, _n) SHMEM_B200_DECL_TEAM_REDUCE(_t, _n, or)
#define SHMEM_B200_D_XOR(_t, _n) SHMEM_B200_DECL_TEAM_REDUCE(_t, _n, xor)
#define SHMEM_B200_D_MIN(_t, _n) SHMEM_B200_DECL_TEAM_REDUCE(_t, _n, min)
#define SHMEM_B200_D_MAX(_t, _n) SHMEM_B200_DECL_TEAM_REDUCE(_t, _n, max)
#define SHMEM_B200_D_SUM(_t, _n) SHMEM_B200_DECL_TEAM_REDUCE(_t, _n, sum)
#define SHMEM_B200_D_PROD(_t, _n) SHMEM_B200_DECL_TEAM_REDUCE(_t, _n, prod)
SHMEM_B200_REDUCE_BITWISE_TYPES(SHMEM_B200_D_AND)
SHMEM_B200_REDUCE_BITWISE_TYPES(SHMEM_B200_D_OR)
SHMEM_B200_REDUCE_BITWISE_TYPES(SHMEM_B200_D_XOR)
SHMEM_B200_REDUCE_MINMAX_TYPES(SHMEM_B200_D_MIN)
SHMEM_B200_REDUCE_MINMAX_TYPES(SHMEM_B200_D_MAX)
SHMEM_B200_REDUCE_ARITH_TYPES(SHMEM_B200_D_SUM)
SHMEM_B200_REDUCE_ARITH_TYPES(SHMEM_B200_D_PROD)
#define SHMEM_B200_T_AND(_t, _n) SHMEM_B200_DECL_TO_ALL(_t, _n, and)
#define SHMEM_B200_T_OR(_t, _n) SHMEM_B200_DECL_TO_ALL(_t, _n, or)
#define SHMEM_B200_T_XOR(_t, _n) SHMEM_B200_DECL_TO_ALL(_t, _n, xor)
#define SHMEM_B200_T_MIN(_t, _n) SHMEM_B200_DECL_TO_ALL(_t, _n, min)
#define SHMEM_B200_T_MAX(_t, _n) SHMEM_B200_DECL_TO_ALL(_t, _n, max)
#define SHMEM_B200_T_SUM(_t, _n) SHMEM_B200_DECL_TO_ALL(_t, _n, sum)
#define SHMEM_B200_T_PROD(_t, _n) SHMEM_B200_DECL_TO_ALL(_t, _n, prod)
SHMEM_B200_TO_ALL_BITWISE_TYPES(SHMEM_B200_T_AND)
SHMEM_B200_TO_ALL_BITWISE_TYPES(SHMEM_B200_T_OR)
SHMEM_B200_TO_ALL_BITWISE_TYPES(SHMEM_B200_T_XOR)
SHMEM_B200_TO_ALL_MINMAX_TYPES(SHMEM_B200_T_MIN)
SHMEM_B200_TO_ALL_MINMAX_TYPES(SHMEM_B200_T_MAX)
SHMEM_B200_TO_ALL_ARITH_TYPES(SHMEM_B200_T_SUM)
SHMEM_B200_TO_ALL_ARITH_TYPES(SHMEM_B200_T_PROD)

/* ---- data movement (shcoll-shim.c:185-702) ------------------------------ */
#define SHMEM_B200_DECL_COPY(_type, _tn)                                        \
  int shmem_##_tn##_fcollect(shmem_team_t team, _type *dest,                   \
                             const _type *source, size_t nelems);               \
  int shmem_##_tn##_collect(shmem_team_t team, _type *dest,                    \
                            const _type *source, size_t nelems);                \
  int shmem_##_tn##_alltoall(shmem_team_t team, _type *dest,                   \
                             const _type *source, size_t nelems);               \
  int shmem_##_tn##_alltoalls(shmem_team_t team, _type *dest,                  \
                              const _type *source, ptrdiff_t dst,               \
                              ptrdiff_t sst, size_t nelems);                    \
  int shmem_##_tn##_broadcast(shmem_team_t team, _type *dest,                  \
                              const _type *source, size_t nelems, int PE_root); \
  void shmem_##_tn##_put(_type *dest, const _type *source, size_t nelems,      \
                         int pe);                                               \
  void shmem_##_tn##_get(_type *dest, const _type *source, size_t nelems,      \
                         int pe);                                               \
  void shmem_##_tn##_p(_type *dest, _type value, int pe);                      \
  _type shmem_##_tn##_g(const _type *source, int pe);                          \
  void shmem_##_tn##_put_nbi(_type *dest, const _type *source, size_t nelems,  \
                             int pe);                                           \
  void shmem_##_tn##_get_nbi(_type *dest, const _type *source, size_t nelems,  \
                             int pe);                                           \
  void shmem_ctx_##_tn##_put(shmem_ctx_t ctx, _type *dest, const _type *source, \
                             size_t nelems, int pe);                            \
  void shmem_ctx_##_tn##_get(shmem_ctx_t ctx, _type *dest, const _type *source, \
                             size_t nelems, int pe);                            \
  void shmem_ctx_##_tn##_p(shmem_ctx_t ctx, _type *dest, _type value, int pe);  \
  _type shmem_ctx_##_tn##_g(shmem_ctx_t ctx, const _type *source, int pe);      \
  void shmem_ctx_##_tn##_put_nbi(shmem_ctx_t ctx, _type *dest,                  \
                                 const _type *source, size_t nelems, int pe);   \
  void shmem_ctx_##_tn##_get_nbi(shmem_ctx_t ctx, _type *dest,                  \
                                 const _type *source, size_t nelems, int pe);
SHMEM_B200_RMA_TYPES(SHMEM_B200_DECL_COPY)
int shmem_fcollectmem(shmem_team_t team, void *dest, const void *source, size_t nelems);
/* collect: each PE passes its own nelems; dest gets the contributions
 * concatenated in member order (shcoll-shim.c:471-560) */
int shmem_collectmem(shmem_team_t team, void *dest, const void *source, size_t nelems);
int shmem_alltoallmem(shmem_team_t team, void *dest, const void *source, size_t nelems);
int shmem_alltoallsmem(shmem_team_t team, void *dest, const void *source, ptrdiff_t dst,
                       ptrdiff_t sst, size_t nelems);
int shmem_broadcastmem(shmem_team_t team, void *dest, const void *source, size_t nelems,
                       int PE_root);
void shmem_fcollect32(void *target, const void *source, size_t nelems, int PE_start,
                      int logPE_stride, int PE_size, long *pSync);
void shmem_fcollect64(void *target, const void *source, size_t nelems, int PE_start,
                      int logPE_stride, int PE_size, long *pSync);
void shmem_collect32(void *target, const void *source, size_t nelems, int PE_start,
                     int logPE_stride, int PE_size, long *pSync);
void shmem_collect64(void *target, const void *source, size_t nelems, int PE_start,
                     int logPE_stride, int PE_size, long *pSync);
void shmem_alltoall32(void *target, const void *source, size_t nelems, int PE_start,
                      int logPE_stride, int PE_size, long *pSync);
void shmem_alltoall64(void *target, const void *source, size_t nelems, int PE_start,
                      int logPE_stride, int PE_size, long *pSync);
void shmem_alltoalls32(void *target, const void *source, ptrdiff_t dst, ptrdiff_t sst,
                       size_t nelems, int PE_start, int logPE_stride, int PE_size, long *pSync);
void shmem_alltoalls64(void *target, const void *source, ptrdiff_t dst, ptrdiff_t sst,
                       size_t nelems, int PE_start, int logPE_stride, int PE_size, long *pSync);
void shmem_broadcast32(void *target, const void *source, size_t nelems, int PE_root,
                       int PE_start, int logPE_stride, int PE_size, long *pSync);
void shmem_broadcast64(void *target, const void *source, size_t nelems, int PE_root,
                       int PE_start, int logPE_stride, int PE_size, long *pSync);

/* ---- atomics (the files of src/api/atomics) ----------------------------- */
#define SHMEM_B200_DECL_AMO_STD(_type, _tn)                                     \
  _type shmem_##_tn##_atomic_fetch_add(_type *dest, _type value, int pe);      \
  void shmem_##_tn##_atomic_add(_type *dest, _type value, int pe);             \
  _type shmem_##_tn##_atomic_fetch_inc(_type *dest, int pe);                   \
  void shmem_##_tn##_atomic_inc(_type *dest, int pe);                          \
  _type shmem_##_tn##_atomic_compare_swap(_type *dest, _type cond,             \
                                          _type value, int pe);                 \
  _type shmem_ctx_##_tn##_atomic_fetch_add(shmem_ctx_t ctx, _type *dest,       \
                                           _type value, int pe);                \
  void shmem_ctx_##_tn##_atomic_add(shmem_ctx_t ctx, _type *dest, _type value, \
                                    int pe);                                    \
  _type shmem_ctx_##_tn##_atomic_fetch_inc(shmem_ctx_t ctx, _type *dest,       \
                                           int pe);                             \
  void shmem_ctx_##_tn##_atomic_inc(shmem_ctx_t ctx, _type *dest, int pe);     \
  _type shmem_ctx_##_tn##_atomic_compare_swap(shmem_ctx_t ctx, _type *dest,    \
                                              _type cond, _type value, int pe);
#define SHMEM_B200_DECL_AMO_EXT(_type, _tn)                                     \
  _type shmem_##_tn##_atomic_swap(_type *dest, _type value, int pe);           \
  void shmem_##_tn##_atomic_set(_type *dest, _type value, int pe);             \
  _type shmem_##_tn##_atomic_fetch(const _type *source, int pe);               \
  _type shmem_ctx_##_tn##_atomic_swap(shmem_ctx_t ctx, _type *dest,            \
                                      _type value, int pe);                     \
  void shmem_ctx_##_tn##_atomic_set(shmem_ctx_t ctx, _type *dest, _type value, \
                                    int pe);                                    \
  _type shmem_ctx_##_tn##_atomic_fetch(shmem_ctx_t ctx, const _type *source,   \
                                       int pe);
#define SHMEM_B200_DECL_AMO_BIT(_type, _tn)                                     \
  _type shmem_##_tn##_atomic_fetch_and(_type *dest, _type value, int pe);      \
  _type shmem_##_tn##_atomic_fetch_or(_type *dest, _type value, int pe);       \
  _type shmem_##_tn##_atomic_fetch_xor(_type *dest, _type value, int pe);      \
  void shmem_##_tn##_atomic_and(_type *dest, _type value, int pe);             \
  void shmem_##_tn##_atomic_or(_type *dest, _type value, int pe);              \
  void shmem_##_tn##_atomic_xor(_type *dest, _type value, int pe);             \
  _type shmem_ctx_##_tn##_atomic_fetch_and(shmem_ctx_t ctx, _type *dest,       \
                                           _type value, int pe);                \
  _type shmem_ctx_##_tn##_atomic_fetch_or(shmem_ctx_t ctx, _type *dest,        \
                                          _type value, int pe);                 \
  _type shmem_ctx_##_tn##_atomic_fetch_xor(shmem_ctx_t ctx, _type *dest,       \
                                           _type value, int pe);                \
  void shmem_ctx_##_tn##_atomic_and(shmem_ctx_t ctx, _type *dest, _type value, \
                                    int pe);                                    \
  void shmem_ctx_##_tn##_atomic_or(shmem_ctx_t ctx, _type *dest, _type value,  \
                                   int pe);                                     \
  void shmem_ctx_##_tn##_atomic_xor(shmem_ctx_t ctx, _type *dest, _type value, \
                                    int pe);
SHMEM_B200_AMO_STANDARD_TYPES(SHMEM_B200_DECL_AMO_STD)
SHMEM_B200_AMO_EXTENDED_TYPES(SHMEM_B200_DECL_AMO_EXT)
SHMEM_B200_AMO_BITWISE_TYPES(SHMEM_B200_DECL_AMO_BIT)

/* Non-blocking fetching atomics (api.h: shmem_<T>_atomic_fetch_add_nbi and
 * the family): *fetch holds the old value after the next shmem_quiet or
 * barrier.  They and the _nbi puts/gets between symmetric objects run
 * through the engine's serving loop. */
#define SHMEM_B200_DECL_AMO_NBI_STD(_type, _tn)                                 \
  void shmem_##_tn##_atomic_fetch_add_nbi(_type *fetch, _type *dest,           \
                                          _type value, int pe);                 \
  void shmem_##_tn##_atomic_fetch_inc_nbi(_type *fetch, _type *dest, int pe);  \
  void shmem_##_tn##_atomic_compare_swap_nbi(_type *fetch, _type *dest,        \
                                             _type cond, _type value, int pe);  \
  void shmem_ctx_##_tn##_atomic_fetch_add_nbi(shmem_ctx_t ctx, _type *fetch,   \
                                              _type *dest, _type value,         \
                                              int pe);                          \
  void shmem_ctx_##_tn##_atomic_fetch_inc_nbi(shmem_ctx_t ctx, _type *fetch,   \
                                              _type *dest, int pe);             \
  void shmem_ctx_##_tn##_atomic_compare_swap_nbi(shmem_ctx_t ctx,              \
                                                 _type *fetch, _type *dest,     \
                                                 _type cond, _type value,       \
                                                 int pe);
#define SHMEM_B200_DECL_AMO_NBI_EXT(_type, _tn)                                 \
  void shmem_##_tn##_atomic_swap_nbi(_type *fetch, _type *dest, _type value,   \
                                     int pe);                                   \
  void shmem_##_tn##_atomic_fetch_nbi(_type *fetch, const _type *source, int pe); \
  void shmem_ctx_##_tn##_atomic_swap_nbi(shmem_ctx_t ctx, _type *fetch,        \
                                         _type *dest, _type value, int pe);     \
  void shmem_ctx_##_tn##_atomic_fetch_nbi(shmem_ctx_t ctx, _type *fetch,       \
                                          const _type *source, int pe);
#define SHMEM_B200_DECL_AMO_NBI_BIT(_type, _tn)                                 \
  void shmem_##_tn##_atomic_fetch_and_nbi(_type *fetch, _type *dest,           \
                                          _type value, int pe);                 \
  void shmem_##_tn##_atomic_fetch_or_nbi(_type *fetch, _type *dest,            \
                                         _type value, int pe);                  \
  void shmem_##_tn##_atomic_fetch_xor_nbi(_type *fetch, _type *dest,           \
                                          _type value, int pe);                 \
  void shmem_ctx_##_tn##_atomic_fetch_and_nbi(shmem_ctx_t ctx, _type *fetch,   \
                                              _type *dest, _type value,         \
                                              int pe);                          \
  void shmem_ctx_##_tn##_atomic_fetch_or_nbi(shmem_ctx_t ctx, _type *fetch,    \
                                             _type *dest, _type value, int pe); \
  void shmem_ctx_##_tn##_atomic_fetch_xor_nbi(shmem_ctx_t ctx, _type *fetch,   \
                                              _type *dest, _type value,         \
                                              int pe);                          \
  /* declared by the reference's api.h with the fetching signature: the same \
   * operation as atomic_fetch_xor_nbi */                                       \
  void shmem_##_tn##_atomic_xor_nbi(_type *fetch, _type *dest, _type value,    \
                                    int pe);                                    \
  void shmem_ctx_##_tn##_atomic_xor_nbi(shmem_ctx_t ctx, _type *fetch,         \
                                        _type *dest, _type value, int pe);
SHMEM_B200_AMO_STANDARD_TYPES(SHMEM_B200_DECL_AMO_NBI_STD)
SHMEM_B200_AMO_EXTENDED_TYPES(SHMEM_B200_DECL_AMO_NBI_EXT)
SHMEM_B200_AMO_BITWISE_TYPES(SHMEM_B200_DECL_AMO_NBI_BIT)

/* ---- strided and signalled RMA (api.h:355-600, 714-1000) ----------------
 * iput/iget: dest[i*tst] = source[i*sst] for i < nelems (strides in
 * elements, >= 1), one side symmetric on `pe`.  put_signal: the data is
 * delivered, then *sig_addr on `pe` is set to or increased by `signal`
 * (sig_op SHMEM_SIGNAL_SET / SHMEM_SIGNAL_ADD); the _nbi forms complete
 * before they return. */
enum { SHMEM_SIGNAL_SET = 0, SHMEM_SIGNAL_ADD };
#define SHMEM_B200_DECL_RMA_STRIDED(_type, _tn)                                 \
  void shmem_##_tn##_iput(_type *dest, const _type *source, ptrdiff_t tst,     \
                          ptrdiff_t sst, size_t nelems, int pe);                \
  void shmem_##_tn##_iget(_type *dest, const _type *source, ptrdiff_t tst,     \
                          ptrdiff_t sst, size_t nelems, int pe);                \
  void shmem_ctx_##_tn##_iput(shmem_ctx_t ctx, _type *dest,                    \
                              const _type *source, ptrdiff_t tst,               \
                              ptrdiff_t sst, size_t nelems, int pe);            \
  void shmem_ctx_##_tn##_iget(shmem_ctx_t ctx, _type *dest,                    \
                              const _type *source, ptrdiff_t tst,               \
                              ptrdiff_t sst, size_t nelems, int pe);            \
  void shmem_##_tn##_put_signal(_type *dest, const _type *source,              \
                                size_t nelems, uint64_t *sig_addr,              \
                                uint64_t signal, int sig_op, int pe);           \
  void shmem_##_tn##_put_signal_nbi(_type *dest, const _type *source,          \
                                    size_t nelems, uint64_t *sig_addr,          \
                                    uint64_t signal, int sig_op, int pe);       \
  void shmem_ctx_##_tn##_put_signal(shmem_ctx_t ctx, _type *dest,              \
                                    const _type *source, size_t nelems,         \
                                    uint64_t *sig_addr, uint64_t signal,        \
                                    int sig_op, int pe);                        \
  void shmem_ctx_##_tn##_put_signal_nbi(shmem_ctx_t ctx, _type *dest,          \
                                        const _type *source, size_t nelems,     \
                                        uint64_t *sig_addr, uint64_t signal,    \
                                        int sig_op, int pe);
SHMEM_B200_RMA_TYPES(SHMEM_B200_DECL_RMA_STRIDED)
#define SHMEM_B200_DECL_RMA_SIZED(_bits)                                        \
  void shmem_put##_bits(void *dest, const void *source, size_t nelems, int pe); \
  void shmem_get##_bits(void *dest, const void *source, size_t nelems, int pe); \
  void shmem_put##_bits##_nbi(void *dest, const void *source, size_t nelems,   \
                              int pe);                                          \
  void shmem_get##_bits##_nbi(void *dest, const void *source, size_t nelems,   \
                              int pe);                                          \
  void shmem_iput##_bits(void *dest, const void *source, ptrdiff_t tst,        \
                         ptrdiff_t sst, size_t nelems, int pe);                 \
  void shmem_iget##_bits(void *dest, const void *source, ptrdiff_t tst,        \
                         ptrdiff_t sst, size_t nelems, int pe);                 \
  void shmem_ctx_put##_bits(shmem_ctx_t ctx, void *dest, const void *source,   \
                            size_t nelems, int pe);                             \
  void shmem_ctx_get##_bits(shmem_ctx_t ctx, void *dest, const void *source,   \
                            size_t nelems, int pe);                             \
  void shmem_ctx_put##_bits##_nbi(shmem_ctx_t ctx, void *dest,                 \
                                  const void *source, size_t nelems, int pe);   \
  void shmem_ctx_get##_bits##_nbi(shmem_ctx_t ctx, void *dest,                 \
                                  const void *source, size_t nelems, int pe);   \
  void shmem_ctx_iput##_bits(shmem_ctx_t ctx, void *dest, const void *source,  \
                             ptrdiff_t tst, ptrdiff_t sst, size_t nelems,       \
                             int pe);                                           \
  void shmem_ctx_iget##_bits(shmem_ctx_t ctx, void *dest, const void *source,  \
                             ptrdiff_t tst, ptrdiff_t sst, size_t nelems,       \
                             int pe);                                           \
  void shmem_put##_bits##_signal(void *dest, const void *source,               \
                                 size_t nelems, uint64_t *sig_addr,             \
                                 uint64_t signal, int sig_op, int pe);          \
  void shmem_put##_bits##_signal_nbi(void *dest, const void *source,           \
                                     size_t nelems, uint64_t *sig_addr,         \
                                     uint64_t signal, int sig_op, int pe);      \
  void shmem_ctx_put##_bits##_signal(shmem_ctx_t ctx, void *dest,              \
                                     const void *source, size_t nelems,         \
                                     uint64_t *sig_addr, uint64_t signal,       \
                                     int sig_op, int pe);                       \
  void shmem_ctx_put##_bits##_signal_nbi(shmem_ctx_t ctx, void *dest,          \
                                         const void *source, size_t nelems,     \
                                         uint64_t *sig_addr, uint64_t signal,   \
                                         int sig_op, int pe);
SHMEM_B200_DECL_RMA_SIZED(8)
SHMEM_B200_DECL_RMA_SIZED(16)
SHMEM_B200_DECL_RMA_SIZED(32)
SHMEM_B200_DECL_RMA_SIZED(64)
SHMEM_B200_DECL_RMA_SIZED(128)
void shmem_putmem_signal(void *dest, const void *source, size_t nelems, uint64_t *sig_addr,
                         uint64_t signal, int sig_op, int pe);
void shmem_putmem_signal_nbi(void *dest, const void *source, size_t nelems, uint64_t *sig_addr,
                             uint64_t signal, int sig_op, int pe);
void shmem_ctx_putmem_signal(shmem_ctx_t ctx, void *dest, const void *source, size_t nelems,
                             uint64_t *sig_addr, uint64_t signal, int sig_op, int pe);
void shmem_ctx_putmem_signal_nbi(shmem_ctx_t ctx, void *dest, const void *source, size_t nelems,
                                 uint64_t *sig_addr, uint64_t signal, int sig_op, int pe);
/* the signal word of the calling PE (api.h:1004-1046) */
uint64_t shmem_signal_fetch(const uint64_t *sig_addr);
uint64_t shmem_signal_wait_until(uint64_t *sig_addr, int cmp, uint64_t cmp_value);

/* ---- point-to-point synchronisation (api.h:1472-2015) --------------------
 * On symmetric variables of the calling PE, compared as their own type.
 * status (may be NULL) excludes element i when status[i] != 0.  test_any
 * and wait_until_any return the lowest index that compares true (SIZE_MAX
 * when there is none, or every element is excluded); test_some and
 * wait_until_some write the indices that compare true and return their
 * count.  The waits block until the condition holds; SHMEM_B200_WAIT_TIMEOUT
 * (seconds) bounds them (then shmemx_b200_last_status() is
 * B200SHM_ERR_TIMEOUT). */
#define SHMEM_B200_SYNC_TYPES(X)                                                \
  X(short, short) X(unsigned short, ushort) SHMEM_B200_AMO_STANDARD_TYPES(X)
#define SHMEM_B200_DECL_SYNC_ONE(_type, _tn)                                    \
  int shmem_##_tn##_test(_type *ivar, int cmp, _type cmp_value);               \
  void shmem_##_tn##_wait_until(_type *ivar, int cmp, _type cmp_value);        \
  void shmem_##_tn##_wait(_type *ivar, _type cmp_value);
#define SHMEM_B200_DECL_SYNC_VEC(_type, _tn)                                    \
  int shmem_##_tn##_test_all(_type *ivars, size_t nelems, const int *status,   \
                             int cmp, _type cmp_value);                         \
  size_t shmem_##_tn##_test_any(_type *ivars, size_t nelems,                   \
                                const int *status, int cmp, _type cmp_value);   \
  size_t shmem_##_tn##_test_some(_type *ivars, size_t nelems, size_t *indices, \
                                 const int *status, int cmp, _type cmp_value);  \
  int shmem_##_tn##_test_all_vector(_type *ivars, size_t nelems,               \
                                    const int *status, int cmp,                 \
                                    _type *cmp_values);                         \
  size_t shmem_##_tn##_test_any_vector(_type *ivars, size_t nelems,            \
                                       const int *status, int cmp,              \
                                       _type *cmp_values);                      \
  size_t shmem_##_tn##_test_some_vector(_type *ivars, size_t nelems,           \
                                        size_t *indices, const int *status,     \
                                        int cmp, _type *cmp_values);            \
  void shmem_##_tn##_wait_until_all(_type *ivars, size_t nelems,               \
                                    const int *status, int cmp,                 \
                                    _type cmp_value);                           \
  size_t shmem_##_tn##_wait_until_any(_type *ivars, size_t nelems,             \
                                      const int *status, int cmp,               \
                                      _type cmp_value);                         \
  size_t shmem_##_tn##_wait_until_some(_type *ivars, size_t nelems,            \
                                       size_t *indices, const int *status,      \
                                       int cmp, _type cmp_value);               \
  void shmem_##_tn##_wait_until_all_vector(_type *ivars, size_t nelems,        \
                                           const int *status, int cmp,          \
                                           _type *cmp_values);                  \
  size_t shmem_##_tn##_wait_until_any_vector(_type *ivars, size_t nelems,      \
                                             const int *status, int cmp,        \
                                             _type *cmp_values);                \
  size_t shmem_##_tn##_wait_until_some_vector(_type *ivars, size_t nelems,     \
                                              size_t *indices,                  \
                                              const int *status, int cmp,       \
                                              _type *cmp_values);
SHMEM_B200_SYNC_TYPES(SHMEM_B200_DECL_SYNC_ONE)
SHMEM_B200_AMO_STANDARD_TYPES(SHMEM_B200_DECL_SYNC_VEC)

/* ---- the atomics' names before OpenSHMEM 1.4 (api.h, deprecated) -------- */
#define SHMEM_B200_DECL_AMO_OLD(_type, _tn)                                     \
  _type shmem_##_tn##_fadd(_type *target, _type value, int pe);                \
  _type shmem_##_tn##_finc(_type *target, int pe);                             \
  void shmem_##_tn##_add(_type *target, _type value, int pe);                  \
  void shmem_##_tn##_inc(_type *target, int pe);                               \
  _type shmem_##_tn##_cswap(_type *target, _type cond, _type value, int pe);   \
  _type shmem_##_tn##_swap(_type *target, _type value, int pe);                \
  _type shmem_##_tn##_fetch(const _type *target, int pe);                      \
  void shmem_##_tn##_set(_type *target, _type value, int pe);
#define SHMEM_B200_DECL_AMO_OLD_EXT(_type, _tn)                                 \
  _type shmem_##_tn##_swap(_type *target, _type value, int pe);                \
  _type shmem_##_tn##_fetch(const _type *target, int pe);                      \
  void shmem_##_tn##_set(_type *target, _type value, int pe);
#define SHMEM_B200_AMO_OLD_TYPES(X) X(int, int) X(long, long) X(long long, longlong)
#define SHMEM_B200_AMO_OLD_EXT_TYPES(X) X(float, float) X(double, double)
SHMEM_B200_AMO_OLD_TYPES(SHMEM_B200_DECL_AMO_OLD)
SHMEM_B200_AMO_OLD_EXT_TYPES(SHMEM_B200_DECL_AMO_OLD_EXT)

#if !defined(__cplusplus) && defined(__STDC_VERSION__) && __STDC_VERSION__ >= 201112L && \
    !defined(SHMEM_B200_NO_GENERICS)
#include "shmem_generics.h"
#endif

#ifdef __cplusplus
}
#endif
#endif
