/*
 * The C11 generic names (include/shmem_generics.h) and the rest of the
 * reference's surface that programs call by name, run as 8 PEs by
 * shmemx_b200_run; the program checks itself, prints one line per failed
 * check and "ok" when there is none.  tests/test_spmd_gpu.py runs it.
 *
 *  - RMA: shmem_put / get / p / g / iput / put_nbi on int, double, long long
 *    and unsigned char objects, with and without a context first;
 *  - atomics: fetch_add / add / inc / fetch / set / compare_swap / swap
 *    (long, float), the bitwise forms (unsigned int), a fetching _nbi form,
 *    a context form, and the pre-1.4 names (shmem_long_fadd, ...);
 *  - collectives: shmem_sum_reduce (float), shmem_max_reduce (long),
 *    shmem_xor_reduce (unsigned int), shmem_sum_to_all (int),
 *    shmem_fcollect / alltoall / broadcast (long long), shmem_sync in both
 *    forms;
 *  - shmem_wait_until / shmem_test on a flag another PE puts;
 *  - shmem_set_lock / shmem_clear_lock around a read-modify-write of a
 *    counter on PE 0 (every increment survives), shmem_test_lock;
 *  - shmem_realloc keeps the first bytes, shmem_addr_accessible,
 *    shmem_team_ptr, the pre-1.2 names, the version and name queries,
 *    shmem_initialized / shmem_finalized.
 */
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "shmem.h"
#include "shmemx.h"

#define NP 8
#define N 32

static int g_fail[NP];

#define CHECK(cond, ...)                                                       \
  do {                                                                         \
    if (!(cond)) {                                                             \
      printf("PE %d: ", me);                                                   \
      printf(__VA_ARGS__);                                                     \
      printf("\n");                                                            \
      g_fail[me]++;                                                            \
    }                                                                          \
  } while (0)

static long psync[SHMEM_REDUCE_SYNC_SIZE];
static int pwrk[SHMEM_REDUCE_MIN_WRKDATA_SIZE + N];

static void pe_main(void *arg) {
  (void)arg;
  shmem_init();
  const int me = shmem_my_pe();
  if (me < 0 || me >= NP) return;
  const int next = (me + 1) % NP, prev = (me + NP - 1) % NP;
  CHECK(shmem_initialized() == 1 && shmem_finalized() == 0, "initialized/finalized");

  /* ---- RMA ---- */
  int *ia = shmem_malloc(N * sizeof(int));
  double *da = shmem_malloc(N * sizeof(double));
  long long *la = shmem_malloc(N * sizeof(long long));
  unsigned char *ua = shmem_malloc(N);
  int isrc[N];
  double dsrc[N];
  unsigned char usrc[N];
  for (int i = 0; i < N; i++) {
    isrc[i] = me * 1000 + i;
    dsrc[i] = me + i * 0.5;
    usrc[i] = (unsigned char)(me * 16 + i);
    la[i] = -1;
  }
  shmem_barrier_all();
  shmem_put(ia, isrc, N, next);                       /* shmem_int_put */
  shmem_put(SHMEM_CTX_DEFAULT, da, dsrc, N, next);    /* shmem_ctx_double_put */
  shmem_put_nbi(ua, usrc, N, next);                   /* shmem_uchar_put_nbi */
  shmem_p(la, (long long)me * 7, next);               /* shmem_longlong_p */
  long long lsrc[4] = {me * 10LL, me * 10LL + 1, me * 10LL + 2, me * 10LL + 3};
  shmem_iput(la + 1, lsrc, 2, 1, 4, next);            /* la[1 + 2i] on next = lsrc[i] */
  shmem_quiet();
  shmem_barrier_all();
  for (int i = 0; i < N; i++) {
    CHECK(ia[i] == prev * 1000 + i, "put int ia[%d] = %d", i, ia[i]);
    CHECK(da[i] == prev + i * 0.5, "ctx put double da[%d]", i);
    CHECK(ua[i] == (unsigned char)(prev * 16 + i), "put_nbi uchar ua[%d]", i);
  }
  CHECK(la[0] == (long long)prev * 7, "p longlong la[0] = %lld", la[0]);
  for (int i = 0; i < 4; i++)
    CHECK(la[1 + 2 * i] == prev * 10LL + i && la[2 + 2 * i] == -1, "iput longlong [%d]", i);
  CHECK(shmem_g(ia, next) == me * 1000, "g int");
  CHECK(shmem_g((const double *)da, next) == me + 0.0, "g const double");
  CHECK(shmem_g(SHMEM_CTX_DEFAULT, ia + 1, next) == me * 1000 + 1, "ctx g int");
  int iget_local[N];
  shmem_get(iget_local, ia, N, prev);
  for (int i = 0; i < N; i++)
    CHECK(iget_local[i] == ((prev + NP - 1) % NP) * 1000 + i, "get int [%d]", i);
  shmem_barrier_all();

  /* ---- atomics ---- */
  long *ctr = shmem_calloc(4, sizeof(long));
  unsigned int *bits = shmem_calloc(1, sizeof(unsigned int));
  float *fw = shmem_calloc(1, sizeof(float));
  shmem_barrier_all();
  const long old = shmem_atomic_fetch_add(ctr, 1L, 0);
  CHECK(old >= 0 && old < NP, "fetch_add old %ld", old);
  shmem_atomic_add(ctr + 1, 2L, 0);
  shmem_atomic_inc(SHMEM_CTX_DEFAULT, ctr + 2, 0);
  shmem_atomic_fetch_xor(bits, 1u << me, 0);
  long nbi_old = -1;
  shmem_atomic_fetch_add_nbi(&nbi_old, ctr + 3, 10L, 0);
  shmem_long_fadd(ctr + 3, 1, 0); /* a pre-1.4 name */
  shmem_quiet();
  CHECK(nbi_old >= 0 && nbi_old <= 11L * NP, "fetch_add_nbi old %ld", nbi_old);
  shmem_barrier_all();
  CHECK(shmem_atomic_fetch(ctr, 0) == NP, "fetch: counter %ld", shmem_atomic_fetch(ctr, 0));
  CHECK(shmem_atomic_fetch((const long *)(ctr + 1), 0) == 2 * NP, "fetch const: add");
  CHECK(shmem_long_fetch(ctr + 2, 0) == NP, "inc via ctx");
  CHECK(shmem_atomic_fetch(ctr + 3, 0) == 11 * NP, "nbi fetch_add + fadd: %ld",
        shmem_atomic_fetch(ctr + 3, 0));
  CHECK(shmem_atomic_fetch(bits, 0) == (1u << NP) - 1, "fetch_xor bits %x",
        shmem_atomic_fetch(bits, 0));
  shmem_barrier_all();
  if (me == 0) {
    shmem_atomic_set(fw, 2.5f, 1);
    CHECK(shmem_atomic_swap(fw, 4.0f, 1) == 2.5f, "float swap");
    CHECK(shmem_atomic_compare_swap(ctr, (long)NP, 100L, 1) == 0, "cswap on PE 1 sees 0");
    CHECK(shmem_atomic_compare_swap(ctr, (long)NP, 100L, 0) == NP, "cswap on PE 0");
    CHECK(shmem_long_cswap(ctr, 100L, 7L, 0) == 100, "pre-1.4 cswap");
  }
  shmem_barrier_all();
  if (me == 1) CHECK(*fw == 4.0f, "float swap left %f", (double)*fw);

  /* ---- collectives ---- */
  float *fs = shmem_malloc(N * sizeof(float)), *fd = shmem_malloc(N * sizeof(float));
  long *ls = shmem_malloc(N * sizeof(long)), *ld = shmem_malloc(N * sizeof(long));
  unsigned int *us = shmem_malloc(N * sizeof(unsigned)), *ud = shmem_malloc(N * sizeof(unsigned));
  int *ts = shmem_malloc(N * sizeof(int)), *td = shmem_malloc(N * sizeof(int));
  long long *cs = shmem_malloc(N * sizeof(long long));
  long long *cd = shmem_malloc(NP * N * sizeof(long long));
  for (int i = 0; i < N; i++) {
    fs[i] = (float)(me + 1) * 0.25f + (float)i;
    ls[i] = (long)((me * 37 + i * 11) % 101) - 50;
    us[i] = (unsigned)(me * 2654435761u + (unsigned)i);
    ts[i] = me * i - 3;
    cs[i] = (long long)me << 32 | (long long)i;
  }
  for (int i = 0; i < SHMEM_REDUCE_SYNC_SIZE; i++) psync[i] = SHMEM_SYNC_VALUE;
  shmem_barrier_all();
  CHECK(shmem_sum_reduce(SHMEM_TEAM_WORLD, fd, fs, N) == 0, "sum_reduce float");
  CHECK(shmem_max_reduce(SHMEM_TEAM_WORLD, ld, ls, N) == 0, "max_reduce long");
  CHECK(shmem_xor_reduce(SHMEM_TEAM_WORLD, ud, us, N) == 0, "xor_reduce uint");
  shmem_sum_to_all(td, ts, N, 0, 0, NP, pwrk, psync);
  for (int i = 0; i < N; i++) {
    float fsum = 0.0f;
    long lmax = -1000;
    unsigned ux = 0;
    int tsum = 0;
    for (int p = 0; p < NP; p++) {
      fsum += (float)(p + 1) * 0.25f + (float)i;
      const long v = (long)((p * 37 + i * 11) % 101) - 50;
      lmax = v > lmax ? v : lmax;
      ux ^= (unsigned)(p * 2654435761u + (unsigned)i);
      tsum += p * i - 3;
    }
    /* quarter steps and small integers: every order of the sum is exact */
    CHECK(fd[i] == fsum, "sum_reduce float [%d] %f != %f", i, (double)fd[i], (double)fsum);
    CHECK(ld[i] == lmax, "max_reduce long [%d]", i);
    CHECK(ud[i] == ux, "xor_reduce uint [%d]", i);
    CHECK(td[i] == tsum, "sum_to_all int [%d]", i);
  }
  shmem_barrier_all();
  CHECK(shmem_fcollect(SHMEM_TEAM_WORLD, cd, cs, N) == 0, "fcollect longlong");
  for (int p = 0; p < NP; p++)
    for (int i = 0; i < N; i++)
      CHECK(cd[p * N + i] == ((long long)p << 32 | (long long)i), "fcollect [%d][%d]", p, i);
  shmem_barrier_all();
  long long *as = shmem_malloc(NP * 4 * sizeof(long long));
  for (int p = 0; p < NP; p++)
    for (int i = 0; i < 4; i++) as[p * 4 + i] = me * 100 + p * 10 + i;
  shmem_barrier_all();
  CHECK(shmem_alltoall(SHMEM_TEAM_WORLD, cd, as, 4) == 0, "alltoall longlong");
  for (int p = 0; p < NP; p++)
    for (int i = 0; i < 4; i++)
      CHECK(cd[p * 4 + i] == p * 100 + me * 10 + i, "alltoall [%d][%d]", p, i);
  shmem_barrier_all();
  CHECK(shmem_broadcast(SHMEM_TEAM_WORLD, cd, cs, N, 3) == 0, "broadcast longlong");
  if (me != 3)
    for (int i = 0; i < N; i++) CHECK(cd[i] == ((3LL << 32) | i), "broadcast [%d]", i);
  shmem_sync(SHMEM_TEAM_WORLD);
  shmem_sync(0, 0, NP, psync);

  /* ---- point-to-point synchronisation ---- */
  int *flag = shmem_calloc(1, sizeof(int));
  shmem_barrier_all();
  shmem_p(flag, me + 1, next);
  shmem_wait_until(flag, SHMEM_CMP_EQ, prev + 1);
  CHECK(shmem_test(flag, SHMEM_CMP_EQ, prev + 1) == 1, "test after wait_until");
  shmem_barrier_all();

  /* ---- locks ---- */
  long *lock = shmem_calloc(1, sizeof(long));
  long *count = shmem_calloc(1, sizeof(long));
  shmem_barrier_all();
  for (int k = 0; k < 3; k++) {
    shmem_set_lock(lock);
    const long c = shmem_g(count, 0); /* a plain read-modify-write, held by the lock */
    shmem_p(count, c + 1, 0);
    shmem_clear_lock(lock);
  }
  shmem_barrier_all();
  CHECK(shmem_g(count, 0) == 3 * NP, "locked increments %ld of %d", shmem_g(count, 0), 3 * NP);
  if (me == 0) {
    CHECK(shmem_test_lock(lock) == 0, "test_lock on a free lock");
    CHECK(shmem_test_lock(lock) == 1, "test_lock on a held lock");
    shmem_clear_lock(lock);
  }
  shmem_barrier_all();

  /* ---- allocation and queries ---- */
  int *r = shmem_malloc(16 * sizeof(int));
  for (int i = 0; i < 16; i++) r[i] = me * 100 + i;
  int *r2 = shmem_realloc(r, 64 * sizeof(int));
  CHECK(r2 != NULL, "realloc");
  if (r2)
    for (int i = 0; i < 16; i++) CHECK(r2[i] == me * 100 + i, "realloc kept [%d]", i);
  CHECK(shmem_addr_accessible(r2, next) == 1, "addr_accessible symmetric");
  CHECK(shmem_team_ptr(SHMEM_TEAM_WORLD, r2, next) == shmem_ptr(r2, next), "team_ptr");
  CHECK(_my_pe() == me && _num_pes() == NP, "pre-1.2 _my_pe / _num_pes");
  long *old_style = shmalloc(8 * sizeof(long));
  CHECK(old_style != NULL, "shmalloc");
  shfree(old_style);
  CHECK(shmem_addr_accessible(isrc, next) == 0, "addr_accessible stack");
  int maj = 0, min = 0, ver = 0;
  char name[SHMEM_MAX_NAME_LEN];
  shmem_info_get_version(&maj, &min);
  shmem_info_get_version_number(&ver);
  shmem_info_get_name(name);
  CHECK(maj == SHMEM_MAJOR_VERSION && min == SHMEM_MINOR_VERSION && ver == maj * 100 + min,
        "version %d.%d (%d)", maj, min, ver);
  CHECK(strcmp(name, SHMEM_VENDOR_STRING) == 0, "name '%s'", name);
  int provided = -1;
  shmem_query_thread(&provided);
  CHECK(provided >= SHMEM_THREAD_SINGLE && provided <= SHMEM_THREAD_MULTIPLE, "query_thread");
  shmem_free(r2);
  shmem_finalize();
  CHECK(shmem_finalized() == 1 && shmem_initialized() == 0, "finalized");
}

int main(void) {
  if (shmemx_b200_run(NP, pe_main, NULL) != 0) {
    fprintf(stderr, "shmemx_b200_run: %s\n", shmemx_b200_last_error());
    return 5;
  }
  int n = 0;
  for (int p = 0; p < NP; p++) n += g_fail[p];
  if (n) {
    printf("%d failed checks\n", n);
    return 1;
  }
  printf("ok\n");
  return 0;
}
