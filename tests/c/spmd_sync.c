/*
 * Point-to-point synchronisation and the strided and signalled puts, run as
 * 8 PEs by shmemx_b200_run; the program checks itself, prints one line per
 * failed check and "ok" when there is none.  tests/test_spmd_gpu.py runs it.
 *
 *  - shmem_int64_iput / iget, shmem_iput32 / shmem_iget128 (strided);
 *  - shmem_int64_put_signal (ADD) and shmem_putmem_signal_nbi (SET) waited
 *    for with shmem_signal_wait_until, read with shmem_signal_fetch;
 *  - shmem_long_test_all/any/some[_vector] and wait_until_all/any/some[_vector]
 *    on flags that the other PEs set one by one, with a status mask;
 *  - shmem_int_wait_until / shmem_int_test on a word another PE puts;
 *  - unsigned comparison (a 64-bit value above 2^63 is greater than 1);
 *  - a collective whose members pass different counts fails on EVERY member
 *    with the same message.
 */
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <time.h>

#include "shmem.h"
#include "shmemx.h"

#define NP 8
#define NI 16
#define NS 64

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

static void nap_ms(int ms) {
  struct timespec ts = {0, ms * 1000000L};
  nanosleep(&ts, NULL);
}

static void pe_main(void *arg) {
  (void)arg;
  shmem_init();
  const int me = shmem_my_pe();
  if (me < 0 || me >= NP) return;
  const int next = (me + 1) % NP, prev = (me + NP - 1) % NP;

  /* ---- strided puts and gets ---- */
  int64_t *src = shmem_malloc(3 * NI * sizeof(int64_t));
  int64_t *dst = shmem_malloc(2 * NI * sizeof(int64_t));
  int32_t *s32 = shmem_malloc(4 * NI * sizeof(int32_t));
  int32_t *d32 = shmem_calloc(2 * NI, sizeof(int32_t));
  for (int i = 0; i < 3 * NI; i++) src[i] = (int64_t)me * 1000 + i;
  for (int i = 0; i < 2 * NI; i++) dst[i] = -1;
  for (int i = 0; i < 4 * NI; i++) s32[i] = me * 100 + i;
  shmem_barrier_all();
  shmem_int64_iput(dst, src, 2, 3, NI, next); /* dst[2i] on next = src[3i] */
  shmem_iput32(d32, s32, 2, 4, NI, next);     /* d32[2i] on next = s32[4i] */
  CHECK(shmemx_b200_last_status() == 0, "iput status %d", shmemx_b200_last_status());
  shmem_barrier_all();
  for (int i = 0; i < NI; i++) {
    CHECK(dst[2 * i] == (int64_t)prev * 1000 + 3 * i, "iput dst[%d] = %lld", 2 * i,
          (long long)dst[2 * i]);
    CHECK(dst[2 * i + 1] == -1, "iput touched dst[%d]", 2 * i + 1);
    CHECK(d32[2 * i] == prev * 100 + 4 * i && d32[2 * i + 1] == 0, "iput32 d32[%d]", 2 * i);
  }
  int64_t loc[NI];
  const int far = (me + 2) % NP;
  shmem_int64_iget(loc, src, 1, 2, NI, far); /* loc[i] = src[2i] on far */
  for (int i = 0; i < NI; i++)
    CHECK(loc[i] == (int64_t)far * 1000 + 2 * i, "iget loc[%d] = %lld", i, (long long)loc[i]);
  int64_t pairs[2 * 4];                      /* 128-bit elements: 2 int64 each */
  shmem_iget128(pairs, src, 1, 3, 4, far);   /* pairs[i] = 128-bit element 3i of src */
  for (int i = 0; i < 4; i++)
    CHECK(pairs[2 * i] == (int64_t)far * 1000 + 6 * i &&
              pairs[2 * i + 1] == (int64_t)far * 1000 + 6 * i + 1,
          "iget128 element %d", i);
  shmem_barrier_all();

  /* ---- put with signal ---- */
  int64_t *sd = shmem_calloc(NS, sizeof(int64_t));
  uint64_t *sig = shmem_calloc(2, sizeof(uint64_t));
  int64_t data[NS];
  for (int i = 0; i < NS; i++) data[i] = (int64_t)me * 7 + i;
  shmem_barrier_all();
  shmem_int64_put_signal(sd, data, NS, &sig[0], 1, SHMEM_SIGNAL_ADD, next);
  const uint64_t seen = shmem_signal_wait_until(&sig[0], SHMEM_CMP_GE, 1);
  CHECK(seen == 1, "signal_wait_until returned %llu", (unsigned long long)seen);
  for (int i = 0; i < NS; i++)
    CHECK(sd[i] == (int64_t)prev * 7 + i, "put_signal data[%d] = %lld", i, (long long)sd[i]);
  shmem_barrier_all();
  shmem_putmem_signal_nbi(sd, data, 8 * sizeof(int64_t), &sig[1], 7, SHMEM_SIGNAL_SET, prev);
  CHECK(shmem_signal_wait_until(&sig[1], SHMEM_CMP_EQ, 7) == 7, "signal SET");
  CHECK(shmem_signal_fetch(&sig[1]) == 7 && shmem_signal_fetch(&sig[0]) == 1, "signal_fetch");
  for (int i = 0; i < 8; i++)
    CHECK(sd[i] == (int64_t)next * 7 + i, "putmem_signal data[%d]", i);
  shmem_barrier_all();

  /* ---- tests and waits on a vector of flags on PE 0 ---- */
  long *flags = shmem_calloc(NP, sizeof(long));
  int *go = shmem_calloc(1, sizeof(int));
  shmem_barrier_all();
  if (me == 0) {
    size_t idx[NP];
    CHECK(shmem_long_test_any(flags, NP, NULL, SHMEM_CMP_GT, 0) == SIZE_MAX, "test_any none");
    CHECK(shmem_long_test_all(flags, NP, NULL, SHMEM_CMP_EQ, 0) == 1, "test_all zero");
    CHECK(shmem_long_test_some(flags, NP, idx, NULL, SHMEM_CMP_NE, 0) == 0, "test_some none");
  }
  shmem_barrier_all();
  if (me != 0) {
    nap_ms(2 * me);
    shmem_long_atomic_set(&flags[me], me + 1, 0);
  } else {
    int status[NP] = {1}; /* flags[0] is never set: excluded */
    const size_t first = shmem_long_wait_until_any(flags, NP, status, SHMEM_CMP_GT, 0);
    CHECK(first >= 1 && first < NP, "wait_until_any returned %zu", first);
    shmem_long_wait_until_all(flags, NP, status, SHMEM_CMP_GT, 0);
    long want[NP];
    for (int i = 0; i < NP; i++) want[i] = i + 1;
    CHECK(shmem_long_test_all_vector(flags, NP, status, SHMEM_CMP_EQ, want) == 1,
          "test_all_vector");
    CHECK(shmem_long_test_all(flags, NP, NULL, SHMEM_CMP_GT, 0) == 0, "test_all unmasked");
    size_t idx[NP];
    const size_t n = shmem_long_wait_until_some(flags, NP, idx, status, SHMEM_CMP_GE, 1);
    CHECK(n == NP - 1, "wait_until_some count %zu", n);
    for (size_t k = 0; k < n; k++) CHECK(idx[k] == k + 1, "wait_until_some index %zu", k);
    want[3] = 99;
    CHECK(shmem_long_test_any_vector(flags, NP, status, SHMEM_CMP_NE, want) == 3,
          "test_any_vector");
    CHECK(shmem_long_test_some_vector(flags, NP, idx, status, SHMEM_CMP_EQ, want) == NP - 2,
          "test_some_vector");
    CHECK(shmem_long_wait_until_any_vector(flags, NP, status, SHMEM_CMP_LT, want) == 3,
          "wait_until_any_vector");
    int all_out[NP];
    for (int i = 0; i < NP; i++) all_out[i] = 1;
    CHECK(shmem_long_wait_until_any(flags, NP, all_out, SHMEM_CMP_GT, 0) == SIZE_MAX,
          "wait_until_any over an all-excluded vector");
    shmem_int_p(go, 5, 1);
  }
  if (me == 1) {
    shmem_int_wait_until(go, SHMEM_CMP_EQ, 5);
    CHECK(shmem_int_test(go, SHMEM_CMP_EQ, 5) == 1 && *go == 5, "int wait_until");
    CHECK(shmem_int_test(go, SHMEM_CMP_LT, 5) == 0, "int test LT");
  }
  shmem_barrier_all();

  /* ---- unsigned comparison ---- */
  uint64_t *u = shmem_malloc(sizeof(uint64_t));
  *u = 0;
  shmem_uint64_p(u, (uint64_t)1 << 63, me);
  CHECK(shmem_uint64_test(u, SHMEM_CMP_GT, 1) == 1, "uint64 compares unsigned");
  shmem_barrier_all();

  /* ---- a collective with mismatched arguments fails everywhere ---- */
  int64_t *r = shmem_calloc(NS, sizeof(int64_t));
  int64_t *rs = shmem_calloc(NS, sizeof(int64_t));
  shmem_barrier_all();
  const int rc = shmem_int64_sum_reduce(SHMEM_TEAM_WORLD, r, rs, me == 3 ? NS - 1 : NS);
  const char *msg = shmemx_b200_last_error();
  CHECK(rc != 0, "mismatched reduce returned 0");
  CHECK(msg && strstr(msg, "different arguments") != NULL, "error message '%s'", msg ? msg : "");
  shmem_barrier_all();
  CHECK(shmem_int64_sum_reduce(SHMEM_TEAM_WORLD, r, rs, NS) == 0, "reduce after a failure");
  shmem_finalize();
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
