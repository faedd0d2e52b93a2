/*
 * The long double reductions of include/shmem.h as an SPMD program sees
 * them, 8 PEs run by shmemx_b200_run: shmem_longdouble_sum_reduce and
 * shmem_longdouble_prod_reduce over SHMEM_TEAM_WORLD, and the active-set
 * form shmem_longdouble_max_to_all.  Inputs (argv[1]): long double
 * in[8][N] for the sums, then mx[8][N] for the max, N = 300.  Output
 * (argv[2]): sum[8][N], prod[8][N], max[8][N] as every PE ends up with
 * them, then int32 status[8].  tests/test_spmd_gpu.py checks the value
 * bytes against the oracle.
 */
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "shmem.h"
#include "shmemx.h"

#define NP 8
#define N 300

static long double in_s[NP][N], in_m[NP][N];
static long double out_sum[NP][N], out_prod[NP][N], out_max[NP][N];
static int32_t status[NP];

static void pe_main(void *arg) {
  (void)arg;
  shmem_init();
  const int me = shmem_my_pe();
  int rc = 0;
  static long pSync[SHMEM_REDUCE_SYNC_SIZE];
  static long double pWrk[SHMEM_REDUCE_MIN_WRKDATA_SIZE];
  long double *src = shmem_malloc(N * sizeof(long double));
  long double *dst = shmem_malloc(N * sizeof(long double));
  memcpy(src, in_s[me], sizeof(in_s[me]));
  rc |= shmem_longdouble_sum_reduce(SHMEM_TEAM_WORLD, dst, src, N);
  memcpy(out_sum[me], dst, sizeof(out_sum[me]));
  rc |= shmem_longdouble_prod_reduce(SHMEM_TEAM_WORLD, dst, src, N);
  memcpy(out_prod[me], dst, sizeof(out_prod[me]));
  memcpy(src, in_m[me], sizeof(in_m[me]));
  shmem_longdouble_max_to_all(dst, src, N, 0, 0, NP, pWrk, pSync);
  rc |= shmemx_b200_last_status();
  memcpy(out_max[me], dst, sizeof(out_max[me]));
  status[me] = rc;
  shmem_free(src);
  shmem_free(dst);
  shmem_finalize();
}

int main(int argc, char **argv) {
  if (argc < 3) return 2;
  FILE *f = fopen(argv[1], "rb");
  if (!f) return 3;
  const size_t ok = fread(in_s, sizeof(in_s), 1, f) + fread(in_m, sizeof(in_m), 1, f);
  fclose(f);
  if (ok != 2) return 4;
  if (shmemx_b200_run(NP, pe_main, NULL) != 0) {
    fprintf(stderr, "shmemx_b200_run: %s\n", shmemx_b200_last_error());
    return 5;
  }
  f = fopen(argv[2], "wb");
  if (!f) return 6;
  fwrite(out_sum, sizeof(out_sum), 1, f);
  fwrite(out_prod, sizeof(out_prod), 1, f);
  fwrite(out_max, sizeof(out_max), 1, f);
  fwrite(status, sizeof(status), 1, f);
  fclose(f);
  return 0;
}
