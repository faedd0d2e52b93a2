/*
 * An OpenSHMEM program written against include/shmem.h only, run as 8 PEs
 * by shmemx_b200_run.  It reads seeded inputs from argv[1], runs the hot-path
 * calls the way an SPMD program does (every PE calls, with its own symmetric
 * pointers), and writes what every PE ends up with to argv[2]; the pytest
 * driver (tests/test_spmd_gpu.py) checks it against the oracle.
 *
 * Layout of the input file (all little-endian, PE-major):
 *   int32  red[8][1024]   config-1 int32 sum_reduce input
 *   int64  fc[8][256]     config-1 fcollect64 input
 *   float  fs[8][4096]    float sum input (rec_dbl order)
 *   double dm[8][512]     double max input (NaN / signed zeros included)
 *   uint8  a2a[8][8*96]   alltoallmem input (96-byte blocks)
 *   int64  as[8][8*5*3]   alltoalls64 input (n=5, sst=3, dst=2)
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "shmem.h"
#include "shmemx.h"

#define NP 8
#define NR 1024
#define NFC 256
#define NFS 4096
#define NDM 512
#define BLK 96
#define NAS 5

static int32_t in_red[NP][NR];
static int64_t in_fc[NP][NFC];
static float in_fs[NP][NFS];
static double in_dm[NP][NDM];
static uint8_t in_a2a[NP][NP * BLK];
static int64_t in_as[NP][NP * NAS * 3];

static struct {
  int32_t red[NP][NR];
  int64_t fc[NP][NP * NFC];
  float fs[NP][NFS];
  double dm[NP][NDM];
  int32_t toall[NP][NR];
  int32_t team_even[NP][NR]; /* rows of odd PEs stay zero */
  uint8_t a2a[NP][NP * BLK];
  int64_t as[NP][NP * NAS * 2];
  int64_t bcast[NP][NFC];
  int64_t amo_final;
  int64_t amo_fetched[NP][4];
  int32_t team_info[NP][4]; /* my_pe in even team, n_pes, x/y of a 2d split */
  int32_t status[NP];
} out;

static void pe_main(void *arg) {
  (void)arg;
  shmem_init();
  const int me = shmem_my_pe();
  int rc = 0;
  static long pSync[SHMEM_REDUCE_SYNC_SIZE]; /* unused by the engine; kept as a real program would */
  static int pWrk[SHMEM_REDUCE_MIN_WRKDATA_SIZE];

  /* config 1: int32 sum_reduce over WORLD, then fcollect64, then barrier_all */
  int32_t *rs = shmem_malloc(NR * sizeof(int32_t));
  int32_t *rd = shmem_malloc(NR * sizeof(int32_t));
  memcpy(rs, in_red[me], sizeof(in_red[me]));
  rc |= shmem_int32_sum_reduce(SHMEM_TEAM_WORLD, rd, rs, NR);
  memcpy(out.red[me], rd, sizeof(out.red[me]));

  int64_t *fs = shmem_malloc(NFC * sizeof(int64_t));
  int64_t *fd = shmem_malloc(NP * NFC * sizeof(int64_t));
  memcpy(fs, in_fc[me], sizeof(in_fc[me]));
  shmem_fcollect64(fd, fs, NFC, 0, 0, NP, pSync);
  rc |= shmemx_b200_last_status();
  memcpy(out.fc[me], fd, sizeof(out.fc[me]));
  shmem_barrier_all();

  /* float sum (rec_dbl order) and double max with NaN / signed zeros */
  float *xs = shmem_malloc(NFS * sizeof(float));
  float *xd = shmem_malloc(NFS * sizeof(float));
  memcpy(xs, in_fs[me], sizeof(in_fs[me]));
  rc |= shmem_float_sum_reduce(SHMEM_TEAM_WORLD, xd, xs, NFS);
  memcpy(out.fs[me], xd, sizeof(out.fs[me]));
  double *ds = shmem_malloc(NDM * sizeof(double));
  double *dd = shmem_malloc(NDM * sizeof(double));
  memcpy(ds, in_dm[me], sizeof(in_dm[me]));
  rc |= shmem_double_max_reduce(SHMEM_TEAM_WORLD, dd, ds, NDM);
  memcpy(out.dm[me], dd, sizeof(out.dm[me]));

  /* active-set form: int sum to_all over all PEs */
  shmem_int_sum_to_all(rd, rs, NR, 0, 0, NP, pWrk, pSync);
  rc |= shmemx_b200_last_status();
  memcpy(out.toall[me], rd, sizeof(out.toall[me]));

  /* a team of the even PEs (split_strided) reduces on its own */
  shmem_team_t even;
  rc |= shmem_team_split_strided(SHMEM_TEAM_WORLD, 0, 2, NP / 2, NULL, 0, &even);
  if (even != SHMEM_TEAM_INVALID) {
    rc |= shmem_int32_sum_reduce(even, rd, rs, NR);
    memcpy(out.team_even[me], rd, sizeof(out.team_even[me]));
    out.team_info[me][0] = shmem_team_my_pe(even);
    out.team_info[me][1] = shmem_team_n_pes(even);
    rc |= shmem_team_sync(even);
  } else {
    out.team_info[me][0] = -1;
    out.team_info[me][1] = -1;
  }
  shmem_team_t xt, yt;
  rc |= shmem_team_split_2d(SHMEM_TEAM_WORLD, 4, NULL, 0, &xt, NULL, 0, &yt);
  out.team_info[me][2] = shmem_team_my_pe(xt) * 100 + shmem_team_n_pes(xt);
  out.team_info[me][3] = shmem_team_my_pe(yt) * 100 + shmem_team_n_pes(yt);

  /* alltoallmem and alltoalls64 */
  uint8_t *as = shmem_malloc(NP * BLK), *ad = shmem_malloc(NP * BLK);
  memcpy(as, in_a2a[me], sizeof(in_a2a[me]));
  rc |= shmem_alltoallmem(SHMEM_TEAM_WORLD, ad, as, BLK);
  memcpy(out.a2a[me], ad, sizeof(out.a2a[me]));
  int64_t *ss = shmem_malloc(sizeof(in_as[me])), *sd = shmem_calloc(NP * NAS * 2, sizeof(int64_t));
  memcpy(ss, in_as[me], sizeof(in_as[me]));
  rc |= shmem_int64_alltoalls(SHMEM_TEAM_WORLD, sd, ss, 2, 3, NAS);
  memcpy(out.as[me], sd, sizeof(out.as[me]));

  /* broadcast from team member 3 */
  int64_t *bd = shmem_calloc(NFC, sizeof(int64_t));
  rc |= shmem_int64_broadcast(SHMEM_TEAM_WORLD, bd, fs, NFC, 3);
  memcpy(out.bcast[me], bd, sizeof(out.bcast[me]));

  /* atomics: every PE adds to a counter on PE 0 */
  int64_t *ctr = shmem_calloc(1, sizeof(int64_t));
  for (int k = 0; k < 4; k++) out.amo_fetched[me][k] = shmem_int64_atomic_fetch_add(ctr, 1, 0);
  shmem_barrier_all();
  if (me == 0) out.amo_final = shmem_int64_atomic_fetch(ctr, 0);

  out.status[me] = rc;
  shmem_free(ctr);
  shmem_finalize();
}

int main(int argc, char **argv) {
  if (argc < 3) return 2;
  FILE *f = fopen(argv[1], "rb");
  if (!f) return 3;
  size_t ok = fread(in_red, sizeof(in_red), 1, f) + fread(in_fc, sizeof(in_fc), 1, f) +
              fread(in_fs, sizeof(in_fs), 1, f) + fread(in_dm, sizeof(in_dm), 1, f) +
              fread(in_a2a, sizeof(in_a2a), 1, f) + fread(in_as, sizeof(in_as), 1, f);
  fclose(f);
  if (ok != 6) return 4;
  if (shmemx_b200_run(NP, pe_main, NULL) != 0) {
    fprintf(stderr, "shmemx_b200_run: %s\n", shmemx_b200_last_error());
    return 5;
  }
  f = fopen(argv[2], "wb");
  if (!f) return 6;
  fwrite(&out, sizeof(out), 1, f);
  fclose(f);
  return 0;
}
