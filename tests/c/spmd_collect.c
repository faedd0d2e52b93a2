/*
 * The three OpenSHMEM collect forms, run as 6 PEs by shmemx_b200_run: each
 * PE contributes its own number of elements (PE i: 3*(i+1) int32 on WORLD,
 * 2*i + 1 int64 over the active set of the even PEs, 5 + i bytes through
 * collectmem on WORLD).  Writes what every PE receives to argv[1]; the
 * pytest driver (tests/test_spmd_gpu.py) checks it against the oracle.
 */
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "shmem.h"
#include "shmemx.h"

#define NP 6
#define W32 (3 * NP * (NP + 1) / 2) /* 63 int32 in all */
#define W64 (1 + 5 + 9)             /* PEs 0, 2, 4 */
#define WM (5 * NP + NP * (NP - 1) / 2)

static struct {
  int32_t c32[NP][W32];
  int64_t c64[NP][W64]; /* rows of odd PEs stay zero */
  uint8_t cm[NP][WM];
  int32_t status[NP];
} out;

static void pe_main(void *arg) {
  (void)arg;
  shmem_init();
  const int me = shmem_my_pe();
  if (me < 0 || me >= NP) return;
  int rc = 0;
  static long pSync[SHMEM_COLLECT_SYNC_SIZE];
  int32_t *s32 = shmem_malloc(3 * NP * sizeof(int32_t));
  int32_t *d32 = shmem_malloc(W32 * sizeof(int32_t));
  for (int i = 0; i < 3 * (me + 1); i++) s32[i] = me * 1000 + i;
  rc |= shmem_int32_collect(SHMEM_TEAM_WORLD, d32, s32, 3 * (me + 1));
  memcpy(out.c32[me], d32, sizeof(out.c32[me]));

  int64_t *s64 = shmem_malloc(NP * 2 * sizeof(int64_t));
  int64_t *d64 = shmem_calloc(W64, sizeof(int64_t));
  for (int i = 0; i < 2 * me + 1; i++) s64[i] = ((int64_t)me << 40) | i;
  shmem_barrier_all();
  if (me % 2 == 0) {
    shmem_collect64(d64, s64, 2 * me + 1, 0, 1, NP / 2, pSync);
    rc |= shmemx_b200_last_status();
    memcpy(out.c64[me], d64, sizeof(out.c64[me]));
  }
  shmem_barrier_all();

  uint8_t *sm = shmem_malloc(5 + NP);
  uint8_t *dm = shmem_malloc(WM);
  for (int i = 0; i < 5 + me; i++) sm[i] = (uint8_t)(me * 16 + i);
  rc |= shmem_collectmem(SHMEM_TEAM_WORLD, dm, sm, 5 + me);
  memcpy(out.cm[me], dm, sizeof(out.cm[me]));
  out.status[me] = rc;
  shmem_finalize();
}

int main(int argc, char **argv) {
  if (argc < 2) return 2;
  if (shmemx_b200_run(NP, pe_main, NULL) != 0) {
    fprintf(stderr, "shmemx_b200_run: %s\n", shmemx_b200_last_error());
    return 5;
  }
  FILE *f = fopen(argv[1], "wb");
  if (!f) return 6;
  fwrite(&out, sizeof(out), 1, f);
  fclose(f);
  return 0;
}
