/*
 * The non-blocking forms, run as 8 PEs by shmemx_b200_run: every PE puts
 * (shmem_int64_put_nbi) its 64-element block into the next PE's dest, adds
 * 1 to a counter on PE 0 sixteen times with shmem_int64_atomic_fetch_add_nbi,
 * quiets, then gets (shmem_int64_get_nbi) the previous PE's source; a put
 * from a non-symmetric local buffer takes the blocking path.  Writes what
 * every PE ends up with to argv[1]; tests/test_spmd_gpu.py checks it.
 */
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "shmem.h"
#include "shmemx.h"

#define NP 8
#define BLK 64
#define NADD 16

static struct {
  int64_t dst[NP][NP * BLK];
  int64_t got[NP][BLK];
  int64_t fetched[NP][NADD];
  uint8_t loc[NP][NP * 32];
  int64_t counter;
  int32_t status[NP];
} out;

static void pe_main(void *arg) {
  (void)arg;
  shmem_init();
  const int me = shmem_my_pe();
  if (me < 0 || me >= NP) return;
  int64_t *src = shmem_malloc(BLK * sizeof(int64_t));
  int64_t *dst = shmem_calloc(NP * BLK, sizeof(int64_t));
  int64_t *got = shmem_calloc(BLK, sizeof(int64_t));
  int64_t *ctr = shmem_calloc(1, sizeof(int64_t));
  uint8_t *loc = shmem_calloc(NP * 32, 1);
  for (int i = 0; i < BLK; i++) src[i] = (int64_t)me * 1000 + i;
  shmem_barrier_all();

  shmem_int64_put_nbi(dst + me * BLK, src, BLK, (me + 1) % NP);
  int64_t fetched[NADD];
  for (int k = 0; k < NADD; k++) shmem_int64_atomic_fetch_add_nbi(&fetched[k], ctr, 1, 0);
  uint8_t tmp[32]; /* not symmetric: the blocking path */
  for (int i = 0; i < 32; i++) tmp[i] = (uint8_t)(me * 32 + i);
  shmem_putmem_nbi(loc + me * 32, tmp, 32, 0);
  shmem_quiet();
  int rc = shmemx_b200_last_status();
  shmem_barrier_all();

  shmem_int64_get_nbi(got, src, BLK, (me + NP - 1) % NP);
  shmem_quiet();
  rc |= shmemx_b200_last_status();

  memcpy(out.dst[me], dst, sizeof(out.dst[me]));
  memcpy(out.got[me], got, sizeof(out.got[me]));
  memcpy(out.fetched[me], fetched, sizeof(out.fetched[me]));
  memcpy(out.loc[me], loc, sizeof(out.loc[me]));
  shmem_barrier_all();
  if (me == 0) out.counter = *ctr;
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
