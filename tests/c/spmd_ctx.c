/*
 * Communication contexts, run as 8 PEs by shmemx_b200_run.  Every PE:
 *  - issues sixteen shmem_ctx_int64_atomic_fetch_add_nbi on context A (a
 *    counter on PE 0) and one shmem_ctx_int64_put_nbi on context B (its
 *    block into the next PE), then quiets A alone: A has nothing pending
 *    and its fetched values are in place, B still holds its put; then
 *    quiets B;
 *  - on the even PEs, makes a context of the team {0,2,4,6}: its PE numbers
 *    are team-relative (a put to team PE k+1, a fetch_or on team PE 1, which
 *    is PE 2), and shmem_ctx_get_team gives the team back; the odd PEs,
 *    outside the team, are refused a context of SHMEM_TEAM_INVALID;
 *  - destroys a context with a fetch_add_nbi still pending: destroying it
 *    completes it;
 *  - uses SHMEM_CTX_INVALID (refused with an error status) and
 *    SHMEM_CTX_DEFAULT (never destroyed), and shmem_ctx_int64_p / _g.
 * Writes what every PE ends up with to argv[1]; tests/test_spmd_gpu.py
 * checks it.
 */
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "shmem.h"
#include "shmemx.h"

#define NP 8
#define BLK 64
#define NADD 16
#define TP 4 /* the even PEs' team */

static struct {
  int64_t dst[NP][NP * BLK];
  int64_t tdst[NP][TP * BLK];
  int64_t fa[NP][NADD];
  int64_t fc[NP];
  int64_t g[NP];
  int64_t counter, counter2, bits;
  int32_t pending[NP][6]; /* A, B before; A, B after quiet(A); B after quiet(B); default */
  int32_t create_rc[NP];  /* shmem_ctx_create of A, B and the destroyed context */
  int32_t team_rc[NP];    /* the team context: 0 on even PEs, nonzero on odd */
  int32_t team_ok[NP];    /* get_team gave the team back, and the handle was valid */
  int32_t invalid_status[NP];
  int32_t status[NP];
} out;

static void pe_main(void *arg) {
  (void)arg;
  shmem_init();
  const int me = shmem_my_pe();
  if (me < 0 || me >= NP) return;
  int64_t *src = shmem_malloc(BLK * sizeof(int64_t));
  int64_t *dst = shmem_calloc(NP * BLK, sizeof(int64_t));
  int64_t *tdst = shmem_calloc(TP * BLK, sizeof(int64_t));
  int64_t *ctr = shmem_calloc(3, sizeof(int64_t)); /* counter, counter2, bits */
  int64_t *gval = shmem_calloc(1, sizeof(int64_t));
  for (int i = 0; i < BLK; i++) src[i] = (int64_t)me * 1000 + i;
  shmem_team_t even = SHMEM_TEAM_INVALID;
  shmem_team_split_strided(SHMEM_TEAM_WORLD, 0, 2, TP, NULL, 0, &even);
  shmem_barrier_all();

  shmem_ctx_t a = SHMEM_CTX_INVALID, b = SHMEM_CTX_INVALID, c = SHMEM_CTX_INVALID;
  int crc = shmem_ctx_create(SHMEM_CTX_PRIVATE, &a);
  crc |= shmem_ctx_create(0, &b);
  int64_t fa[NADD];
  for (int k = 0; k < NADD; k++) shmem_ctx_int64_atomic_fetch_add_nbi(a, &fa[k], ctr, 1, 0);
  shmem_ctx_int64_put_nbi(b, dst + me * BLK, src, BLK, (me + 1) % NP);
  out.pending[me][0] = shmemx_b200_ctx_pending(a);
  out.pending[me][1] = shmemx_b200_ctx_pending(b);
  shmem_ctx_quiet(a);
  int rc = shmemx_b200_last_status();
  memcpy(out.fa[me], fa, sizeof(fa)); /* complete now: A was quieted */
  out.pending[me][2] = shmemx_b200_ctx_pending(a);
  out.pending[me][3] = shmemx_b200_ctx_pending(b);
  shmem_ctx_quiet(b);
  rc |= shmemx_b200_last_status();
  out.pending[me][4] = shmemx_b200_ctx_pending(b);
  shmem_barrier_all();

  shmem_ctx_t t = SHMEM_CTX_INVALID;
  out.team_rc[me] = shmem_team_create_ctx(even, 0, &t);
  if (out.team_rc[me] == 0) {
    shmem_team_t back = SHMEM_TEAM_INVALID;
    const int tme = shmem_team_my_pe(even);
    out.team_ok[me] = shmem_ctx_get_team(t, &back) == 0 && back == even && tme == me / 2;
    shmem_ctx_int64_put_nbi(t, tdst + tme * BLK, src, BLK, (tme + 1) % TP);
    shmem_ctx_int64_atomic_fetch_or(t, ctr + 2, (int64_t)1 << me, 1);
    rc |= shmemx_b200_last_status();
    shmem_ctx_quiet(t);
    rc |= shmemx_b200_last_status();
    shmem_ctx_destroy(t);
  } else {
    out.team_ok[me] = t == SHMEM_CTX_INVALID;
  }

  crc |= shmem_ctx_create(0, &c);
  int64_t fc = -1;
  shmem_ctx_int64_atomic_fetch_add_nbi(c, &fc, ctr + 1, 1, 0);
  shmem_ctx_destroy(c); /* completes the fetch_add */
  out.fc[me] = fc;
  out.create_rc[me] = crc;

  shmem_ctx_putmem_nbi(SHMEM_CTX_INVALID, dst, src, 8, (me + 1) % NP);
  out.invalid_status[me] = shmemx_b200_last_status();
  if (shmemx_b200_ctx_pending(SHMEM_CTX_INVALID) != -1) out.invalid_status[me] = 0;
  shmem_ctx_destroy(SHMEM_CTX_DEFAULT);
  out.pending[me][5] = shmemx_b200_ctx_pending(SHMEM_CTX_DEFAULT);

  shmem_ctx_int64_p(SHMEM_CTX_DEFAULT, gval, me, (me + 1) % NP);
  shmem_barrier_all();
  out.g[me] = shmem_ctx_int64_g(a, gval, (me + 1) % NP);
  rc |= shmemx_b200_last_status();
  shmem_ctx_destroy(a);
  shmem_ctx_destroy(b);

  memcpy(out.dst[me], dst, sizeof(out.dst[me]));
  memcpy(out.tdst[me], tdst, sizeof(out.tdst[me]));
  shmem_barrier_all();
  if (me == 0) {
    out.counter = ctr[0];
    out.counter2 = ctr[1];
  }
  if (me == 2) out.bits = ctr[2];
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
