/*
 * shmemx.h -- extensions of the B200 engine's OpenSHMEM surface.
 */
#ifndef B200_SHMEMX_H
#define B200_SHMEMX_H

#include "shmem.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Run pe_main(arg) on npes PEs, each a host thread of this process, over a
 * symmetric heap of SHMEM_SYMMETRIC_SIZE bytes per PE (default 64M; K/M/G
 * suffixes) on the current CUDA device.  SHMEM_B200_HEAP=device puts the
 * heap in device memory instead of the default CUDA managed memory (then
 * only shmem_put/get and the collectives touch it).  Plays the role of
 * oshrun + shmem_init for an SPMD program.  Returns 0, or non-zero if the
 * engine could not start (shmemx_b200_last_error() says why). */
int shmemx_b200_run(int npes, void (*pe_main)(void *arg), void *arg);

/* Last error of the calling thread (engine or surface). */
const char *shmemx_b200_last_error(void);

/* Return code of the last collective this PE completed: 0, or a negative
 * b200shm_status (the void-returning OpenSHMEM forms cannot report it). */
int shmemx_b200_last_status(void);

/* Non-blocking operations of a context that its next shmem_ctx_quiet will
 * complete (-1 for a context that is not valid). */
int shmemx_b200_ctx_pending(shmem_ctx_t ctx);

/* Wall-clock seconds (shmemx_wtime, include/shmemx.h of the reference). */
double shmemx_wtime(void);

#ifdef __cplusplus
}
#endif
#endif
