/*
 * b200shm.h -- C ABI of the B200 OpenSHMEM collective and atomic engine.
 *
 * Model.  `npes` PEs are emulated on one GPU.  Each PE's symmetric heap is
 * the slice [pe * slice, (pe + 1) * slice) of one HBM arena, so a symmetric
 * object is one offset `off` that is valid in every slice.  A team (or an
 * active set) is the member list pe_start + i * pe_stride, i < pe_size.
 * A collective is issued ONCE for the whole team, not once per PE: the
 * per-PE OpenSHMEM calls (include/shmem.h, include/shcoll_b200.h) aggregate
 * the members' calls into one of these entry points.
 *
 * Streams.  `stream` is a cudaStream_t passed as void*.  NULL means the
 * library's own stream and a blocking call (the call returns when the
 * result is in every member's dest, as the OpenSHMEM routines do).  A
 * non-NULL stream makes the call stream-ordered and asynchronous.
 *
 * Errors.  Every int-returning entry point returns B200SHM_OK (0) or a
 * negative enum b200shm_status; b200shm_last_error() describes the last
 * failure of the calling thread.
 *
 * Each declaration cites the reference (BTMichalowicz/osss-ucx) interface
 * it replaces.
 */
#ifndef B200SHM_H
#define B200SHM_H

#include <stddef.h>
#include <stdint.h>

#include "../osss-ucx_b200/csrc/b200shm_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------------- */
/* lifecycle and heap                                                      */
/* ---------------------------------------------------------------------- */

#define B200SHM_INIT_MANAGED 0x1 /* arena in CUDA managed memory (host-visible) */

/* Create the arena of npes slices of heap_bytes_per_pe (rounded up to
 * 2 MiB) on the current CUDA device.  Replaces shmemc_heaps_init
 * (src/shmemc/heaps.c:33-52) and register_symmetric_heap
 * (src/shmemc/ucx/init.c:174-218); the heap size plays the role of
 * SHMEM_SYMMETRIC_SIZE (src/shmemc/env.c:117-119). */
int b200shm_init(int npes, uint64_t heap_bytes_per_pe, int flags);
/* Release everything (src/shmemc/init.c shmemc_finalize). */
int b200shm_finalize(void);
int b200shm_initialized(void);
int b200shm_n_pes(void);                 /* shmem_n_pes, src/api/info.c */
uint64_t b200shm_heap_slice(void);       /* bytes per PE slice */
void *b200shm_heap_base(void);           /* device address of slice 0 */
/* Device address of offset `off` in PE `pe`'s slice; NULL if out of range.
 * Plays the role of shmem_ptr (src/api/ptr.c) and of the region lookup
 * translate_region_address (src/shmemc/ucx/comms.c:99-112). */
void *b200shm_ptr(int pe, uint64_t off);
const char *b200shm_last_error(void);
/* Wait for all work on the library stream (shmem_quiet semantics for the
 * device, src/shmemc/ucx/comms.c:205-227). */
int b200shm_quiet(void);
/* Number of kernels this library has launched since it was loaded. */
unsigned long long b200shm_launch_count(void);
/* The library stream, as a cudaStream_t. */
void *b200shm_stream(void);

/* Symmetric allocation: the same offset in every slice.  Replaces
 * shmem_malloc / shmem_align / shmem_free (src/api/shmalloc.c:47-195) and
 * the dlmalloc mspace behind them (src/api/allocator/memalloc.c:29-93). */
int b200shm_malloc(uint64_t bytes, uint64_t align, uint64_t *off);
int b200shm_free(uint64_t off);
uint64_t b200shm_heap_free_bytes(void);

/* Host <-> symmetric heap copies for pe_count PEs pe_start + i*pe_stride:
 * host row i (bytes_per_pe bytes) <-> offset `off` of member i.  These are
 * how host buffers enter and leave the arena (the put/get of
 * src/shmemc/ucx/comms.c:677-737 with a host-side peer). */
int b200shm_put_host(int pe_start, int pe_stride, int pe_count, uint64_t off,
                     const void *host_src, uint64_t bytes_per_pe, void *stream);
int b200shm_get_host(void *host_dst, int pe_start, int pe_stride, int pe_count,
                     uint64_t off, uint64_t bytes_per_pe, void *stream);
/* Copy between any two addresses the device can see (heap, device, managed
 * or host memory); blocking when stream is NULL.  Backs shmem_putmem /
 * shmem_getmem (src/shmemc/ucx/comms.c:677-737). */
int b200shm_memcpy(void *dst, const void *src, uint64_t bytes, void *stream);
/* Strided copy of nelems elements of elem_bytes: dst[i*dst_stride] =
 * src[i*src_stride] (strides in elements, >= 1), between any memory the
 * device can see; blocking when stream is NULL.  Backs shmem_<T>_iput /
 * iget and shmem_iput/iget{8,16,32,64,128} (src/api/rma/putget.h:131-220,
 * which issue one UCX put or get per element). */
int b200shm_memcpy_strided(void *dst, int64_t dst_stride, const void *src, int64_t src_stride,
                           uint64_t elem_bytes, uint64_t nelems, void *stream);
/* Compare nelems symmetric words of `dtype` (a 2-, 4- or 8-byte integer
 * type, compared as that type) at offset `off` of PE `pe` with cmp
 * (SHMEM_CMP_EQ/NE/GT/LE/LT/GE = 0..5) against *cmp_value, or against
 * cmp_values[i] when cmp_values is not NULL (host arrays of the element
 * type).  out[i] (host) receives 1 when element i compares true, 0 when
 * not, 2 when status (may be NULL) is non-zero at i; loaded (may be NULL)
 * receives the bits each element held when it was compared.  One device
 * pass with acquire loads, so words written by the engine's puts, atomics
 * and serving loop are seen.  Blocking.  Backs shmem_<T>_test,
 * test_all/any/some[_vector], and in a polling loop wait_until,
 * wait_until_all/any/some[_vector] and shmem_signal_wait_until
 * (src/shmemc/ucx/test.c:10-170, waituntil.c:18-320). */
int b200shm_test_words(int cmp, int dtype, int pe, uint64_t off, uint64_t nelems,
                       const int *status, const void *cmp_value, const void *cmp_values,
                       uint8_t *out, uint64_t *loaded);
/* Fill bytes_per_pe bytes at `off` of pe_count members with `byte`. */
int b200shm_memset(int pe_start, int pe_stride, int pe_count, uint64_t off,
                   int byte, uint64_t bytes_per_pe, void *stream);

/* ---------------------------------------------------------------------- */
/* collectives (one call per team)                                         */
/* ---------------------------------------------------------------------- */

/* All-reduce of nelems elements: every member's dest gets the reduction of
 * all members' sources, computed in the combine order of `algo`.
 * Replaces reduce_helper_<T>_<op>_{linear,binomial,rec_dbl,rabenseifner,
 * rabenseifner2} (src/shcoll/src/reduce.c:55-724) behind
 * shcoll_<T>_<op>_reduce_<algo> (reduce.c:1078-1102) and
 * shcoll_<T>_<op>_to_all_<algo> (reduce.c:931-955).  dest_off == src_off
 * (in place) is allowed; other overlaps are rejected.  Long double
 * (B200SHM_F80, MIN/MAX/SUM/PROD) runs on a software x87 whose bits equal
 * an x86 host's; its MIN/MAX teams are limited to 2048 members. */
int b200shm_reduce(int op, int dtype, int algo, int pe_start, int pe_stride,
                   int pe_size, uint64_t dest_off, uint64_t src_off,
                   uint64_t nelems, void *stream);

/* The all-reduce of host rows: member i's source row is host_src +
 * i*src_pitch and its result row host_dest + i*dest_pitch (bytes); the rows
 * pass through the symmetric objects at src_off / dest_off.  The same as
 * b200shm_put_host(src rows) + b200shm_reduce + b200shm_get_host(dest rows),
 * and bit-identical to it, but pipelined: the elements go in chunks whose
 * copy in, reduction and copy out overlap on three streams, so both PCIe
 * directions and the GPU work at once (pinned host rows are needed for the
 * copies to overlap).  Replaces the reference's put + shcoll reduce + get
 * sequence of a host-resident caller (src/shmemc/ucx/comms.c:677-737,
 * src/shcoll/src/reduce.c:1078-1102). */
int b200shm_reduce_host(int op, int dtype, int algo, int pe_start, int pe_stride,
                        int pe_size, void *host_dest, uint64_t dest_pitch,
                        const void *host_src, uint64_t src_pitch, uint64_t dest_off,
                        uint64_t src_off, uint64_t nelems, void *stream);

/* The same all-reduce for callers that cannot allocate device memory (a
 * runtime that owns every device allocation through its own pool, or code
 * that may not call cudaMalloc at all).  No counterpart in the reference.
 * It needs no b200shm_init and allocates nothing: member i's rows are the
 * caller's device buffers source + i*source_stride and dest + i*dest_stride
 * (the strides may differ).  The dest rows must be the source rows
 * themselves (in place: dest == source, equal strides) or lie wholly apart
 * from every source row; any other overlap is rejected with
 * B200SHM_ERR_ARG.  Grids are sized for the current device.
 * Float MIN/MAX keeps its list of order-dependent elements in a file-scope
 * static device array (2 MiB + 256 bytes per GPU that loads the library,
 * held until exit), so float MIN/MAX is limited to 2^18 elements per
 * member; larger sizes are rejected with B200SHM_ERR_UNSUPPORTED.  All
 * calls share that array: calls that overlap on the GPU race.  The first
 * call on a device resolves the array's device address (set-up), so make
 * it before any stream capture.  The call blocks until the result is in
 * every dest (on `stream`, or the default stream when NULL). */
int b200shm_reduce_noalloc(int op, int dtype, int algo, int npes, void *dest,
                           uint64_t dest_stride, const void *source,
                           uint64_t source_stride, uint64_t nelems, void *stream);

/* Fixed-size allgather: member j's dest[k*nbytes ..] = member k's source.
 * Replaces fcollect_helper_* (src/shcoll/src/fcollect.c:32-484) behind
 * shcoll_fcollect{32,64}_<algo>, shcoll_<T>_fcollect_<algo> and
 * shcoll_fcollectmem_<algo> (fcollect.c:492-653). */
int b200shm_fcollect(int pe_start, int pe_stride, int pe_size,
                     uint64_t dest_off, uint64_t src_off, uint64_t nbytes,
                     void *stream);

/* Variable-size allgather: member k contributes nbytes[k] bytes (host
 * array of pe_size sizes) from src_off; every member's dest holds the
 * contributions concatenated in member order (member k's block at the sum
 * of nbytes[0..k)).  Replaces collect_helper_* (src/shcoll/src/collect.c:
 * 35-591) behind shcoll_collect{32,64}_<algo>, shcoll_<T>_collect_<algo> and
 * shcoll_collectmem_<algo> (collect.c:593-738), where each PE passes its own
 * count. */
int b200shm_collect(int pe_start, int pe_stride, int pe_size, uint64_t dest_off,
                    uint64_t src_off, const uint64_t *nbytes, void *stream);

/* All-to-all of nbytes blocks: member j's dest block k = member k's source
 * block j.  Replaces alltoall_helper_* (src/shcoll/src/alltoall.c:75-201)
 * behind shcoll_alltoall{32,64}_<algo>, shcoll_<T>_alltoall_<algo> and
 * shcoll_alltoallmem_<algo> (alltoall.c:242-387). */
int b200shm_alltoall(int pe_start, int pe_stride, int pe_size,
                     uint64_t dest_off, uint64_t src_off, uint64_t nbytes,
                     void *stream);

/* Strided all-to-all: element t from member k to member l moves
 * src_k[(l*nelems + t)*sst] -> dest_l[(k*nelems + t)*dst] (elements of
 * elem_size bytes); other dest elements are untouched.  Replaces
 * alltoalls_helper_* (src/shcoll/src/alltoalls.c:54-297, index rule 39-50)
 * behind shcoll_alltoalls{32,64}_<algo> and shcoll_<T>_alltoalls_<algo>
 * (alltoalls.c:303-435). */
int b200shm_alltoalls(int pe_start, int pe_stride, int pe_size,
                      uint64_t dest_off, uint64_t src_off, int64_t dst,
                      int64_t sst, uint64_t nelems, uint64_t elem_size,
                      void *stream);

/* Broadcast nbytes from member `root`'s source to every other member's
 * dest (the root's dest is left untouched).  Replaces broadcast_helper_*
 * (src/shcoll/src/broadcast.c:58-599). */
int b200shm_broadcast(int root, int pe_start, int pe_stride, int pe_size,
                      uint64_t dest_off, uint64_t src_off, uint64_t nbytes,
                      void *stream);

/* Barrier among the members, run on the device by one PE context per
 * member over flag words with the given algorithm's message pattern, with
 * a bounded spin.  Replaces barrier_sync_helper_* (src/shcoll/src/
 * barrier.c:56-266) behind shcoll_barrier[_all]_<algo>, shcoll_sync[_all]
 * and shcoll_team_sync_<algo> (barrier.c:279-366).  Returns
 * B200SHM_ERR_TIMEOUT if a member's wait ran out of budget. */
int b200shm_barrier(int algo, int pe_start, int pe_stride, int pe_size,
                    void *stream);

/* Set the budget of every device-side barrier wait to `ns` nanoseconds
 * (0 restores the default of 2 s); returns the previous budget.  The
 * reference's waits (shmem_long_wait_until, src/shmemc/ucx/waituntil.c:
 * 18-51) spin without bound; here a member that does not arrive within the
 * budget turns the barrier into B200SHM_ERR_TIMEOUT. */
uint64_t b200shm_set_wait_budget(uint64_t ns);

/* Failure injection for failure-detection tests: barrier `algo` over the
 * team with member `absent` never arriving (its PE context is not
 * started).  Every wait that depends on it runs out of its budget, the call
 * returns B200SHM_ERR_TIMEOUT with the flag lines cleared, and the team's
 * next barrier works.  No reference counterpart (a missing PE hangs the
 * reference's barrier_sync_helper_*, src/shcoll/src/barrier.c:56-266). */
int b200shm_barrier_absent(int algo, int pe_start, int pe_stride, int pe_size, int absent,
                           void *stream);

/* Number of barrier flag words that are not zero (every barrier returns its
 * flags to zero, as the reference returns pSync to SHMEM_SYNC_VALUE,
 * src/shcoll/src/barrier.c:56-266); for tests of the recovery path. */
int64_t b200shm_barrier_flags_nonzero(void);

/* ---------------------------------------------------------------------- */
/* teams that span GPUs (one process and one engine per GPU)               */
/* ---------------------------------------------------------------------- */

/* The arena's CUDA IPC handle (64 bytes into `handle`), for the other
 * GPUs' processes to map it with b200shm_peer_open.  Every engine of a
 * spanning job is initialised with the same npes and heap size (the
 * symmetric heap's own rule), and not in managed memory.  The reference
 * reaches other PEs' heaps through UCX rkeys (src/shmemc/ucx/comms.c:58-112);
 * here another GPU's arena is one mapped address range. */
int b200shm_ipc_handle(void *handle);
/* Map another engine's arena from its IPC handle; *peer_base receives the
 * device address of its slice 0.  A handle opened again shares the first
 * mapping (each open wants a close); b200shm_finalize closes the mappings
 * still open. */
int b200shm_peer_open(const void *handle, void **peer_base);
int b200shm_peer_close(void *peer_base);

/* Every address the span calls below take (a partial vector, a rank's
 * arena base) must lie, with everything the call reads through it, inside
 * this engine's arena or inside an arena mapped with b200shm_peer_open and
 * still open (a peer arena having this one's npes and slice size); any
 * other address is refused with B200SHM_ERR_ARG before anything is
 * launched, zero-size calls included. */

/* The cross-GPU half of a reduction over a team of G x pe_count members
 * (pe_count on each of G GPUs, G a power of two up to 16), fused with its
 * write-back: element by element, the G ranks' partial vectors -- each the
 * reduction over one GPU's members, at the device addresses partials[g]
 * (this rank's own, the others' through b200shm_peer_open) -- combined as
 * rank `rank` combines them in the butterfly (round j pairs rank r with
 * r ^ 2^j, keeping op(own, partner): src/shcoll/src/reduce.c:250-272), the
 * result written to this GPU's members pe_start + i*pe_stride at dest_off.
 * Plain loads of the peers' memory.  The caller separates the phases with a
 * barrier across the processes: all partials written before any rank
 * combines, all combines done before any partial is overwritten.  Every
 * dtype but long double; complex for SUM and PROD only. */
int b200shm_span_combine(int op, int dtype, int G, int rank, const uint64_t *partials,
                         int pe_start, int pe_stride, int pe_count, uint64_t dest_off,
                         uint64_t nelems, void *stream);
/* fcollect over the same team: member m = g*pe_count + k is PE
 * pe_start + k*pe_stride of GPU g's engine (the same local PEs on every
 * GPU) and sends nbytes from src_off; every local member's dest holds the
 * G*pe_count blocks in member order.  bases[g] = GPU g's arena base (this rank's own
 * b200shm_heap_base, the others' mapped).  Replaces fcollect_helper_*
 * (src/shcoll/src/fcollect.c:32-484) for a team across GPUs. */
int b200shm_span_fcollect(int G, int rank, const uint64_t *bases, int pe_start, int pe_stride,
                          int pe_count, uint64_t dest_off, uint64_t src_off, uint64_t nbytes,
                          void *stream);
/* alltoall over the same team: local member j's dest block m = member m's
 * source block rank*pe_count + j, wherever member m lives.  Replaces
 * alltoall_helper_* (src/shcoll/src/alltoall.c:75-201) across GPUs. */
int b200shm_span_alltoall(int G, int rank, const uint64_t *bases, int pe_start, int pe_stride,
                          int pe_count, uint64_t dest_off, uint64_t src_off, uint64_t nbytes,
                          void *stream);

/* One-sided atomics over the same team: op k on member member[k] (on GPU
 * member[k] / pe_count) at byte offset off[k], run by this GPU as a
 * system-scope atomic on the owner's arena -- the other GPUs' through
 * b200shm_peer_open, over NVLink -- with no other rank taking part; the
 * old values land in fetched[k] (device arrays, as b200shm_amo_batch).
 * Ops of different GPUs on one word are applied atomically in an
 * unspecified order, as concurrent AMOs of different PEs are in OpenSHMEM
 * (src/shmemc/ucx/comms.c:409-671).  A target outside the team or the
 * slice fails the call with B200SHM_ERR_ARG after the others ran. */
int b200shm_span_amo(int amo, int dtype, int G, const uint64_t *bases, int pe_start,
                     int pe_stride, int pe_count, uint64_t nops, const int32_t *member,
                     const uint64_t *off, const void *value, const void *cond, void *fetched,
                     void *stream);

/* ---------------------------------------------------------------------- */
/* batched reductions                                                      */
/* ---------------------------------------------------------------------- */

/* algo value that lets the library choose (rec_dbl, the reference's
 * default, src/shcoll/src/defaults.h:71) */
#define B200SHM_ALGO_AUTO (-1)

/* One reduction of a batch: the arguments of b200shm_reduce.  `lanes` and
 * `tile` are outputs of b200shm_batch_create: the lanes per 16-byte column
 * and the units per tile the autotuner chose (0 = this reduction runs as
 * its own launch because the batch kernels do not cover its
 * (dtype, op, algo, size)); `algo` is rewritten when it was AUTO. */
typedef struct b200shm_reduce_desc {
  int32_t op, dtype, algo;
  int32_t pe_start, pe_stride, pe_size;
  uint64_t dest_off, src_off, nelems;
  int32_t lanes, tile;
} b200shm_reduce_desc;

typedef struct b200shm_batch b200shm_batch;

#define B200SHM_BATCH_NO_TUNE 0x1 /* the heuristic plan (or cached choices) only */
#define B200SHM_BATCH_GRAPH 0x2   /* capture the run into a CUDA graph     */
#define B200SHM_BATCH_TUNE 0x4    /* tune (the default unless NO_TUNE)     */

/* Plan a batch of n independent reductions: validate every descriptor,
 * choose lanes per column, columns per lane and tile size per shape (the
 * autotuner's cached choice for the shape's class, else a measured
 * heuristic), then -- unless B200SHM_BATCH_NO_TUNE, or a descriptor runs
 * in place -- tune: for the shape classes that carry the most bytes and
 * have no cached choice, try the other (lanes, tile) plans and time the
 * whole batch as it runs, keeping what makes it faster; the choices are
 * cached for the process.  Tuning runs the batch, so the dests are written
 * at create time (with the values a run writes).  The reductions run
 * concurrently, so a descriptor whose dest touches another descriptor's
 * source or dest (in any member) is rejected with B200SHM_ERR_ARG; sharing
 * a source, and a descriptor in place, are fine.  Replaces n separate
 * shcoll_<T>_<op>_reduce_<algo> calls (src/shcoll/src/reduce.c:1078-1102),
 * which the reference can only issue one after the other.  Every result is
 * bit-identical to b200shm_reduce on the same descriptor, whatever the
 * plan. */
int b200shm_batch_create(b200shm_reduce_desc *descs, uint64_t n, int flags,
                         b200shm_batch **out);
/* Run the whole batch: one persistent launch per (type, op, combine order)
 * group, the groups overlapping on side streams, plus one launch that
 * replays order-dependent float MIN/MAX elements and one launch per
 * reduction the batch kernels do not cover.  With B200SHM_BATCH_GRAPH the
 * run is a single CUDA graph launch.  Runs of one batch must not overlap
 * on the GPU (they share its tile counters). */
int b200shm_batch_run(b200shm_batch *batch, void *stream);
int b200shm_batch_destroy(b200shm_batch *batch);
/* create + run + destroy. */
int b200shm_reduce_batch(b200shm_reduce_desc *descs, uint64_t n, void *stream);

/* ---------------------------------------------------------------------- */
/* serving loop                                                            */
/* ---------------------------------------------------------------------- */

/* Request kinds of the serving loop. */
enum b200shm_req_kind {
  B200SHM_REQ_REDUCE = 0, /* all-reduce over the team, as b200shm_reduce      */
  B200SHM_REQ_FCOLLECT,   /* as b200shm_fcollect, n = bytes per member        */
  B200SHM_REQ_ALLTOALL,   /* as b200shm_alltoall, n = bytes per block         */
  B200SHM_REQ_PUT,        /* n bytes from PE pe_start's src_off to PE pe's dest_off */
  B200SHM_REQ_GET,        /* n bytes from PE pe's src_off to PE pe_start's dest_off */
  B200SHM_REQ_AMO,        /* op = b200shm_amo on (pe, dest_off), as b200shm_amo */
  B200SHM_REQ_NKIND
};

/* One request.  REDUCE: op/dtype/algo/team/dest/src/n = nelems, as
 * b200shm_reduce (dtype one of I32, U32, I64, U64, F32, F64).  AMO: op is
 * a b200shm_amo, dtype a 4- or 8-byte type, value/cond hold the operand
 * bits, the old value comes back through b200shm_serve_poll.  Any other
 * kind may pass dest_off = B200SHM_SERVE_ALLOC: the loop then allocates the
 * dest from the symmetric heap (the bytes one member's dest spans) when it
 * admits the request, so the request waits in the ring, in arrival order,
 * until the heap has room; b200shm_serve_poll / _wait return the offset it
 * got, and the caller releases it with b200shm_free.  A request waiting for
 * room keeps the loop awake, and b200shm_serve_stop waits (bounded) for it
 * to be admitted.  The per-call replays take no such request. */
#define B200SHM_SERVE_ALLOC (~(uint64_t)0)
typedef struct b200shm_request {
  int32_t kind, op, dtype, algo;
  int32_t pe_start, pe_stride, pe_size, pe;
  uint64_t dest_off, src_off, n;
  uint64_t value, cond;
} b200shm_request;

typedef struct b200shm_server b200shm_server;

/* Start the serving loop: a persistent kernel of `ctas` CTAs (0 = two per
 * SM, as many as fit at once) on its own stream that drains a ring of
 * queue_slots requests kept in mapped host memory.  Requests are cut into
 * tiles, and a request's tiles into at most one share per CTA, which idle
 * CTAs claim, so a large request spreads over the GPU while small ones pass
 * it; each request reports completion through a word in host memory.  When
 * no new request has arrived for idle_seconds (0 = 0.25 s) the CTAs exit;
 * the next enqueue, poll or wait relaunches the kernel, so the loop holds
 * the GPU only while it is used.  Replaces the reference's issue-one-call-and-wait model
 * (shmem_* -> shcoll / shmemc_ctx_* round trips, src/shcoll/src/ files,
 * src/shmemc/ucx/comms.c) for streams of small operations.  Requests in
 * flight together may run in any order and concurrently, as non-blocking
 * (_nbi) operations do: a request that depends on another's result must
 * be enqueued after that one completed.  While a server runs, calls that
 * synchronise the whole device (cudaDeviceSynchronize, cudaFree, and so
 * b200shm_finalize) wait for it to go idle; the library's other entry
 * points use stream-ordered memory and do not.  The first launch of a
 * kernel that CUDA has not loaded yet (lazy module loading, the default)
 * also waits for the loop to go idle (at most idle_seconds; 0 = 0.25 s):
 * run CUDA_MODULE_LOADING=EAGER, or use the calls once before starting the
 * loop, where that matters. */
int b200shm_serve_start(uint32_t queue_slots, int ctas, double idle_seconds,
                        b200shm_server **out);
/* The same, with admission by symmetric-heap bytes: requests are opened to
 * the GPU in arrival order only while the heap bytes that the admitted,
 * incomplete ones write (over all their members: a reduction n*size*P, an
 * fcollect or alltoall block*P*P, a put or get n, an atomic 8) stay within
 * heap_budget (0 = no limit); a later request waits in the ring until
 * completions free enough, and a request larger than the whole budget is
 * refused at enqueue.  Accounting is on the device (one counter raised by
 * the CTA that admits, lowered by the CTA that completes).  No reference
 * counterpart: the reference runs each call to completion. */
int b200shm_serve_start_budget(uint32_t queue_slots, int ctas, double idle_seconds,
                               uint64_t heap_budget, b200shm_server **out);
/* Validate and publish one request; *ticket identifies it.  Returns
 * B200SHM_ERR_BUSY when all queue slots hold requests not yet complete. */
int b200shm_serve_enqueue(b200shm_server *srv, const b200shm_request *req,
                          uint64_t *ticket);
/* 1 when the request completed, 0 while it is pending, < 0 on an error.
 * *fetched (may be NULL) receives an AMO's old value, and for the other
 * kinds the dest offset the request wrote to (the one the loop allocated,
 * for B200SHM_SERVE_ALLOC). */
int b200shm_serve_poll(b200shm_server *srv, uint64_t ticket, uint64_t *fetched);
/* Device clock stamps (globaltimer, ns) of a completed request still in
 * its slot: copied from the ring into device memory, its last tiles
 * claimed, complete.  1 when available, 0 otherwise. */
int b200shm_serve_trace(b200shm_server *srv, uint64_t ticket, uint64_t stamps[3]);
/* Block until the request completes or timeout_seconds pass
 * (B200SHM_ERR_TIMEOUT). */
int b200shm_serve_wait(b200shm_server *srv, uint64_t ticket, double timeout_seconds,
                       uint64_t *fetched);
/* Let the loop drain, wait (bounded) for its kernel to exit, free it. */
int b200shm_serve_stop(b200shm_server *srv);
/* Open-loop replay of n requests: request k is issued at arrival_s[k]
 * seconds after the call starts (through the server when srv is non-NULL,
 * else as one blocking per-call entry point each: b200shm_reduce,
 * _fcollect, _alltoall, _memcpy, _amo), and latency_s[k] receives the time
 * from its arrival to the observed completion.  fetched (may be NULL)
 * receives AMO old values.  The measuring tool behind the serving
 * benchmark and its per-call comparison. */
int b200shm_serve_replay(b200shm_server *srv, const b200shm_request *reqs, uint64_t n,
                         const double *arrival_s, double *latency_s, uint64_t *fetched);
/* The per-call comparison in stream order: every request through its
 * per-call entry point on `stream` (NULL = the library stream) with no
 * synchronisation between requests -- b200shm_reduce, _fcollect,
 * _alltoall, a device copy for put/get, one single-operation atomic kernel
 * -- then one synchronisation.  *seconds (may be NULL) receives the time
 * from the first issue to the last completion, fetched (may be NULL) the
 * AMO old values.  Requests must not depend on each other's results (they
 * complete in stream order).  The reference has no stream-ordered form: a
 * measuring tool for the serving benchmark. */
int b200shm_serve_replay_ordered(const b200shm_request *reqs, uint64_t n, void *stream,
                                 double *seconds, uint64_t *fetched);

/* Fill nelems elements of `dtype` at `off` in pe_count members with seeded
 * pseudo-random values: integers uniform in [lo, hi], floats uniform in
 * [lo, hi) (the value depends only on seed, global PE and index).  Input
 * generation on the device for tests and benchmarks. */
int b200shm_fill_uniform(int pe_start, int pe_stride, int pe_count, uint64_t off,
                         int dtype, uint64_t nelems, uint64_t seed, double lo,
                         double hi, void *stream);

/* ---------------------------------------------------------------------- */
/* atomics                                                                 */
/* ---------------------------------------------------------------------- */

/* A batch of nops atomic operations on symmetric objects of `dtype`
 * (4- or 8-byte integers; F32/F64 for SWAP/SET/FETCH): operation k acts on
 * the element at offset off[k] (bytes) of PE pe[k].  value/cond/fetched are
 * arrays of nops elements (cond only for CSWAP; fetched may be NULL for the
 * non-fetching forms).  All arrays are DEVICE pointers.  Replaces one
 * shmem_<T>_atomic_<op> per element (the src/api/atomics files ->
 * shmemc_ctx_{fadd,add,swap,cswap,fetch,set,and,or,xor}, src/shmemc/ucx/
 * comms.c:409-671), each of which is a blocking round trip there. */
int b200shm_amo_batch(int amo, int dtype, uint64_t nops, const int32_t *pe,
                      const uint64_t *off, const void *value, const void *cond,
                      void *fetched, void *stream);

/* One atomic operation issued from the host: the per-call path behind
 * shmem_[ctx_]<T>_atomic_<op> (shmemc_ctx_fadd & co., src/shmemc/ucx/
 * comms.c:409-671).  value/cond are passed by value (4 or 8 bytes read from
 * the pointers), the old value is written to *fetched (may be NULL).
 * Blocking: one kernel launch and one stream synchronisation per call, so
 * batch with b200shm_amo_batch wherever there is more than one. */
int b200shm_amo(int amo, int dtype, int pe, uint64_t off, const void *value,
                const void *cond, void *fetched);

#ifdef __cplusplus
}
#endif
#endif
