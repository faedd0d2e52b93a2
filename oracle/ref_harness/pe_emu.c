/*
 * pe_emu.c -- in-process PE emulator that runs the reference's own shcoll
 * algorithm code (the C files of BTMichalowicz/osss-ucx src/shcoll/src, compiled
 * unmodified) on the CPU.  TEST INFRASTRUCTURE ONLY: this is the parity
 * checker and the timed CPU baseline, never part of the product path.
 *
 * Each emulated PE is one pthread with a thread-local PE number.  The
 * symmetric heap of PE p is the slice [p*slice, (p+1)*slice) of one host
 * arena, so a symmetric address is translated by keeping its offset inside
 * the caller's slice and moving it to the target PE's slice.
 *
 * The reference reaches its transport through ~25 OpenSHMEM primitives
 * (the undefined symbols of the shcoll objects).  They are restated here
 * with the semantics of src/shmemc/ucx/comms.c:
 *   put/get (comms.c:677-737) and their nbi forms (748-762)  -> memmove,
 *     completed before return, so fence/quiet ordering is trivially kept;
 *   p (single-element put)                                   -> release store;
 *   atomic add/inc/fetch/fetch_add/set (comms.c:409-671)      -> __atomic_*;
 *   wait_until (src/shmemc/ucx/waituntil.c:18-51)             -> acquire spin
 *     with sched_yield, bounded by a wall-clock limit;
 *   fence/quiet (comms.c:192-227)                             -> seq_cst fence;
 *   shmem_malloc (src/api/shmalloc.c:47-77)                   -> per-PE bump
 *     allocation from the PE's slice.  The reference also runs
 *     shmem_barrier_all inside shmem_malloc/shmem_free; the emulator does
 *     not, because the only caller on the collective path (the team reduce
 *     wrapper, reduce.c:1090-1100) allocates an unused pWrk, and a WORLD
 *     barrier there would deadlock sub-team reductions in which non-members
 *     never call.  Allocation stays symmetric because every member
 *     allocates in the same order.
 *   team pSync lookup/reset (src/shmemc/teams.c:156-239)     -> per-PE
 *     translated pointers into a reserved region of each slice.
 *
 * The driver entry point (ref_run) is called from Python through
 * ctypes by the parity tests and by the CPU baseline leg of the benchmark.
 */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <errno.h>
#include <pthread.h>
#include <sched.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#include <shmem.h>
#include "shmemc.h"

/* ------------------------------------------------------------------------ */
/* arena layout inside every PE slice                                        */
/* ------------------------------------------------------------------------ */
#define EMU_PSYNC_OFF 0               /* user pSync for active-set forms */
#define EMU_PSYNC_LONGS 1024
#define EMU_TEAM_PSYNC_OFF (EMU_PSYNC_OFF + EMU_PSYNC_LONGS * sizeof(long))
#define EMU_TEAM_PSYNC_LONGS 256      /* per pSync kind (max is 128) */
#define EMU_TEAM_PSYNC_BYTES (SHMEMC_NUM_PSYNCS * EMU_TEAM_PSYNC_LONGS * sizeof(long))
#define EMU_HEAP_OFF (EMU_TEAM_PSYNC_OFF + EMU_TEAM_PSYNC_BYTES)
#define EMU_HEAP_BYTES ((size_t)1 << 16)
#define EMU_DATA_OFF (EMU_HEAP_OFF + EMU_HEAP_BYTES)

static char *g_arena = NULL;
static size_t g_slice = 0;
static int g_npes = 0;
static double g_wait_limit_s = 120.0;
static volatile int g_failed = 0;

static __thread int t_me = -1;
static __thread size_t t_brk = 0;

static void emu_die(const char *msg) {
  fprintf(stderr, "pe_emu: PE %d: %s\n", t_me, msg);
  fflush(stderr);
  abort();
}

static inline char *xlate(const void *sym, int pe) {
  const char *p = (const char *)sym;
  const char *mine = g_arena + (size_t)t_me * g_slice;
  if (p < mine || p >= mine + g_slice) {
    emu_die("address is not inside the caller's symmetric slice");
  }
  if (pe < 0 || pe >= g_npes) {
    emu_die("target PE out of range");
  }
  return g_arena + (size_t)pe * g_slice + (size_t)(p - mine);
}

static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* ------------------------------------------------------------------------ */
/* OpenSHMEM primitives used by the shcoll objects                           */
/* ------------------------------------------------------------------------ */
int shmem_my_pe(void) { return t_me; }
int shmem_n_pes(void) { return g_npes; }

void shmem_putmem(void *dest, const void *source, size_t nelems, int pe) {
  memmove(xlate(dest, pe), source, nelems);
  __atomic_thread_fence(__ATOMIC_RELEASE);
}
void shmem_putmem_nbi(void *dest, const void *source, size_t nelems, int pe) {
  shmem_putmem(dest, source, nelems, pe);
}
void shmem_getmem(void *dest, const void *source, size_t nelems, int pe) {
  __atomic_thread_fence(__ATOMIC_ACQUIRE);
  memmove(dest, xlate(source, pe), nelems);
}
void shmem_getmem_nbi(void *dest, const void *source, size_t nelems, int pe) {
  shmem_getmem(dest, source, nelems, pe);
}
void shmem_fence(void) { __atomic_thread_fence(__ATOMIC_SEQ_CST); }
void shmem_quiet(void) { __atomic_thread_fence(__ATOMIC_SEQ_CST); }

void shmem_long_p(long *addr, long value, int pe) {
  __atomic_store_n((long *)xlate(addr, pe), value, __ATOMIC_RELEASE);
}
void shmem_size_p(size_t *addr, size_t value, int pe) {
  __atomic_store_n((size_t *)xlate(addr, pe), value, __ATOMIC_RELEASE);
}
void shmem_uint64_p(uint64_t *addr, uint64_t value, int pe) {
  __atomic_store_n((uint64_t *)xlate(addr, pe), value, __ATOMIC_RELEASE);
}

void shmem_long_atomic_inc(long *dest, int pe) {
  __atomic_fetch_add((long *)xlate(dest, pe), 1L, __ATOMIC_SEQ_CST);
}
void shmem_long_atomic_add(long *dest, long value, int pe) {
  __atomic_fetch_add((long *)xlate(dest, pe), value, __ATOMIC_SEQ_CST);
}
long shmem_long_atomic_fetch_add(long *dest, long value, int pe) {
  return __atomic_fetch_add((long *)xlate(dest, pe), value, __ATOMIC_SEQ_CST);
}
long shmem_long_atomic_fetch(const long *source, int pe) {
  return __atomic_load_n((long *)xlate(source, pe), __ATOMIC_SEQ_CST);
}
void shmem_size_atomic_add(size_t *dest, size_t value, int pe) {
  __atomic_fetch_add((size_t *)xlate(dest, pe), value, __ATOMIC_SEQ_CST);
}
void shmem_size_atomic_set(size_t *dest, size_t value, int pe) {
  __atomic_store_n((size_t *)xlate(dest, pe), value, __ATOMIC_SEQ_CST);
}

#define EMU_CMP(_cmp, _a, _b)                                                  \
  ((_cmp) == SHMEM_CMP_EQ   ? (_a) == (_b)                                     \
   : (_cmp) == SHMEM_CMP_NE ? (_a) != (_b)                                     \
   : (_cmp) == SHMEM_CMP_GT ? (_a) > (_b)                                      \
   : (_cmp) == SHMEM_CMP_LE ? (_a) <= (_b)                                     \
   : (_cmp) == SHMEM_CMP_LT ? (_a) < (_b)                                      \
                            : (_a) >= (_b))

#define EMU_WAIT(_type, _ivar, _cmp, _value)                                   \
  do {                                                                         \
    const double t0 = now_s();                                                 \
    unsigned spins = 0;                                                        \
    for (;;) {                                                                 \
      _type cur = __atomic_load_n((_ivar), __ATOMIC_ACQUIRE);                  \
      if (EMU_CMP((_cmp), cur, (_value))) break;                               \
      if (g_failed) emu_die("another PE failed");                              \
      if ((++spins & 63u) == 0 && now_s() - t0 > g_wait_limit_s) {             \
        g_failed = 1;                                                          \
        emu_die("wait_until exceeded the wall-clock limit");                   \
      }                                                                        \
      sched_yield();                                                           \
    }                                                                          \
  } while (0)

void shmem_long_wait_until(long *ivar, int cmp, long cmp_value) {
  EMU_WAIT(long, ivar, cmp, cmp_value);
}
void shmem_size_wait_until(size_t *ivar, int cmp, size_t cmp_value) {
  EMU_WAIT(size_t, ivar, cmp, cmp_value);
}

void *shmem_malloc(size_t size) {
  size_t off = (t_brk + 63) & ~(size_t)63;
  if (off + size > EMU_HEAP_BYTES) emu_die("emulated heap exhausted");
  t_brk = off + size;
  return g_arena + (size_t)t_me * g_slice + EMU_HEAP_OFF + off;
}
void shmem_free(void *ptr) { (void)ptr; }

/* Team pSync arrays: the team struct is shared by all emulated PEs, so the
 * pointer handed out is the calling PE's own copy (teams.c:218-239). */
long *shmemc_team_get_psync(shmemc_team_h th, int psync_type) {
  (void)th;
  if (psync_type < 0 || psync_type >= SHMEMC_NUM_PSYNCS) return NULL;
  return (long *)(g_arena + (size_t)t_me * g_slice + EMU_TEAM_PSYNC_OFF +
                  (size_t)psync_type * EMU_TEAM_PSYNC_LONGS * sizeof(long));
}
int shmemc_team_reset_psync(shmemc_team_h th, unsigned psync_idx) {
  long *ps = shmemc_team_get_psync(th, (int)psync_idx);
  if (ps == NULL) return -1;
  for (size_t i = 0; i < EMU_TEAM_PSYNC_LONGS; i++) ps[i] = SHMEM_SYNC_VALUE;
  return 0;
}

/* shmem_team_sync dispatches to the default team_sync algorithm
 * (binomial_tree, src/api/collectives/defaults.h). */
extern int shcoll_team_sync_binomial_tree(shmem_team_t team);
int shmem_team_sync(shmem_team_t team) {
  return shcoll_team_sync_binomial_tree(team);
}

/* ------------------------------------------------------------------------ */
/* driver                                                                    */
/* ------------------------------------------------------------------------ */
enum ref_kind {
  REF_REDUCE_TEAM = 0,   /* int f(team, T*, const T*, size_t)                 */
  REF_TO_ALL = 1,        /* void f(T*, const T*, int, int, int, int, T*, long*) */
  REF_SIZED = 2,         /* void f(void*, const void*, size_t, int,int,int,long*) */
  REF_TEAM_COPY = 3,     /* int f(team, void*, const void*, size_t)           */
  REF_ALLTOALLS_SIZED = 4, /* void f(void*, const void*, ptrdiff_t, ptrdiff_t,
                              size_t, int, int, int, long*)                  */
  REF_ALLTOALLS_TEAM = 5,  /* int f(team, T*, const T*, ptrdiff_t, ptrdiff_t,
                              size_t)                                        */
  REF_BARRIER = 6,       /* void f(int, int, int, long*)                      */
  REF_BARRIER_ALL = 7,   /* void f(long*)                                     */
  REF_TEAM_SYNC = 8,     /* int f(team)                                       */
  REF_BROADCAST_SIZED = 9, /* void f(void*, const void*, size_t, int root,
                              int, int, int, long*)                          */
  REF_BROADCAST_TEAM = 10, /* int f(team, T*, const T*, size_t, int root)     */
  REF_COLLECT_SIZED = 11,  /* void f(void*, const void*, size_t, int,int,int,long*)
                              with each member's own count (below)           */
  REF_COLLECT_TEAM = 12,   /* int f(team, void*, const void*, size_t), own count */
};

struct ref_job;
static size_t collect_count(const struct ref_job *j, int as);

struct ref_job {
  int kind;
  void *fn;
  int pe_start, log_stride, pe_size; /* active set (team: start/stride) */
  size_t nelems;                     /* the call's element/byte count arg */
  long a, b;                         /* dst/sst strides, or root           */
  size_t src_bytes, dst_bytes;       /* per member                         */
  const char *in;                    /* [pe_size][src_bytes]               */
  char *out;                         /* [pe_size][dst_bytes] in/out        */
  int warmup, iters;
  double *times;                     /* [iters] seconds, written by PE 0   */
  shmemc_team_t team;
  pthread_barrier_t bar;
  int pin;
};

/* Collect takes a different count on every member: member i passes
 * nelems + (i * a) % (b + 1) (a rule the caller knows, so it can size and
 * check the result). */
static size_t collect_count(const struct ref_job *j, int as) {
  return j->nelems + (size_t)(((long)as * j->a) % (j->b + 1));
}

static int member_index(const struct ref_job *j, int pe) {
  const int stride = 1 << j->log_stride;
  if (pe < j->pe_start) return -1;
  if ((pe - j->pe_start) % stride) return -1;
  const int as = (pe - j->pe_start) / stride;
  return as < j->pe_size ? as : -1;
}

static void call_once(struct ref_job *j, char *src, char *dst, long *psync) {
  const int stride_log = j->log_stride;
  shmem_team_t team = (shmem_team_t)&j->team;
  switch (j->kind) {
  case REF_REDUCE_TEAM:
  case REF_TEAM_COPY:
    ((int (*)(shmem_team_t, void *, const void *, size_t))j->fn)(team, dst, src,
                                                                  j->nelems);
    break;
  case REF_TO_ALL: {
    void *pwrk = shmem_malloc(4096);
    ((void (*)(void *, const void *, int, int, int, int, void *, long *))j->fn)(
        dst, src, (int)j->nelems, j->pe_start, stride_log, j->pe_size, pwrk,
        psync);
    break;
  }
  case REF_SIZED:
    ((void (*)(void *, const void *, size_t, int, int, int, long *))j->fn)(
        dst, src, j->nelems, j->pe_start, stride_log, j->pe_size, psync);
    break;
  case REF_ALLTOALLS_SIZED:
    ((void (*)(void *, const void *, ptrdiff_t, ptrdiff_t, size_t, int, int,
               int, long *))j->fn)(dst, src, (ptrdiff_t)j->a, (ptrdiff_t)j->b,
                                   j->nelems, j->pe_start, stride_log,
                                   j->pe_size, psync);
    break;
  case REF_ALLTOALLS_TEAM:
    ((int (*)(shmem_team_t, void *, const void *, ptrdiff_t, ptrdiff_t,
              size_t))j->fn)(team, dst, src, (ptrdiff_t)j->a, (ptrdiff_t)j->b,
                             j->nelems);
    break;
  case REF_BARRIER:
    ((void (*)(int, int, int, long *))j->fn)(j->pe_start, stride_log,
                                             j->pe_size, psync);
    break;
  case REF_BARRIER_ALL:
    ((void (*)(long *))j->fn)(psync);
    break;
  case REF_TEAM_SYNC:
    ((int (*)(shmem_team_t))j->fn)(team);
    break;
  case REF_BROADCAST_SIZED:
    ((void (*)(void *, const void *, size_t, int, int, int, int, long *))j->fn)(
        dst, src, j->nelems, (int)j->a, j->pe_start, stride_log, j->pe_size,
        psync);
    break;
  case REF_BROADCAST_TEAM:
    ((int (*)(shmem_team_t, void *, const void *, size_t, int))j->fn)(
        team, dst, src, j->nelems, (int)j->a);
    break;
  case REF_COLLECT_SIZED:
    ((void (*)(void *, const void *, size_t, int, int, int, long *))j->fn)(
        dst, src, collect_count(j, member_index(j, t_me)), j->pe_start, stride_log,
        j->pe_size, psync);
    break;
  case REF_COLLECT_TEAM:
    ((int (*)(shmem_team_t, void *, const void *, size_t))j->fn)(
        team, dst, src, collect_count(j, member_index(j, t_me)));
    break;
  default:
    emu_die("unknown job kind");
  }
}

struct pe_arg {
  struct ref_job *job;
  int pe;
};

static void *pe_main(void *argp) {
  struct pe_arg *arg = (struct pe_arg *)argp;
  struct ref_job *j = arg->job;
  t_me = arg->pe;
  t_brk = 0;
  if (j->pin) {
    long ncpu = sysconf(_SC_NPROCESSORS_ONLN);
    if (ncpu > 0) {
      cpu_set_t set;
      CPU_ZERO(&set);
      CPU_SET((int)(t_me % ncpu), &set);
      pthread_setaffinity_np(pthread_self(), sizeof(set), &set);
    }
  }
  char *base = g_arena + (size_t)t_me * g_slice;
  char *src = base + EMU_DATA_OFF;
  char *dst = src + ((j->src_bytes + 4095) & ~(size_t)4095);
  long *psync = (long *)(base + EMU_PSYNC_OFF);
  const int as = member_index(j, t_me);
  const int all_call = (j->kind == REF_BARRIER_ALL);
  const int total = j->warmup + j->iters;

  for (int it = 0; it < total; it++) {
    /* every iteration starts from the same inputs and clear sync words */
    for (size_t i = 0; i < EMU_PSYNC_LONGS; i++) psync[i] = SHMEM_SYNC_VALUE;
    long *tps = (long *)(base + EMU_TEAM_PSYNC_OFF);
    for (size_t i = 0; i < EMU_TEAM_PSYNC_BYTES / sizeof(long); i++)
      tps[i] = SHMEM_SYNC_VALUE;
    if (as >= 0) {
      memcpy(src, j->in + (size_t)as * j->src_bytes, j->src_bytes);
      memcpy(dst, j->out + (size_t)as * j->dst_bytes, j->dst_bytes);
    }
    t_brk = 0;
    pthread_barrier_wait(&j->bar);
    double t0 = now_s();
    if (as >= 0 || all_call) call_once(j, src, dst, psync);
    pthread_barrier_wait(&j->bar);
    double t1 = now_s();
    if (t_me == 0 && it >= j->warmup && j->times) j->times[it - j->warmup] = t1 - t0;
    if (it == total - 1 && as >= 0) {
      /* results are copied out only after the last iteration */
    }
  }
  pthread_barrier_wait(&j->bar);
  if (as >= 0) memcpy(j->out + (size_t)as * j->dst_bytes, dst, j->dst_bytes);
  return NULL;
}

static int setup_arena(int npes, size_t data_bytes) {
  size_t need = EMU_DATA_OFF + data_bytes + 8192;
  need = (need + 4095) & ~(size_t)4095;
  free(g_arena);
  g_arena = NULL;
  if (posix_memalign((void **)&g_arena, 4096, need * (size_t)npes) != 0)
    return -1;
  memset(g_arena, 0, need * (size_t)npes);
  g_slice = need;
  g_npes = npes;
  g_failed = 0;
  return 0;
}

/*
 * Run one shcoll function `fname` over `npes` emulated PEs.
 * Active set / team = {pe_start + i * 2^log_stride : i < pe_size}.
 * in:  [pe_size][src_bytes] source contents of every member.
 * out: [pe_size][dst_bytes] initial dest contents on entry, results on exit.
 * times: optional [iters] per-iteration seconds (between two barriers).
 * Returns 0 on success, negative on a setup error.
 */
int ref_run(int kind, const char *fname, int npes, int pe_start,
            int log_stride, int pe_size, size_t nelems, long a, long b,
            const void *in, size_t src_bytes, void *out, size_t dst_bytes,
            int warmup, int iters, double *times, int pin) {
  void *fn = dlsym(RTLD_DEFAULT, fname);
  if (fn == NULL) return -2;
  if (npes <= 0 || pe_size <= 0 || iters < 1) return -3;
  if (pe_start + (long)(pe_size - 1) * (1L << log_stride) >= npes) return -4;
  if (setup_arena(npes, ((src_bytes + 4095) & ~(size_t)4095) + dst_bytes) != 0)
    return -5;

  struct ref_job job;
  memset(&job, 0, sizeof(job));
  job.kind = kind;
  job.fn = fn;
  job.pe_start = pe_start;
  job.log_stride = log_stride;
  job.pe_size = pe_size;
  job.nelems = nelems;
  job.a = a;
  job.b = b;
  job.src_bytes = src_bytes;
  job.dst_bytes = dst_bytes;
  job.in = (const char *)in;
  job.out = (char *)out;
  job.warmup = warmup;
  job.iters = iters;
  job.times = times;
  job.pin = pin;
  job.team.name = "emulated";
  job.team.rank = -1;
  job.team.nranks = pe_size;
  job.team.start = pe_start;
  job.team.stride = 1 << log_stride;
  pthread_barrier_init(&job.bar, NULL, (unsigned)npes);

  pthread_t *th = (pthread_t *)calloc((size_t)npes, sizeof(pthread_t));
  struct pe_arg *args = (struct pe_arg *)calloc((size_t)npes, sizeof(*args));
  for (int p = 0; p < npes; p++) {
    args[p].job = &job;
    args[p].pe = p;
    if (pthread_create(&th[p], NULL, pe_main, &args[p]) != 0) emu_die("pthread_create");
  }
  for (int p = 0; p < npes; p++) pthread_join(th[p], NULL);
  pthread_barrier_destroy(&job.bar);
  free(th);
  free(args);
  return 0;
}

void ref_set_wait_limit(double seconds) { g_wait_limit_s = seconds; }
