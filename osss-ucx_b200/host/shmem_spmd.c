/*
 * shmem_spmd.c -- the OpenSHMEM calls of the collective and atomic hot path
 * (include/shmem.h), for SPMD programs whose PEs are host threads, backed by
 * the B200 engine (include/b200shm.h).
 *
 * In the reference every PE is an OS process and every collective runs its
 * algorithm as rounds of UCX puts between them (src/shcoll/src, reached via
 * src/api/collectives/shcoll-shim.c).  Here every PE is a thread started by
 * shmemx_b200_run, all symmetric heaps are slices of one GPU arena, and a
 * collective is ONE device call for the whole team: each team (and each
 * active set of the deprecated forms) has an arrival point; members record
 * their arguments there, the last to arrive checks that every member passed
 * the same symmetric offsets and counts and issues the b200shm_* call, and
 * all members return when it has completed -- so every collective is also a
 * barrier among its members, as in the reference.
 *
 * Algorithm names are read from the reference's environment variables
 * (src/shmemc/env.c:186-312): SHMEM_<OP>_REDUCE_ALGO / SHMEM_<OP>_TO_ALL_ALGO
 * choose the combine order (linear, binomial, rec_dbl, rabenseifner,
 * rabenseifner2; default rec_dbl, src/api/collectives/defaults.h) and
 * SHMEM_BARRIER[_ALL]_ALGO, SHMEM_SYNC[_ALL]_ALGO, SHMEM_TEAM_SYNC_ALGO the
 * barrier pattern (default binomial_tree).  fcollect / alltoall(s) /
 * broadcast produce the same bytes whatever their algorithm name, so those
 * names are accepted and ignored.
 */
#include <errno.h>
#include <pthread.h>
#include <sched.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

/* the library defines the functions themselves: no generic-name macros */
#define SHMEM_B200_NO_GENERICS 1
#include "../../include/b200shm.h"
#include "../../include/shmem.h"
#include "../../include/shmemx.h"

/* ---- sizes of the live symmetric objects (for shmem_realloc) --------------- */
static pthread_mutex_t g_sz_mu = PTHREAD_MUTEX_INITIALIZER;
static uint64_t *g_sz_off, *g_sz_len;
static size_t g_sz_n, g_sz_cap;

static void size_note(uint64_t off, uint64_t len) {
  pthread_mutex_lock(&g_sz_mu);
  if (g_sz_n == g_sz_cap) {
    const size_t cap = g_sz_cap ? 2 * g_sz_cap : 64;
    uint64_t *o = (uint64_t *)realloc(g_sz_off, cap * sizeof(uint64_t));
    if (o) g_sz_off = o;
    uint64_t *l = (uint64_t *)realloc(g_sz_len, cap * sizeof(uint64_t));
    if (l) g_sz_len = l;
    if (o && l) g_sz_cap = cap;
  }
  if (g_sz_n < g_sz_cap) {
    g_sz_off[g_sz_n] = off;
    g_sz_len[g_sz_n] = len;
    g_sz_n++;
  }
  pthread_mutex_unlock(&g_sz_mu);
}
static void size_forget(uint64_t off) {
  pthread_mutex_lock(&g_sz_mu);
  for (size_t i = 0; i < g_sz_n; i++)
    if (g_sz_off[i] == off) {
      g_sz_off[i] = g_sz_off[g_sz_n - 1];
      g_sz_len[i] = g_sz_len[g_sz_n - 1];
      g_sz_n--;
      break;
    }
  pthread_mutex_unlock(&g_sz_mu);
}
/* bytes of the object at `off`; 0 if none starts there */
static uint64_t size_of_object(uint64_t off) {
  uint64_t len = 0;
  pthread_mutex_lock(&g_sz_mu);
  for (size_t i = 0; i < g_sz_n; i++)
    if (g_sz_off[i] == off) {
      len = g_sz_len[i];
      break;
    }
  pthread_mutex_unlock(&g_sz_mu);
  return len;
}

/* ---- errors ---------------------------------------------------------------- */
static __thread char t_err[512];
static __thread int t_status;

static int set_err(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(t_err, sizeof(t_err), fmt, ap);
  va_end(ap);
  return code;
}
const char *shmemx_b200_last_error(void) { return t_err[0] ? t_err : b200shm_last_error(); }
int shmemx_b200_last_status(void) { return t_status; }
static int engine_err(int rc) {
  if (rc) set_err(rc, "%s", b200shm_last_error());
  return rc;
}

double shmemx_wtime(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* ---- PEs -------------------------------------------------------------------- */
static int g_npes;           /* PEs of the running job (world size) */
static char *g_base;         /* arena base */
static uint64_t g_slice;     /* bytes per PE slice */
static uint64_t g_scratch;   /* per-PE scratch offset (AMO operands) */
static __thread int t_pe = -1;

/* ---- arrival points ----------------------------------------------------- */
enum { K_NONE, K_MALLOC, K_FREE, K_BARRIER, K_REDUCE, K_FCOLLECT, K_ALLTOALL, K_ALLTOALLS,
       K_BROADCAST, K_SPLIT, K_SPLIT2D, K_DESTROY, K_COLLECT };

typedef struct coll {
  int kind, op, dtype, algo, root;
  uint64_t dest, src, n, esize;
  int64_t a, b;
} coll_t;

typedef struct agg {
  pthread_mutex_t mu;
  pthread_cond_t cv;
  int arrived, mismatch, rc;
  unsigned long gen;
  coll_t req;
  uint64_t out;
  void *outp, *outq;
  uint64_t *counts; /* collect: each member's own byte count, by team index */
  int counts_cap;
  char msg[512];    /* the failure of the last launch, for every member */
} agg_t;

typedef struct b200_team {
  int start, stride, size; /* global PEs start + i*stride, i < size */
  int valid;
  agg_t agg;
  struct b200_team *next; /* every team ever made, freed at exit */
} b200_team_t;

static b200_team_t g_world;
static pthread_mutex_t g_teams_mu = PTHREAD_MUTEX_INITIALIZER;
static b200_team_t *g_teams;    /* split teams */
static b200_team_t *g_actsets;  /* arrival points of the active-set forms */

shmem_team_t SHMEM_TEAM_WORLD = &g_world;
shmem_team_t SHMEM_TEAM_SHARED = &g_world;
shmem_team_t SHMEM_TEAM_INVALID = NULL;
static char g_ctx_invalid; /* a handle no context has */
shmem_ctx_t SHMEM_CTX_DEFAULT = NULL;
shmem_ctx_t SHMEM_CTX_INVALID = &g_ctx_invalid;

static void agg_init(agg_t *g) {
  pthread_mutex_init(&g->mu, NULL);
  pthread_cond_init(&g->cv, NULL);
  g->arrived = g->mismatch = g->rc = 0;
  g->gen = 0;
}

static b200_team_t *team_new(int start, int stride, int size) {
  b200_team_t *t = (b200_team_t *)calloc(1, sizeof(*t));
  if (!t) return NULL;
  t->start = start;
  t->stride = size > 1 ? stride : 1;
  t->size = size;
  t->valid = 1;
  agg_init(&t->agg);
  pthread_mutex_lock(&g_teams_mu);
  t->next = g_teams;
  g_teams = t;
  pthread_mutex_unlock(&g_teams_mu);
  return t;
}

/* index of global PE `pe` in team t, or -1 */
static int team_index(const b200_team_t *t, int pe) {
  if (!t || !t->valid || pe < t->start) return -1;
  const int d = pe - t->start;
  if (d % t->stride) return -1;
  return d / t->stride < t->size ? d / t->stride : -1;
}

/* arrival point of the active set (PE_start, 2^logPE_stride, PE_size) */
static b200_team_t *active_set(int start, int logstride, int size) {
  const int stride = 1 << logstride;
  pthread_mutex_lock(&g_teams_mu);
  b200_team_t *t = g_actsets;
  for (; t; t = t->next)
    if (t->start == start && t->stride == (size > 1 ? stride : 1) && t->size == size) break;
  if (!t) {
    t = (b200_team_t *)calloc(1, sizeof(*t));
    if (t) {
      t->start = start;
      t->stride = size > 1 ? stride : 1;
      t->size = size;
      t->valid = 1;
      agg_init(&t->agg);
      t->next = g_actsets;
      g_actsets = t;
    }
  }
  pthread_mutex_unlock(&g_teams_mu);
  return t;
}

static int same_req(const coll_t *x, const coll_t *y) {
  /* collect is the one collective whose count differs between members */
  return x->kind == y->kind && x->op == y->op && x->dtype == y->dtype && x->algo == y->algo &&
         x->root == y->root && x->dest == y->dest && x->src == y->src &&
         (x->n == y->n || x->kind == K_COLLECT) && x->esize == y->esize && x->a == y->a &&
         x->b == y->b;
}

static int launch(b200_team_t *t, agg_t *g);

/* Record this member's arguments; the last member to arrive launches. */
static int arrive(b200_team_t *t, const coll_t *mine) {
  if (t_pe < 0) return set_err(B200SHM_ERR_STATE, "not a PE thread (start PEs with shmemx_b200_run)");
  if (!t || !t->valid) return set_err(B200SHM_ERR_ARG, "invalid team");
  if (team_index(t, t_pe) < 0)
    return set_err(B200SHM_ERR_ARG, "PE %d is not a member of the team/active set", t_pe);
  agg_t *g = &t->agg;
  pthread_mutex_lock(&g->mu);
  const unsigned long gen = g->gen;
  if (g->arrived == 0) {
    g->req = *mine;
    g->mismatch = 0;
  } else if (!same_req(&g->req, mine)) {
    g->mismatch = 1;
  }
  if (mine->kind == K_COLLECT) {
    if (g->counts_cap < t->size) {
      uint64_t *c = (uint64_t *)realloc(g->counts, (size_t)t->size * sizeof(uint64_t));
      if (!c) g->mismatch = 1;
      else {
        g->counts = c;
        g->counts_cap = t->size;
      }
    }
    if (g->counts_cap >= t->size) g->counts[team_index(t, t_pe)] = mine->n;
  }
  if (++g->arrived == t->size) {
    t_err[0] = 0;
    g->rc = g->mismatch ? set_err(B200SHM_ERR_ARG,
                                  "members passed different arguments (non-symmetric "
                                  "addresses or counts)")
                        : launch(t, g);
    /* every member reports the same failure, whichever thread launched */
    if (g->rc) snprintf(g->msg, sizeof(g->msg), "%s", t_err[0] ? t_err : b200shm_last_error());
    else g->msg[0] = 0;
    g->arrived = 0;
    g->gen++;
    pthread_cond_broadcast(&g->cv);
  } else {
    while (gen == g->gen) pthread_cond_wait(&g->cv, &g->mu);
  }
  const int rc = g->rc;
  if (rc) set_err(rc, "%s", g->msg);
  pthread_mutex_unlock(&g->mu);
  t_status = rc;
  return rc;
}

/* ---- algorithm names ------------------------------------------------------ */
static int parse_algo(const char *env, const char *const *names, int n, int dflt) {
  const char *e = getenv(env);
  if (!e || !*e) return dflt;
  char buf[64];
  snprintf(buf, sizeof(buf), "%s", e);
  char *colon = strchr(buf, ':'); /* "rec_dbl:int32" names a typed entry */
  if (colon) *colon = 0;
  for (int i = 0; i < n; i++)
    if (strcmp(buf, names[i]) == 0) return i;
  fprintf(stderr, "shmem_b200: unknown %s=%s, using the default\n", env, e);
  return dflt;
}
static const char *const k_reduce_names[] = {"linear", "binomial", "rec_dbl", "rabenseifner",
                                             "rabenseifner2"};
static const char *const k_barrier_names[] = {"linear", "complete_tree", "binomial_tree",
                                              "knomial_tree", "dissemination"};
static const char *const k_op_env[] = {"AND", "OR", "XOR", "MIN", "MAX", "SUM", "PROD"};
static int g_reduce_algo[2][7]; /* [0] team form, [1] to_all form */
static int g_barrier_algo, g_barrier_all_algo, g_sync_algo, g_sync_all_algo, g_team_sync_algo;

static void read_env(void) {
  char name[64];
  for (int op = 0; op < 7; op++) {
    snprintf(name, sizeof(name), "SHMEM_%s_REDUCE_ALGO", k_op_env[op]);
    g_reduce_algo[0][op] = parse_algo(name, k_reduce_names, 5, B200SHM_REC_DBL);
    snprintf(name, sizeof(name), "SHMEM_%s_TO_ALL_ALGO", k_op_env[op]);
    g_reduce_algo[1][op] = parse_algo(name, k_reduce_names, 5, B200SHM_REC_DBL);
  }
  g_barrier_algo = parse_algo("SHMEM_BARRIER_ALGO", k_barrier_names, 5, B200SHM_BAR_BINOMIAL_TREE);
  g_barrier_all_algo = parse_algo("SHMEM_BARRIER_ALL_ALGO", k_barrier_names, 5, B200SHM_BAR_BINOMIAL_TREE);
  g_sync_algo = parse_algo("SHMEM_SYNC_ALGO", k_barrier_names, 5, B200SHM_BAR_BINOMIAL_TREE);
  g_sync_all_algo = parse_algo("SHMEM_SYNC_ALL_ALGO", k_barrier_names, 5, B200SHM_BAR_BINOMIAL_TREE);
  g_team_sync_algo = parse_algo("SHMEM_TEAM_SYNC_ALGO", k_barrier_names, 5, B200SHM_BAR_BINOMIAL_TREE);
}

/* ---- the single device call of a collective -------------------------------- */
static int launch(b200_team_t *t, agg_t *g) {
  const coll_t *r = &g->req;
  switch (r->kind) {
  case K_MALLOC: {
    uint64_t off = 0;
    int rc = b200shm_malloc(r->n, r->a, &off);
    g->out = off;
    if (rc == 0) size_note(off, r->n);
    return engine_err(rc);
  }
  case K_FREE:
    size_forget(r->dest);
    return engine_err(b200shm_free(r->dest));
  case K_BARRIER: return engine_err(b200shm_barrier(r->algo, t->start, t->stride, t->size, NULL));
  case K_REDUCE:
    return engine_err(b200shm_reduce(r->op, r->dtype, r->algo, t->start, t->stride, t->size,
                                     r->dest, r->src, r->n, NULL));
  case K_FCOLLECT:
    return engine_err(b200shm_fcollect(t->start, t->stride, t->size, r->dest, r->src, r->n, NULL));
  case K_ALLTOALL:
    return engine_err(b200shm_alltoall(t->start, t->stride, t->size, r->dest, r->src, r->n, NULL));
  case K_COLLECT:
    return engine_err(b200shm_collect(t->start, t->stride, t->size, r->dest, r->src, g->counts,
                                      NULL));
  case K_ALLTOALLS:
    return engine_err(b200shm_alltoalls(t->start, t->stride, t->size, r->dest, r->src, r->a, r->b,
                                        r->n, r->esize, NULL));
  case K_BROADCAST:
    return engine_err(b200shm_broadcast(r->root, t->start, t->stride, t->size, r->dest, r->src,
                                        r->n, NULL));
  case K_SPLIT: { /* (start, stride, size) relative to the parent team */
    const int start = (int)r->a, stride = (int)r->b, size = (int)r->n;
    if (size < 1 || start < 0 || (size > 1 && stride < 1) ||
        start + (int64_t)(size - 1) * (size > 1 ? stride : 0) >= t->size)
      return set_err(B200SHM_ERR_ARG, "team_split_strided: (%d, %d, %d) outside the parent", start,
                     stride, size);
    b200_team_t *n = team_new(t->start + start * t->stride, t->stride * (size > 1 ? stride : 1), size);
    g->outp = n;
    return n ? 0 : set_err(B200SHM_ERR_NOMEM, "team_split_strided: out of memory");
  }
  case K_SPLIT2D: { /* x teams: runs of xrange members; y teams: members with equal i%xrange */
    const int xr = (int)r->a, n = t->size;
    if (xr < 1) return set_err(B200SHM_ERR_ARG, "team_split_2d: xrange %d < 1", xr);
    const int nx = (n + xr - 1) / xr, ny = xr < n ? xr : n;
    b200_team_t **xs = (b200_team_t **)calloc((size_t)nx, sizeof(*xs));
    b200_team_t **ys = (b200_team_t **)calloc((size_t)ny, sizeof(*ys));
    if (!xs || !ys) return set_err(B200SHM_ERR_NOMEM, "team_split_2d: out of memory");
    for (int k = 0; k < nx; k++) {
      const int sz = (n - k * xr) < xr ? (n - k * xr) : xr;
      xs[k] = team_new(t->start + k * xr * t->stride, t->stride, sz);
    }
    for (int j = 0; j < ny; j++)
      ys[j] = team_new(t->start + j * t->stride, t->stride * xr, (n - j + xr - 1) / xr);
    g->outp = xs;
    g->outq = ys;
    return 0;
  }
  case K_DESTROY: t->valid = 0; return 0;
  default: return set_err(B200SHM_ERR_ARG, "unknown collective");
  }
}

/* ---- symmetric addresses ------------------------------------------------- */
static int sym_off(const void *p, uint64_t *off) {
  const char *mine = g_base + (uint64_t)t_pe * g_slice;
  if ((const char *)p < mine || (const char *)p >= mine + g_slice)
    return set_err(B200SHM_ERR_ARG, "address %p is not in PE %d's symmetric heap", p, t_pe);
  *off = (uint64_t)((const char *)p - mine);
  return 0;
}

/* ---- start-up --------------------------------------------------------------- */
static uint64_t parse_size(const char *s, uint64_t dflt) {
  if (!s || !*s) return dflt;
  char *end = NULL;
  double v = strtod(s, &end);
  if (end && *end) {
    switch (*end) {
    case 'k': case 'K': v *= 1024.0; break;
    case 'm': case 'M': v *= 1024.0 * 1024.0; break;
    case 'g': case 'G': v *= 1024.0 * 1024.0 * 1024.0; break;
    default: break;
    }
  }
  return v > 0 ? (uint64_t)v : dflt;
}

static int engine_up(int npes) {
  if (b200shm_initialized()) {
    if (b200shm_n_pes() < npes)
      return set_err(B200SHM_ERR_STATE, "engine already started with %d PEs (< %d)",
                     b200shm_n_pes(), npes);
  } else {
    const uint64_t heap = parse_size(getenv("SHMEM_SYMMETRIC_SIZE"), 64ull << 20);
    const char *kind = getenv("SHMEM_B200_HEAP");
    const int flags = (kind && strcmp(kind, "device") == 0) ? 0 : B200SHM_INIT_MANAGED;
    int rc = b200shm_init(npes, heap, flags);
    if (rc) return engine_err(rc);
    uint64_t off = 0;
    if ((rc = b200shm_malloc(256, 256, &off))) return engine_err(rc);
    g_scratch = off;
  }
  g_base = (char *)b200shm_heap_base();
  g_slice = b200shm_heap_slice();
  g_npes = npes;
  g_world.start = 0;
  g_world.stride = 1;
  g_world.size = npes;
  g_world.valid = 1;
  agg_init(&g_world.agg);
  read_env();
  return 0;
}

struct pe_arg {
  void (*fn)(void *);
  void *arg;
  int pe;
};
static void *pe_trampoline(void *p) {
  struct pe_arg *a = (struct pe_arg *)p;
  t_pe = a->pe;
  t_err[0] = 0;
  a->fn(a->arg);
  return NULL;
}

static void stop_job_server(void);

int shmemx_b200_run(int npes, void (*pe_main)(void *), void *arg) {
  if (npes < 1 || !pe_main) return set_err(B200SHM_ERR_ARG, "shmemx_b200_run: bad arguments");
  int rc = engine_up(npes);
  if (rc) return rc;
  pthread_t *th = (pthread_t *)calloc((size_t)npes, sizeof(*th));
  struct pe_arg *args = (struct pe_arg *)calloc((size_t)npes, sizeof(*args));
  if (!th || !args) return set_err(B200SHM_ERR_NOMEM, "shmemx_b200_run: out of memory");
  for (int p = 0; p < npes; p++) {
    args[p].fn = pe_main;
    args[p].arg = arg;
    args[p].pe = p;
    if (pthread_create(&th[p], NULL, pe_trampoline, &args[p]) != 0)
      return set_err(B200SHM_ERR_STATE, "shmemx_b200_run: cannot start PE %d", p);
  }
  for (int p = 0; p < npes; p++) pthread_join(th[p], NULL);
  free(th);
  free(args);
  stop_job_server();
  return 0;
}

/* ---- setup / query ----------------------------------------------------------- */
static __thread int t_finalized;
static int g_thread_level = SHMEM_THREAD_SINGLE;
void shmem_init(void) {
  if (t_pe >= 0) return; /* PE threads are set up by shmemx_b200_run */
  if (engine_up(1) == 0) t_pe = 0; /* a lone thread becomes a 1-PE job */
}
int shmem_init_thread(int requested, int *provided) {
  shmem_init();
  if (requested >= SHMEM_THREAD_SINGLE && requested <= SHMEM_THREAD_MULTIPLE)
    g_thread_level = requested; /* every level is provided */
  if (provided) *provided = g_thread_level;
  return t_pe >= 0 ? 0 : -1;
}
void shmem_finalize(void) {
  shmem_barrier_all();
  t_finalized = 1;
}
int shmem_initialized(void) { return t_pe >= 0 && !t_finalized; }
int shmem_finalized(void) { return t_finalized; }
void shmem_query_thread(int *provided) {
  if (provided) *provided = g_thread_level;
}
void shmem_info_get_version(int *major, int *minor) {
  if (major) *major = SHMEM_MAJOR_VERSION;
  if (minor) *minor = SHMEM_MINOR_VERSION;
}
void shmem_info_get_name(char *name) {
  if (!name) return;
  strncpy(name, SHMEM_VENDOR_STRING, SHMEM_MAX_NAME_LEN - 1);
  name[SHMEM_MAX_NAME_LEN - 1] = '\0';
}
/* major * 100 + minor, and that * 100 + patch for the vendor's */
void shmem_info_get_version_number(int *version) {
  if (version) *version = SHMEM_MAJOR_VERSION * 100 + SHMEM_MINOR_VERSION;
}
void shmem_info_get_vendor_version(int *major, int *minor, int *patch) {
  if (major) *major = SHMEM_VENDOR_MAJOR_VERSION;
  if (minor) *minor = SHMEM_VENDOR_MINOR_VERSION;
  if (patch) *patch = SHMEM_VENDOR_PATCH_VERSION;
}
void shmem_info_get_vendor_version_number(int *version) {
  if (version)
    *version = (SHMEM_VENDOR_MAJOR_VERSION * 100 + SHMEM_VENDOR_MINOR_VERSION) * 100 +
               SHMEM_VENDOR_PATCH_VERSION;
}
void shmem_pcontrol(const int level, ...) { (void)level; /* no profiling levels */ }
int shmem_my_pe(void) { return t_pe; }
int shmem_n_pes(void) { return g_npes; }
int shmem_pe_accessible(int pe) { return pe >= 0 && pe < g_npes; }
void shmem_global_exit(int status) { exit(status); }

/* ---- symmetric heap ---------------------------------------------------------- */
void *shmem_align(size_t alignment, size_t size) {
  coll_t r = {0};
  r.kind = K_MALLOC;
  r.n = size;
  r.a = (int64_t)(alignment ? alignment : 256);
  if (arrive(&g_world, &r)) return NULL;
  return g_base + (uint64_t)t_pe * g_slice + g_world.agg.out;
}
void *shmem_malloc(size_t size) { return shmem_align(256, size); }
void *shmem_calloc(size_t count, size_t size) {
  char *p = (char *)shmem_malloc(count * size);
  if (p) {
    const uint64_t off = (uint64_t)(p - (g_base + (uint64_t)t_pe * g_slice));
    b200shm_memset(t_pe, 1, 1, off, 0, count * size, NULL);
    shmem_barrier_all();
  }
  return p;
}
void shmem_free(void *ptr) {
  if (!ptr) return;
  coll_t r = {0};
  r.kind = K_FREE;
  if (sym_off(ptr, &r.dest)) return;
  arrive(&g_world, &r);
}
void *shmem_malloc_with_hints(size_t size, long hints) {
  (void)hints; /* every object is reachable by atomics and signals alike */
  return shmem_malloc(size);
}
/* Collective, like shmem_malloc: a new object of `size` bytes, this PE's
 * first min(old, new) bytes copied into it, the old object freed. */
void *shmem_realloc(void *ptr, size_t size) {
  if (!ptr) return shmem_malloc(size);
  uint64_t off = 0;
  if (sym_off(ptr, &off)) {
    t_status = set_err(B200SHM_ERR_ARG, "shmem_realloc: %p is not a symmetric object", ptr);
    return NULL;
  }
  if (size == 0) {
    shmem_free(ptr);
    return NULL;
  }
  const uint64_t old = size_of_object(off);
  char *p = (char *)shmem_malloc(size);
  if (!p) return NULL; /* the old object stays */
  const uint64_t keep = old < size ? old : size;
  if (keep) t_status = engine_err(b200shm_memcpy(p, ptr, keep, NULL));
  shmem_free(ptr); /* collective: every member's copy is done before it returns */
  return p;
}
void *shmem_team_ptr(shmem_team_t team, const void *dest, int pe) {
  const b200_team_t *t = (const b200_team_t *)team;
  if (!t || !t->valid || pe < 0 || pe >= t->size) return NULL;
  return shmem_ptr(dest, t->start + pe * t->stride);
}
/* names before OpenSHMEM 1.2 */
void start_pes(int npes) {
  (void)npes; /* the job's size is shmemx_b200_run's */
  shmem_init();
}
int _my_pe(void) { return shmem_my_pe(); }
int _num_pes(void) { return shmem_n_pes(); }
void *shmalloc(size_t size) { return shmem_malloc(size); }
void shfree(void *ptr) { shmem_free(ptr); }
void *shrealloc(void *ptr, size_t size) { return shmem_realloc(ptr, size); }
void *shmemalign(size_t alignment, size_t size) { return shmem_align(alignment, size); }
void shmem_set_cache_inv(void) {}
void shmem_set_cache_line_inv(void *dest) { (void)dest; }
void shmem_clear_cache_inv(void) {}
void shmem_clear_cache_line_inv(void *dest) { (void)dest; }
void shmem_udcflush(void) {}
void shmem_udcflush_line(void *dest) { (void)dest; }
int shmem_addr_accessible(const void *addr, int pe) {
  uint64_t off = 0;
  return sym_off(addr, &off) == 0 && pe >= 0 && pe < g_npes;
}
void *shmem_ptr(const void *dest, int pe) {
  uint64_t off = 0;
  if (sym_off(dest, &off) || pe < 0 || pe >= g_npes) return NULL;
  return b200shm_ptr(pe, off);
}

/* ---- RMA ----------------------------------------------------------------------- */
/* ---- non-blocking operations: the serving loop ------------------------------ */
/* A _nbi put/get between two symmetric objects, and a fetching _nbi atomic,
 * is a request to the job's serving loop (b200shm_serve_*, started by the
 * first such call); the PE thread keeps its tickets, and shmem_quiet (and
 * every barrier, which implies quiet) waits for them and writes the fetched
 * values.  A put or get whose local buffer is not symmetric takes the
 * blocking path, which is complete on return as well. */
static pthread_mutex_t g_srv_mu = PTHREAD_MUTEX_INITIALIZER;
static b200shm_server *g_srv;
typedef struct {
  uint64_t ticket;
  void *fetch;
  int size;
} nbi_t;
/* the outstanding requests of one context */
typedef struct {
  nbi_t *v;
  int n, cap;
} nbi_list_t;
/* a context made by shmem_ctx_create: its own outstanding requests on the
 * job's one serving loop (contexts share the loop; they are completed, and
 * quieted, independently) */
typedef struct {
  unsigned magic;
  long options;
  b200_team_t *team; /* PE numbers are relative to this team (NULL: the world) */
  nbi_list_t list;
} b200_ctx_t;
#define B200_CTX_MAGIC 0xC0DE5EEDu
static __thread nbi_list_t t_default; /* SHMEM_CTX_DEFAULT of this PE */
#define t_nbi_n (t_default.n)

static b200shm_server *job_server(void) {
  pthread_mutex_lock(&g_srv_mu);
  if (!g_srv && b200shm_serve_start(4096, 0, 0.25, &g_srv) != 0) g_srv = NULL;
  b200shm_server *s = g_srv;
  pthread_mutex_unlock(&g_srv_mu);
  return s;
}

static void stop_job_server(void) {
  pthread_mutex_lock(&g_srv_mu);
  if (g_srv) b200shm_serve_stop(g_srv);
  g_srv = NULL;
  pthread_mutex_unlock(&g_srv_mu);
}

/* Complete the outstanding requests of one context. */
static int nbi_quiet_list(nbi_list_t *l) {
  int rc = 0;
  for (int i = 0; i < l->n; i++) {
    uint64_t f = 0;
    const int r = b200shm_serve_wait(g_srv, l->v[i].ticket, 60.0, &f);
    if (r) rc = engine_err(r);
    else if (l->v[i].fetch) memcpy(l->v[i].fetch, &f, (size_t)l->v[i].size);
  }
  l->n = 0;
  return rc;
}
static int nbi_quiet(void) { return nbi_quiet_list(&t_default); }

static b200_ctx_t *ctx_obj(shmem_ctx_t ctx) {
  if (!ctx || ctx == SHMEM_CTX_INVALID) return NULL;
  b200_ctx_t *c = (b200_ctx_t *)ctx;
  return c->magic == B200_CTX_MAGIC ? c : NULL;
}
/* the request list of a context handle (SHMEM_CTX_DEFAULT: this PE's own) */
static nbi_list_t *ctx_list(shmem_ctx_t ctx) {
  if (ctx == SHMEM_CTX_DEFAULT) return &t_default;
  b200_ctx_t *c = ctx_obj(ctx);
  return c ? &c->list : NULL;
}
/* the global PE of a context's PE number (-1 when it names none, which the
 * engine then refuses) */
static int ctx_pe(shmem_ctx_t ctx, int pe) {
  if (ctx == SHMEM_CTX_DEFAULT) return pe;
  const b200_ctx_t *c = ctx_obj(ctx);
  if (!c) return -1;
  if (!c->team) return pe;
  if (!c->team->valid || pe < 0 || pe >= c->team->size) return -1;
  return c->team->start + pe * c->team->stride;
}

/* 0 when queued, 1 when the loop is unavailable (take the blocking path), <0 on error. */
static int nbi_enqueue_on(nbi_list_t *l, const b200shm_request *r, void *fetch, int size) {
  if (!l) return set_err(B200SHM_ERR_ARG, "invalid context");
  b200shm_server *s = job_server();
  if (!s) return 1;
  uint64_t tk = 0;
  const double t0 = shmemx_wtime();
  for (;;) {
    const int rc = b200shm_serve_enqueue(s, r, &tk);
    if (rc == 0) break;
    if (rc != B200SHM_ERR_BUSY) return engine_err(rc);
    if (l->n) nbi_quiet_list(l); /* free slots held by this context */
    else sched_yield();          /* other slots free as the GPU completes them */
    if (shmemx_wtime() - t0 > 60.0) return set_err(B200SHM_ERR_TIMEOUT, "nbi: no free slot");
  }
  if (l->n == l->cap) {
    const int cap = l->cap ? 2 * l->cap : 64;
    nbi_t *n = (nbi_t *)realloc(l->v, (size_t)cap * sizeof(nbi_t));
    if (!n) {
      uint64_t f = 0;
      b200shm_serve_wait(s, tk, 60.0, &f);
      if (fetch) memcpy(fetch, &f, (size_t)size);
      return 0;
    }
    l->v = n;
    l->cap = cap;
  }
  l->v[l->n].ticket = tk;
  l->v[l->n].fetch = fetch;
  l->v[l->n].size = size;
  l->n++;
  return 0;
}
static int nbi_enqueue(const b200shm_request *r, void *fetch, int size) {
  return nbi_enqueue_on(&t_default, r, fetch, size);
}

/* put (kind PUT) or get (kind GET) of n bytes between this PE and `pe`; 1 if
 * an address is not symmetric */
static int nbi_rma(nbi_list_t *l, int kind, void *dest, const void *source, size_t n, int pe) {
  if (!l) return set_err(B200SHM_ERR_ARG, "invalid context");
  uint64_t doff, soff;
  const char *mine = g_base + (uint64_t)t_pe * g_slice;
  const char *d = (const char *)dest, *sp = (const char *)source;
  if (d < mine || d >= mine + g_slice || sp < mine || sp >= mine + g_slice) return 1;
  doff = (uint64_t)(d - mine);
  soff = (uint64_t)(sp - mine);
  b200shm_request r;
  memset(&r, 0, sizeof(r));
  r.kind = kind;
  r.pe_start = t_pe;
  r.pe_stride = 1;
  r.pe_size = 1;
  r.pe = pe;
  r.dest_off = doff;
  r.src_off = soff;
  r.n = n;
  return nbi_enqueue_on(l, &r, NULL, 0);
}

static void nbi_amo(nbi_list_t *l, int op, int dtype, const void *dest, int pe,
                    const void *value, const void *cond, void *fetch, int size) {
  uint64_t off = 0;
  if (sym_off(dest, &off)) {
    t_status = B200SHM_ERR_ARG;
    return;
  }
  b200shm_request r;
  memset(&r, 0, sizeof(r));
  r.kind = B200SHM_REQ_AMO;
  r.op = op;
  r.dtype = dtype;
  r.pe = pe;
  r.dest_off = off;
  if (value) memcpy(&r.value, value, (size_t)size);
  if (cond) memcpy(&r.cond, cond, (size_t)size);
  const int rc = nbi_enqueue_on(l, &r, fetch, size);
  if (rc == 1) /* no serving loop: the blocking form */
    t_status = engine_err(b200shm_amo(op, dtype, pe, off, value, cond, fetch));
  else
    t_status = rc;
}

void shmem_putmem(void *dest, const void *source, size_t nelems, int pe) {
  uint64_t off = 0;
  if (sym_off(dest, &off) == 0) t_status = engine_err(b200shm_memcpy(b200shm_ptr(pe, off), source, nelems, NULL));
}
void shmem_getmem(void *dest, const void *source, size_t nelems, int pe) {
  uint64_t off = 0;
  if (sym_off(source, &off) == 0) t_status = engine_err(b200shm_memcpy(dest, b200shm_ptr(pe, off), nelems, NULL));
}
void shmem_ctx_putmem_nbi(shmem_ctx_t ctx, void *dest, const void *source, size_t nelems,
                          int pe) {
  const int g = ctx_pe(ctx, pe);
  const int rc = nbi_rma(ctx_list(ctx), B200SHM_REQ_PUT, dest, source, nelems, g);
  if (rc == 1) shmem_putmem(dest, source, nelems, g);
  else t_status = rc;
}
void shmem_ctx_getmem_nbi(shmem_ctx_t ctx, void *dest, const void *source, size_t nelems,
                          int pe) {
  const int g = ctx_pe(ctx, pe);
  const int rc = nbi_rma(ctx_list(ctx), B200SHM_REQ_GET, dest, source, nelems, g);
  if (rc == 1) shmem_getmem(dest, source, nelems, g);
  else t_status = rc;
}
void shmem_putmem_nbi(void *dest, const void *source, size_t nelems, int pe) {
  shmem_ctx_putmem_nbi(SHMEM_CTX_DEFAULT, dest, source, nelems, pe);
}
void shmem_getmem_nbi(void *dest, const void *source, size_t nelems, int pe) {
  shmem_ctx_getmem_nbi(SHMEM_CTX_DEFAULT, dest, source, nelems, pe);
}
void shmem_ctx_putmem(shmem_ctx_t ctx, void *dest, const void *source, size_t nelems, int pe) {
  shmem_putmem(dest, source, nelems, ctx_pe(ctx, pe));
}
void shmem_ctx_getmem(shmem_ctx_t ctx, void *dest, const void *source, size_t nelems, int pe) {
  shmem_getmem(dest, source, nelems, ctx_pe(ctx, pe));
}

/* ---- contexts (api.h: shmem_ctx_create / destroy / quiet / fence) ---------- */
static int ctx_make(b200_team_t *team, long options, shmem_ctx_t *ctxp) {
  if (!ctxp) return -1;
  *ctxp = SHMEM_CTX_INVALID;
  if (team && !team->valid) return -1;
  b200_ctx_t *c = (b200_ctx_t *)calloc(1, sizeof(*c));
  if (!c) return -1;
  c->magic = B200_CTX_MAGIC;
  c->options = options;
  c->team = team == &g_world ? NULL : team;
  *ctxp = (shmem_ctx_t)c;
  return 0;
}
int shmem_ctx_create(long options, shmem_ctx_t *ctxp) { return ctx_make(NULL, options, ctxp); }
int shmem_team_create_ctx(shmem_team_t team, long options, shmem_ctx_t *ctxp) {
  if (!team) {
    if (ctxp) *ctxp = SHMEM_CTX_INVALID;
    return -1;
  }
  return ctx_make((b200_team_t *)team, options, ctxp);
}
int shmem_ctx_get_team(shmem_ctx_t ctx, shmem_team_t *team) {
  if (!team) return -1;
  if (ctx == SHMEM_CTX_DEFAULT) {
    *team = SHMEM_TEAM_WORLD;
    return 0;
  }
  const b200_ctx_t *c = ctx_obj(ctx);
  if (!c) {
    *team = SHMEM_TEAM_INVALID;
    return -1;
  }
  *team = c->team ? (shmem_team_t)c->team : SHMEM_TEAM_WORLD;
  return 0;
}
void shmem_ctx_quiet(shmem_ctx_t ctx) {
  nbi_list_t *l = ctx_list(ctx);
  if (!l) {
    t_status = set_err(B200SHM_ERR_ARG, "invalid context");
    return;
  }
  const int rc = l->n ? nbi_quiet_list(l) : 0;
  const int r2 = b200shm_quiet();
  t_status = rc ? rc : engine_err(r2);
}
void shmem_ctx_fence(shmem_ctx_t ctx) { shmem_ctx_quiet(ctx); }
int shmemx_b200_ctx_pending(shmem_ctx_t ctx) {
  const nbi_list_t *l = ctx_list(ctx);
  return l ? l->n : -1;
}
void shmem_ctx_destroy(shmem_ctx_t ctx) {
  b200_ctx_t *c = ctx_obj(ctx);
  if (!c) return; /* the default and invalid contexts are not destroyed */
  shmem_ctx_quiet(ctx); /* destroying a context completes its operations */
  free(c->list.v);
  c->magic = 0;
  free(c);
}
/* Requests in flight may complete in any order, so fence (ordering of this
 * PE's puts to one PE) is as strong as quiet here. */
void shmem_fence(void) { shmem_quiet(); }
void shmem_quiet(void) {
  int rc = t_nbi_n ? nbi_quiet() : 0;
  const int r2 = b200shm_quiet();
  t_status = rc ? rc : engine_err(r2);
}

#define DEF_RMA(_type, _tn)                                                    \
  void shmem_##_tn##_put(_type *dest, const _type *source, size_t nelems,      \
                         int pe) {                                             \
    shmem_putmem(dest, source, nelems * sizeof(_type), pe);                    \
  }                                                                            \
  void shmem_##_tn##_get(_type *dest, const _type *source, size_t nelems,      \
                         int pe) {                                             \
    shmem_getmem(dest, source, nelems * sizeof(_type), pe);                    \
  }                                                                            \
  void shmem_##_tn##_p(_type *dest, _type value, int pe) {                     \
    shmem_putmem(dest, &value, sizeof(_type), pe);                             \
  }                                                                            \
  _type shmem_##_tn##_g(const _type *source, int pe) {                         \
    _type v;                                                                   \
    memset(&v, 0, sizeof(v));                                                  \
    shmem_getmem(&v, source, sizeof(_type), pe);                               \
    return v;                                                                  \
  }                                                                            \
  void shmem_##_tn##_put_nbi(_type *dest, const _type *source, size_t nelems,  \
                             int pe) {                                         \
    shmem_putmem_nbi(dest, source, nelems * sizeof(_type), pe);                \
  }                                                                            \
  void shmem_##_tn##_get_nbi(_type *dest, const _type *source, size_t nelems,  \
                             int pe) {                                         \
    shmem_getmem_nbi(dest, source, nelems * sizeof(_type), pe);                \
  }                                                                            \
  void shmem_ctx_##_tn##_put(shmem_ctx_t ctx, _type *dest,                     \
                             const _type *source,                              \
                             size_t nelems, int pe) {                          \
    shmem_ctx_putmem(ctx, dest, source, nelems * sizeof(_type), pe);           \
  }                                                                            \
  void shmem_ctx_##_tn##_get(shmem_ctx_t ctx, _type *dest,                     \
                             const _type *source,                              \
                             size_t nelems, int pe) {                          \
    shmem_ctx_getmem(ctx, dest, source, nelems * sizeof(_type), pe);           \
  }                                                                            \
  void shmem_ctx_##_tn##_p(shmem_ctx_t ctx, _type *dest, _type value,          \
                           int pe) {                                           \
    shmem_ctx_putmem(ctx, dest, &value, sizeof(_type), pe);                    \
  }                                                                            \
  _type shmem_ctx_##_tn##_g(shmem_ctx_t ctx, const _type *source, int pe) {    \
    _type v;                                                                   \
    memset(&v, 0, sizeof(v));                                                  \
    shmem_ctx_getmem(ctx, &v, source, sizeof(_type), pe);                      \
    return v;                                                                  \
  }                                                                            \
  void shmem_ctx_##_tn##_put_nbi(shmem_ctx_t ctx, _type *dest,                 \
                                 const _type *source, size_t nelems, int pe) { \
    shmem_ctx_putmem_nbi(ctx, dest, source, nelems * sizeof(_type), pe);       \
  }                                                                            \
  void shmem_ctx_##_tn##_get_nbi(shmem_ctx_t ctx, _type *dest,                 \
                                 const _type *source, size_t nelems, int pe) { \
    shmem_ctx_getmem_nbi(ctx, dest, source, nelems * sizeof(_type), pe);       \
  }
SHMEM_B200_RMA_TYPES(DEF_RMA)

/* ---- synchronisation ---------------------------------------------------------- */
static int barrier_on(b200_team_t *t, int algo) {
  if (t_nbi_n) nbi_quiet(); /* a barrier completes this PE's outstanding requests */
  coll_t r = {0};
  r.kind = K_BARRIER;
  r.algo = algo;
  return arrive(t, &r);
}
void shmem_barrier_all(void) { barrier_on(&g_world, g_barrier_all_algo); }
void shmem_sync_all(void) { barrier_on(&g_world, g_sync_all_algo); }
void shmem_barrier(int PE_start, int logPE_stride, int PE_size, long *pSync) {
  (void)pSync; /* the engine owns its flag words */
  barrier_on(active_set(PE_start, logPE_stride, PE_size), g_barrier_algo);
}
void shmem_sync(int PE_start, int logPE_stride, int PE_size, long *pSync) {
  (void)pSync;
  barrier_on(active_set(PE_start, logPE_stride, PE_size), g_sync_algo);
}
void shmem_sync_deprecated(int PE_start, int logPE_stride, int PE_size, long *pSync) {
  shmem_sync(PE_start, logPE_stride, PE_size, pSync);
}
int shmem_team_sync(shmem_team_t team) {
  return barrier_on((b200_team_t *)team, g_team_sync_algo);
}

/* ---- teams --------------------------------------------------------------------- */
int shmem_team_my_pe(shmem_team_t team) { return team_index((b200_team_t *)team, t_pe); }
int shmem_team_n_pes(shmem_team_t team) {
  b200_team_t *t = (b200_team_t *)team;
  return (t && t->valid) ? t->size : -1;
}
int shmem_team_translate_pe(shmem_team_t src_team, int src_pe, shmem_team_t dest_team) {
  b200_team_t *s = (b200_team_t *)src_team;
  if (!s || !s->valid || src_pe < 0 || src_pe >= s->size) return -1;
  return team_index((b200_team_t *)dest_team, s->start + src_pe * s->stride);
}
int shmem_team_get_config(shmem_team_t team, long config_mask, shmem_team_config_t *config) {
  (void)config_mask;
  if (!team || !config) return -1;
  config->num_contexts = 0;
  return 0;
}
int shmem_team_split_strided(shmem_team_t parent_team, int start, int stride, int size,
                             const shmem_team_config_t *config, long config_mask,
                             shmem_team_t *new_team) {
  (void)config;
  (void)config_mask;
  b200_team_t *p = (b200_team_t *)parent_team;
  coll_t r = {0};
  r.kind = K_SPLIT;
  r.a = start;
  r.b = stride;
  r.n = (uint64_t)size;
  int rc = arrive(p, &r);
  if (new_team) *new_team = SHMEM_TEAM_INVALID;
  if (rc) return -1;
  b200_team_t *n = (b200_team_t *)p->agg.outp;
  if (new_team && team_index(n, t_pe) >= 0) *new_team = n;
  return 0;
}
int shmem_team_split_2d(shmem_team_t parent_team, int xrange,
                        const shmem_team_config_t *xaxis_config, long xaxis_mask,
                        shmem_team_t *xaxis_team, const shmem_team_config_t *yaxis_config,
                        long yaxis_mask, shmem_team_t *yaxis_team) {
  (void)xaxis_config;
  (void)xaxis_mask;
  (void)yaxis_config;
  (void)yaxis_mask;
  b200_team_t *p = (b200_team_t *)parent_team;
  coll_t r = {0};
  r.kind = K_SPLIT2D;
  r.a = xrange;
  if (xaxis_team) *xaxis_team = SHMEM_TEAM_INVALID;
  if (yaxis_team) *yaxis_team = SHMEM_TEAM_INVALID;
  if (arrive(p, &r)) return -1;
  const int i = team_index(p, t_pe);
  b200_team_t **xs = (b200_team_t **)p->agg.outp, **ys = (b200_team_t **)p->agg.outq;
  if (xaxis_team) *xaxis_team = xs[i / xrange];
  if (yaxis_team) *yaxis_team = ys[i % xrange];
  return 0;
}
void shmem_team_destroy(shmem_team_t team) {
  coll_t r = {0};
  r.kind = K_DESTROY;
  if (team && team != SHMEM_TEAM_WORLD) arrive((b200_team_t *)team, &r);
}

/* ---- reductions --------------------------------------------------------------- */
#define B200_DTYPE_OF(_type)                                                   \
  _Generic((_type)0, char: B200SHM_I8, signed char: B200SHM_I8,                \
           unsigned char: B200SHM_U8, short: B200SHM_I16,                      \
           unsigned short: B200SHM_U16, int: B200SHM_I32,                      \
           unsigned int: B200SHM_U32, long: B200SHM_I64,                       \
           unsigned long: B200SHM_U64, long long: B200SHM_I64,                 \
           unsigned long long: B200SHM_U64, float: B200SHM_F32,                \
           double: B200SHM_F64, long double: B200SHM_F80,                      \
           float _Complex: B200SHM_C32, double _Complex: B200SHM_C64)

static int reduce_on(b200_team_t *t, int op, int dtype, int form, void *dest, const void *source,
                     size_t n) {
  coll_t r = {0};
  r.kind = K_REDUCE;
  r.op = op;
  r.dtype = dtype;
  r.algo = g_reduce_algo[form][op];
  r.n = n;
  if (sym_off(dest, &r.dest) || sym_off(source, &r.src)) return t_status = B200SHM_ERR_ARG;
  return arrive(t, &r);
}

#define DEF_TEAM_REDUCE(_type, _tn, _op, _OP)                                  \
  int shmem_##_tn##_##_op##_reduce(shmem_team_t team, _type *dest,             \
                                   const _type *source, size_t nreduce) {      \
    return reduce_on((b200_team_t *)team, _OP, B200_DTYPE_OF(_type), 0, dest,  \
                     source, nreduce);                                         \
  }
#define DEF_TO_ALL(_type, _tn, _op, _OP)                                       \
  void shmem_##_tn##_##_op##_to_all(_type *dest, const _type *source,          \
                                    int nreduce, int PE_start,                 \
                                    int logPE_stride, int PE_size,             \
                                    _type *pWrk, long *pSync) {                \
    (void)pWrk;                                                                \
    (void)pSync;                                                               \
    reduce_on(active_set(PE_start, logPE_stride, PE_size), _OP,                \
              B200_DTYPE_OF(_type), 1, dest, source,                           \
              nreduce > 0 ? (size_t)nreduce : 0);                              \
  }
#define R_AND(_t, _n) DEF_TEAM_REDUCE(_t, _n, and, B200SHM_AND)
#define R_OR(_t, _n) DEF_TEAM_REDUCE(_t, _n, or, B200SHM_OR)
#define R_XOR(_t, _n) DEF_TEAM_REDUCE(_t, _n, xor, B200SHM_XOR)
#define R_MIN(_t, _n) DEF_TEAM_REDUCE(_t, _n, min, B200SHM_MIN)
#define R_MAX(_t, _n) DEF_TEAM_REDUCE(_t, _n, max, B200SHM_MAX)
#define R_SUM(_t, _n) DEF_TEAM_REDUCE(_t, _n, sum, B200SHM_SUM)
#define R_PROD(_t, _n) DEF_TEAM_REDUCE(_t, _n, prod, B200SHM_PROD)
SHMEM_B200_REDUCE_BITWISE_TYPES(R_AND)
SHMEM_B200_REDUCE_BITWISE_TYPES(R_OR)
SHMEM_B200_REDUCE_BITWISE_TYPES(R_XOR)
SHMEM_B200_REDUCE_MINMAX_TYPES(R_MIN)
SHMEM_B200_REDUCE_MINMAX_TYPES(R_MAX)
SHMEM_B200_REDUCE_ARITH_TYPES(R_SUM)
SHMEM_B200_REDUCE_ARITH_TYPES(R_PROD)
#define A_AND(_t, _n) DEF_TO_ALL(_t, _n, and, B200SHM_AND)
#define A_OR(_t, _n) DEF_TO_ALL(_t, _n, or, B200SHM_OR)
#define A_XOR(_t, _n) DEF_TO_ALL(_t, _n, xor, B200SHM_XOR)
#define A_MIN(_t, _n) DEF_TO_ALL(_t, _n, min, B200SHM_MIN)
#define A_MAX(_t, _n) DEF_TO_ALL(_t, _n, max, B200SHM_MAX)
#define A_SUM(_t, _n) DEF_TO_ALL(_t, _n, sum, B200SHM_SUM)
#define A_PROD(_t, _n) DEF_TO_ALL(_t, _n, prod, B200SHM_PROD)
SHMEM_B200_TO_ALL_BITWISE_TYPES(A_AND)
SHMEM_B200_TO_ALL_BITWISE_TYPES(A_OR)
SHMEM_B200_TO_ALL_BITWISE_TYPES(A_XOR)
SHMEM_B200_TO_ALL_MINMAX_TYPES(A_MIN)
SHMEM_B200_TO_ALL_MINMAX_TYPES(A_MAX)
SHMEM_B200_TO_ALL_ARITH_TYPES(A_SUM)
SHMEM_B200_TO_ALL_ARITH_TYPES(A_PROD)

/* ---- data movement -------------------------------------------------------------- */
static int copy_on(b200_team_t *t, int kind, void *dest, const void *source, uint64_t n,
                   int64_t a, int64_t b, uint64_t esize, int root) {
  coll_t r = {0};
  r.kind = kind;
  r.n = n;
  r.a = a;
  r.b = b;
  r.esize = esize;
  r.root = root;
  if (sym_off(dest, &r.dest) || sym_off(source, &r.src)) return t_status = B200SHM_ERR_ARG;
  return arrive(t, &r);
}

#define DEF_COPY(_type, _tn)                                                   \
  int shmem_##_tn##_fcollect(shmem_team_t team, _type *dest,                   \
                             const _type *source, size_t nelems) {             \
    return copy_on((b200_team_t *)team, K_FCOLLECT, dest, source,              \
                   nelems * sizeof(_type), 0, 0, 0, 0);                        \
  }                                                                            \
  int shmem_##_tn##_collect(shmem_team_t team, _type *dest,                    \
                            const _type *source, size_t nelems) {              \
    return copy_on((b200_team_t *)team, K_COLLECT, dest, source,               \
                   nelems * sizeof(_type), 0, 0, 0, 0);                        \
  }                                                                            \
  int shmem_##_tn##_alltoall(shmem_team_t team, _type *dest,                   \
                             const _type *source, size_t nelems) {             \
    return copy_on((b200_team_t *)team, K_ALLTOALL, dest, source,              \
                   nelems * sizeof(_type), 0, 0, 0, 0);                        \
  }                                                                            \
  int shmem_##_tn##_alltoalls(shmem_team_t team, _type *dest,                  \
                              const _type *source, ptrdiff_t dst,              \
                              ptrdiff_t sst, size_t nelems) {                  \
    return copy_on((b200_team_t *)team, K_ALLTOALLS, dest, source, nelems,     \
                   dst, sst, sizeof(_type), 0);                                \
  }                                                                            \
  int shmem_##_tn##_broadcast(shmem_team_t team, _type *dest,                  \
                              const _type *source, size_t nelems,              \
                              int PE_root) {                                   \
    return copy_on((b200_team_t *)team, K_BROADCAST, dest, source,             \
                   nelems * sizeof(_type), 0, 0, 0, PE_root);                  \
  }
SHMEM_B200_RMA_TYPES(DEF_COPY)

int shmem_fcollectmem(shmem_team_t team, void *dest, const void *source, size_t nelems) {
  return copy_on((b200_team_t *)team, K_FCOLLECT, dest, source, nelems, 0, 0, 0, 0);
}
int shmem_collectmem(shmem_team_t team, void *dest, const void *source, size_t nelems) {
  return copy_on((b200_team_t *)team, K_COLLECT, dest, source, nelems, 0, 0, 0, 0);
}
int shmem_alltoallmem(shmem_team_t team, void *dest, const void *source, size_t nelems) {
  return copy_on((b200_team_t *)team, K_ALLTOALL, dest, source, nelems, 0, 0, 0, 0);
}
int shmem_alltoallsmem(shmem_team_t team, void *dest, const void *source, ptrdiff_t dst,
                       ptrdiff_t sst, size_t nelems) {
  /* one element of nelems bytes per PE pair (alltoalls.c:397-435) */
  return copy_on((b200_team_t *)team, K_ALLTOALLS, dest, source, 1, dst, sst, nelems, 0);
}
int shmem_broadcastmem(shmem_team_t team, void *dest, const void *source, size_t nelems,
                       int PE_root) {
  return copy_on((b200_team_t *)team, K_BROADCAST, dest, source, nelems, 0, 0, 0, PE_root);
}

#define DEF_SIZED(_bits)                                                       \
  void shmem_fcollect##_bits(void *target, const void *source, size_t nelems,  \
                             int PE_start, int logPE_stride, int PE_size,      \
                             long *pSync) {                                    \
    (void)pSync;                                                               \
    copy_on(active_set(PE_start, logPE_stride, PE_size), K_FCOLLECT, target,   \
            source, nelems * (_bits / 8), 0, 0, 0, 0);                         \
  }                                                                            \
  void shmem_collect##_bits(void *target, const void *source, size_t nelems,   \
                            int PE_start, int logPE_stride, int PE_size,       \
                            long *pSync) {                                     \
    (void)pSync;                                                               \
    copy_on(active_set(PE_start, logPE_stride, PE_size), K_COLLECT, target,    \
            source, nelems * (_bits / 8), 0, 0, 0, 0);                         \
  }                                                                            \
  void shmem_alltoall##_bits(void *target, const void *source, size_t nelems,  \
                             int PE_start, int logPE_stride, int PE_size,      \
                             long *pSync) {                                    \
    (void)pSync;                                                               \
    copy_on(active_set(PE_start, logPE_stride, PE_size), K_ALLTOALL, target,   \
            source, nelems * (_bits / 8), 0, 0, 0, 0);                         \
  }                                                                            \
  void shmem_alltoalls##_bits(void *target, const void *source, ptrdiff_t dst, \
                              ptrdiff_t sst, size_t nelems, int PE_start,      \
                              int logPE_stride, int PE_size, long *pSync) {    \
    (void)pSync;                                                               \
    copy_on(active_set(PE_start, logPE_stride, PE_size), K_ALLTOALLS, target,  \
            source, nelems, dst, sst, _bits / 8, 0);                           \
  }                                                                            \
  void shmem_broadcast##_bits(void *target, const void *source, size_t nelems, \
                              int PE_root, int PE_start, int logPE_stride,     \
                              int PE_size, long *pSync) {                      \
    (void)pSync;                                                               \
    copy_on(active_set(PE_start, logPE_stride, PE_size), K_BROADCAST, target,  \
            source, nelems * (_bits / 8), 0, 0, 0, PE_root);                   \
  }
DEF_SIZED(32)
DEF_SIZED(64)

/* ---- atomics ------------------------------------------------------------------ */
static void amo(int op, int dtype, const void *dest, int pe, const void *value, const void *cond,
                void *fetched) {
  uint64_t off = 0;
  if (sym_off(dest, &off)) {
    t_status = B200SHM_ERR_ARG;
    return;
  }
  t_status = engine_err(b200shm_amo(op, dtype, pe, off, value, cond, fetched));
}

#define DEF_AMO_STD(_type, _tn)                                                \
  _type shmem_##_tn##_atomic_fetch_add(_type *dest, _type value, int pe) {     \
    _type old = 0;                                                             \
    amo(B200SHM_AMO_FETCH_ADD, B200_DTYPE_OF(_type), dest, pe, &value, NULL,   \
        &old);                                                                 \
    return old;                                                                \
  }                                                                            \
  void shmem_##_tn##_atomic_add(_type *dest, _type value, int pe) {            \
    amo(B200SHM_AMO_ADD, B200_DTYPE_OF(_type), dest, pe, &value, NULL, NULL);  \
  }                                                                            \
  _type shmem_##_tn##_atomic_fetch_inc(_type *dest, int pe) {                  \
    _type old = 0;                                                             \
    amo(B200SHM_AMO_FETCH_INC, B200_DTYPE_OF(_type), dest, pe, NULL, NULL,     \
        &old);                                                                 \
    return old;                                                                \
  }                                                                            \
  void shmem_##_tn##_atomic_inc(_type *dest, int pe) {                         \
    amo(B200SHM_AMO_INC, B200_DTYPE_OF(_type), dest, pe, NULL, NULL, NULL);    \
  }                                                                            \
  _type shmem_##_tn##_atomic_compare_swap(_type *dest, _type cond,             \
                                          _type value, int pe) {               \
    _type old = 0;                                                             \
    amo(B200SHM_AMO_CSWAP, B200_DTYPE_OF(_type), dest, pe, &value, &cond,      \
        &old);                                                                 \
    return old;                                                                \
  }                                                                            \
  _type shmem_ctx_##_tn##_atomic_fetch_add(shmem_ctx_t ctx, _type *dest,       \
                                           _type value, int pe) {              \
    return shmem_##_tn##_atomic_fetch_add(dest, value, ctx_pe(ctx, pe));       \
  }                                                                            \
  void shmem_ctx_##_tn##_atomic_add(shmem_ctx_t ctx, _type *dest, _type value, \
                                    int pe) {                                  \
    shmem_##_tn##_atomic_add(dest, value, ctx_pe(ctx, pe));                    \
  }                                                                            \
  _type shmem_ctx_##_tn##_atomic_fetch_inc(shmem_ctx_t ctx, _type *dest,       \
                                           int pe) {                           \
    return shmem_##_tn##_atomic_fetch_inc(dest, ctx_pe(ctx, pe));              \
  }                                                                            \
  void shmem_ctx_##_tn##_atomic_inc(shmem_ctx_t ctx, _type *dest, int pe) {    \
    shmem_##_tn##_atomic_inc(dest, ctx_pe(ctx, pe));                           \
  }                                                                            \
  _type shmem_ctx_##_tn##_atomic_compare_swap(shmem_ctx_t ctx, _type *dest,    \
                                              _type cond, _type value,         \
                                              int pe) {                        \
    return shmem_##_tn##_atomic_compare_swap(dest, cond, value, ctx_pe(ctx, pe)); \
  }
#define DEF_AMO_EXT(_type, _tn)                                                \
  _type shmem_##_tn##_atomic_swap(_type *dest, _type value, int pe) {          \
    _type old = 0;                                                             \
    amo(B200SHM_AMO_SWAP, B200_DTYPE_OF(_type), dest, pe, &value, NULL, &old); \
    return old;                                                                \
  }                                                                            \
  void shmem_##_tn##_atomic_set(_type *dest, _type value, int pe) {            \
    amo(B200SHM_AMO_SET, B200_DTYPE_OF(_type), dest, pe, &value, NULL, NULL);  \
  }                                                                            \
  _type shmem_##_tn##_atomic_fetch(const _type *source, int pe) {              \
    _type old = 0;                                                             \
    amo(B200SHM_AMO_FETCH, B200_DTYPE_OF(_type), source, pe, NULL, NULL,       \
        &old);                                                                 \
    return old;                                                                \
  }                                                                            \
  _type shmem_ctx_##_tn##_atomic_swap(shmem_ctx_t ctx, _type *dest,            \
                                      _type value, int pe) {                   \
    return shmem_##_tn##_atomic_swap(dest, value, ctx_pe(ctx, pe));            \
  }                                                                            \
  void shmem_ctx_##_tn##_atomic_set(shmem_ctx_t ctx, _type *dest, _type value, \
                                    int pe) {                                  \
    shmem_##_tn##_atomic_set(dest, value, ctx_pe(ctx, pe));                    \
  }                                                                            \
  _type shmem_ctx_##_tn##_atomic_fetch(shmem_ctx_t ctx, const _type *source,   \
                                       int pe) {                               \
    return shmem_##_tn##_atomic_fetch(source, ctx_pe(ctx, pe));                \
  }
#define DEF_AMO_BIT(_type, _tn)                                                \
  _type shmem_##_tn##_atomic_fetch_and(_type *dest, _type value, int pe) {     \
    _type old = 0;                                                             \
    amo(B200SHM_AMO_FETCH_AND, B200_DTYPE_OF(_type), dest, pe, &value, NULL,   \
        &old);                                                                 \
    return old;                                                                \
  }                                                                            \
  _type shmem_##_tn##_atomic_fetch_or(_type *dest, _type value, int pe) {      \
    _type old = 0;                                                             \
    amo(B200SHM_AMO_FETCH_OR, B200_DTYPE_OF(_type), dest, pe, &value, NULL,    \
        &old);                                                                 \
    return old;                                                                \
  }                                                                            \
  _type shmem_##_tn##_atomic_fetch_xor(_type *dest, _type value, int pe) {     \
    _type old = 0;                                                             \
    amo(B200SHM_AMO_FETCH_XOR, B200_DTYPE_OF(_type), dest, pe, &value, NULL,   \
        &old);                                                                 \
    return old;                                                                \
  }                                                                            \
  void shmem_##_tn##_atomic_and(_type *dest, _type value, int pe) {            \
    amo(B200SHM_AMO_AND, B200_DTYPE_OF(_type), dest, pe, &value, NULL, NULL);  \
  }                                                                            \
  void shmem_##_tn##_atomic_or(_type *dest, _type value, int pe) {             \
    amo(B200SHM_AMO_OR, B200_DTYPE_OF(_type), dest, pe, &value, NULL, NULL);   \
  }                                                                            \
  void shmem_##_tn##_atomic_xor(_type *dest, _type value, int pe) {            \
    amo(B200SHM_AMO_XOR, B200_DTYPE_OF(_type), dest, pe, &value, NULL, NULL);  \
  }                                                                            \
  _type shmem_ctx_##_tn##_atomic_fetch_and(shmem_ctx_t ctx, _type *dest,       \
                                           _type value,                        \
                                          int pe) {                            \
    return shmem_##_tn##_atomic_fetch_and(dest, value, ctx_pe(ctx, pe));       \
  }                                                                            \
  void shmem_ctx_##_tn##_atomic_and(shmem_ctx_t ctx, _type *dest,              \
                                    _type value, int pe) {                     \
    shmem_##_tn##_atomic_and(dest, value, ctx_pe(ctx, pe));                    \
  }                                                                            \
  _type shmem_ctx_##_tn##_atomic_fetch_or(shmem_ctx_t ctx, _type *dest,        \
                                          _type value,                         \
                                          int pe) {                            \
    return shmem_##_tn##_atomic_fetch_or(dest, value, ctx_pe(ctx, pe));        \
  }                                                                            \
  void shmem_ctx_##_tn##_atomic_or(shmem_ctx_t ctx, _type *dest,               \
                                   _type value, int pe) {                      \
    shmem_##_tn##_atomic_or(dest, value, ctx_pe(ctx, pe));                     \
  }                                                                            \
  _type shmem_ctx_##_tn##_atomic_fetch_xor(shmem_ctx_t ctx, _type *dest,       \
                                           _type value,                        \
                                          int pe) {                            \
    return shmem_##_tn##_atomic_fetch_xor(dest, value, ctx_pe(ctx, pe));       \
  }                                                                            \
  void shmem_ctx_##_tn##_atomic_xor(shmem_ctx_t ctx, _type *dest,              \
                                    _type value, int pe) {                     \
    shmem_##_tn##_atomic_xor(dest, value, ctx_pe(ctx, pe));                    \
  }
SHMEM_B200_AMO_STANDARD_TYPES(DEF_AMO_STD)
SHMEM_B200_AMO_EXTENDED_TYPES(DEF_AMO_EXT)
SHMEM_B200_AMO_BITWISE_TYPES(DEF_AMO_BIT)

/* the fetching atomics' _nbi forms: the old value lands in *fetch at quiet */
#define DEF_AMO_NBI_STD(_type, _tn)                                            \
  void shmem_ctx_##_tn##_atomic_fetch_add_nbi(shmem_ctx_t ctx, _type *fetch,   \
                                              _type *dest, _type value,        \
                                              int pe) {                        \
    nbi_amo(ctx_list(ctx), B200SHM_AMO_FETCH_ADD, B200_DTYPE_OF(_type),        \
            dest, ctx_pe(ctx, pe), &value, NULL, fetch, sizeof(_type));        \
  }                                                                            \
  void shmem_##_tn##_atomic_fetch_add_nbi(_type *fetch, _type *dest,           \
                                          _type value, int pe) {               \
    shmem_ctx_##_tn##_atomic_fetch_add_nbi(SHMEM_CTX_DEFAULT, fetch, dest,     \
                                           value, pe);                         \
  }                                                                            \
  void shmem_ctx_##_tn##_atomic_fetch_inc_nbi(shmem_ctx_t ctx, _type *fetch,   \
                                              _type *dest, int pe) {           \
    nbi_amo(ctx_list(ctx), B200SHM_AMO_FETCH_INC, B200_DTYPE_OF(_type),        \
            dest, ctx_pe(ctx, pe), NULL, NULL, fetch, sizeof(_type));          \
  }                                                                            \
  void shmem_##_tn##_atomic_fetch_inc_nbi(_type *fetch, _type *dest, int pe) { \
    shmem_ctx_##_tn##_atomic_fetch_inc_nbi(SHMEM_CTX_DEFAULT, fetch, dest,     \
                                           pe);                                \
  }                                                                            \
  void shmem_ctx_##_tn##_atomic_compare_swap_nbi(shmem_ctx_t ctx,              \
                                                 _type *fetch, _type *dest,    \
                                                 _type cond, _type value,      \
                                                 int pe) {                     \
    nbi_amo(ctx_list(ctx), B200SHM_AMO_CSWAP, B200_DTYPE_OF(_type), dest,      \
            ctx_pe(ctx, pe), &value, &cond, fetch, sizeof(_type));             \
  }                                                                            \
  void shmem_##_tn##_atomic_compare_swap_nbi(_type *fetch, _type *dest,        \
                                             _type cond, _type value,          \
                                             int pe) {                         \
    shmem_ctx_##_tn##_atomic_compare_swap_nbi(SHMEM_CTX_DEFAULT, fetch,        \
                                              dest, cond, value, pe);          \
  }
#define DEF_AMO_NBI_EXT(_type, _tn)                                            \
  void shmem_ctx_##_tn##_atomic_swap_nbi(shmem_ctx_t ctx, _type *fetch,        \
                                         _type *dest, _type value, int pe) {   \
    nbi_amo(ctx_list(ctx), B200SHM_AMO_SWAP, B200_DTYPE_OF(_type), dest,       \
            ctx_pe(ctx, pe), &value, NULL, fetch, sizeof(_type));              \
  }                                                                            \
  void shmem_##_tn##_atomic_swap_nbi(_type *fetch, _type *dest, _type value,   \
                                     int pe) {                                 \
    shmem_ctx_##_tn##_atomic_swap_nbi(SHMEM_CTX_DEFAULT, fetch, dest, value,   \
                                      pe);                                     \
  }                                                                            \
  void shmem_ctx_##_tn##_atomic_fetch_nbi(shmem_ctx_t ctx, _type *fetch,       \
                                          const _type *source, int pe) {       \
    nbi_amo(ctx_list(ctx), B200SHM_AMO_FETCH, B200_DTYPE_OF(_type), source,    \
            ctx_pe(ctx, pe), NULL, NULL, fetch, sizeof(_type));                \
  }                                                                            \
  void shmem_##_tn##_atomic_fetch_nbi(_type *fetch, const _type *source,       \
                                      int pe) {                                \
    shmem_ctx_##_tn##_atomic_fetch_nbi(SHMEM_CTX_DEFAULT, fetch, source, pe);  \
  }
#define DEF_AMO_NBI_BIT(_type, _tn)                                            \
  void shmem_ctx_##_tn##_atomic_fetch_and_nbi(shmem_ctx_t ctx, _type *fetch,   \
                                              _type *dest, _type value,        \
                                              int pe) {                        \
    nbi_amo(ctx_list(ctx), B200SHM_AMO_FETCH_AND, B200_DTYPE_OF(_type),        \
            dest, ctx_pe(ctx, pe), &value, NULL, fetch, sizeof(_type));        \
  }                                                                            \
  void shmem_##_tn##_atomic_fetch_and_nbi(_type *fetch, _type *dest,           \
                                          _type value, int pe) {               \
    shmem_ctx_##_tn##_atomic_fetch_and_nbi(SHMEM_CTX_DEFAULT, fetch, dest,     \
                                           value, pe);                         \
  }                                                                            \
  void shmem_ctx_##_tn##_atomic_fetch_or_nbi(shmem_ctx_t ctx, _type *fetch,    \
                                             _type *dest, _type value,         \
                                             int pe) {                         \
    nbi_amo(ctx_list(ctx), B200SHM_AMO_FETCH_OR, B200_DTYPE_OF(_type), dest,   \
            ctx_pe(ctx, pe), &value, NULL, fetch, sizeof(_type));              \
  }                                                                            \
  void shmem_##_tn##_atomic_fetch_or_nbi(_type *fetch, _type *dest,            \
                                         _type value, int pe) {                \
    shmem_ctx_##_tn##_atomic_fetch_or_nbi(SHMEM_CTX_DEFAULT, fetch, dest,      \
                                          value, pe);                          \
  }                                                                            \
  void shmem_ctx_##_tn##_atomic_fetch_xor_nbi(shmem_ctx_t ctx, _type *fetch,   \
                                              _type *dest, _type value,        \
                                              int pe) {                        \
    nbi_amo(ctx_list(ctx), B200SHM_AMO_FETCH_XOR, B200_DTYPE_OF(_type),        \
            dest, ctx_pe(ctx, pe), &value, NULL, fetch, sizeof(_type));        \
  }                                                                            \
  void shmem_##_tn##_atomic_fetch_xor_nbi(_type *fetch, _type *dest,           \
                                          _type value, int pe) {               \
    shmem_ctx_##_tn##_atomic_fetch_xor_nbi(SHMEM_CTX_DEFAULT, fetch, dest,     \
                                           value, pe);                         \
  }                                                                            \
  void shmem_ctx_##_tn##_atomic_xor_nbi(shmem_ctx_t ctx, _type *fetch,         \
                                        _type *dest, _type value, int pe) {    \
    shmem_ctx_##_tn##_atomic_fetch_xor_nbi(ctx, fetch, dest, value, pe);       \
  }                                                                            \
  void shmem_##_tn##_atomic_xor_nbi(_type *fetch, _type *dest, _type value,    \
                                    int pe) {                                  \
    shmem_ctx_##_tn##_atomic_fetch_xor_nbi(SHMEM_CTX_DEFAULT, fetch, dest,     \
                                           value, pe);                         \
  }
SHMEM_B200_AMO_STANDARD_TYPES(DEF_AMO_NBI_STD)
SHMEM_B200_AMO_EXTENDED_TYPES(DEF_AMO_NBI_EXT)
SHMEM_B200_AMO_BITWISE_TYPES(DEF_AMO_NBI_BIT)

/* ---- strided and signalled RMA (src/api/rma/putget.h:131-220, 420;
 *      put_signal.h:28-98, put_signal.c:67-285) ------------------------------- */
static void iput_bytes(void *dest, const void *source, ptrdiff_t tst, ptrdiff_t sst,
                       size_t nelems, size_t esize, int pe) {
  uint64_t off = 0;
  if (sym_off(dest, &off)) {
    t_status = B200SHM_ERR_ARG;
    return;
  }
  void *remote = b200shm_ptr(pe, off);
  if (!remote) {
    t_status = set_err(B200SHM_ERR_ARG, "iput: PE %d is not in the job", pe);
    return;
  }
  t_status = engine_err(b200shm_memcpy_strided(remote, tst, source, sst, esize, nelems, NULL));
}
static void iget_bytes(void *dest, const void *source, ptrdiff_t tst, ptrdiff_t sst,
                       size_t nelems, size_t esize, int pe) {
  uint64_t off = 0;
  if (sym_off(source, &off)) {
    t_status = B200SHM_ERR_ARG;
    return;
  }
  const void *remote = b200shm_ptr(pe, off);
  if (!remote) {
    t_status = set_err(B200SHM_ERR_ARG, "iget: PE %d is not in the job", pe);
    return;
  }
  t_status = engine_err(b200shm_memcpy_strided(dest, tst, remote, sst, esize, nelems, NULL));
}

/* The data is delivered (a blocking copy) before the signal word is set
 * or added to, so a PE that sees the signal sees the data; the _nbi forms
 * complete the same way before they return. */
static void put_signal(void *dest, const void *source, size_t nbytes, uint64_t *sig_addr,
                       uint64_t signal, int sig_op, int pe) {
  if (sig_op != SHMEM_SIGNAL_SET && sig_op != SHMEM_SIGNAL_ADD) {
    t_status = set_err(B200SHM_ERR_ARG, "put_signal: unknown signal operation %d", sig_op);
    return;
  }
  shmem_putmem(dest, source, nbytes, pe);
  if (t_status) return;
  amo(sig_op == SHMEM_SIGNAL_ADD ? B200SHM_AMO_ADD : B200SHM_AMO_SET, B200SHM_U64, sig_addr, pe,
      &signal, NULL, NULL);
}

#define DEF_RMA_STRIDED(_type, _tn)                                            \
  void shmem_##_tn##_iput(_type *dest, const _type *source, ptrdiff_t tst,     \
                          ptrdiff_t sst, size_t nelems, int pe) {              \
    iput_bytes(dest, source, tst, sst, nelems, sizeof(_type), pe);             \
  }                                                                            \
  void shmem_##_tn##_iget(_type *dest, const _type *source, ptrdiff_t tst,     \
                          ptrdiff_t sst, size_t nelems, int pe) {              \
    iget_bytes(dest, source, tst, sst, nelems, sizeof(_type), pe);             \
  }                                                                            \
  void shmem_ctx_##_tn##_iput(shmem_ctx_t ctx, _type *dest,                    \
                              const _type *source, ptrdiff_t tst,              \
                              ptrdiff_t sst, size_t nelems, int pe) {          \
    iput_bytes(dest, source, tst, sst, nelems, sizeof(_type), ctx_pe(ctx, pe)); \
  }                                                                            \
  void shmem_ctx_##_tn##_iget(shmem_ctx_t ctx, _type *dest,                    \
                              const _type *source, ptrdiff_t tst,              \
                              ptrdiff_t sst, size_t nelems, int pe) {          \
    iget_bytes(dest, source, tst, sst, nelems, sizeof(_type), ctx_pe(ctx, pe)); \
  }                                                                            \
  void shmem_##_tn##_put_signal(_type *dest, const _type *source,              \
                                size_t nelems, uint64_t *sig_addr,             \
                                uint64_t signal, int sig_op, int pe) {         \
    put_signal(dest, source, nelems * sizeof(_type), sig_addr, signal, sig_op, \
               pe);                                                            \
  }                                                                            \
  void shmem_##_tn##_put_signal_nbi(_type *dest, const _type *source,          \
                                    size_t nelems, uint64_t *sig_addr,         \
                                    uint64_t signal, int sig_op, int pe) {     \
    put_signal(dest, source, nelems * sizeof(_type), sig_addr, signal, sig_op, \
               pe);                                                            \
  }                                                                            \
  void shmem_ctx_##_tn##_put_signal(shmem_ctx_t ctx, _type *dest,              \
                                    const _type *source, size_t nelems,        \
                                    uint64_t *sig_addr, uint64_t signal,       \
                                    int sig_op, int pe) {                      \
    put_signal(dest, source, nelems * sizeof(_type), sig_addr, signal, sig_op, \
               ctx_pe(ctx, pe));                                               \
  }                                                                            \
  void shmem_ctx_##_tn##_put_signal_nbi(shmem_ctx_t ctx, _type *dest,          \
                                        const _type *source, size_t nelems,    \
                                        uint64_t *sig_addr, uint64_t signal,   \
                                        int sig_op, int pe) {                  \
    put_signal(dest, source, nelems * sizeof(_type), sig_addr, signal, sig_op, \
               ctx_pe(ctx, pe));                                               \
  }
SHMEM_B200_RMA_TYPES(DEF_RMA_STRIDED)

#define DEF_RMA_SIZED(_bits)                                                   \
  void shmem_put##_bits(void *dest, const void *source, size_t nelems, int pe) { \
    shmem_putmem(dest, source, nelems * (_bits / 8), pe);                      \
  }                                                                            \
  void shmem_get##_bits(void *dest, const void *source, size_t nelems, int pe) { \
    shmem_getmem(dest, source, nelems * (_bits / 8), pe);                      \
  }                                                                            \
  void shmem_put##_bits##_nbi(void *dest, const void *source, size_t nelems,   \
                              int pe) {                                        \
    shmem_putmem_nbi(dest, source, nelems * (_bits / 8), pe);                  \
  }                                                                            \
  void shmem_get##_bits##_nbi(void *dest, const void *source, size_t nelems,   \
                              int pe) {                                        \
    shmem_getmem_nbi(dest, source, nelems * (_bits / 8), pe);                  \
  }                                                                            \
  void shmem_iput##_bits(void *dest, const void *source, ptrdiff_t tst,        \
                         ptrdiff_t sst, size_t nelems, int pe) {               \
    iput_bytes(dest, source, tst, sst, nelems, _bits / 8, pe);                 \
  }                                                                            \
  void shmem_iget##_bits(void *dest, const void *source, ptrdiff_t tst,        \
                         ptrdiff_t sst, size_t nelems, int pe) {               \
    iget_bytes(dest, source, tst, sst, nelems, _bits / 8, pe);                 \
  }                                                                            \
  void shmem_ctx_put##_bits(shmem_ctx_t ctx, void *dest, const void *source,   \
                            size_t nelems, int pe) {                           \
    shmem_ctx_putmem(ctx, dest, source, nelems * (_bits / 8), pe);             \
  }                                                                            \
  void shmem_ctx_get##_bits(shmem_ctx_t ctx, void *dest, const void *source,   \
                            size_t nelems, int pe) {                           \
    shmem_ctx_getmem(ctx, dest, source, nelems * (_bits / 8), pe);             \
  }                                                                            \
  void shmem_ctx_put##_bits##_nbi(shmem_ctx_t ctx, void *dest,                 \
                                  const void *source, size_t nelems, int pe) { \
    shmem_ctx_putmem_nbi(ctx, dest, source, nelems * (_bits / 8), pe);         \
  }                                                                            \
  void shmem_ctx_get##_bits##_nbi(shmem_ctx_t ctx, void *dest,                 \
                                  const void *source, size_t nelems, int pe) { \
    shmem_ctx_getmem_nbi(ctx, dest, source, nelems * (_bits / 8), pe);         \
  }                                                                            \
  void shmem_ctx_iput##_bits(shmem_ctx_t ctx, void *dest, const void *source,  \
                             ptrdiff_t tst, ptrdiff_t sst, size_t nelems,      \
                             int pe) {                                         \
    iput_bytes(dest, source, tst, sst, nelems, _bits / 8, ctx_pe(ctx, pe));    \
  }                                                                            \
  void shmem_ctx_iget##_bits(shmem_ctx_t ctx, void *dest, const void *source,  \
                             ptrdiff_t tst, ptrdiff_t sst, size_t nelems,      \
                             int pe) {                                         \
    iget_bytes(dest, source, tst, sst, nelems, _bits / 8, ctx_pe(ctx, pe));    \
  }                                                                            \
  void shmem_put##_bits##_signal(void *dest, const void *source,               \
                                 size_t nelems, uint64_t *sig_addr,            \
                                 uint64_t signal, int sig_op, int pe) {        \
    put_signal(dest, source, nelems * (_bits / 8), sig_addr, signal, sig_op,   \
               pe);                                                            \
  }                                                                            \
  void shmem_put##_bits##_signal_nbi(void *dest, const void *source,           \
                                     size_t nelems, uint64_t *sig_addr,        \
                                     uint64_t signal, int sig_op, int pe) {    \
    put_signal(dest, source, nelems * (_bits / 8), sig_addr, signal, sig_op,   \
               pe);                                                            \
  }                                                                            \
  void shmem_ctx_put##_bits##_signal(shmem_ctx_t ctx, void *dest,              \
                                     const void *source, size_t nelems,        \
                                     uint64_t *sig_addr, uint64_t signal,      \
                                     int sig_op, int pe) {                     \
    put_signal(dest, source, nelems * (_bits / 8), sig_addr, signal, sig_op,   \
               ctx_pe(ctx, pe));                                               \
  }                                                                            \
  void shmem_ctx_put##_bits##_signal_nbi(shmem_ctx_t ctx, void *dest,          \
                                         const void *source, size_t nelems,    \
                                         uint64_t *sig_addr, uint64_t signal,  \
                                         int sig_op, int pe) {                 \
    put_signal(dest, source, nelems * (_bits / 8), sig_addr, signal, sig_op,   \
               ctx_pe(ctx, pe));                                               \
  }
DEF_RMA_SIZED(8)
DEF_RMA_SIZED(16)
DEF_RMA_SIZED(32)
DEF_RMA_SIZED(64)
DEF_RMA_SIZED(128)

void shmem_putmem_signal(void *dest, const void *source, size_t nelems, uint64_t *sig_addr,
                         uint64_t signal, int sig_op, int pe) {
  put_signal(dest, source, nelems, sig_addr, signal, sig_op, pe);
}
void shmem_putmem_signal_nbi(void *dest, const void *source, size_t nelems, uint64_t *sig_addr,
                             uint64_t signal, int sig_op, int pe) {
  put_signal(dest, source, nelems, sig_addr, signal, sig_op, pe);
}
void shmem_ctx_putmem_signal(shmem_ctx_t ctx, void *dest, const void *source, size_t nelems,
                             uint64_t *sig_addr, uint64_t signal, int sig_op, int pe) {
  put_signal(dest, source, nelems, sig_addr, signal, sig_op, ctx_pe(ctx, pe));
}
void shmem_ctx_putmem_signal_nbi(shmem_ctx_t ctx, void *dest, const void *source, size_t nelems,
                                 uint64_t *sig_addr, uint64_t signal, int sig_op, int pe) {
  put_signal(dest, source, nelems, sig_addr, signal, sig_op, ctx_pe(ctx, pe));
}

/* ---- point-to-point synchronisation (the src/api/pt2pt_synch files over
 *      src/shmemc/ucx/test.c and waituntil.c) -------------------------------
 * Every pass is one device comparison of the whole vector
 * (b200shm_test_words); the waits repeat passes, yielding between them.
 * The reference's waits spin without bound; here SHMEM_B200_WAIT_TIMEOUT
 * (seconds) may bound them: a wait that runs out returns with the status
 * B200SHM_ERR_TIMEOUT (shmemx_b200_last_status), wait_until_any with
 * SIZE_MAX. */
typedef struct {
  size_t ntrue, nlive, first;
} pass_t;

static double wait_limit(void) {
  const char *e = getenv("SHMEM_B200_WAIT_TIMEOUT");
  const double v = e ? atof(e) : 0.0;
  return v > 0.0 ? v : -1.0;
}

/* one comparison pass; indices (may be NULL) receive the true elements */
static int pass(int cmp, int dtype, const void *ivars, size_t n, const int *status,
                const void *value, const void *values, size_t *indices, uint64_t *loaded,
                pass_t *p) {
  p->ntrue = p->nlive = 0;
  p->first = SIZE_MAX;
  if (n == 0) return 0;
  uint64_t off = 0;
  if (sym_off(ivars, &off)) return t_status = B200SHM_ERR_ARG;
  uint8_t small[256];
  uint8_t *out = n <= sizeof(small) ? small : (uint8_t *)malloc(n);
  if (!out) return t_status = set_err(B200SHM_ERR_NOMEM, "test: out of host memory");
  const int rc = engine_err(b200shm_test_words(cmp, dtype, t_pe, off, n, status, value, values,
                                               out, loaded));
  if (rc == 0) {
    for (size_t i = 0; i < n; i++) {
      if (out[i] == 2) continue;
      p->nlive++;
      if (out[i] == 1) {
        if (p->first == SIZE_MAX) p->first = i;
        if (indices) indices[p->ntrue] = i;
        p->ntrue++;
      }
    }
  }
  if (out != small) free(out);
  return t_status = rc;
}

enum { W_ONE, W_ALL, W_ANY, W_SOME };
/* repeat passes until the wait's condition holds (or the bound runs out) */
static int wait_pass(int kind, int cmp, int dtype, const void *ivars, size_t n,
                     const int *status, const void *value, const void *values, size_t *indices,
                     uint64_t *loaded, pass_t *p) {
  const double limit = wait_limit(), t0 = shmemx_wtime();
  for (unsigned it = 0;; it++) {
    if (pass(cmp, dtype, ivars, n, status, value, values, indices, loaded, p)) return t_status;
    if (kind == W_ALL ? p->ntrue == p->nlive : (p->ntrue > 0 || p->nlive == 0)) return 0;
    if (limit > 0 && shmemx_wtime() - t0 > limit)
      return t_status = set_err(B200SHM_ERR_TIMEOUT, "wait_until: not satisfied after %.3f s",
                                limit);
    if (it > 16) sched_yield();
  }
}

#define DEF_SYNC_ONE(_type, _tn)                                               \
  int shmem_##_tn##_test(_type *ivar, int cmp, _type cmp_value) {              \
    pass_t p;                                                                  \
    pass(cmp, B200_DTYPE_OF(_type), ivar, 1, NULL, &cmp_value, NULL, NULL,     \
         NULL, &p);                                                            \
    return p.ntrue ? 1 : 0;                                                    \
  }                                                                            \
  void shmem_##_tn##_wait_until(_type *ivar, int cmp, _type cmp_value) {       \
    pass_t p;                                                                  \
    wait_pass(W_ONE, cmp, B200_DTYPE_OF(_type), ivar, 1, NULL, &cmp_value,     \
              NULL, NULL, NULL, &p);                                           \
  }                                                                            \
  void shmem_##_tn##_wait(_type *ivar, _type cmp_value) {                      \
    shmem_##_tn##_wait_until(ivar, SHMEM_CMP_NE, cmp_value);                   \
  }
#define DEF_SYNC_VEC(_type, _tn)                                               \
  int shmem_##_tn##_test_all(_type *ivars, size_t nelems, const int *status,   \
                             int cmp, _type cmp_value) {                       \
    pass_t p;                                                                  \
    if (pass(cmp, B200_DTYPE_OF(_type), ivars, nelems, status, &cmp_value,     \
             NULL, NULL, NULL, &p))                                            \
      return 0;                                                                \
    return p.ntrue == p.nlive ? 1 : 0;                                         \
  }                                                                            \
  size_t shmem_##_tn##_test_any(_type *ivars, size_t nelems,                   \
                                const int *status, int cmp, _type cmp_value) { \
    pass_t p;                                                                  \
    pass(cmp, B200_DTYPE_OF(_type), ivars, nelems, status, &cmp_value, NULL,   \
         NULL, NULL, &p);                                                      \
    return p.first;                                                            \
  }                                                                            \
  size_t shmem_##_tn##_test_some(_type *ivars, size_t nelems, size_t *indices, \
                                 const int *status, int cmp,                   \
                                 _type cmp_value) {                            \
    pass_t p;                                                                  \
    pass(cmp, B200_DTYPE_OF(_type), ivars, nelems, status, &cmp_value, NULL,   \
         indices, NULL, &p);                                                   \
    return p.ntrue;                                                            \
  }                                                                            \
  int shmem_##_tn##_test_all_vector(_type *ivars, size_t nelems,               \
                                    const int *status, int cmp,                \
                                    _type *cmp_values) {                       \
    pass_t p;                                                                  \
    if (pass(cmp, B200_DTYPE_OF(_type), ivars, nelems, status, NULL,           \
             cmp_values, NULL, NULL, &p))                                      \
      return 0;                                                                \
    return p.ntrue == p.nlive ? 1 : 0;                                         \
  }                                                                            \
  size_t shmem_##_tn##_test_any_vector(_type *ivars, size_t nelems,            \
                                       const int *status, int cmp,             \
                                       _type *cmp_values) {                    \
    pass_t p;                                                                  \
    pass(cmp, B200_DTYPE_OF(_type), ivars, nelems, status, NULL, cmp_values,   \
         NULL, NULL, &p);                                                      \
    return p.first;                                                            \
  }                                                                            \
  size_t shmem_##_tn##_test_some_vector(_type *ivars, size_t nelems,           \
                                        size_t *indices, const int *status,    \
                                        int cmp, _type *cmp_values) {          \
    pass_t p;                                                                  \
    pass(cmp, B200_DTYPE_OF(_type), ivars, nelems, status, NULL, cmp_values,   \
         indices, NULL, &p);                                                   \
    return p.ntrue;                                                            \
  }                                                                            \
  void shmem_##_tn##_wait_until_all(_type *ivars, size_t nelems,               \
                                    const int *status, int cmp,                \
                                    _type cmp_value) {                         \
    pass_t p;                                                                  \
    wait_pass(W_ALL, cmp, B200_DTYPE_OF(_type), ivars, nelems, status,         \
              &cmp_value, NULL, NULL, NULL, &p);                               \
  }                                                                            \
  size_t shmem_##_tn##_wait_until_any(_type *ivars, size_t nelems,             \
                                      const int *status, int cmp,              \
                                      _type cmp_value) {                       \
    pass_t p;                                                                  \
    if (wait_pass(W_ANY, cmp, B200_DTYPE_OF(_type), ivars, nelems, status,     \
                  &cmp_value, NULL, NULL, NULL, &p))                           \
      return SIZE_MAX;                                                         \
    return p.first;                                                            \
  }                                                                            \
  size_t shmem_##_tn##_wait_until_some(_type *ivars, size_t nelems,            \
                                       size_t *indices, const int *status,     \
                                       int cmp, _type cmp_value) {             \
    pass_t p;                                                                  \
    if (wait_pass(W_SOME, cmp, B200_DTYPE_OF(_type), ivars, nelems, status,    \
                  &cmp_value, NULL, indices, NULL, &p))                        \
      return 0;                                                                \
    return p.ntrue;                                                            \
  }                                                                            \
  void shmem_##_tn##_wait_until_all_vector(_type *ivars, size_t nelems,        \
                                           const int *status, int cmp,         \
                                           _type *cmp_values) {                \
    pass_t p;                                                                  \
    wait_pass(W_ALL, cmp, B200_DTYPE_OF(_type), ivars, nelems, status, NULL,   \
              cmp_values, NULL, NULL, &p);                                     \
  }                                                                            \
  size_t shmem_##_tn##_wait_until_any_vector(_type *ivars, size_t nelems,      \
                                             const int *status, int cmp,       \
                                             _type *cmp_values) {              \
    pass_t p;                                                                  \
    if (wait_pass(W_ANY, cmp, B200_DTYPE_OF(_type), ivars, nelems, status,     \
                  NULL, cmp_values, NULL, NULL, &p))                           \
      return SIZE_MAX;                                                         \
    return p.first;                                                            \
  }                                                                            \
  size_t shmem_##_tn##_wait_until_some_vector(_type *ivars, size_t nelems,     \
                                              size_t *indices,                 \
                                              const int *status, int cmp,      \
                                              _type *cmp_values) {             \
    pass_t p;                                                                  \
    if (wait_pass(W_SOME, cmp, B200_DTYPE_OF(_type), ivars, nelems, status,    \
                  NULL, cmp_values, indices, NULL, &p))                        \
      return 0;                                                                \
    return p.ntrue;                                                            \
  }
SHMEM_B200_SYNC_TYPES(DEF_SYNC_ONE)
SHMEM_B200_AMO_STANDARD_TYPES(DEF_SYNC_VEC)

uint64_t shmem_signal_fetch(const uint64_t *sig_addr) {
  uint64_t v = 0;
  amo(B200SHM_AMO_FETCH, B200SHM_U64, sig_addr, t_pe, NULL, NULL, &v);
  return v;
}
uint64_t shmem_signal_wait_until(uint64_t *sig_addr, int cmp, uint64_t cmp_value) {
  pass_t p;
  uint64_t seen = 0;
  wait_pass(W_ONE, cmp, B200SHM_U64, sig_addr, 1, NULL, &cmp_value, NULL, NULL, &seen, &p);
  return seen;
}

/* ---- locks (src/api/lock.c) ---------------------------------------------------
 * A lock is a symmetric long, 0 when free.  Its word on one owner PE (spread
 * over the PEs by the lock's offset) holds 0 or the holder's PE + 1, and
 * changes only by compare-and-swap through the engine's atomics.  set_lock
 * retries until its swap wins, yielding the thread between tries; test_lock
 * tries once; clear_lock completes the holder's outstanding puts first
 * (shmem_quiet), then swaps its PE + 1 back to 0. */
static long *lock_word(long *lock, int *owner) {
  uint64_t off = 0;
  if (sym_off(lock, &off)) {
    t_status = set_err(B200SHM_ERR_ARG, "lock %p is not a symmetric object", (void *)lock);
    return NULL;
  }
  *owner = (int)((off >> 3) % (uint64_t)g_npes);
  return lock;
}
static int lock_try(long *lock) {
  int owner = 0;
  long *w = lock_word(lock, &owner);
  if (!w) return -1;
  const long old = shmem_long_atomic_compare_swap(w, 0, (long)t_pe + 1, owner);
  if (t_status) return -1;
  return old == 0;
}
void shmem_set_lock(long *lock) {
  for (;;) {
    const int got = lock_try(lock);
    if (got != 0) return; /* taken, or an error left in t_status */
    sched_yield();
  }
}
int shmem_test_lock(long *lock) {
  const int got = lock_try(lock);
  return got == 1 ? 0 : 1; /* 0: the lock is now this PE's */
}
void shmem_clear_lock(long *lock) {
  int owner = 0;
  long *w = lock_word(lock, &owner);
  if (!w) return;
  shmem_quiet();
  const long old = shmem_long_atomic_compare_swap(w, (long)t_pe + 1, 0, owner);
  if (!t_status && old != (long)t_pe + 1)
    t_status = set_err(B200SHM_ERR_STATE, "shmem_clear_lock: PE %d does not hold the lock", t_pe);
}

/* ---- the atomics' names before OpenSHMEM 1.4 ------------------------------------ */
#define DEF_AMO_OLD(_type, _tn)                                                \
  _type shmem_##_tn##_fadd(_type *target, _type value, int pe) {               \
    return shmem_##_tn##_atomic_fetch_add(target, value, pe);                  \
  }                                                                            \
  _type shmem_##_tn##_finc(_type *target, int pe) {                            \
    return shmem_##_tn##_atomic_fetch_inc(target, pe);                         \
  }                                                                            \
  void shmem_##_tn##_add(_type *target, _type value, int pe) {                 \
    shmem_##_tn##_atomic_add(target, value, pe);                               \
  }                                                                            \
  void shmem_##_tn##_inc(_type *target, int pe) { shmem_##_tn##_atomic_inc(target, pe); } \
  _type shmem_##_tn##_cswap(_type *target, _type cond, _type value, int pe) {  \
    return shmem_##_tn##_atomic_compare_swap(target, cond, value, pe);         \
  }
#define DEF_AMO_OLD_EXT(_type, _tn)                                            \
  _type shmem_##_tn##_swap(_type *target, _type value, int pe) {               \
    return shmem_##_tn##_atomic_swap(target, value, pe);                       \
  }                                                                            \
  _type shmem_##_tn##_fetch(const _type *target, int pe) {                     \
    return shmem_##_tn##_atomic_fetch(target, pe);                             \
  }                                                                            \
  void shmem_##_tn##_set(_type *target, _type value, int pe) {                 \
    shmem_##_tn##_atomic_set(target, value, pe);                               \
  }
SHMEM_B200_AMO_OLD_TYPES(DEF_AMO_OLD)
SHMEM_B200_AMO_OLD_TYPES(DEF_AMO_OLD_EXT)
SHMEM_B200_AMO_OLD_EXT_TYPES(DEF_AMO_OLD_EXT)
