/*
 * b200shm_types.h -- enumerations shared by the C host layer, the CUDA
 * kernels and the public C ABI (include/b200shm.h).
 */
#ifndef B200SHM_TYPES_H
#define B200SHM_TYPES_H

/* Machine element types.  The OpenSHMEM type names of
 * include/shmem/api_types.h map onto these (x86-64 LP64: char and schar are
 * I8, long/longlong/ptrdiff are I64, size/ulong/ulonglong are U64). */
enum b200shm_dtype {
  B200SHM_I8 = 0, B200SHM_I16, B200SHM_I32, B200SHM_I64,
  B200SHM_U8, B200SHM_U16, B200SHM_U32, B200SHM_U64,
  B200SHM_F32, B200SHM_F64,
  B200SHM_F80, /* long double: accepted by the API, rejected on the GPU */
  B200SHM_C32, /* float _Complex  */
  B200SHM_C64, /* double _Complex */
  B200SHM_NDTYPE
};

/* Reduction operators, in the order of reduce.c:730-736. */
enum b200shm_op {
  B200SHM_AND = 0, B200SHM_OR, B200SHM_XOR, B200SHM_MIN, B200SHM_MAX,
  B200SHM_SUM, B200SHM_PROD, B200SHM_NOP
};

/* Reduction algorithms of src/shcoll/src/reduce.c.  The algorithm fixes the
 * combine order, and so the exact floating-point result; the data movement
 * is always one pass. */
enum b200shm_algo {
  B200SHM_LINEAR = 0, B200SHM_BINOMIAL, B200SHM_REC_DBL, B200SHM_RABENSEIFNER,
  B200SHM_RABENSEIFNER2, B200SHM_NALGO
};

/* Barrier algorithms of src/shcoll/src/barrier.c. */
enum b200shm_barrier_algo {
  B200SHM_BAR_LINEAR = 0, B200SHM_BAR_COMPLETE_TREE, B200SHM_BAR_BINOMIAL_TREE,
  B200SHM_BAR_KNOMIAL_TREE, B200SHM_BAR_DISSEMINATION, B200SHM_BAR_NALGO
};

/* Atomic memory operations (src/api/atomics, src/shmemc/ucx/comms.c). */
enum b200shm_amo {
  B200SHM_AMO_FETCH_ADD = 0, B200SHM_AMO_ADD, B200SHM_AMO_FETCH_INC,
  B200SHM_AMO_INC, B200SHM_AMO_SWAP, B200SHM_AMO_CSWAP, B200SHM_AMO_SET,
  B200SHM_AMO_FETCH, B200SHM_AMO_FETCH_AND, B200SHM_AMO_AND,
  B200SHM_AMO_FETCH_OR, B200SHM_AMO_OR, B200SHM_AMO_FETCH_XOR,
  B200SHM_AMO_XOR, B200SHM_AMO_NOP
};

/* Return codes of every b200shm_* entry point. */
enum b200shm_status {
  B200SHM_OK = 0,
  B200SHM_ERR_ARG = -1,       /* invalid argument (team, size, overlap, ...) */
  B200SHM_ERR_UNSUPPORTED = -2, /* (op, dtype, algo) not available          */
  B200SHM_ERR_NOMEM = -3,     /* symmetric heap or device memory exhausted  */
  B200SHM_ERR_CUDA = -4,      /* a CUDA call failed                         */
  B200SHM_ERR_STATE = -5,     /* not initialised / already initialised      */
  B200SHM_ERR_TIMEOUT = -6,   /* a device wait ran out of its spin budget   */
  B200SHM_ERR_BUSY = -7       /* queue full / no free slot                  */
};

#endif
