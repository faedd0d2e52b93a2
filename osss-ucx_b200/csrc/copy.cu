/*
 * copy.cu -- the data-movement collectives: fcollect, collect, alltoall,
 * strided alltoall and broadcast.
 *
 * In the reference every byte crosses a process boundary as a UCX put
 * (fcollect: log2(P) Bruck rounds plus an in-place byte rotation,
 * src/shcoll/src/fcollect.c:370-403 and util/rotate.c:22-54; alltoall:
 * P-1 puts per PE, alltoall.c:75-110; strided alltoall: one put per
 * element, alltoalls.c:54-90).  The result of each is a fixed permutation
 * of bytes that does not depend on the algorithm, so here each collective
 * is one copy kernel that moves every byte once from its source slice to
 * its final place: no rounds, no intermediate copies, no rotation.
 *
 * Copies run in 16-byte vectors when every base offset and size is a
 * multiple of 16, else in bytes (or elements for the strided form).
 */
#include <stdint.h>
#include <stdlib.h>

#include <vector>

#include "internal.cuh"

namespace b200 {
namespace {

__device__ __forceinline__ uint4 ld16(const char *p) {
  uint4 u;
  asm("ld.global.nc.L1::no_allocate.v4.u32 {%0,%1,%2,%3}, [%4];"
      : "=r"(u.x), "=r"(u.y), "=r"(u.z), "=r"(u.w)
      : "l"(p));
  return u;
}
__device__ __forceinline__ void st16(char *p, uint4 u) {
  asm volatile("st.global.v4.u32 [%0], {%1,%2,%3,%4};" ::"l"(p), "r"(u.x), "r"(u.y), "r"(u.z),
               "r"(u.w)
               : "memory");
}

/* streaming store (evict-first in L2): for data this kernel does not read
 * again, such as fcollect's P copies of each source vector */
__device__ __forceinline__ void st16cs(char *p, uint4 u) {
  asm volatile("st.global.cs.v4.u32 [%0], {%1,%2,%3,%4};" ::"l"(p), "r"(u.x), "r"(u.y), "r"(u.z),
               "r"(u.w)
               : "memory");
}

/* fcollect: member j's dest[k*nbytes + b] = member k's src[b].
 * blockIdx.y = source member k; each thread reads one vector of k's
 * source once and writes it into every member's dest (streaming stores:
 * 5.99 against 5.92 TB/s with write-back stores, and 5.93 with each CTA
 * starting at its own member, on 128 members x 32 KiB). */
template <bool VEC>
__global__ void __launch_bounds__(256) k_fcollect(const char *src0, char *dst0, uint64_t step,
                                                  int P, uint64_t nbytes) {
  const int k = blockIdx.y;
  const char *src = src0 + (uint64_t)k * step;
  char *dst = dst0 + (uint64_t)k * nbytes;
  const uint64_t n = VEC ? nbytes / 16 : nbytes;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (uint64_t)gridDim.x * blockDim.x) {
    if constexpr (VEC) {
      const uint4 u = ld16(src + v * 16);
      for (int j = 0; j < P; j++) st16cs(dst + (uint64_t)j * step + v * 16, u);
    } else {
      const char c = src[v];
      for (int j = 0; j < P; j++) dst[(uint64_t)j * step + v] = c;
    }
  }
}

/* fcollect staged through shared memory with the bulk-copy engine: a CTA
 * brings a tile of source k into shared memory with one cp.async.bulk load
 * (completion counted on an mbarrier), then issues one cp.async.bulk store
 * of the tile to each member's dest, so the P writes of every byte are
 * issued by the copy engine rather than by P store instructions per thread.
 * Two buffers: the load of the next tile overlaps the stores of this one.
 * Needs 16-byte aligned offsets, step and size (the vector path's rule).
 * Every wait is bounded; one that runs out sets the TIMEOUT status bit and
 * the CTA stops issuing. */
constexpr unsigned kFcBulkTile = 8192; /* bytes per tile */
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ bool mbar_wait(uint64_t *m, unsigned phase) {
  for (unsigned i = 0; i < (1u << 24); i++) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(m)), "r"(phase)
        : "memory");
    if (ok) return true;
    __nanosleep(32);
  }
  return false;
}
__device__ __forceinline__ void bulk_load(void *dst_smem, const char *src, unsigned bytes,
                                          uint64_t *m) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(m)),
               "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_addr(dst_smem)),
      "l"(src), "r"(bytes), "r"(smem_addr(m))
      : "memory");
}

__global__ void __launch_bounds__(256) k_fcollect_bulk(const char *src0, char *dst0,
                                                       uint64_t step, int P, uint64_t nbytes,
                                                       int *status) {
  __shared__ __align__(128) char buf[2][kFcBulkTile];
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ int s_ok;
  const int k = blockIdx.y;
  const char *src = src0 + (uint64_t)k * step;
  const uint64_t ntiles = (nbytes + kFcBulkTile - 1) / kFcBulkTile;
  uint64_t t = blockIdx.x;
  if (t >= ntiles) return;
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&mbar[0])) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&mbar[1])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_ok = 1;
  }
  __syncthreads();
  auto tile_bytes = [&](uint64_t tt) {
    const uint64_t off = tt * kFcBulkTile;
    return (unsigned)(nbytes - off < kFcBulkTile ? nbytes - off : kFcBulkTile);
  };
  if (threadIdx.x == 0) bulk_load(buf[0], src + t * kFcBulkTile, tile_bytes(t), &mbar[0]);
  unsigned phase[2] = {0, 0};
  bool issued = false;
  for (int b = 0; t < ntiles; t += gridDim.x, b ^= 1) {
    const uint64_t off = t * kFcBulkTile;
    const unsigned bytes = tile_bytes(t);
    /* every thread that stores waits for the tile itself */
    const bool ready = mbar_wait(&mbar[b], phase[b]);
    phase[b] ^= 1;
    if (!ready) {
      if (threadIdx.x == 0) atomicOr(status, (int)B200SHM_STATUS_TIMEOUT);
      s_ok = 0;
    }
    __syncthreads();
    if (!s_ok) break;
    for (int j = threadIdx.x; j < P; j += blockDim.x) {
      char *d = dst0 + (uint64_t)j * step + (uint64_t)k * nbytes + off;
      asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(d),
                   "r"(smem_addr(buf[b])), "r"(bytes)
                   : "memory");
      issued = true;
    }
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
    /* the stores of the previous tile (the other buffer) have read it */
    asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0 && t + gridDim.x < ntiles)
      bulk_load(buf[b ^ 1], src + (t + gridDim.x) * kFcBulkTile, tile_bytes(t + gridDim.x),
                &mbar[b ^ 1]);
  }
  /* this thread's stores complete before the CTA ends */
  if (issued) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
  __syncthreads();
}

/* collect: member k contributes sizes[k] bytes; member j's
 * dest[prefix[k] + b] = member k's src[b] (collect.c:35-591: the
 * contributions concatenated in member order).  blockIdx.y = source member
 * k; each thread reads one word of k's contribution once and writes it
 * into every member's dest.  W is a width every offset and size divides. */
template <class W>
__global__ void __launch_bounds__(256) k_collect(const char *src0, char *dst0, uint64_t step,
                                                 int P, const uint64_t *sizes,
                                                 const uint64_t *prefix) {
  const int k = blockIdx.y;
  const W *src = (const W *)(src0 + (uint64_t)k * step);
  char *dst = dst0 + prefix[k];
  const uint64_t n = sizes[k] / sizeof(W);
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (uint64_t)gridDim.x * blockDim.x) {
    const W u = src[v];
    for (int j = 0; j < P; j++) ((W *)(dst + (uint64_t)j * step))[v] = u;
  }
}

/* alltoall: member j's dest[k*B + b] = member k's src[j*B + b].
 * Pairs k*P + j are spread over blockIdx.y (grid-stride when there are more
 * pairs than the grid's y extent); blockIdx.x strides over the block. */
template <bool VEC>
__global__ void __launch_bounds__(256) k_alltoall(const char *src0, char *dst0, uint64_t step,
                                                  int P, uint64_t B) {
  const uint64_t pairs = (uint64_t)P * (uint64_t)P;
  const uint64_t n = VEC ? B / 16 : B;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t pr = blockIdx.y; pr < pairs; pr += gridDim.y) {
    const uint64_t k = pr / (uint64_t)P, j = pr % (uint64_t)P;
    const char *src = src0 + k * step + j * B;
    char *dst = dst0 + j * step + k * B;
    uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if constexpr (VEC) {
      /* four vectors in flight per thread */
      for (; v + 3 * stride < n; v += 4 * stride) {
        uint4 u0 = ld16(src + v * 16), u1 = ld16(src + (v + stride) * 16);
        uint4 u2 = ld16(src + (v + 2 * stride) * 16), u3 = ld16(src + (v + 3 * stride) * 16);
        st16(dst + v * 16, u0);
        st16(dst + (v + stride) * 16, u1);
        st16(dst + (v + 2 * stride) * 16, u2);
        st16(dst + (v + 3 * stride) * 16, u3);
      }
      for (; v < n; v += stride) st16(dst + v * 16, ld16(src + v * 16));
    } else {
      for (; v < n; v += stride) dst[v] = src[v];
    }
  }
}

/* alltoall of small blocks (fewer words per pair than a CTA has threads):
 * one thread per word of the flattened [pair][word] space, so a CTA spans
 * many pairs instead of idling most of its threads on one. */
template <class W>
__global__ void __launch_bounds__(256) k_alltoall_flat(const char *src0, char *dst0,
                                                       uint64_t step, int P, uint64_t nw) {
  const uint64_t total = (uint64_t)P * (uint64_t)P * nw;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t pr = i / nw, w = i - pr * nw;
    const uint64_t k = pr / (uint64_t)P, j = pr - k * (uint64_t)P;
    ((W *)(dst0 + j * step))[k * nw + w] = ((const W *)(src0 + k * step))[j * nw + w];
  }
}

/* strided alltoall (alltoalls.c:39-50, 78-83): element t from member k to
 * member l: src_k[(l*n + t)*sst] -> dest_l[(k*n + t)*dst].
 * Pairs k*P + l over blockIdx.y, grid-stride as in k_alltoall. */
template <class E>
__global__ void __launch_bounds__(256) k_alltoalls(const char *src0, char *dst0, uint64_t step,
                                                   int P, uint64_t n, int64_t dst, int64_t sst) {
  const uint64_t pairs = (uint64_t)P * (uint64_t)P;
  for (uint64_t pr = blockIdx.y; pr < pairs; pr += gridDim.y) {
    const uint64_t k = pr / (uint64_t)P, l = pr % (uint64_t)P;
    const E *src = (const E *)(src0 + k * step) + l * n * (uint64_t)sst;
    E *d = (E *)(dst0 + l * step) + k * n * (uint64_t)dst;
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (uint64_t)gridDim.x * blockDim.x)
      d[t * (uint64_t)dst] = src[t * (uint64_t)sst];
  }
}

/* strided alltoall with few elements per pair: one thread per element of
 * the flattened [pair][element] space */
template <class E>
__global__ void __launch_bounds__(256) k_alltoalls_flat(const char *src0, char *dst0,
                                                        uint64_t step, int P, uint64_t n,
                                                        int64_t dst, int64_t sst) {
  const uint64_t total = (uint64_t)P * (uint64_t)P * n;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t pr = i / n, t = i - pr * n;
    const uint64_t k = pr / (uint64_t)P, l = pr - k * (uint64_t)P;
    const E *src = (const E *)(src0 + k * step);
    E *d = (E *)(dst0 + l * step);
    d[(k * n + t) * (uint64_t)dst] = src[(l * n + t) * (uint64_t)sst];
  }
}

/* strided alltoall with an element size that is not 1/2/4/8/16 bytes */
__global__ void __launch_bounds__(256) k_alltoalls_bytes(const char *src0, char *dst0,
                                                         uint64_t step, int P, uint64_t n,
                                                         int64_t dst, int64_t sst, uint64_t es) {
  const uint64_t pairs = (uint64_t)P * (uint64_t)P;
  for (uint64_t pr = blockIdx.y; pr < pairs; pr += gridDim.y) {
    const uint64_t k = pr / (uint64_t)P, l = pr % (uint64_t)P;
    const char *src = src0 + k * step + l * n * (uint64_t)sst * es;
    char *d = dst0 + l * step + k * n * (uint64_t)dst * es;
    for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < n * es;
         x += (uint64_t)gridDim.x * blockDim.x) {
      const uint64_t t = x / es, b = x % es;
      d[t * (uint64_t)dst * es + b] = src[t * (uint64_t)sst * es + b];
    }
  }
}

/* broadcast: every member but the root gets the root's source */
template <bool VEC>
__global__ void __launch_bounds__(256) k_broadcast(const char *src, char *dst0, uint64_t step,
                                                   int P, int root, uint64_t nbytes) {
  const uint64_t n = VEC ? nbytes / 16 : nbytes;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (uint64_t)gridDim.x * blockDim.x) {
    if constexpr (VEC) {
      const uint4 u = ld16(src + v * 16);
      for (int j = 0; j < P; j++)
        if (j != root) st16(dst0 + (uint64_t)j * step + v * 16, u);
    } else {
      const char c = src[v];
      for (int j = 0; j < P; j++)
        if (j != root) dst0[(uint64_t)j * step + v] = c;
    }
  }
}

/* Pairs of an all-to-all beyond this many loop over blockIdx.y. */
constexpr uint64_t kMaxGridY = 65535;
/* Blocks of fewer words than this per pair take the flattened kernels. */
constexpr uint64_t kFlatWords = 64;

/* CTAs along x for a per-pair / per-member extent of n work items, so that
 * the whole grid is about `want` CTAs. */
unsigned x_blocks(uint64_t n, uint64_t ypairs, uint64_t want) {
  uint64_t per = (n + 255) / 256;
  uint64_t cap = want / (ypairs ? ypairs : 1);
  if (cap < 1) cap = 1;
  if (per > cap) per = cap;
  return (unsigned)(per < 1 ? 1 : per);
}

}  // namespace

int fcollect_launch(int pe_start, int pe_stride, int P, uint64_t dest_off, uint64_t src_off,
                    uint64_t nbytes, cudaStream_t s) {
  int rc = check_team(pe_start, pe_stride, P);
  if (rc) return rc;
  if (nbytes > st().slice / (uint64_t)P) return fail(B200SHM_ERR_ARG, "fcollect: too large");
  if ((rc = check_extent(src_off, nbytes, "fcollect source"))) return rc;
  if ((rc = check_extent(dest_off, nbytes * (uint64_t)P, "fcollect dest"))) return rc;
  if (overlaps(dest_off, nbytes * (uint64_t)P, src_off, nbytes))
    return fail(B200SHM_ERR_ARG, "fcollect: dest and source overlap");
  if (nbytes == 0) return B200SHM_OK;
  if (P > 65535) return fail(B200SHM_ERR_UNSUPPORTED, "fcollect: more than 65535 members");
  Members m = members(pe_start, pe_stride, P);
  const bool vec = ((src_off | dest_off | nbytes | m.step) & 15u) == 0;
  const uint64_t n = vec ? nbytes / 16 : nbytes;
  static const bool bulk = getenv("B200SHM_FCOLLECT_BULK") && atoi(getenv("B200SHM_FCOLLECT_BULK")) > 0;
  if (vec && bulk) { /* the staged form, selected for measurement */
    const uint64_t ntiles = (nbytes + kFcBulkTile - 1) / kFcBulkTile;
    const uint64_t cap = (8ull * st().sm_count + P - 1) / (uint64_t)P;
    dim3 g((unsigned)(ntiles < cap ? ntiles : (cap ? cap : 1)), P);
    k_fcollect_bulk<<<g, 256, 0, s>>>(m.first + src_off, m.first + dest_off, m.step, P, nbytes,
                                      st().d_status);
    count_launch();
    return B200SHM_OK;
  }
  dim3 grid(x_blocks(n, P, 8ull * st().sm_count * 4), P);
  if (vec)
    k_fcollect<true><<<grid, 256, 0, s>>>(m.first + src_off, m.first + dest_off, m.step, P, nbytes);
  else
    k_fcollect<false><<<grid, 256, 0, s>>>(m.first + src_off, m.first + dest_off, m.step, P, nbytes);
  count_launch();
  return B200SHM_OK;
}

int collect_launch(int pe_start, int pe_stride, int P, uint64_t dest_off, uint64_t src_off,
                   const uint64_t *nbytes, cudaStream_t s) {
  int rc = check_team(pe_start, pe_stride, P);
  if (rc) return rc;
  if (!nbytes) return fail(B200SHM_ERR_ARG, "collect: null size array");
  if (P > 65535) return fail(B200SHM_ERR_UNSUPPORTED, "collect: more than 65535 members");
  std::vector<uint64_t> host(2 * (size_t)P);
  uint64_t total = 0, biggest = 0, bits = 0;
  for (int k = 0; k < P; k++) {
    if (nbytes[k] > st().slice || total + nbytes[k] > st().slice)
      return fail(B200SHM_ERR_ARG, "collect: contributions larger than a heap slice");
    host[k] = nbytes[k];
    host[P + k] = total;
    total += nbytes[k];
    if (nbytes[k] > biggest) biggest = nbytes[k];
    bits |= nbytes[k];
  }
  if ((rc = check_extent(src_off, biggest, "collect source"))) return rc;
  if ((rc = check_extent(dest_off, total, "collect dest"))) return rc;
  if (overlaps(dest_off, total, src_off, biggest))
    return fail(B200SHM_ERR_ARG, "collect: dest and source overlap");
  if (total == 0) return B200SHM_OK;
  Members m = members(pe_start, pe_stride, P);
  bits |= src_off | dest_off | m.step;
  const uint64_t w = bits & 15 ? (bits & 7 ? (bits & 3 ? 1 : 4) : 8) : 16;
  uint64_t *dev = nullptr;
  B200_CK(cudaMallocAsync((void **)&dev, host.size() * sizeof(uint64_t), s));
  B200_CK(cudaMemcpyAsync(dev, host.data(), host.size() * sizeof(uint64_t),
                          cudaMemcpyHostToDevice, s));
  dim3 grid(x_blocks(biggest / w, P, 8ull * st().sm_count * 4), P);
  const char *src = m.first + src_off;
  char *dst = m.first + dest_off;
  switch (w) {
  case 16: k_collect<uint4><<<grid, 256, 0, s>>>(src, dst, m.step, P, dev, dev + P); break;
  case 8: k_collect<unsigned long long><<<grid, 256, 0, s>>>(src, dst, m.step, P, dev, dev + P); break;
  case 4: k_collect<unsigned><<<grid, 256, 0, s>>>(src, dst, m.step, P, dev, dev + P); break;
  default: k_collect<unsigned char><<<grid, 256, 0, s>>>(src, dst, m.step, P, dev, dev + P); break;
  }
  count_launch();
  B200_CK(cudaFreeAsync(dev, s));
  return B200SHM_OK;
}

int alltoall_launch(int pe_start, int pe_stride, int P, uint64_t dest_off, uint64_t src_off,
                    uint64_t B, cudaStream_t s) {
  int rc = check_team(pe_start, pe_stride, P);
  if (rc) return rc;
  if (B > st().slice / (uint64_t)P) return fail(B200SHM_ERR_ARG, "alltoall: too large");
  if ((rc = check_extent(src_off, B * (uint64_t)P, "alltoall source"))) return rc;
  if ((rc = check_extent(dest_off, B * (uint64_t)P, "alltoall dest"))) return rc;
  if (overlaps(dest_off, B * (uint64_t)P, src_off, B * (uint64_t)P))
    return fail(B200SHM_ERR_ARG, "alltoall: dest and source overlap");
  if (B == 0) return B200SHM_OK;
  Members m = members(pe_start, pe_stride, P);
  const char *sp = m.first + src_off;
  char *dp = m.first + dest_off;
  const uint64_t pairs = (uint64_t)P * P;
  const uint64_t bits = src_off | dest_off | B | m.step;
  const uint64_t w = bits & 15 ? (bits & 7 ? (bits & 3 ? 1 : 4) : 8) : 16;
  if (B / w < kFlatWords) {
    /* small blocks: threads over the flattened [pair][word] space */
    const uint64_t nw = B / w;
    const unsigned g = grid_for(pairs * nw, 256, 8);
    switch (w) {
    case 16: k_alltoall_flat<uint4><<<g, 256, 0, s>>>(sp, dp, m.step, P, nw); break;
    case 8: k_alltoall_flat<unsigned long long><<<g, 256, 0, s>>>(sp, dp, m.step, P, nw); break;
    case 4: k_alltoall_flat<unsigned><<<g, 256, 0, s>>>(sp, dp, m.step, P, nw); break;
    default: k_alltoall_flat<unsigned char><<<g, 256, 0, s>>>(sp, dp, m.step, P, nw); break;
    }
    count_launch();
    return B200SHM_OK;
  }
  const bool vec = w == 16;
  const uint64_t n = vec ? B / 16 : B;
  const unsigned gy = (unsigned)(pairs < kMaxGridY ? pairs : kMaxGridY);
  dim3 grid(x_blocks(vec ? (n + 3) / 4 : n, gy, 8ull * st().sm_count * 4), gy);
  if (vec)
    k_alltoall<true><<<grid, 256, 0, s>>>(sp, dp, m.step, P, B);
  else
    k_alltoall<false><<<grid, 256, 0, s>>>(sp, dp, m.step, P, B);
  count_launch();
  return B200SHM_OK;
}

int alltoalls_launch(int pe_start, int pe_stride, int P, uint64_t dest_off, uint64_t src_off,
                     int64_t dst, int64_t sst, uint64_t n, uint64_t es, cudaStream_t s) {
  int rc = check_team(pe_start, pe_stride, P);
  if (rc) return rc;
  if (dst < 1 || sst < 1 || es < 1)
    return fail(B200SHM_ERR_ARG, "alltoalls: strides and element size must be positive");
  const uint64_t lim = st().slice;
  /* extent touched: (P*n - 1)*stride + 1 elements */
  if (n > lim / es / (uint64_t)P) return fail(B200SHM_ERR_ARG, "alltoalls: too large");
  if (n == 0) return B200SHM_OK;
  const uint64_t cnt = (uint64_t)P * n;
  if ((uint64_t)dst > lim / cnt || (uint64_t)sst > lim / cnt)
    return fail(B200SHM_ERR_ARG, "alltoalls: stride too large");
  const uint64_t dbytes = ((cnt - 1) * (uint64_t)dst + 1) * es;
  const uint64_t sbytes = ((cnt - 1) * (uint64_t)sst + 1) * es;
  if ((rc = check_extent(src_off, sbytes, "alltoalls source"))) return rc;
  if ((rc = check_extent(dest_off, dbytes, "alltoalls dest"))) return rc;
  if (overlaps(dest_off, dbytes, src_off, sbytes))
    return fail(B200SHM_ERR_ARG, "alltoalls: dest and source overlap");
  Members m = members(pe_start, pe_stride, P);
  const uint64_t pairs = (uint64_t)P * P;
  const char *sp = m.first + src_off;
  char *dp = m.first + dest_off;
  const bool al = ((src_off | dest_off | m.step) % es) == 0;
  const bool typed = es == 1 || (al && (es == 2 || es == 4 || es == 8 || es == 16));
  if (typed && n < kFlatWords) {
    /* few elements per pair: threads over the flattened [pair][element] space */
    const unsigned g = grid_for(pairs * n, 256, 8);
    switch (es) {
    case 8: k_alltoalls_flat<uint64_t><<<g, 256, 0, s>>>(sp, dp, m.step, P, n, dst, sst); break;
    case 4: k_alltoalls_flat<uint32_t><<<g, 256, 0, s>>>(sp, dp, m.step, P, n, dst, sst); break;
    case 2: k_alltoalls_flat<uint16_t><<<g, 256, 0, s>>>(sp, dp, m.step, P, n, dst, sst); break;
    case 16: k_alltoalls_flat<uint4><<<g, 256, 0, s>>>(sp, dp, m.step, P, n, dst, sst); break;
    default: k_alltoalls_flat<uint8_t><<<g, 256, 0, s>>>(sp, dp, m.step, P, n, dst, sst); break;
    }
    count_launch();
    return B200SHM_OK;
  }
  const unsigned gy = (unsigned)(pairs < kMaxGridY ? pairs : kMaxGridY);
  dim3 grid(x_blocks(n, gy, 8ull * st().sm_count * 4), gy);
  if (al && es == 8)
    k_alltoalls<uint64_t><<<grid, 256, 0, s>>>(sp, dp, m.step, P, n, dst, sst);
  else if (al && es == 4)
    k_alltoalls<uint32_t><<<grid, 256, 0, s>>>(sp, dp, m.step, P, n, dst, sst);
  else if (al && es == 2)
    k_alltoalls<uint16_t><<<grid, 256, 0, s>>>(sp, dp, m.step, P, n, dst, sst);
  else if (es == 1)
    k_alltoalls<uint8_t><<<grid, 256, 0, s>>>(sp, dp, m.step, P, n, dst, sst);
  else if (al && es == 16)
    k_alltoalls<uint4><<<grid, 256, 0, s>>>(sp, dp, m.step, P, n, dst, sst);
  else {
    dim3 g2(x_blocks(n * es, gy, 8ull * st().sm_count * 4), gy);
    k_alltoalls_bytes<<<g2, 256, 0, s>>>(sp, dp, m.step, P, n, dst, sst, es);
  }
  count_launch();
  return B200SHM_OK;
}

int broadcast_launch(int root, int pe_start, int pe_stride, int P, uint64_t dest_off,
                     uint64_t src_off, uint64_t nbytes, cudaStream_t s) {
  int rc = check_team(pe_start, pe_stride, P);
  if (rc) return rc;
  if (root < 0 || root >= P) return fail(B200SHM_ERR_ARG, "broadcast: root %d not a member", root);
  if ((rc = check_extent(src_off, nbytes, "broadcast source"))) return rc;
  if ((rc = check_extent(dest_off, nbytes, "broadcast dest"))) return rc;
  if (dest_off != src_off && overlaps(dest_off, nbytes, src_off, nbytes))
    return fail(B200SHM_ERR_ARG, "broadcast: dest and source overlap");
  if (nbytes == 0 || P == 1) return B200SHM_OK;
  Members m = members(pe_start, pe_stride, P);
  const bool vec = ((src_off | dest_off | nbytes | m.step) & 15u) == 0;
  const uint64_t n = vec ? nbytes / 16 : nbytes;
  const char *src = m.first + (uint64_t)root * m.step + src_off;
  if (vec)
    k_broadcast<true><<<grid_for(n, 256, 8), 256, 0, s>>>(src, m.first + dest_off, m.step, P, root, nbytes);
  else
    k_broadcast<false><<<grid_for(n, 256, 8), 256, 0, s>>>(src, m.first + dest_off, m.step, P, root, nbytes);
  count_launch();
  return B200SHM_OK;
}

}  // namespace b200

using namespace b200;

extern "C" {

int b200shm_fcollect(int pe_start, int pe_stride, int pe_size, uint64_t dest_off,
                     uint64_t src_off, uint64_t nbytes, void *stream) {
  int rc = fcollect_launch(pe_start, pe_stride, pe_size, dest_off, src_off, nbytes,
                           pick_stream(stream));
  return rc ? rc : finish(stream, "b200shm_fcollect");
}

int b200shm_collect(int pe_start, int pe_stride, int pe_size, uint64_t dest_off,
                    uint64_t src_off, const uint64_t *nbytes, void *stream) {
  int rc = collect_launch(pe_start, pe_stride, pe_size, dest_off, src_off, nbytes,
                          pick_stream(stream));
  return rc ? rc : finish(stream, "b200shm_collect");
}

int b200shm_alltoall(int pe_start, int pe_stride, int pe_size, uint64_t dest_off,
                     uint64_t src_off, uint64_t nbytes, void *stream) {
  int rc = alltoall_launch(pe_start, pe_stride, pe_size, dest_off, src_off, nbytes,
                           pick_stream(stream));
  return rc ? rc : finish(stream, "b200shm_alltoall");
}

int b200shm_alltoalls(int pe_start, int pe_stride, int pe_size, uint64_t dest_off,
                      uint64_t src_off, int64_t dst, int64_t sst, uint64_t nelems,
                      uint64_t elem_size, void *stream) {
  int rc = alltoalls_launch(pe_start, pe_stride, pe_size, dest_off, src_off, dst, sst, nelems,
                            elem_size, pick_stream(stream));
  return rc ? rc : finish(stream, "b200shm_alltoalls");
}

int b200shm_broadcast(int root, int pe_start, int pe_stride, int pe_size, uint64_t dest_off,
                      uint64_t src_off, uint64_t nbytes, void *stream) {
  int rc = broadcast_launch(root, pe_start, pe_stride, pe_size, dest_off, src_off, nbytes,
                            pick_stream(stream));
  return rc ? rc : finish(stream, "b200shm_broadcast");
}

}  // extern "C"
