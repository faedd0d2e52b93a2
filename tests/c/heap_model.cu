/*
 * Host build of the symmetric-heap allocator's bookkeeping
 * (osss-ucx_b200/csrc/heap_core.cuh; the device runs the same functions
 * under its lock).  A seeded random sequence of allocations (sizes, and
 * alignments, of many scales) and frees, with the whole structure checked
 * after every operation:
 *  - the blocks tile [0, N) exactly, with consistent back links;
 *  - no two free blocks are adjacent (frees merge at once);
 *  - every free block is in the list of its size class, the bitmaps say
 *    exactly which lists are non-empty, free_units is the sum;
 *  - live allocations never overlap, are aligned as asked, and only their
 *    owner's free releases them (a second free is refused);
 *  - an allocation fails only when no free block can hold it;
 * then exhaustion (allocate until refused) and a full free back to one
 * block.  Prints "ok" or the first broken rule.  Run by tests/test_heap_cpu.py.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <map>
#include <random>
#include <vector>

#include "heap_core.cuh"

using namespace b200;

#define REQUIRE(c, ...)                                                        \
  do {                                                                         \
    if (!(c)) {                                                                \
      printf(__VA_ARGS__);                                                     \
      printf("\n");                                                            \
      exit(1);                                                                 \
    }                                                                          \
  } while (0)

struct Model {
  unsigned N;
  HeapCtl ctl;
  std::vector<unsigned> size, prev_phys, next_free, prev_free;
  std::vector<unsigned char> flags;
  HeapDev h;
  explicit Model(unsigned n) : N(n), size(n), prev_phys(n), next_free(n), prev_free(n), flags(n) {
    memset(&ctl, 0, sizeof(ctl));
    for (int i = 0; i < kHeapFL; i++)
      for (int j = 0; j < kHeapSL; j++) ctl.head[i][j] = kHeapNil;
    ctl.nunits = n;
    ctl.unit_shift = 8;
    h.ctl = &ctl;
    h.size = size.data();
    h.prev_phys = prev_phys.data();
    h.next_free = next_free.data();
    h.prev_free = prev_free.data();
    h.flags = flags.data();
    h.free_bytes_host = nullptr;
    size[0] = n;
    prev_phys[0] = kHeapNil;
    heap_link(h, 0);
  }
  unsigned largest_free() const {
    unsigned best = 0;
    for (unsigned b = 0; b < N; b += size[b])
      if ((flags[b] & kBlkFree) && size[b] > best) best = size[b];
    return best;
  }
  void check(const std::map<unsigned, unsigned> &live) const {
    unsigned long long free_sum = 0;
    unsigned prev = kHeapNil;
    bool prev_free_blk = false;
    unsigned nfree = 0;
    for (unsigned b = 0; b < N;) {
      REQUIRE(flags[b] & kBlkStart, "unit %u is not a block start", b);
      REQUIRE(size[b] >= 1 && b + size[b] <= N, "block %u has size %u", b, size[b]);
      REQUIRE(prev_phys[b] == prev, "block %u: back link %u, want %u", b, prev_phys[b], prev);
      const bool fr = flags[b] & kBlkFree;
      REQUIRE(!(fr && prev_free_blk), "free blocks %u and %u are adjacent", prev, b);
      if (fr) {
        free_sum += size[b];
        nfree++;
        int fl, sl;
        heap_class(size[b], fl, sl);
        bool found = false;
        for (unsigned x = ctl.head[fl][sl]; x != kHeapNil; x = next_free[x]) found |= x == b;
        REQUIRE(found, "free block %u (size %u) is not in its list", b, size[b]);
        REQUIRE(!live.count(b), "live block %u is marked free", b);
      } else {
        auto it = live.find(b);
        REQUIRE(it != live.end(), "allocated block %u is not live", b);
        REQUIRE(size[b] == it->second, "live block %u: size %u, want %u", b, size[b], it->second);
      }
      for (unsigned u = b + 1; u < b + size[b] && u < b + 4; u++)
        REQUIRE(!(flags[u] & kBlkStart), "unit %u inside block %u is a start", u, b);
      prev = b;
      prev_free_blk = fr;
      b += size[b];
    }
    REQUIRE(free_sum == ctl.free_units, "free units %llu, counted %llu",
            (unsigned long long)ctl.free_units, free_sum);
    unsigned listed = 0;
    for (int i = 0; i < kHeapFL; i++) {
      REQUIRE(((ctl.fl_map >> i) & 1) == (ctl.sl_map[i] != 0), "first-level bit %d", i);
      for (int j = 0; j < kHeapSL; j++) {
        const bool nonempty = ctl.head[i][j] != kHeapNil;
        REQUIRE(((ctl.sl_map[i] >> j) & 1) == (unsigned)nonempty, "second-level bit %d/%d", i, j);
        unsigned p = kHeapNil;
        for (unsigned x = ctl.head[i][j]; x != kHeapNil; x = next_free[x]) {
          REQUIRE(prev_free[x] == p, "list %d/%d: back link of %u", i, j, x);
          p = x;
          listed++;
          REQUIRE(listed <= N, "list cycle");
        }
      }
    }
    REQUIRE(listed == nfree, "%u blocks listed, %u free", listed, nfree);
    REQUIRE(ctl.blocks_used == live.size(), "blocks_used %llu, live %zu",
            (unsigned long long)ctl.blocks_used, live.size());
  }
};

int main(int argc, char **argv) {
  const unsigned long long seed = argc > 1 ? strtoull(argv[1], nullptr, 0) : 1;
  std::mt19937_64 rng(seed);
  unsigned long long allocs = 0, refused = 0, frees = 0;
  for (unsigned N : {1u, 17u, 4096u, 98304u, 1u << 20}) {
    Model m(N);
    std::map<unsigned, unsigned> live;
    m.check(live);
    const int ops = N < 100 ? 200 : 6000;
    for (int op = 0; op < ops; op++) {
      const bool do_alloc = live.empty() || rng() % 100 < 55;
      if (do_alloc) {
        unsigned units;
        const int scale = (int)(rng() % 5);
        if (scale == 0) units = 1 + rng() % 4;
        else if (scale == 1) units = 1 + rng() % 64;
        else if (scale == 2) units = 1 + rng() % 1024;
        else if (scale == 3) units = 1 + rng() % (N / 8 + 1);
        else units = 1 + rng() % (N / 2 + 1);
        const unsigned align = rng() % 4 == 0 ? 1u << (rng() % 6) : 1u;
        const unsigned largest = m.largest_free();
        const unsigned b = heap_alloc_locked(m.h, units, align);
        if (b == kHeapNil) {
          refused++;
          REQUIRE((unsigned long long)units + align - 1 > largest,
                  "N=%u: %u units (align %u) refused with a free block of %u", N, units, align,
                  largest);
        } else {
          REQUIRE(b % align == 0, "block %u not aligned to %u", b, align);
          REQUIRE(b + units <= N, "block %u + %u beyond %u", b, units, N);
          auto it = live.lower_bound(b);
          if (it != live.end()) REQUIRE(b + units <= it->first, "overlaps block %u", it->first);
          if (it != live.begin()) {
            --it;
            REQUIRE(it->first + it->second <= b, "overlaps block %u", it->first);
          }
          live[b] = units;
          allocs++;
        }
      } else {
        auto it = live.begin();
        std::advance(it, rng() % live.size());
        const unsigned b = it->first;
        live.erase(it);
        REQUIRE(heap_free_locked(m.h, b) == kHeapOk, "free of live block %u refused", b);
        frees++;
        REQUIRE(heap_free_locked(m.h, b) == kHeapBadFree, "second free of %u accepted", b);
      }
      if (N <= 4096 || op % 50 == 0) m.check(live);
    }
    m.check(live);
    REQUIRE(heap_free_locked(m.h, N) == kHeapBadFree, "free beyond the heap accepted");
    /* exhaustion: fill with small blocks until refused, then free everything */
    for (;;) {
      const unsigned units = 1 + rng() % 8;
      const unsigned b = heap_alloc_locked(m.h, units, 1);
      if (b == kHeapNil) {
        REQUIRE(m.largest_free() < units, "refused with room");
        break;
      }
      live[b] = units;
    }
    m.check(live);
    for (auto &kv : live) REQUIRE(heap_free_locked(m.h, kv.first) == kHeapOk, "final free");
    live.clear();
    m.check(live);
    REQUIRE(m.size[0] == N && (m.flags[0] & kBlkFree) && m.ctl.free_units == N,
            "N=%u: not one free block after freeing everything", N);
  }
  printf("%llu allocations, %llu refused, %llu frees\nok\n", allocs, refused, frees);
  return 0;
}
