// Checks the software x87 arithmetic of osss-ucx_b200/csrc/f80.cuh (host
// build of the same functions the GPU kernels run) against this machine's
// own long double, which gcc evaluates on the x87 unit: add, multiply and
// the two comparisons, on random operands of every encoding class and on
// operand pairs aimed at cancellation, rounding ties, overflow and gradual
// underflow.  Prints the mismatch count and exits non-zero on any mismatch.
//
//   g++ -O2 -std=c++17 -I osss-ucx_b200/csrc tests/c/f80_model.cpp -o f80_model
//   ./f80_model [operand pairs per class pair, default 200000] [seed]
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "f80.cuh"

using b200::f80;

static uint64_t g_state = 0x9E3779B97F4A7C15ull;  // seed: argv[2] when given
static uint64_t rnd() { /* splitmix64 */
  uint64_t z = (g_state += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static long double to_ld(const f80 &a) {
  long double x;
  memset(&x, 0, sizeof(x));
  memcpy(&x, &a.sig, 8);
  memcpy((char *)&x + 8, &a.se, 2);
  return x;
}
static f80 from_ld(long double x) {
  f80 r = b200::f80_make(0, 0);
  memcpy(&r.sig, &x, 8);
  memcpy(&r.se, (char *)&x + 8, 2);
  return r;
}

// operands of one class: 0 normal (any exponent), 1 normal near exponent
// `near`, 2 denormal, 3 pseudo-denormal, 4 zero, 5 infinity, 6 quiet NaN,
// 7 signalling NaN, 8 unnormal / pseudo-NaN / pseudo-infinity, 9 normal
// with a short significand (exact results and ties), 10 extreme exponents
static f80 operand(int cls, int near) {
  const uint16_t s = (uint16_t)((rnd() & 1) << 15);
  switch (cls) {
  case 0: return b200::f80_make(s | (uint16_t)(1 + rnd() % 0x7FFE), b200::kF80J | rnd());
  case 1: {
    int e = near + (int)(rnd() % 140) - 70;
    if (e < 1) e = 1;
    if (e > 0x7FFE) e = 0x7FFE;
    return b200::f80_make(s | (uint16_t)e, b200::kF80J | rnd());
  }
  case 2: return b200::f80_make(s, (rnd() >> (rnd() % 64)) & ~b200::kF80J);
  case 3: return b200::f80_make(s, b200::kF80J | (rnd() >> (rnd() % 64)));
  case 4: return b200::f80_make(s, 0);
  case 5: return b200::f80_make(s | 0x7FFF, b200::kF80J);
  case 6: return b200::f80_make(s | 0x7FFF, b200::kF80J | b200::kF80Quiet | (rnd() & 0xFFFF));
  case 7: return b200::f80_make(s | 0x7FFF, b200::kF80J | (1 + (rnd() & 0xFFFF)));
  case 8: {
    const uint16_t e = (rnd() & 1) ? 0x7FFF : (uint16_t)(1 + rnd() % 0x7FFE);
    return b200::f80_make(s | e, rnd() & ~b200::kF80J);
  }
  case 9: {
    int e = near + (int)(rnd() % 130) - 65;
    if (e < 1) e = 1;
    if (e > 0x7FFE) e = 0x7FFE;
    const int keep = 1 + (int)(rnd() % 64);
    return b200::f80_make(s | (uint16_t)e, b200::kF80J | ((rnd() >> (64 - keep)) << (64 - keep)));
  }
  default: {
    const uint16_t e = (rnd() & 1) ? (uint16_t)(1 + rnd() % 80) : (uint16_t)(0x7FFE - rnd() % 80);
    return b200::f80_make(s | e, b200::kF80J | rnd());
  }
  }
}

static bool same(const f80 &a, const f80 &b) { return a.sig == b.sig && a.se == b.se; }

int main(int argc, char **argv) {
  const long per = argc > 1 ? atol(argv[1]) : 200000;
  if (argc > 2) g_state = strtoull(argv[2], nullptr, 0);
  long bad = 0, n = 0;
  for (int ca = 0; ca <= 10; ca++) {
    for (int cb = 0; cb <= 10; cb++) {
      for (long i = 0; i < per / 8; i++) {
        const int near = (int)(rnd() % 0x7FFF);
        const f80 a = operand(ca, near), b = operand(cb, near);
        volatile long double x = to_ld(a), y = to_ld(b);
        const f80 s_ref = from_ld(x + y), p_ref = from_ld(x * y);
        const bool lt_ref = x < y, gt_ref = x > y;
        const f80 s = b200::f80_add(a, b), p = b200::f80_mul(a, b);
        const bool lt = b200::f80_lt(a, b), gt = b200::f80_gt(a, b);
        n++;
        if (!same(s, s_ref) || !same(p, p_ref) || lt != lt_ref || gt != gt_ref) {
          if (bad < 12)
            printf("mismatch cls %d/%d: a=%04x:%016llx b=%04x:%016llx add %04x:%016llx "
                   "(x87 %04x:%016llx) mul %04x:%016llx (x87 %04x:%016llx) lt %d/%d gt %d/%d\n",
                   ca, cb, a.se, (unsigned long long)a.sig, b.se, (unsigned long long)b.sig,
                   s.se, (unsigned long long)s.sig, s_ref.se, (unsigned long long)s_ref.sig,
                   p.se, (unsigned long long)p.sig, p_ref.se, (unsigned long long)p_ref.sig, lt,
                   lt_ref, gt, gt_ref);
          bad++;
        }
      }
    }
  }
  printf("f80 model: %ld operand pairs, %ld mismatches\n", n, bad);
  return bad ? 1 : 0;
}
