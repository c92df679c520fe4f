/* CPU check of the LU-SGS sweeps' division by a precomputed reciprocal
 * (div_by_recip in minifs_b200/csrc/mfg_kernels.cuh): the same steps with
 * the C library's fma, against the division, on pseudo-random pairs.
 * Usage: div_by_recip_check N SEED; prints the count of differing results. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static uint64_t splitmix64(uint64_t *x) {
  uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static double bits_to_double(uint64_t u) {
  double d;
  memcpy(&d, &u, 8);
  return d;
}

static uint64_t double_to_bits(double d) {
  uint64_t u;
  memcpy(&u, &d, 8);
  return u;
}

static double draw(uint64_t *x, int all_ones) {
  const uint64_t r = splitmix64(x), e = splitmix64(x);
  const uint64_t mant = all_ones ? 0xFFFFFFFFFFFFFull : (r & 0xFFFFFFFFFFFFFull);
  const uint64_t expo = (uint64_t)(1023 - 600 + (int64_t)(e % 1201));
  return bits_to_double(((r >> 63) << 63) | (expo << 52) | mant);
}

static double div_by_recip(double a, double b, double y) {
  const int ea = (int)((double_to_bits(a) >> 52) & 0x7FF);
  const int eb = (int)((double_to_bits(b) >> 52) & 0x7FF);
  if (ea < 523 || ea > 1523 || eb < 523 || eb > 1523) return a / b;
  const double q0 = a * y;
  const double r0 = fma(-b, q0, a);
  const double q1 = fma(r0, y, q0);
  const double r1 = fma(-b, q1, a);
  return fma(r1, y, q1);
}

int main(int argc, char **argv) {
  const long long n = argc > 1 ? atoll(argv[1]) : 10000000;
  const uint64_t seed = argc > 2 ? strtoull(argv[2], NULL, 10) : 1;
  long long bad = 0;
  for (long long i = 0; i < n; i++) {
    uint64_t x = seed ^ ((uint64_t)i * 0xD1B54A32D192ED03ull);
    const double a = draw(&x, 0);
    const double b = draw(&x, (i & 3) == 3);
    const double q = div_by_recip(a, b, 1.0 / b);
    if (double_to_bits(q) != double_to_bits(a / b)) bad++;
  }
  printf("%lld\n", bad);
  return 0;
}
