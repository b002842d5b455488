/* The division-free x / 60 of the MP5 reconstruction (div60 in
 * asterx_b200/csrc/axb_recon.cuh: Markstein's FMA correction step against the
 * correctly rounded reciprocal) against the correctly rounded quotient x / 60,
 * bit for bit: random mantissas over exponents -600..600, integers, and
 * scaled integers (multiples of 15 among them).  Exit status 0 when every
 * result matches. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static uint64_t state = 88172645463325252ull;
static uint64_t xorshift(void) {
  state ^= state << 13;
  state ^= state >> 7;
  state ^= state << 17;
  return state;
}

static double div60(double x) {
  const double r = 1.0 / 60.0;
  const double q = x * r;
  const double aq = fabs(q);
  if (!(aq >= 0x1p-960 && aq <= 0x1p1000))
    return x / 60.0;
  const double rem = fma(-q, 60.0, x);
  return fma(rem, r, q);
}

static long check(double x) {
  const double a = x / 60.0, c = div60(x);
  return memcmp(&a, &c, sizeof a) != 0;
}

int main(int argc, char **argv) {
  const long n = argc > 1 ? atol(argv[1]) : 20000000L;
  long bad = 0, total = 0;
  for (long i = 0; i < n; ++i) {
    uint64_t b = xorshift();
    b = (b & 0x800FFFFFFFFFFFFFull) | ((uint64_t)(1023 + (int)(xorshift() % 1200) - 600) << 52);
    double x;
    memcpy(&x, &b, sizeof x);
    bad += check(x);
    ++total;
  }
  for (long m = -1000000; m <= 1000000; ++m) {
    bad += check((double)m) + check((double)m * 0x1p-40) + check((double)m * 0x1p+37);
    total += 3;
  }
  printf("%ld checked, %ld mismatches\n", total, bad);
  return bad != 0;
}
