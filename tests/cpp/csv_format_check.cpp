// Checks the CSV entry formatter of form_factors_b200/csrc/ffb_csv.cuh, built
// as plain C++, against the C library's "%g" (what the reference's
// `std::ostream << float` prints through libstdc++).  Usage:
//   csv_format_check <n_random> <seed>
// Prints the number of mismatches and the first few; exit status 1 on any.
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>

#include "ffb_csv.cuh"

static long g_bad = 0, g_checked = 0;

static void check(float f)
{
  char want[64], got[32];
  snprintf(want, sizeof want, "%g", (double)f);
  const int n = ffb::csv::format_g6(f, got);
  got[n] = 0;
  ++g_checked;
  if (strcmp(want, got) != 0) {
    if (g_bad < 10) {
      unsigned u;
      memcpy(&u, &f, 4);
      printf("mismatch bits=0x%08x want=%s got=%s\n", u, want, got);
    }
    ++g_bad;
  }
}

int main(int argc, char** argv)
{
  const long n_random = argc > 1 ? atol(argv[1]) : 1000000;
  const unsigned seed = argc > 2 ? (unsigned)atol(argv[2]) : 1u;
  // special values and edges
  const float specials[] = {0.f, -0.f, 1.f, -1.f, 0.5f, 0.1f, 1e-4f, 9.99999e-5f, 1e-5f, 100000.f, 999999.f,
                            999999.5f, 1e6f, 1234567.f, FLT_MAX, -FLT_MAX, FLT_MIN, FLT_TRUE_MIN, -FLT_TRUE_MIN,
                            INFINITY, -INFINITY, NAN, -NAN, 0.000976562f, 3.0517578125e-05f, 16777216.f, 8388607.5f};
  for (float f : specials)
    check(f);
  // exact ties at the seventh significant digit: powers of two
  for (int e = -149; e <= 127; ++e)
    check(ldexpf(1.f, e));
  // count / outgoing as the normalisation computes it
  for (int out = 1; out <= 4000; ++out) {
    const float r = 1.f / (float)out;
    for (int c = 0; c <= out; c += 1 + out / 200)
      check((float)c * r);
  }
  // every float with a random bit pattern
  std::mt19937 rng(seed);
  for (long i = 0; i < n_random; ++i) {
    unsigned u = rng();
    float f;
    memcpy(&f, &u, 4);
    check(f);
  }
  // all floats of a few binades in full
  for (int e = -30; e <= 25; e += 11) {
    const float lo = ldexpf(1.f, e);
    for (unsigned k = 0; k < (1u << 23); k += 7) {
      unsigned u;
      memcpy(&u, &lo, 4);
      u += k;
      float f;
      memcpy(&f, &u, 4);
      check(f);
    }
  }
  printf("checked %ld, mismatches %ld\n", g_checked, g_bad);
  return g_bad ? 1 : 0;
}
