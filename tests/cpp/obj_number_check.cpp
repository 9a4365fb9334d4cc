// Checks the OBJ number conversions of form_factors_b200/csrc/ffb_obj.cuh,
// built as plain C++, against the C library that the reference's importer
// calls (sscanf "%f" = strtof, "%d"; import_export/obj_import.cpp:193-224).
// Usage: obj_number_check <n_random> <seed>; exit status 1 on any mismatch.
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>

#include "ffb_obj.cuh"

static long g_bad = 0, g_checked = 0;

static void check_float(const std::string& text)
{
  ++g_checked;
  float want = 0.f;
  int n_want = 0;
  const int r = sscanf(text.c_str(), "%f%n", &want, &n_want);
  float got = 0.f;
  const int n_got = ffb::obj::parse_float(text.c_str(), (int)text.size(), &got);
  bool ok;
  if (r != 1)
    ok = n_got == 0;
  else {
    uint32_t a, b;
    memcpy(&a, &want, 4);
    memcpy(&b, &got, 4);
    ok = n_got == n_want && (a == b || (std::isnan(want) && std::isnan(got) && ((a ^ b) >> 31) == 0));
  }
  if (!ok) {
    if (g_bad < 12)
      printf("float mismatch '%s': want %a (%d chars, r=%d) got %a (%d chars)\n", text.c_str(), want, n_want, r, got,
             n_got);
    ++g_bad;
  }
}

static void check_face(const std::string& line)
{
  ++g_checked;
  int d, i0 = 0, i1 = 0, i2 = 0;
  const char* s = line.c_str();
  bool want = sscanf(s, "%d %d %d", &i0, &i1, &i2) == 3 ||
              sscanf(s, "%d//%d %d//%d %d//%d", &i0, &d, &i1, &d, &i2, &d) == 6 ||
              sscanf(s, "%d/%d/%d %d/%d/%d %d/%d/%d", &i0, &d, &d, &i1, &d, &d, &i2, &d, &d) == 9;
  long long idx[3] = {0, 0, 0};
  bool got = ffb::obj::scan_face(s, (int)line.size(), idx);
  bool ok = want == got && (!want || (idx[0] == i0 && idx[1] == i1 && idx[2] == i2));
  if (!ok) {
    if (g_bad < 12)
      printf("face mismatch '%s': want %d (%d %d %d) got %d (%lld %lld %lld)\n", s, want, i0, i1, i2, got, idx[0],
             idx[1], idx[2]);
    ++g_bad;
  }
}

int main(int argc, char** argv)
{
  const long n_random = argc > 1 ? atol(argv[1]) : 200000;
  std::mt19937_64 rng(argc > 2 ? atol(argv[2]) : 1);
  const char* fixed[] = {"0", "-0", "1", "+1.5", "  3.25", "1e10", "1E-5", ".5", "5.", "-.25e+2", "inf", "-INF",
                         "Infinity", "nan", "-nan", "nan(123)", "NaN(abc_1)", "0x1.8p3", "-0x.8p-2", "0X1P-149",
                         "0x1p-150", "0x1.000001p0", "0x1.0000018p0", "3.4028235e38", "3.4028236e38", "1e39",
                         "1.4e-45", "7e-46", "7.1e-46", "1.17549435e-38", "1.1754942e-38", "9.999999e-5",
                         "16777217", "16777219", "8388608.5", "0.1", "0.2", "0.3", "1.00000005960464477539",
                         "1.000000059604644775390625", "1.0000000596046447753906250000001", "x", "", "-", "e5",
                         "1e", "1e+", "0x", "123456789012345678901234567890", "0.000000000000000000000000000001",
                         "2.5e-45", "1.401298464324817e-45", "7.006492321624086e-46"};
  for (const char* f : fixed)
    check_float(f);
  // exact float values, their neighbours and midpoints printed with many digits
  std::uniform_int_distribution<uint32_t> u32;
  char buf[128];
  for (long i = 0; i < n_random; ++i) {
    uint32_t bits = u32(rng) & 0x7FFFFFFFu;
    if ((bits >> 23) == 0xFF)
      continue;
    float f;
    memcpy(&f, &bits, 4);
    const double mid = (double)f + ((double)std::nextafter(f, INFINITY) - (double)f) / 2;
    const int prec = (int)(rng() % 12) + 1;
    snprintf(buf, sizeof buf, "%.*g", prec, (double)f);
    check_float(buf);
    snprintf(buf, sizeof buf, "%.17g", mid);  // near a midpoint
    check_float(buf);
    snprintf(buf, sizeof buf, "%.40e", mid);  // the midpoint, exactly
    check_float(buf);
    snprintf(buf, sizeof buf, "%a", (double)f * (1.0 + 1e-9 * (double)(rng() % 3)));
    check_float(buf);
    snprintf(buf, sizeof buf, "%.*f", (int)(rng() % 8), (double)(rng() % 2000000) / 1000.0 - 1000.0);
    check_float(buf);
  }
  // face lines in the three formats, with junk
  const char* faces[] = {" 1 2 3", " 1 2 3 4", " 1//4 2//5 3//6", " 1/2/3 4/5/6 7/8/9", " 1/2 3/4 5/6",
                         "\t-1 -2 -3", " 1// 2//3 4//5", " 1/2/3", " a b c", " 10  20\t30", " 1//2 3//4",
                         " 1/2/3 4/5/6 7/8", " +1 +2 +3", " 1 2", " 1//2  3//4  5//6", " 1 / 2 3"};
  for (const char* f : faces)
    check_face(f);
  for (long i = 0; i < n_random / 10; ++i) {
    const int form = (int)(rng() % 3);
    std::string line;
    for (int k = 0; k < 3; ++k) {
      line += " " + std::to_string(rng() % 100000 + 1);
      if (form == 1)
        line += "//" + std::to_string(rng() % 1000);
      if (form == 2)
        line += "/" + std::to_string(rng() % 1000) + "/" + std::to_string(rng() % 1000);
    }
    check_face(line);
  }
  printf("checked %ld, mismatches %ld\n", g_checked, g_bad);
  return g_bad ? 1 : 0;
}
