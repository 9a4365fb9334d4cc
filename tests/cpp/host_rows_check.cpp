// Checks the host-side row expansion of packed count blocks
// (form_factors_b200/csrc/ffb_host_rows.cpp) against a plain dense
// construction: random sparse rows (ascending columns, some empty, some
// full), row widths 1..300 and a few thousand, destinations at every 4-byte
// offset from a 64-byte boundary, 1 to 5 threads, jobs back to back on one
// pool; pairs of two words and of one; counts as they are, and normalised to
// floats (float)count * inv with finite, infinite and negative factors.  Exits non-zero on the first
// difference (bit for bit).
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

#include "ffb_internal.h"

int ffb_set_error(int code, const char*) { return code; }

int main()
{
  std::mt19937_64 rng(12345);
  int cases = 0;
  for (int threads = 1; threads <= 5; threads += 2) {
    ffb_host_pool* pool = ffb_host_pool_create(threads);
    for (int rep = 0; rep < 60; ++rep) {
      const int n_cols = rep % 3 == 0 ? 1 + (int)(rng() % 300) : 1000 + (int)(rng() % 4000);
      const int rows = 1 + (int)(rng() % 40);
      const int shift = (int)(rng() % 16);  // destination offset in words from a 64-byte boundary
      // one-word pairs (column | count << 16) on half the cases
      const bool narrow = rep % 4 >= 2;
      const size_t words = narrow ? 1 : 2;
      std::vector<uint32_t> first(rows), count(rows), pairs;
      std::vector<uint32_t> want((size_t)rows * n_cols, 0u);
      for (int r = 0; r < rows; ++r) {
        first[r] = (uint32_t)(pairs.size() / words);
        const int kind = (int)(rng() % 4);  // empty, sparse, dense, full
        const double p = kind == 0 ? 0.0 : kind == 1 ? 0.02 : kind == 2 ? 0.5 : 1.0;
        std::bernoulli_distribution take(p);
        for (int c = 0; c < n_cols; ++c)
          if (take(rng)) {
            const uint32_t v = 1u + (uint32_t)(rng() % (narrow ? 0xFFFFull : 0xFFFFFFFEull));
            if (narrow) {
              pairs.push_back((uint32_t)c | (v << 16));
            } else {
              pairs.push_back((uint32_t)c);
              pairs.push_back(v);
            }
            want[(size_t)r * n_cols + c] = v;
          }
        count[r] = (uint32_t)(pairs.size() / words) - first[r];
      }
      // the normalised form on every other case: one factor per row, among
      // them the non-finite and negative ones (zeros become NaN or -0)
      const bool norm = rep % 2 == 1;
      std::vector<float> inv(rows);
      if (norm) {
        for (int r = 0; r < rows; ++r) {
          const int pick = (int)(rng() % 8);
          const int32_t outgoing = pick == 0 ? 0 : pick == 1 ? -3 : 1 + (int32_t)(rng() % 100000);
          inv[r] = 1.f / (float)outgoing;
          for (int c = 0; c < n_cols; ++c) {
            const float v = (float)want[(size_t)r * n_cols + c] * inv[r];
            std::memcpy(&want[(size_t)r * n_cols + c], &v, sizeof v);
          }
        }
      }
      std::vector<uint32_t> mem((size_t)rows * n_cols + 64, 0xDEADBEEFu);
      uint32_t* base = mem.data();
      while ((uintptr_t)base & 63u)
        ++base;
      uint32_t* dst = base + shift;
      if (norm)
        ffb_host_expand_norm_start(pool, reinterpret_cast<float*>(dst), rows, n_cols, first.data(), count.data(),
                                   pairs.data(), narrow, inv.data());
      else
        ffb_host_expand_start(pool, dst, rows, n_cols, first.data(), count.data(), pairs.data(), narrow);
      ffb_host_expand_join(pool);
      for (size_t i = 0; i < want.size(); ++i)
        if (dst[i] != want[i]) {
          std::printf("FAIL threads=%d n_cols=%d rows=%d shift=%d entry %zu: %u != %u\n", threads, n_cols, rows,
                      shift, i, dst[i], want[i]);
          return 1;
        }
      // nothing outside the rows is written
      for (uint32_t* q = mem.data(); q < dst; ++q)
        if (*q != 0xDEADBEEFu) {
          std::printf("FAIL: write before the destination\n");
          return 1;
        }
      for (uint32_t* q = dst + want.size(); q < mem.data() + mem.size(); ++q)
        if (*q != 0xDEADBEEFu) {
          std::printf("FAIL: write after the destination\n");
          return 1;
        }
      ++cases;
    }
    ffb_host_pool_destroy(pool);
  }
  std::printf("OK %d cases\n", cases);
  return 0;
}
