// ffb_host_rows.cpp -- host threads that write count-matrix rows into a
// caller's host buffer from the (column, count) pairs of their nonzero
// entries (ffb_internal.h).
//
// A form-factor count matrix is mostly zeros (the closed 22 080-face
// enclosure at 1000 rays per face fills 4 % of its entries), so a host
// output is cheaper to move as the pairs of its nonzeros: the device packs
// each finished row block, the pairs cross PCIe, and these threads expand
// them into the dense rows.  A thread writes a row front to back, segment by
// segment, with non-temporal stores (no read-for-ownership of the
// destination lines): the destination is written once, in full, at the
// host's streaming-store bandwidth.
#include <immintrin.h>

#include <algorithm>
#include <cstdlib>
#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <functional>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include "ffb_internal.h"

struct ffb_host_pool {
  std::vector<std::thread> workers;
  std::mutex mu;
  std::condition_variable wake, idle;
  uint64_t generation = 0;
  bool stop = false;
  int busy = 0;  // workers still on the current job
  std::function<void(int, int)> task;  // (task, worker)
  int n_tasks = 0;
  std::atomic<int> next{0};
  std::vector<uint32_t*> seg;  // one zeroed 64-byte aligned scratch segment per worker
  bool avx2 = false;
  bool avx512 = false;
};

namespace {

void worker_main(ffb_host_pool* p, int id)
{
  uint64_t seen = 0;
  for (;;) {
    std::function<void(int, int)> task;
    {
      std::unique_lock<std::mutex> lk(p->mu);
      p->wake.wait(lk, [&] { return p->stop || p->generation != seen; });
      if (p->stop)
        return;
      seen = p->generation;
      task = p->task;
    }
    for (int t = p->next.fetch_add(1); t < p->n_tasks; t = p->next.fetch_add(1))
      task(t, id);
    _mm_sfence();  // the streaming stores are globally visible before the job counts as done
    std::lock_guard<std::mutex> lk(p->mu);
    if (--p->busy == 0)
      p->idle.notify_all();
  }
}

// Row r of the block from its pairs, which come in ascending column order.
// The row is built in segments of kSeg words in a zeroed scratch segment of
// the thread's (16 KB, L1 resident): the segment's few pairs are stored
// into it, the segment is streamed to the destination with non-temporal
// stores, and the stored words are cleared again.  Words before the
// destination's first 32-byte boundary are written with plain stores, so
// the streaming stores are aligned; so is the tail after the last whole
// vector.  With kNorm the row holds floats, count * inv as
// (float)count * inv (one rounding each, the device normalisation's
// operations); its zeros are 0.f * inv, all-zero bits unless inv is not
// finite or negative, which rows take word by word.
constexpr int kSeg = 4096;

inline uint32_t bits_of(float x)
{
  uint32_t u;
  std::memcpy(&u, &x, sizeof u);
  return u;
}

template <bool kNorm>
inline uint32_t entry_bits(uint32_t count, float inv)
{
  return kNorm ? bits_of((float)count * inv) : count;
}

// Pair k of a row: two words (column, count), or with kNarrow one word
// column | count << 16.
template <bool kNarrow>
inline uint32_t pair_col(const uint32_t* pairs, uint32_t k)
{
  return kNarrow ? pairs[k] & 0xFFFFu : pairs[2 * k];
}
template <bool kNarrow>
inline uint32_t pair_val(const uint32_t* pairs, uint32_t k)
{
  return kNarrow ? pairs[k] >> 16 : pairs[2 * k + 1];
}

template <bool kNorm, bool kNarrow>
void expand_row_words(uint32_t* __restrict__ dst, int n_cols, const uint32_t* __restrict__ pairs, uint32_t n, float inv)
{
  const uint32_t zero = entry_bits<kNorm>(0u, inv);
  uint32_t k = 0;
  for (int i = 0; i < n_cols; ++i)
    dst[i] = (k < n && pair_col<kNarrow>(pairs, k) == (uint32_t)i) ? entry_bits<kNorm>(pair_val<kNarrow>(pairs, k++), inv) : zero;
}

template <bool kNorm, bool kNarrow>
void expand_row_sse2(uint32_t* __restrict__ dst, int n_cols, const uint32_t* __restrict__ pairs, uint32_t n,
                     uint32_t* __restrict__ seg, float inv)
{
  if (kNorm && entry_bits<true>(0u, inv) != 0u)
    return expand_row_words<kNorm, kNarrow>(dst, n_cols, pairs, n, inv);
  uint32_t k = 0;
  int head = (int)(((32u - ((uint32_t)(uintptr_t)dst & 31u)) & 31u) >> 2);
  head = std::min(head, n_cols);
  for (int i = 0; i < head; ++i)
    dst[i] = (k < n && pair_col<kNarrow>(pairs, k) == (uint32_t)i) ? entry_bits<kNorm>(pair_val<kNarrow>(pairs, k++), inv) : 0u;
  for (int i0 = head; i0 < n_cols; i0 += kSeg) {
    const int len = std::min(kSeg, n_cols - i0);
    const uint32_t k0 = k;
    while (k < n && pair_col<kNarrow>(pairs, k) < (uint32_t)(i0 + len)) {
      seg[pair_col<kNarrow>(pairs, k) - (uint32_t)i0] = entry_bits<kNorm>(pair_val<kNarrow>(pairs, k), inv);
      ++k;
    }
    uint32_t* d = dst + i0;
    int j = 0;
    for (; j + 8 <= len; j += 8) {
      _mm_stream_si128(reinterpret_cast<__m128i*>(d + j), _mm_load_si128(reinterpret_cast<const __m128i*>(seg + j)));
      _mm_stream_si128(reinterpret_cast<__m128i*>(d + j + 4),
                       _mm_load_si128(reinterpret_cast<const __m128i*>(seg + j + 4)));
    }
    for (; j < len; ++j)
      d[j] = seg[j];
    for (uint32_t q = k0; q < k; ++q)
      seg[pair_col<kNarrow>(pairs, q) - (uint32_t)i0] = 0u;
  }
}

template <bool kNorm, bool kNarrow>
__attribute__((target("avx2"))) void expand_row_avx2(uint32_t* __restrict__ dst, int n_cols,
                                                     const uint32_t* __restrict__ pairs, uint32_t n,
                                                     uint32_t* __restrict__ seg, float inv)
{
  if (kNorm && entry_bits<true>(0u, inv) != 0u)
    return expand_row_words<kNorm, kNarrow>(dst, n_cols, pairs, n, inv);
  uint32_t k = 0;
  int head = (int)(((32u - ((uint32_t)(uintptr_t)dst & 31u)) & 31u) >> 2);
  head = std::min(head, n_cols);
  for (int i = 0; i < head; ++i)
    dst[i] = (k < n && pair_col<kNarrow>(pairs, k) == (uint32_t)i) ? entry_bits<kNorm>(pair_val<kNarrow>(pairs, k++), inv) : 0u;
  for (int i0 = head; i0 < n_cols; i0 += kSeg) {
    const int len = std::min(kSeg, n_cols - i0);
    const uint32_t k0 = k;
    while (k < n && pair_col<kNarrow>(pairs, k) < (uint32_t)(i0 + len)) {
      seg[pair_col<kNarrow>(pairs, k) - (uint32_t)i0] = entry_bits<kNorm>(pair_val<kNarrow>(pairs, k), inv);
      ++k;
    }
    uint32_t* d = dst + i0;
    int j = 0;
    for (; j + 16 <= len; j += 16) {
      _mm256_stream_si256(reinterpret_cast<__m256i*>(d + j),
                          _mm256_load_si256(reinterpret_cast<const __m256i*>(seg + j)));
      _mm256_stream_si256(reinterpret_cast<__m256i*>(d + j + 8),
                          _mm256_load_si256(reinterpret_cast<const __m256i*>(seg + j + 8)));
    }
    for (; j < len; ++j)
      d[j] = seg[j];
    for (uint32_t q = k0; q < k; ++q)
      seg[pair_col<kNarrow>(pairs, q) - (uint32_t)i0] = 0u;
  }
}

template <bool kNorm, bool kNarrow>
__attribute__((target("avx512f"))) void expand_row_avx512(uint32_t* __restrict__ dst, int n_cols,
                                                     const uint32_t* __restrict__ pairs, uint32_t n,
                                                     uint32_t* __restrict__ seg, float inv)
{
  if (kNorm && entry_bits<true>(0u, inv) != 0u)
    return expand_row_words<kNorm, kNarrow>(dst, n_cols, pairs, n, inv);
  uint32_t k = 0;
  int head = (int)(((32u - ((uint32_t)(uintptr_t)dst & 31u)) & 31u) >> 2);
  head = std::min(head, n_cols);
  for (int i = 0; i < head; ++i)
    dst[i] = (k < n && pair_col<kNarrow>(pairs, k) == (uint32_t)i) ? entry_bits<kNorm>(pair_val<kNarrow>(pairs, k++), inv) : 0u;
  for (int i0 = head; i0 < n_cols; i0 += kSeg) {
    const int len = std::min(kSeg, n_cols - i0);
    const uint32_t k0 = k;
    while (k < n && pair_col<kNarrow>(pairs, k) < (uint32_t)(i0 + len)) {
      seg[pair_col<kNarrow>(pairs, k) - (uint32_t)i0] = entry_bits<kNorm>(pair_val<kNarrow>(pairs, k), inv);
      ++k;
    }
    uint32_t* d = dst + i0;
    int j = 0;
    // 64-byte stores from a 32-byte boundary: one 32-byte store first when
    // the destination is not 64-byte aligned
    if (j + 8 <= len && ((uintptr_t)(d + j) & 63u) != 0) {
      _mm256_stream_si256(reinterpret_cast<__m256i*>(d + j),
                          _mm256_load_si256(reinterpret_cast<const __m256i*>(seg + j)));
      j += 8;
    }
    for (; j + 16 <= len; j += 16)
      _mm512_stream_si512(reinterpret_cast<__m512i*>(d + j), _mm512_loadu_si512(seg + j));
    for (; j < len; ++j)
      d[j] = seg[j];
    for (uint32_t q = k0; q < k; ++q)
      seg[pair_col<kNarrow>(pairs, q) - (uint32_t)i0] = 0u;
  }
}

}  // namespace

ffb_host_pool* ffb_host_pool_create(int threads)
{
  ffb_host_pool* p = new (std::nothrow) ffb_host_pool;
  if (!p)
    return nullptr;
  threads = std::max(threads, 1);
  p->avx2 = __builtin_cpu_supports("avx2");
  p->avx512 = p->avx2 && __builtin_cpu_supports("avx512f");
  for (int i = 0; i < threads; ++i) {
    uint32_t* sg = static_cast<uint32_t*>(std::aligned_alloc(64, sizeof(uint32_t) * kSeg));
    if (!sg) {
      ffb_host_pool_destroy(p);
      return nullptr;
    }
    std::memset(sg, 0, sizeof(uint32_t) * kSeg);
    p->seg.push_back(sg);
  }
  try {
    for (int i = 0; i < threads; ++i)
      p->workers.emplace_back(worker_main, p, i);
  } catch (...) {  // no more threads: the threads started so far are stopped
    ffb_host_pool_destroy(p);
    return nullptr;
  }
  return p;
}

void ffb_host_pool_destroy(ffb_host_pool* p)
{
  if (!p)
    return;
  {
    std::lock_guard<std::mutex> lk(p->mu);
    p->stop = true;
  }
  p->wake.notify_all();
  for (std::thread& t : p->workers)
    t.join();
  for (uint32_t* sg : p->seg)
    std::free(sg);
  delete p;
}

int ffb_host_pool_threads(const ffb_host_pool* p) { return p ? (int)p->workers.size() : 0; }

namespace {

// Hands rows [0, rows) to the pool; inv: one factor per row (kNorm), or null.
template <bool kNorm, bool kNarrow>
void expand_start(ffb_host_pool* p, uint32_t* dst, int rows, int n_cols, const uint32_t* first, const uint32_t* count,
                  const uint32_t* pairs, const float* inv)
{
  // tasks of 8 rows: a few hundred KB of destination each
  constexpr int kRowsPerTask = 8;
  constexpr size_t kWords = kNarrow ? 1 : 2;  // words per pair
  std::lock_guard<std::mutex> lk(p->mu);
  p->task = [p, dst, rows, n_cols, first, count, pairs, inv](int t, int w) {
    uint32_t* sg = p->seg[(size_t)w];
    const int r1 = std::min(rows, (t + 1) * kRowsPerTask);
    for (int r = t * kRowsPerTask; r < r1; ++r) {
      // the next row's pairs lie elsewhere (rows reserve their pairs in any
      // order): fetch them into the cache while this row is written
      if (r + 1 < rows) {
        const char* q = reinterpret_cast<const char*>(pairs + kWords * first[r + 1]);
        for (size_t b = 0; b < 4 * kWords * count[r + 1]; b += 64)
          _mm_prefetch(q + b, _MM_HINT_T0);
      }
      uint32_t* d = dst + (size_t)r * (size_t)n_cols;
      const float f = kNorm ? inv[r] : 0.f;
      const uint32_t* pr = pairs + kWords * first[r];
      if (p->avx512)
        expand_row_avx512<kNorm, kNarrow>(d, n_cols, pr, count[r], sg, f);
      else if (p->avx2)
        expand_row_avx2<kNorm, kNarrow>(d, n_cols, pr, count[r], sg, f);
      else
        expand_row_sse2<kNorm, kNarrow>(d, n_cols, pr, count[r], sg, f);
    }
  };
  p->n_tasks = (rows + kRowsPerTask - 1) / kRowsPerTask;
  p->next.store(0);
  p->busy = (int)p->workers.size();
  ++p->generation;
  p->wake.notify_all();
}

}  // namespace

void ffb_host_expand_start(ffb_host_pool* p, uint32_t* dst, int rows, int n_cols, const uint32_t* first,
                           const uint32_t* count, const uint32_t* pairs, int narrow)
{
  if (narrow)
    expand_start<false, true>(p, dst, rows, n_cols, first, count, pairs, nullptr);
  else
    expand_start<false, false>(p, dst, rows, n_cols, first, count, pairs, nullptr);
}

void ffb_host_expand_norm_start(ffb_host_pool* p, float* dst, int rows, int n_cols, const uint32_t* first,
                                const uint32_t* count, const uint32_t* pairs, int narrow, const float* inv)
{
  uint32_t* d = reinterpret_cast<uint32_t*>(dst);
  if (narrow)
    expand_start<true, true>(p, d, rows, n_cols, first, count, pairs, inv);
  else
    expand_start<true, false>(p, d, rows, n_cols, first, count, pairs, inv);
}

void ffb_host_expand_join(ffb_host_pool* p)
{
  std::unique_lock<std::mutex> lk(p->mu);
  p->idle.wait(lk, [&] { return p->busy == 0; });
}
