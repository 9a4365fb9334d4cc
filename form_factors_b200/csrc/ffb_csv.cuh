// ffb_csv.cuh -- the form-factor matrix as the reference's CSV text
// (csv_export::export_csv, import_export/csv_export.cpp:26-46): row i holds
// the n entries of matrix row i, each written by `std::ostream << float`,
// separated by ';' and ended by '\n' (std::endl).  `ostream << float` prints
// the value widened to double with "%g" at precision 6: six significant
// digits of the exact binary value, rounded to nearest with ties to even,
// trailing zeros (and a bare decimal point) removed, exponent form when the
// decimal exponent is below -4 or at least 6.
//
// The conversion below is exact integer arithmetic on the float's mantissa
// and exponent: a 64-bit path for values in [2^-36, 2^24) (every form factor
// count / outgoing with outgoing < 2^31 lands there) and a multi-word path
// for the rest of the finite floats.
#pragma once

#include <stdint.h>

#ifndef __CUDACC__
#ifndef __host__
#define __host__
#endif
#ifndef __device__
#define __device__
#endif
#endif

namespace ffb {
namespace csv {

constexpr int kMaxEntry = 16;  // longest entry with its separator is 13 bytes ("-1.17549e-38;")

// Value m * 2^q (m > 0, m < 2^24) rounded to six significant digits:
// value ~= digits * 10^(exp10 - 5), digits in [100000, 999999].
struct Dec6 {
  uint32_t digits;
  int exp10;
};

__host__ __device__ inline Dec6 round6_from_7(uint64_t n7, bool rest, int exp10)
{
  uint32_t n6 = (uint32_t)(n7 / 10u);
  const uint32_t r = (uint32_t)(n7 % 10u);
  if (r > 5u || (r == 5u && (rest || (n6 & 1u))))
    ++n6;
  if (n6 == 1000000u) {
    n6 = 100000u;
    ++exp10;
  }
  return Dec6{n6, exp10};
}

// Number of decimal digits of v > 0.
__host__ __device__ inline int n_digits(uint64_t v)
{
  int n = 1;
  while (v >= 10u) {
    v /= 10u;
    ++n;
  }
  return n;
}

__host__ __device__ inline uint64_t pow10_u64(int k)
{
  uint64_t p = 1;
  for (int i = 0; i < k; ++i)
    p *= 10u;
  return p;
}

// Fast path: s = -q in [1, 59].  Integer part I = m >> s (< 2^24), fraction
// F / 2^s; fraction digits come from F * 10 (< 2^63).
__host__ __device__ inline Dec6 round6_small(uint32_t m, int s)
{
  const uint64_t mask = (s >= 64) ? ~0ull : ((1ull << s) - 1ull);
  const uint64_t I = s >= 32 ? 0ull : (uint64_t)(m >> s);
  uint64_t F = (uint64_t)m & mask;
  uint64_t n7 = 0;
  int got = 0, exp10;
  if (I > 0) {
    const int nI = n_digits(I);
    exp10 = nI - 1;
    if (nI >= 7) {
      const uint64_t p = pow10_u64(nI - 7);
      return round6_from_7(I / p, (I % p) != 0 || F != 0, exp10);
    }
    n7 = I;
    got = nI;
  } else {
    // leading zeros after the point
    exp10 = -1;
    for (;;) {
      F *= 10u;
      const uint64_t d = F >> s;
      F &= mask;
      if (d) {
        n7 = d;
        got = 1;
        break;
      }
      --exp10;
    }
  }
  while (got < 7) {
    F *= 10u;
    n7 = n7 * 10u + (F >> s);
    F &= mask;
    ++got;
  }
  return round6_from_7(n7, F != 0, exp10);
}

// General path: any finite positive value m * 2^q, with 32-bit limbs
// (little endian).  Integer part m << q has at most 128 bits; a fraction
// F / 2^s has s <= 149 bits and grows by 4 bits per digit.
constexpr int kLimbs = 6;

__host__ __device__ inline bool big_zero(const uint32_t* a)
{
  uint32_t o = 0;
  for (int i = 0; i < kLimbs; ++i)
    o |= a[i];
  return o == 0;
}

// a /= 10, returns the remainder
__host__ __device__ inline uint32_t big_div10(uint32_t* a)
{
  uint64_t r = 0;
  for (int i = kLimbs - 1; i >= 0; --i) {
    const uint64_t cur = (r << 32) | a[i];
    a[i] = (uint32_t)(cur / 10u);
    r = cur % 10u;
  }
  return (uint32_t)r;
}

// a *= 10, then returns and clears the bits at and above bit s
__host__ __device__ inline uint32_t big_mul10_take(uint32_t* a, int s)
{
  uint64_t c = 0;
  for (int i = 0; i < kLimbs; ++i) {
    const uint64_t cur = (uint64_t)a[i] * 10u + c;
    a[i] = (uint32_t)cur;
    c = cur >> 32;
  }
  // digit = a >> s (below 10), then a &= 2^s - 1.  a < 2^(s+4) after the
  // multiplication, so the digit's bits lie in limbs w and (for b > 28) w+1.
  const int w = s >> 5, b = s & 31;
  uint32_t d = a[w] >> b;
  if (b > 28 && w + 1 < kLimbs) {
    d |= a[w + 1] << (32 - b);
    a[w + 1] = 0;
  }
  a[w] &= b ? ((1u << b) - 1u) : 0u;
  return d;
}

__host__ __device__ inline Dec6 round6_general(uint32_t m, int q)
{
  uint32_t a[kLimbs];
  for (int i = 0; i < kLimbs; ++i)
    a[i] = 0;
  if (q >= 0) {
    // integer: m << q (q <= 104), decimal digits by repeated division
    const int w = q >> 5, b = q & 31;
    a[w] = m << b;
    if (b && w + 1 < kLimbs)
      a[w + 1] = m >> (32 - b);
    uint8_t dig[40];
    int n = 0;
    while (!big_zero(a))
      dig[n++] = (uint8_t)big_div10(a);
    // dig[n-1] is the leading digit
    uint64_t n7 = 0;
    const int take = n < 7 ? n : 7;
    for (int i = 0; i < take; ++i)
      n7 = n7 * 10u + dig[n - 1 - i];
    for (int i = take; i < 7; ++i)
      n7 *= 10u;
    bool rest = false;
    for (int i = 0; i < n - 7; ++i)
      rest |= dig[i] != 0;
    return round6_from_7(n7, rest, n - 1);
  }
  // pure fraction (s >= 60, so m >> s == 0): digits of m / 2^s
  const int s = -q;
  a[0] = m;
  int exp10 = -1;
  uint32_t d;
  for (;;) {
    d = big_mul10_take(a, s);
    if (d)
      break;
    --exp10;
  }
  uint64_t n7 = d;
  for (int i = 1; i < 7; ++i)
    n7 = n7 * 10u + big_mul10_take(a, s);
  return round6_from_7(n7, !big_zero(a), exp10);
}

__host__ __device__ inline int put_text(char* out, const char* t)
{
  int n = 0;
  while (t[n]) {
    out[n] = t[n];
    ++n;
  }
  return n;
}

// Writes "%g" of f (precision 6) to out (no terminator); returns the length
// (at most 12).
__host__ __device__ inline int format_g6(float f, char* out)
{
  uint32_t bits;
#ifdef __CUDA_ARCH__
  bits = __float_as_uint(f);
#else
  __builtin_memcpy(&bits, &f, 4);
#endif
  const bool neg = bits >> 31;
  const uint32_t ex = (bits >> 23) & 0xFFu, fr = bits & 0x7FFFFFu;
  int n = 0;
  if (ex == 0xFFu)
    return put_text(out, fr ? (neg ? "-nan" : "nan") : (neg ? "-inf" : "inf"));
  if (neg)
    out[n++] = '-';
  if (ex == 0 && fr == 0) {
    out[n++] = '0';
    return n;
  }
  const uint32_t m = ex ? (fr | 0x800000u) : fr;
  const int q = ex ? (int)ex - 150 : -149;
  const Dec6 d = (q < 0 && q >= -59) ? round6_small(m, -q) : round6_general(m, q);
  char dg[6];
  uint32_t v = d.digits;
  for (int i = 5; i >= 0; --i) {
    dg[i] = (char)('0' + v % 10u);
    v /= 10u;
  }
  int last = 5;  // last significant digit kept after stripping trailing zeros
  while (last > 0 && dg[last] == '0')
    --last;
  const int X = d.exp10;
  if (X < -4 || X >= 6) {
    out[n++] = dg[0];
    if (last > 0) {
      out[n++] = '.';
      for (int i = 1; i <= last; ++i)
        out[n++] = dg[i];
    }
    out[n++] = 'e';
    out[n++] = X < 0 ? '-' : '+';
    const int ax = X < 0 ? -X : X;
    if (ax >= 100)
      out[n++] = (char)('0' + ax / 100);
    out[n++] = (char)('0' + (ax / 10) % 10);
    out[n++] = (char)('0' + ax % 10);
    return n;
  }
  if (X >= 0) {
    for (int i = 0; i <= X; ++i)
      out[n++] = dg[i];
    if (last > X) {
      out[n++] = '.';
      for (int i = X + 1; i <= last; ++i)
        out[n++] = dg[i];
    }
    return n;
  }
  out[n++] = '0';
  out[n++] = '.';
  for (int i = 0; i < -X - 1; ++i)
    out[n++] = '0';
  for (int i = 0; i <= last; ++i)
    out[n++] = dg[i];
  return n;
}

#ifdef __CUDACC__
// ---------------------------------------------------------------------------
// Kernels.  The matrix is processed in segments of consecutive entries
// (row-major); a segment is cut into tiles of kTile entries, one block each.
//  1. k_csv_len: the text length of every tile (entries + separators).
//  2. k_csv_scan: exclusive prefix sums of the tile lengths (64-bit) and the
//     segment's total.
//  3. k_csv_write: each block formats its tile again into shared memory at
//     its block-local offsets (a block-wide scan of the entry lengths), then
//     copies the tile's text to its global offset with 16-byte stores.  The
//     shared buffer starts at the destination's offset modulo 16, so shared
//     and global addresses line up for the vector copy; only the ragged head
//     and tail go byte by byte.
// Reads: the 4-byte entry twice (plus the row's outgoing count); writes: the
// text once.
// ---------------------------------------------------------------------------
constexpr int kThreads = 256;
constexpr int kPerThread = 16;
constexpr int kTile = kThreads * kPerThread;            // entries per block
constexpr int kTileBytes = kTile * (kMaxEntry - 3) + 16;  // 13 bytes per entry at most, + alignment shift

// Entries [e0, e0 + n_entries) of an n x n matrix: floats, or counts
// normalised by their row's outgoing rays as ffb_normalise does
// ((float)count * (1.f / (float)outgoing[row]), cpu_system.cpp:193-195).
struct Source {
  const float* __restrict__ ff;
  const uint32_t* __restrict__ counts;
  const int32_t* __restrict__ outgoing;
  int n;
  long long e0, n_entries;
};

__device__ __forceinline__ float entry_value(const Source& s, long long e, int row)
{
  if (s.ff)
    return __ldg(s.ff + e);
  const float ratio = 1.f / (float)__ldg(s.outgoing + row);
  return (float)__ldg(s.counts + e) * ratio;
}

__global__ void __launch_bounds__(kThreads) k_csv_len(Source s, unsigned long long* __restrict__ tile_len)
{
  __shared__ uint32_t warp_sum[kThreads / 32];
  const long long t0 = (long long)blockIdx.x * kTile;
  const long long g0 = s.e0 + t0;
  const int r0 = (int)(g0 / s.n), c0 = (int)(g0 - (long long)r0 * s.n);
  uint32_t sum = 0;
  char buf[kMaxEntry];
  for (int k = 0; k < kPerThread; ++k) {
    const int o = k * kThreads + (int)threadIdx.x;
    if (t0 + o < s.n_entries) {
      const int row = r0 + (c0 + o) / s.n;
      sum += (uint32_t)format_g6(entry_value(s, g0 + o, row), buf) + 1u;
    }
  }
  for (int off = 16; off > 0; off >>= 1)
    sum += __shfl_xor_sync(0xFFFFFFFFu, sum, off);
  if ((threadIdx.x & 31) == 0)
    warp_sum[threadIdx.x >> 5] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (int w = 0; w < kThreads / 32; ++w)
      t += warp_sum[w];
    tile_len[blockIdx.x] = t;
  }
}

// Exclusive scan of n tile lengths (one block; each thread a contiguous run)
// into out[0..n), and the total into out[n].
constexpr int kScanThreads = 1024;
__global__ void __launch_bounds__(kScanThreads) k_csv_scan(const unsigned long long* __restrict__ in, int n,
                                                           unsigned long long* __restrict__ out)
{
  __shared__ unsigned long long warp_sum[kScanThreads / 32];
  const int per = (n + kScanThreads - 1) / kScanThreads;
  const int b = (int)threadIdx.x * per, e = min(n, b + per);
  unsigned long long s = 0;
  for (int i = b; i < e; ++i)
    s += in[i];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned long long incl = s;
  for (int off = 1; off < 32; off <<= 1) {
    const unsigned long long y = __shfl_up_sync(0xFFFFFFFFu, incl, off);
    if (lane >= off)
      incl += y;
  }
  if (lane == 31)
    warp_sum[warp] = incl;
  __syncthreads();
  unsigned long long before = 0;
  for (int w = 0; w < warp; ++w)
    before += warp_sum[w];
  unsigned long long run = before + incl - s;
  for (int i = b; i < e; ++i) {
    out[i] = run;
    run += in[i];
  }
  if (threadIdx.x == kScanThreads - 1)
    out[n] = run;
}

__global__ void __launch_bounds__(kThreads) k_csv_write(Source s, const unsigned long long* __restrict__ tile_off,
                                                        char* __restrict__ text)
{
  extern __shared__ __align__(16) unsigned char sbuf[];
  __shared__ uint32_t warp_sum[kThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long t0 = (long long)blockIdx.x * kTile;
  const long long g0 = s.e0 + t0;
  const int r0 = (int)(g0 / s.n), c0 = (int)(g0 - (long long)r0 * s.n);
  char* dst = text + tile_off[blockIdx.x];
  const uint32_t shift = (uint32_t)((uintptr_t)dst & 15u);
  uint32_t run = shift;  // next free byte of sbuf
  char buf[kMaxEntry];
  for (int k = 0; k < kPerThread; ++k) {
    const int o = k * kThreads + (int)threadIdx.x;
    uint32_t len = 0;
    if (t0 + o < s.n_entries) {
      const int cc = c0 + o;
      const int row = r0 + cc / s.n, col = cc % s.n;
      len = (uint32_t)format_g6(entry_value(s, g0 + o, row), buf);
      buf[len++] = col == s.n - 1 ? '\n' : ';';
    }
    uint32_t incl = len;
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, off);
      if (lane >= off)
        incl += y;
    }
    if (lane == 31)
      warp_sum[warp] = incl;
    __syncthreads();
    uint32_t before = 0, total = 0;
    for (int w = 0; w < kThreads / 32; ++w) {
      const uint32_t u = warp_sum[w];
      before += w < warp ? u : 0u;
      total += u;
    }
    const uint32_t pos = run + before + incl - len;
    for (uint32_t i = 0; i < len; ++i)
      sbuf[pos + i] = (unsigned char)buf[i];
    run += total;
    __syncthreads();
  }
  // copy [shift, run) of sbuf to dst: ragged head, 16-byte body, ragged tail
  const uint32_t L = run - shift;
  const uint32_t head = min(L, (16u - shift) & 15u);
  const uint32_t body = (L - head) >> 4;
  for (uint32_t i = threadIdx.x; i < head; i += kThreads)
    dst[i] = (char)sbuf[shift + i];
  const uint4* sv = reinterpret_cast<const uint4*>(sbuf + shift + head);
  uint4* dv = reinterpret_cast<uint4*>(dst + head);
  for (uint32_t i = threadIdx.x; i < body; i += kThreads)
    dv[i] = sv[i];
  for (uint32_t i = head + 16u * body + threadIdx.x; i < L; i += kThreads)
    dst[i] = (char)sbuf[shift + i];
}
#endif  // __CUDACC__

}  // namespace csv
}  // namespace ffb
