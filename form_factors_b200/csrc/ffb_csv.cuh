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

// Text sinks of the formatter: a pointer (host buffers, shared memory) or a
// counter (lengths only; the compiler drops the character work).
struct PtrOut {
  char* p;
  int n;
  __host__ __device__ void put(char c) { p[n++] = c; }
};
struct CountOut {
  int n;
  __host__ __device__ void put(char) { ++n; }
};

template <class Out>
__host__ __device__ inline void put_text(Out& out, const char* t)
{
  for (int i = 0; t[i]; ++i)
    out.put(t[i]);
}

// Appends "%g" of f (precision 6) to out: at most 12 characters.
template <class Out>
__host__ __device__ inline void format_g6_to(float f, Out& out)
{
  uint32_t bits;
#ifdef __CUDA_ARCH__
  bits = __float_as_uint(f);
#else
  __builtin_memcpy(&bits, &f, 4);
#endif
  const bool neg = bits >> 31;
  const uint32_t ex = (bits >> 23) & 0xFFu, fr = bits & 0x7FFFFFu;
  if (ex == 0xFFu) {
    put_text(out, fr ? (neg ? "-nan" : "nan") : (neg ? "-inf" : "inf"));
    return;
  }
  if (neg)
    out.put('-');
  if (ex == 0 && fr == 0) {
    out.put('0');
    return;
  }
  const uint32_t m = ex ? (fr | 0x800000u) : fr;
  const int q = ex ? (int)ex - 150 : -149;
  const Dec6 d = (q < 0 && q >= -59) ? round6_small(m, -q) : round6_general(m, q);
  // digits of d.digits, most significant first, without trailing zeros
  uint32_t v = d.digits;
  int last = 5;
  while (last > 0 && v % 10u == 0u) {
    v /= 10u;
    --last;
  }
  // v now holds digits 0..last; divisor picks them from the top
  uint32_t div = 1;
  for (int i = 0; i < last; ++i)
    div *= 10u;
  const int X = d.exp10;
  auto next_digit = [&]() {
    const uint32_t dg = v / div;
    v -= dg * div;
    div /= 10u;
    return (char)('0' + dg);
  };
  if (X < -4 || X >= 6) {
    out.put(next_digit());
    if (last > 0) {
      out.put('.');
      for (int i = 1; i <= last; ++i)
        out.put(next_digit());
    }
    out.put('e');
    out.put(X < 0 ? '-' : '+');
    const int ax = X < 0 ? -X : X;
    if (ax >= 100)
      out.put((char)('0' + ax / 100));
    out.put((char)('0' + (ax / 10) % 10));
    out.put((char)('0' + ax % 10));
    return;
  }
  if (X >= 0) {
    // integer digits 0..X (digits past `last` are zeros)
    for (int i = 0; i <= X; ++i)
      out.put(i <= last ? next_digit() : '0');
    if (last > X) {
      out.put('.');
      for (int i = X + 1; i <= last; ++i)
        out.put(next_digit());
    }
    return;
  }
  out.put('0');
  out.put('.');
  for (int i = 0; i < -X - 1; ++i)
    out.put('0');
  for (int i = 0; i <= last; ++i)
    out.put(next_digit());
}

// Writes "%g" of f to out (no terminator); returns the length.
__host__ __device__ inline int format_g6(float f, char* out)
{
  PtrOut o{out, 0};
  format_g6_to(f, o);
  return o.n;
}

__host__ __device__ inline int format_g6_len(float f)
{
  CountOut o{0};
  format_g6_to(f, o);
  return o.n;
}

#ifdef __CUDACC__
// ---------------------------------------------------------------------------
// Kernels.  The matrix (row-major entries) is cut into tiles of kTile
// entries, one block each.  A device buffer gets its text from k_csv_fused
// (one pass, below); lengths, host buffers and files use:
//  1. k_csv_len: the text length of every tile.
//  2. k_csv_scan: exclusive prefix sums of the tile lengths (64-bit) and the
//     total.
//  3. k_csv_write: each block lays its tile's text out in shared memory and
//     copies it to its global offset with 16-byte stores (the shared buffer
//     starts at the destination's offset modulo 16, so both sides line up;
//     only the ragged head and tail go byte by byte).
// In both passes an entry that is +0 costs a load and a compare ("0" plus
// separator); the other entries go to a per-block queue and are formatted by
// all threads together, so that a sparse matrix does not leave warps running
// the formatter with one lane.  Per-entry offsets come from a block scan of
// the entry lengths (16-bit: a tile's text is below 64 KB).
// ---------------------------------------------------------------------------
constexpr int kThreads = 256;
constexpr int kPerThread = 16;
constexpr int kTile = kThreads * kPerThread;            // entries per block
constexpr int kTileBytes = kTile * (kMaxEntry - 3) + 16;  // 13 bytes per entry at most, + alignment shift
constexpr size_t kIndexSmem = 2 * sizeof(uint16_t) * kTile;  // offsets + queue of k_csv_write
// Dynamic shared memory of k_csv_write for tiles of at most max_tile bytes.
__host__ __device__ inline size_t write_smem(unsigned long long max_tile)
{
  return (size_t)((max_tile + 16u + 15u) & ~15ull) + kIndexSmem;
}

// The n x n matrix: floats, or counts normalised by their row's outgoing
// rays as ffb_normalise does ((float)count * (1.f / (float)outgoing[row]),
// cpu_system.cpp:193-195).
struct Source {
  const float* __restrict__ ff;
  const uint32_t* __restrict__ counts;
  const int32_t* __restrict__ outgoing;
  int n;
  long long n_entries;
};

__device__ __forceinline__ float row_ratio(const Source& s, int row)
{
  return s.ff ? 1.f : 1.f / (float)__ldg(s.outgoing + row);
}

__device__ __forceinline__ float entry_value(const Source& s, long long e, float ratio)
{
  return s.ff ? __ldg(s.ff + e) : (float)__ldg(s.counts + e) * ratio;
}

// A thread's entries o = k * kThreads + tid of one tile, held in registers
// for both walks of a kernel: the 16 loads are issued together.
struct TileRegs {
  float v[kPerThread];
  int col0;  // column of the first entry
};

__device__ __forceinline__ void load_tile(const Source& s, long long tile, TileRegs& r)
{
  const long long e0 = tile * kTile + threadIdx.x;
  uint32_t raw[kPerThread];
#pragma unroll
  for (int k = 0; k < kPerThread; ++k) {
    const long long e = e0 + (long long)k * kThreads;
    raw[k] = 0u;
    if (e < s.n_entries)
      raw[k] = s.ff ? __float_as_uint(__ldg(s.ff + e)) : __ldg(s.counts + e);
  }
  int row = (int)(e0 / s.n), col = (int)(e0 - (long long)row * s.n);
  r.col0 = col;
  float ratio = (!s.ff && row < s.n) ? row_ratio(s, row) : 1.f;
#pragma unroll
  for (int k = 0; k < kPerThread; ++k) {
    r.v[k] = s.ff ? __uint_as_float(raw[k]) : (float)raw[k] * ratio;
    col += kThreads;
    if (col >= s.n) {
      while (col >= s.n) {
        col -= s.n;
        ++row;
      }
      if (!s.ff && row < s.n)
        ratio = row_ratio(s, row);
    }
  }
}

// fn(o, valid, value, col) for the thread's entries; it runs on every lane
// of the warp each step (callers use warp votes); entries past the matrix end
// come with valid = false.
template <class Fn>
__device__ __forceinline__ void walk_tile(const Source& s, long long tile, const TileRegs& r, Fn fn)
{
  int col = r.col0;
#pragma unroll
  for (int k = 0; k < kPerThread; ++k) {
    const int o = k * kThreads + (int)threadIdx.x;
    fn(o, tile * kTile + o < s.n_entries, r.v[k], col);
    col += kThreads;
    while (col >= s.n)
      col -= s.n;
  }
}

// Value and column of entry o of the tile (queue work, one division).
__device__ __forceinline__ float tile_value(const Source& s, long long tile, int o, int* col)
{
  const long long e = tile * kTile + o;
  const int row = (int)(e / s.n);
  *col = (int)(e - (long long)row * s.n);
  return entry_value(s, e, row_ratio(s, row));
}

__device__ __forceinline__ void enqueue(uint16_t* queue, uint32_t* qn, bool take, int o)
{
  const unsigned mask = __ballot_sync(0xFFFFFFFFu, take);
  if (!mask)
    return;
  const int lane = threadIdx.x & 31;
  uint32_t base = 0;
  if (lane == __ffs(mask) - 1)
    base = atomicAdd(qn, (uint32_t)__popc(mask));
  base = __shfl_sync(0xFFFFFFFFu, base, __ffs(mask) - 1);
  if (take)
    queue[base + __popc(mask & ((1u << lane) - 1u))] = (uint16_t)o;
}

__global__ void __launch_bounds__(kThreads, 4) k_csv_len(Source s, unsigned long long* __restrict__ tile_len)
{
  __shared__ uint16_t queue[kTile];
  __shared__ uint32_t qn;
  __shared__ uint32_t warp_sum[kThreads / 32];
  if (threadIdx.x == 0)
    qn = 0;
  __syncthreads();
  uint32_t sum = 0;
  TileRegs r;
  load_tile(s, blockIdx.x, r);
  walk_tile(s, blockIdx.x, r, [&](int o, bool valid, float v, int) {
    const bool zero = __float_as_uint(v) == 0u;
    sum += valid && zero ? 2u : 0u;
    enqueue(queue, &qn, valid && !zero, o);
  });
  __syncthreads();
  const uint32_t n_q = qn;
  for (uint32_t q = threadIdx.x; q < n_q; q += kThreads) {
    int col;
    sum += (uint32_t)format_g6_len(tile_value(s, blockIdx.x, queue[q], &col)) + 1u;
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
// into out[0..n), the total into out[n] and the longest tile into out[n + 1].
constexpr int kScanThreads = 1024;
__global__ void __launch_bounds__(kScanThreads) k_csv_scan(const unsigned long long* __restrict__ in, int n,
                                                           unsigned long long* __restrict__ out)
{
  __shared__ unsigned long long warp_sum[kScanThreads / 32];
  __shared__ unsigned long long warp_max[kScanThreads / 32];
  const int per = (n + kScanThreads - 1) / kScanThreads;
  const int b = (int)threadIdx.x * per, e = min(n, b + per);
  unsigned long long s = 0, mx = 0;
  for (int i = b; i < e; ++i) {
    const unsigned long long x = in[i];
    s += x;
    mx = x > mx ? x : mx;
  }
  for (int off = 16; off > 0; off >>= 1) {
    const unsigned long long y = __shfl_xor_sync(0xFFFFFFFFu, mx, off);
    mx = y > mx ? y : mx;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned long long incl = s;
  for (int off = 1; off < 32; off <<= 1) {
    const unsigned long long y = __shfl_up_sync(0xFFFFFFFFu, incl, off);
    if (lane >= off)
      incl += y;
  }
  if (lane == 31)
    warp_sum[warp] = incl;
  if (lane == 0)
    warp_max[warp] = mx;
  __syncthreads();
  unsigned long long before = 0;
  for (int w = 0; w < warp; ++w)
    before += warp_sum[w];
  unsigned long long run = before + incl - s;
  for (int i = b; i < e; ++i) {
    out[i] = run;
    run += in[i];
  }
  if (threadIdx.x == kScanThreads - 1) {
    out[n] = run;
    unsigned long long m = 0;
    for (int w = 0; w < kScanThreads / 32; ++w)
      m = warp_max[w] > m ? warp_max[w] : m;
    out[n + 1] = m;
  }
}

// Writes tiles tile0 + blockIdx.x; their text goes to text + (tile_off[t] -
// base).  The dynamic shared memory is write_smem(longest tile): the text
// region first (text_region bytes), then offsets and queue.
__global__ void __launch_bounds__(kThreads, 4) k_csv_write(Source s, const unsigned long long* __restrict__ tile_off,
                                                        long long tile0, unsigned long long base, uint32_t text_region,
                                                        char* __restrict__ text)
{
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned char* sbuf = smem;                                         // text_region bytes
  uint16_t* off = reinterpret_cast<uint16_t*>(smem + text_region);    // per entry: length, then offset
  uint16_t* queue = off + kTile;
  __shared__ uint32_t qn;
  __shared__ uint32_t warp_sum[kThreads / 32];
  const long long tile = tile0 + blockIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0)
    qn = 0;
  for (int o = threadIdx.x; o < kTile; o += kThreads)
    off[o] = 0;  // entries past the matrix end
  __syncthreads();
  // 1. lengths: zeros directly, the others through the queue
  TileRegs r;
  load_tile(s, tile, r);
  walk_tile(s, tile, r, [&](int o, bool valid, float v, int) {
    const bool zero = __float_as_uint(v) == 0u;
    if (valid && zero)
      off[o] = 2;
    enqueue(queue, &qn, valid && !zero, o);
  });
  __syncthreads();
  const uint32_t n_q = qn;
  for (uint32_t q = threadIdx.x; q < n_q; q += kThreads) {
    const int o = queue[q];
    int col;
    off[o] = (uint16_t)(format_g6_len(tile_value(s, tile, o, &col)) + 1);
  }
  __syncthreads();
  // 2. offsets: thread t scans entries [16t, 16t + 16)
  char* dst = text + (tile_off[tile] - base);
  const uint32_t shift = (uint32_t)((uintptr_t)dst & 15u);
  uint32_t mine = 0;
  for (int i = 0; i < kPerThread; ++i)
    mine += off[threadIdx.x * kPerThread + i];
  uint32_t incl = mine;
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
    if (lane >= d)
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
  uint32_t run = shift + before + incl - mine;
  for (int i = 0; i < kPerThread; ++i) {
    const int o = threadIdx.x * kPerThread + i;
    const uint32_t len = off[o];
    off[o] = (uint16_t)run;  // below 64 KB
    run += len;
  }
  __syncthreads();
  // 3. text: zeros, then the queued entries
  walk_tile(s, tile, r, [&](int o, bool valid, float v, int col) {
    if (valid && __float_as_uint(v) == 0u) {
      sbuf[off[o]] = '0';
      sbuf[off[o] + 1] = col == s.n - 1 ? '\n' : ';';
    }
  });
  for (uint32_t q = threadIdx.x; q < n_q; q += kThreads) {
    const int o = queue[q];
    int col;
    const float v = tile_value(s, tile, o, &col);
    PtrOut w{reinterpret_cast<char*>(sbuf + off[o]), 0};
    format_g6_to(v, w);
    w.put(col == s.n - 1 ? '\n' : ';');
  }
  __syncthreads();
  // 4. copy [shift, shift + total) of sbuf to dst
  const uint32_t L = total;
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

// ---------------------------------------------------------------------------
// Single pass into a device buffer (decoupled look-back).  Each block takes
// the next tile by ticket, so every tile it waits for already runs and waits
// only for earlier tiles.  Thread t holds entries [16t, 16t + 16) of its
// tile, so its text is one contiguous run whose offset comes from a block
// scan of 16-entry sums; +0 entries ("0" and the separator) are written by
// their thread, the others formatted densely through the block queue (once
// for the length, once for the text).  The tile publishes its length and
// lays its text out in shared memory; then it sums the lengths and prefixes
// the preceding tiles published (bounded polls), publishes its inclusive
// prefix and stores its text with 16-byte writes.  A tile whose text would
// pass the end of the buffer writes nothing and sets kFusedOverflow; the
// last tile writes the text length.
// ---------------------------------------------------------------------------
constexpr unsigned long long kTileAgg = 1ull << 62;     // status: the tile's own length
constexpr unsigned long long kTilePrefix = 2ull << 62;  // status: the inclusive prefix
constexpr unsigned long long kTileValue = (1ull << 62) - 1;
constexpr unsigned kLookbackPolls = 1u << 22;           // polls of one status word before giving up
enum : unsigned { kFusedTimeout = 1u, kFusedOverflow = 2u };
constexpr int kRun = 16;  // consecutive entries per thread
#ifndef FFB_CSV_THREADS
#define FFB_CSV_THREADS 256
#endif
#ifndef FFB_CSV_BLOCKS
#define FFB_CSV_BLOCKS 3
#endif
constexpr int kFusedThreads = FFB_CSV_THREADS;
constexpr int kFusedTile = kRun * kFusedThreads;              // entries per tile, one run per thread
constexpr int kFusedText = kFusedTile * (kMaxEntry - 3) + 16;  // staged text of a tile at most, + one word read past it
static_assert(kFusedText % 16 == 0, "the length bytes start 16-byte aligned");
constexpr size_t kFusedSmem =
    kFusedText + kFusedTile * (sizeof(uint8_t) + sizeof(uint16_t)) + kFusedThreads * sizeof(uint32_t);

struct FusedSink {
  char* text;
  unsigned long long cap;
  unsigned long long* status;  // one word per tile, zero before the launch
  unsigned int* ticket;        // zero before the launch
  unsigned int* err;           // kFused* bits, zero before the launch
  unsigned long long* total;   // the text length, written by the last tile
  long long n_tiles;
};

__device__ __forceinline__ unsigned long long ld_relaxed(const unsigned long long* p)
{
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_relaxed(unsigned long long* p, unsigned long long v)
{
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Exclusive prefix of `tile` from the status words of the tiles before it;
// run by one full warp after the tile's own length was published.
__device__ __forceinline__ unsigned long long look_back(const FusedSink& out, long long tile, int lane)
{
  unsigned long long excl = 0;
  for (long long j = tile - 1;; j -= 32) {
    const long long idx = j - lane;
    unsigned long long w = kTilePrefix;  // before the first tile: prefix 0
    if (idx >= 0) {
      unsigned polls = 0;
      do {
        w = ld_relaxed(out.status + idx);
      } while ((w >> 62) == 0 && ++polls < kLookbackPolls);
    }
    if (__any_sync(0xFFFFFFFFu, (w >> 62) == 0)) {  // a tile never published: give up
      if (lane == 0)
        atomicOr(out.err, kFusedTimeout);
      return excl;
    }
    // lane 0 is the nearest tile; stop at the nearest one with a prefix
    const unsigned pm = __ballot_sync(0xFFFFFFFFu, (w >> 62) == 2);
    unsigned long long v = w & kTileValue;
    if (pm && lane > __ffs(pm) - 1)
      v = 0;
    for (int d = 16; d > 0; d >>= 1)
      v += __shfl_xor_sync(0xFFFFFFFFu, v, d);
    excl += v;
    if (pm)
      return excl;
  }
}

// Value and column of entry o of a fused tile (queue work, one division).
__device__ __forceinline__ float fused_value(const Source& s, long long tile, int o, int* col)
{
  const long long e = tile * kFusedTile + o;
  const int row = (int)(e / s.n);
  *col = (int)(e - (long long)row * s.n);
  return entry_value(s, e, row_ratio(s, row));
}

__global__ void __launch_bounds__(kFusedThreads, FFB_CSV_BLOCKS) k_csv_fused(Source s, FusedSink out)
{
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned char* sbuf = smem;                                         // staged text
  uint8_t* len = smem + kFusedText;                                   // entry lengths, run by run
  uint16_t* queue = reinterpret_cast<uint16_t*>(len + kFusedTile);    // nonzero entries
  uint32_t* toff = reinterpret_cast<uint32_t*>(queue + kFusedTile);  // staged offset of each run
  __shared__ uint32_t qn;
  __shared__ long long s_tile;
  __shared__ unsigned long long s_prefix;
  __shared__ uint32_t warp_sum[kFusedThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) {
    qn = 0;
    s_tile = (long long)atomicAdd(out.ticket, 1u);
  }
  __syncthreads();
  const long long tile = s_tile;
  // 1. the run's entries, their +0 / row-end flags and the +0 lengths
  const int o0 = kRun * (int)threadIdx.x;
  const long long e0 = tile * kFusedTile + o0;
  const uint32_t* words = s.ff ? reinterpret_cast<const uint32_t*>(s.ff) : s.counts;
  uint32_t raw[kRun];
  if (e0 + kRun <= s.n_entries && ((uintptr_t)(words + e0) & 15u) == 0) {
    const uint4* p = reinterpret_cast<const uint4*>(words + e0);
#pragma unroll
    for (int j = 0; j < kRun / 4; ++j) {
      const uint4 w = __ldg(p + j);
      raw[4 * j] = w.x;
      raw[4 * j + 1] = w.y;
      raw[4 * j + 2] = w.z;
      raw[4 * j + 3] = w.w;
    }
  } else {
#pragma unroll
    for (int k = 0; k < kRun; ++k)
      raw[k] = e0 + k < s.n_entries ? __ldg(words + e0 + k) : 0u;
  }
  int row = (int)(e0 / s.n), col = (int)(e0 - (long long)row * s.n);
  float ratio = (!s.ff && row < s.n) ? row_ratio(s, row) : 1.f;
  uint32_t zero_mask = 0, end_mask = 0, lens[kRun / 4] = {0u, 0u, 0u, 0u};
#pragma unroll
  for (int k = 0; k < kRun; ++k) {
    const bool valid = e0 + k < s.n_entries;
    const float v = s.ff ? __uint_as_float(raw[k]) : (float)raw[k] * ratio;
    const bool zero = valid && __float_as_uint(v) == 0u;
    zero_mask |= zero ? 1u << k : 0u;
    end_mask |= col == s.n - 1 ? 1u << k : 0u;
    lens[k >> 2] |= zero ? 2u << (8 * (k & 3)) : 0u;
    enqueue(queue, &qn, valid && !zero, o0 + k);
    if (++col == s.n) {
      col = 0;
      ++row;
      if (!s.ff && row < s.n)
        ratio = row_ratio(s, row);
    }
  }
  *reinterpret_cast<uint4*>(len + o0) = make_uint4(lens[0], lens[1], lens[2], lens[3]);
  __syncthreads();
  const uint32_t n_q = qn;
  for (uint32_t q = threadIdx.x; q < n_q; q += kFusedThreads) {
    const int o = queue[q];
    int c;
    len[o] = (uint8_t)(format_g6_len(fused_value(s, tile, o, &c)) + 1);
  }
  __syncthreads();
  // 2. run lengths, the tile's length and each run's offset in the tile
  const uint4 lw = *reinterpret_cast<const uint4*>(len + o0);
  const uint32_t run_len[4] = {lw.x, lw.y, lw.z, lw.w};  // four entry lengths per word
  const uint32_t mine = __dp4a(lw.x, 0x01010101u, __dp4a(lw.y, 0x01010101u, __dp4a(lw.z, 0x01010101u,
                                                                                  __dp4a(lw.w, 0x01010101u, 0u))));
  uint32_t incl = mine;
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
    if (lane >= d)
      incl += y;
  }
  if (lane == 31)
    warp_sum[warp] = incl;
  __syncthreads();
  uint32_t before = 0, total = 0;
  for (int w = 0; w < kFusedThreads / 32; ++w) {
    const uint32_t u = warp_sum[w];
    before += w < warp ? u : 0u;
    total += u;
  }
  // 3. publish the tile's length; its text is staged from offset 0 while
  // the tiles before it finish
  if (threadIdx.x == 0)
    st_relaxed(out.status + tile, (tile == 0 ? kTilePrefix : kTileAgg) | total);
  uint32_t pos = before + incl - mine;
  toff[threadIdx.x] = pos;
  if (zero_mask == 0xFFFFu && (pos & 1u) == 0u) {
    // a run of sixteen +0 entries at an even offset (the common case of a
    // sparse matrix): its 32 bytes "0;0;...0;" as word stores (a halfword at
    // each end when the run starts two bytes into a word), then the
    // newlines of any row ends: 9 or 10 shared stores instead of 32 byte
    // stores at a 32-byte stride, which put eight lanes on one bank
    constexpr uint32_t kZeroSemi = 0x3B303B30u;  // "0;0;" little-endian
    uint32_t p = pos;
    if (p & 2u) {
      *reinterpret_cast<uint16_t*>(sbuf + p) = (uint16_t)kZeroSemi;
      p += 2;
    }
    const uint32_t words = (pos + 32u - p) >> 2;
#pragma unroll 8
    for (uint32_t w = 0; w < words; ++w)
      reinterpret_cast<uint32_t*>(sbuf + p)[w] = kZeroSemi;
    p += 4u * words;
    if (p < pos + 32u)
      *reinterpret_cast<uint16_t*>(sbuf + p) = (uint16_t)kZeroSemi;
    for (uint32_t m = end_mask; m; m &= m - 1u)
      sbuf[pos + 2u * (uint32_t)(__ffs(m) - 1) + 1u] = '\n';
  } else {
#pragma unroll
    for (int k = 0; k < kRun; ++k) {
      if ((zero_mask >> k) & 1u) {
        sbuf[pos] = '0';
        sbuf[pos + 1] = ((end_mask >> k) & 1u) ? '\n' : ';';
      }
      pos += (run_len[k >> 2] >> (8 * (k & 3))) & 0xFFu;
    }
  }
  __syncthreads();
  for (uint32_t q = threadIdx.x; q < n_q; q += kFusedThreads) {
    const int o = queue[q];
    const int t = o / kRun;
    uint32_t at = toff[t];
    for (int j = t * kRun; j < o; ++j)
      at += len[j];
    int c;
    const float v = fused_value(s, tile, o, &c);
    PtrOut w{reinterpret_cast<char*>(sbuf + at), 0};
    format_g6_to(v, w);
    w.put(c == s.n - 1 ? '\n' : ';');
  }
  // 4. the tile's place in the text
  if (warp == 0) {
    unsigned long long excl = 0;
    if (tile > 0) {
      excl = look_back(out, tile, lane);
      if (lane == 0)
        st_relaxed(out.status + tile, kTilePrefix | (excl + total));
    }
    if (lane == 0) {
      s_prefix = excl;
      if (tile == out.n_tiles - 1)
        *out.total = excl + total;
    }
  }
  __syncthreads();
  const unsigned long long P = s_prefix;
  if (P + total > out.cap) {
    if (threadIdx.x == 0)
      atomicOr(out.err, kFusedOverflow);
    return;
  }
  // 5. copy the staged text to text + P: bytes up to the first 16-byte
  // boundary, then 16-byte stores assembled from 32-bit shared words
  // (funnel shifts by the staged offset's misalignment), then the tail
  char* dst = out.text + P;
  const uint32_t head = min(total, (uint32_t)((16u - ((uintptr_t)dst & 15u)) & 15u));
  const uint32_t body = (total - head) >> 4;
  for (uint32_t i = threadIdx.x; i < head; i += kFusedThreads)
    dst[i] = (char)sbuf[i];
  const uint32_t r8 = 8u * (head & 3u);
  const uint32_t* sw = reinterpret_cast<const uint32_t*>(sbuf) + (head >> 2);
  uint4* dv = reinterpret_cast<uint4*>(dst + head);
  for (uint32_t i = threadIdx.x; i < body; i += kFusedThreads) {
    const uint32_t* w = sw + 4 * i;
    const uint32_t a0 = w[0], a1 = w[1], a2 = w[2], a3 = w[3], a4 = w[4];
    dv[i] = make_uint4(__funnelshift_r(a0, a1, r8), __funnelshift_r(a1, a2, r8), __funnelshift_r(a2, a3, r8),
                       __funnelshift_r(a3, a4, r8));
  }
  for (uint32_t i = head + 16u * body + threadIdx.x; i < total; i += kFusedThreads)
    dst[i] = (char)sbuf[i];
}
#endif  // __CUDACC__

}  // namespace csv
}  // namespace ffb
