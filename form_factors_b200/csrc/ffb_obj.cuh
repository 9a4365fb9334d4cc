// ffb_obj.cuh -- Wavefront OBJ geometry parsed on the GPU, with the results
// of the reference's importer (import_export/obj_import.cpp:167-340).  The
// reference reads each line with getline and converts it with sscanf:
//   vertex  "v x y z"   sscanf(line + 1, "%f %f %f")
//   face    "f a b c"   "%d %d %d", else "%d//%d %d//%d %d//%d",
//                       else "%d/%d/%d %d/%d/%d %d/%d/%d"
// This header holds the conversions as exact integer arithmetic (usable as
// plain C++ for tests): %f is strtof's correctly rounded decimal (or
// hexadecimal) conversion, ties to even, including subnormals, infinities and
// NaNs; %d is a decimal integer with optional sign.
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
namespace obj {

__host__ __device__ inline bool is_space(char c)
{
  return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r';
}

__host__ __device__ inline bool is_digit(char c) { return c >= '0' && c <= '9'; }

__host__ __device__ inline char lower(char c) { return (c >= 'A' && c <= 'Z') ? (char)(c + 32) : c; }

__host__ __device__ inline uint32_t f2u(float f)
{
#ifdef __CUDA_ARCH__
  return __float_as_uint(f);
#else
  uint32_t u;
  __builtin_memcpy(&u, &f, 4);
  return u;
#endif
}

__host__ __device__ inline float u2f(uint32_t u)
{
#ifdef __CUDA_ARCH__
  return __uint_as_float(u);
#else
  float f;
  __builtin_memcpy(&f, &u, 4);
  return f;
#endif
}

__host__ __device__ inline int bit_length64(uint64_t v)
{
  int n = 0;
  while (v) {
    ++n;
    v >>= 1;
  }
  return n;
}

// A float from the binary value (mant + f) * 2^e2, 0 <= f < 1, rounded to
// nearest with ties to even; `sticky` says f > 0.  mant > 0 must carry at
// least two bits below the float's last kept bit whenever sticky can be set,
// so that f alone never decides a rounding.  Handles the subnormal range
// (quantum 2^-149) and overflow to infinity.
__host__ __device__ inline float round_to_float(uint64_t mant, int e2, bool sticky, bool neg)
{
  const uint32_t sign = neg ? 0x80000000u : 0u;
  const int E = e2 + bit_length64(mant) - 1;  // exponent of the leading bit
  if (E > 127)
    return u2f(sign | 0x7F800000u);
  const int qe = E >= -126 ? E - 23 : -149;  // exponent of the last kept bit
  const int drop = qe - e2;
  uint64_t q;
  if (drop <= 0) {
    q = mant << (-drop);  // exact (drop >= -63 for every caller)
  } else if (drop > 64) {
    q = 0;  // below half a quantum
  } else {
    q = drop == 64 ? 0 : (mant >> drop);
    const uint64_t rem = drop == 64 ? mant : (mant & ((1ull << drop) - 1ull));
    const uint64_t half = 1ull << (drop - 1);
    if (rem > half || (rem == half && (sticky || (q & 1ull))))
      ++q;
  }
  if (qe == -149)  // subnormal; q = 2^23 after a carry is the smallest normal
    return u2f(sign | (uint32_t)q);
  int exp = E;
  if (q >> 24) {  // carry out of the mantissa
    q >>= 1;
    ++exp;
    if (exp > 127)
      return u2f(sign | 0x7F800000u);
  }
  return u2f(sign | ((uint32_t)(exp + 127) << 23) | ((uint32_t)q & 0x7FFFFFu));
}

// ---------------------------------------------------------------------------
// Small big integers (little-endian 32-bit limbs) for the exact paths.
// ---------------------------------------------------------------------------
// 512 bits: up to 120 significant decimal digits times 2^60 over 5^166.
constexpr int kBig = 16;
// Significant decimal digits kept exactly.  A float midpoint has at most
// about 113 significant digits, so the digits beyond these only act as a
// sticky bit.
constexpr int kMaxDigits = 120;

struct Big {
  uint32_t l[kBig];
};

__host__ __device__ inline void big_set(Big& a, uint64_t v)
{
  for (int i = 0; i < kBig; ++i)
    a.l[i] = 0;
  a.l[0] = (uint32_t)v;
  a.l[1] = (uint32_t)(v >> 32);
}

__host__ __device__ inline void big_mul_small(Big& a, uint32_t m)
{
  uint64_t c = 0;
  for (int i = 0; i < kBig; ++i) {
    const uint64_t t = (uint64_t)a.l[i] * m + c;
    a.l[i] = (uint32_t)t;
    c = t >> 32;
  }
}

__host__ __device__ inline void big_add_small(Big& a, uint32_t v)
{
  uint64_t c = v;
  for (int i = 0; i < kBig && c; ++i) {
    const uint64_t t = (uint64_t)a.l[i] + c;
    a.l[i] = (uint32_t)t;
    c = t >> 32;
  }
}

__host__ __device__ inline int big_bits(const Big& a)
{
  for (int i = kBig - 1; i >= 0; --i)
    if (a.l[i]) {
      int b = 0;
      uint32_t v = a.l[i];
      while (v) {
        ++b;
        v >>= 1;
      }
      return 32 * i + b;
    }
  return 0;
}

__host__ __device__ inline bool big_bit(const Big& a, int k) { return (a.l[k >> 5] >> (k & 31)) & 1u; }

// the bits [lo, lo + n) as an integer (n <= 64)
__host__ __device__ inline uint64_t big_bits_at(const Big& a, int lo, int n)
{
  uint64_t v = 0;
  for (int i = n - 1; i >= 0; --i)
    v = (v << 1) | (uint64_t)big_bit(a, lo + i);
  return v;
}

__host__ __device__ inline bool big_any_below(const Big& a, int k)
{
  for (int i = 0; i < k; ++i)
    if (big_bit(a, i))
      return true;
  return false;
}

__host__ __device__ inline void big_shl(Big& a, int s)
{
  if (s <= 0)
    return;
  const int w = s >> 5, b = s & 31;
  for (int i = kBig - 1; i >= 0; --i) {
    uint32_t v = 0;
    if (i - w >= 0) {
      v = a.l[i - w] << b;
      if (b && i - w - 1 >= 0)
        v |= a.l[i - w - 1] >> (32 - b);
    }
    a.l[i] = v;
  }
}

__host__ __device__ inline int big_cmp(const Big& a, const Big& b)
{
  for (int i = kBig - 1; i >= 0; --i)
    if (a.l[i] != b.l[i])
      return a.l[i] < b.l[i] ? -1 : 1;
  return 0;
}

__host__ __device__ inline void big_sub(Big& a, const Big& b)
{
  int64_t br = 0;
  for (int i = 0; i < kBig; ++i) {
    int64_t t = (int64_t)a.l[i] - b.l[i] - br;
    br = t < 0;
    a.l[i] = (uint32_t)(t + (br << 32));
  }
}

__host__ __device__ inline bool big_is_zero(const Big& a)
{
  uint32_t o = 0;
  for (int i = 0; i < kBig; ++i)
    o |= a.l[i];
  return o == 0;
}

// Exact W * 10^q (W > 0 with nsig significant digits; `more` = nonzero
// digits were dropped after W) rounded to float.
__host__ __device__ inline float decimal_exact(Big a, int nsig, int q, bool more, bool neg)
{
  if (nsig - 1 + q >= 39)  // at least 10^39 > FLT_MAX
    return u2f((neg ? 0x80000000u : 0u) | 0x7F800000u);
  if (nsig + q < -46)  // below 10^-46 < 2^-150
    return u2f(neg ? 0x80000000u : 0u);
  if (q >= 0) {
    for (int i = 0; i < q; ++i)
      big_mul_small(a, 10);
    // value = a (an integer below 10^39); `more` adds less than one unit
    const int n = big_bits(a);
    const int take = n < 60 ? n : 60;
    const uint64_t top = big_bits_at(a, n - take, take);
    if (n - take < 2 && more) {
      // not enough bits below the float's precision: widen with zeros
      return round_to_float(top << 2, n - take - 2, true, neg);
    }
    return round_to_float(top, n - take, more || big_any_below(a, n - take), neg);
  }
  // value = W / 10^-q = W / (5^-q * 2^-q): quot = floor(W * 2^s / 5^-q) with
  // about 60 bits, the remainder (and dropped digits) as sticky
  Big d;
  big_set(d, 1);
  for (int i = 0; i < -q; ++i)
    big_mul_small(d, 5);
  // a quotient of about 60 bits: shift W up, or the divisor when W is long
  const int s = 60 + big_bits(d) - big_bits(a);
  const int sh = s > 0 ? s : 0;
  const int dsh = s < 0 ? -s : 0;
  big_shl(a, sh);
  big_shl(d, dsh);
  uint64_t quot = 0;
  Big r;
  big_set(r, 0);
  const int n = big_bits(a);
  for (int i = n - 1; i >= 0; --i) {
    big_shl(r, 1);
    r.l[0] |= (uint32_t)big_bit(a, i);
    quot <<= 1;
    if (big_cmp(r, d) >= 0) {
      big_sub(r, d);
      quot |= 1;
    }
  }
  // value = quot * 2^(q - sh + dsh)   (the 2^q of 10^q and the shifts)
  return round_to_float(quot, q - sh + dsh, !big_is_zero(r) || more, neg);
}

// 10^k, exact in double for k <= 22
__host__ __device__ inline double pow10_exact(int k)
{
  double p = 1.0;
  for (int i = 0; i < k; ++i)
    p *= 10.0;
  return p;
}

// Parses a %f conversion of scanf (strtof) at s[0..n): leading white space,
// sign, then "inf"/"infinity", "nan"/"nan(...)", a hexadecimal or a decimal
// number.  Returns the characters consumed (0: no conversion) and the value.
__host__ __device__ inline int parse_float(const char* s, int n, float* out)
{
  int i = 0;
  while (i < n && is_space(s[i]))
    ++i;
  bool neg = false;
  if (i < n && (s[i] == '+' || s[i] == '-')) {
    neg = s[i] == '-';
    ++i;
  }
  const uint32_t sign = neg ? 0x80000000u : 0u;
  // infinity / nan
  if (i < n && (lower(s[i]) == 'i' || lower(s[i]) == 'n')) {
    const char* inf = "infinity";
    int k = 0;
    while (k < 8 && i + k < n && lower(s[i + k]) == inf[k])
      ++k;
    if (k >= 3) {
      *out = u2f(sign | 0x7F800000u);
      return i + (k == 8 ? 8 : 3);
    }
    const char* nan = "nan";
    k = 0;
    while (k < 3 && i + k < n && lower(s[i + k]) == nan[k])
      ++k;
    if (k == 3) {  // scanf stops after "nan" (no parenthesised payload)
      *out = u2f(sign | 0x7FC00000u);
      return i + 3;
    }
    return 0;
  }
  // hexadecimal: 0x h.hhh p[+-]d
  if (i + 1 < n && s[i] == '0' && lower(s[i + 1]) == 'x') {
    int j = i + 2;
    uint64_t m = 0;
    int shift = 0;  // binary exponent adjustment
    bool any = false, more = false;
    auto hexval = [](char c) -> int {
      if (c >= '0' && c <= '9') return c - '0';
      c = lower(c);
      if (c >= 'a' && c <= 'f') return c - 'a' + 10;
      return -1;
    };
    while (j < n && hexval(s[j]) >= 0) {
      any = true;
      if (m >> 56)
        shift += 4, more |= hexval(s[j]) != 0;
      else
        m = (m << 4) | (uint64_t)hexval(s[j]);
      ++j;
    }
    if (j < n && s[j] == '.') {
      ++j;
      while (j < n && hexval(s[j]) >= 0) {
        any = true;
        if (m >> 56) {
          more |= hexval(s[j]) != 0;
        } else {
          m = (m << 4) | (uint64_t)hexval(s[j]);
          shift -= 4;
        }
        ++j;
      }
    }
    if (!any)  // "0x" without digits: scanf converts nothing
      return 0;
    if (j < n && lower(s[j]) == 'p') {
      int t = j + 1;
      bool eneg = false;
      if (t < n && (s[t] == '+' || s[t] == '-')) {
        eneg = s[t] == '-';
        ++t;
      }
      if (t < n && is_digit(s[t])) {
        int e = 0;
        while (t < n && is_digit(s[t])) {
          if (e < 100000)
            e = e * 10 + (s[t] - '0');
          ++t;
        }
        shift += eneg ? -e : e;
        j = t;
      }
    }
    *out = m ? round_to_float(m, shift, more, neg) : u2f(sign);
    return j;
  }
  // decimal: the first kMaxDigits significant digits kept exactly
  int j = i;
  uint64_t w = 0;  // the first 19 of them, for the fast path
  Big W;
  big_set(W, 0);
  int nsig = 0, exp10 = 0;
  bool any = false, more = false;
  auto digit = [&](char c, bool frac) {
    any = true;
    if (nsig == 0 && c == '0') {  // leading zero
      if (frac)
        --exp10;
      return;
    }
    if (nsig < kMaxDigits) {
      if (nsig < 19)
        w = w * 10 + (uint64_t)(c - '0');
      big_mul_small(W, 10);
      big_add_small(W, (uint32_t)(c - '0'));
      ++nsig;
      if (frac)
        --exp10;
    } else {
      more |= c != '0';
      if (!frac)
        ++exp10;
    }
  };
  while (j < n && is_digit(s[j]))
    digit(s[j++], false);
  if (j < n && s[j] == '.') {
    ++j;
    while (j < n && is_digit(s[j]))
      digit(s[j++], true);
  }
  if (!any)
    return 0;
  if (j < n && lower(s[j]) == 'e') {
    // scanf takes the 'e' and a sign even when no digit follows
    int t = j + 1;
    bool eneg = false;
    if (t < n && (s[t] == '+' || s[t] == '-')) {
      eneg = s[t] == '-';
      ++t;
    }
    int e = 0;
    while (t < n && is_digit(s[t])) {
      if (e < 100000)
        e = e * 10 + (s[t] - '0');
      ++t;
    }
    exp10 += eneg ? -e : e;
    j = t;
  }
  if (nsig == 0) {
    *out = u2f(sign);
    return j;
  }
  // Clinger's fast path: w and 10^|q| exact in double, one correctly rounded
  // operation; rounding that double to float is right unless the double is
  // exactly a float midpoint (then the exact path decides)
  if (nsig <= 19 && w < (1ull << 53) && exp10 >= -22 && exp10 <= 22) {
    const double d = exp10 >= 0 ? (double)w * pow10_exact(exp10) : (double)w / pow10_exact(-exp10);
    uint64_t bits;
#ifdef __CUDA_ARCH__
    bits = (uint64_t)__double_as_longlong(d);
#else
    __builtin_memcpy(&bits, &d, 8);
#endif
    const int be = (int)((bits >> 52) & 0x7FF) - 1023;
    const bool normal = be >= -126 && be <= 127;  // a normal float: 29 bits below its precision
    const uint64_t low = bits & ((1ull << 29) - 1ull);
    if (normal && low != (1ull << 28)) {
      const float f = (float)d;
      *out = neg ? -f : f;
      return j;
    }
  }
  *out = decimal_exact(W, nsig, exp10, more, neg);
  return j;
}

// Parses a %d conversion of scanf: white space, optional sign, digits.
// Returns the characters consumed (0: no conversion).
__host__ __device__ inline int parse_int(const char* s, int n, long long* out)
{
  int i = 0;
  while (i < n && is_space(s[i]))
    ++i;
  bool neg = false;
  if (i < n && (s[i] == '+' || s[i] == '-')) {
    neg = s[i] == '-';
    ++i;
  }
  if (i >= n || !is_digit(s[i]))
    return 0;
  long long v = 0;
  while (i < n && is_digit(s[i])) {
    if (v < (1ll << 40))
      v = v * 10 + (s[i] - '0');
    ++i;
  }
  *out = neg ? -v : v;
  return i;
}

// sscanf(line, "%f %f %f"): the number of conversions (0..3).
__host__ __device__ inline int scan_3f(const char* s, int n, float* v)
{
  int pos = 0;
  for (int k = 0; k < 3; ++k) {
    const int c = parse_float(s + pos, n - pos, v + k);
    if (!c)
      return k;
    pos += c;
  }
  return 3;
}

// The face formats of obj_import.cpp:209-224 tried in order; returns true and
// the three vertex numbers (1-based, as written) for the first that converts
// fully.  A space in a scanf format matches any white space (none included).
__host__ __device__ inline bool scan_face(const char* s, int n, long long* idx)
{
  // format 0: "%d %d %d"
  {
    int pos = 0, k = 0;
    for (; k < 3; ++k) {
      const int c = parse_int(s + pos, n - pos, idx + k);
      if (!c)
        break;
      pos += c;
    }
    if (k == 3)
      return true;
  }
  // formats 1 and 2: "%d//%d" and "%d/%d/%d" per vertex
  for (int form = 1; form <= 2; ++form) {
    int pos = 0;
    bool ok = true;
    for (int k = 0; k < 3 && ok; ++k) {
      long long other;
      int c = parse_int(s + pos, n - pos, idx + k);
      if (!c) {
        ok = false;
        break;
      }
      pos += c;
      if (form == 1) {
        if (pos + 1 < n && s[pos] == '/' && s[pos + 1] == '/')
          pos += 2;
        else
          ok = false;
        if (ok && !(c = parse_int(s + pos, n - pos, &other)))
          ok = false;
        pos += ok ? c : 0;
      } else {
        for (int r = 0; r < 2 && ok; ++r) {
          if (pos < n && s[pos] == '/')
            ++pos;
          else
            ok = false;
          if (ok && !(c = parse_int(s + pos, n - pos, &other)))
            ok = false;
          pos += ok ? c : 0;
        }
      }
      // the space between vertex groups in the format skips white space
      while (ok && k < 2 && pos < n && is_space(s[pos]))
        ++pos;
    }
    if (ok)
      return true;
  }
  return false;
}

#ifdef __CUDACC__
// ---------------------------------------------------------------------------
// Kernels.  The file's bytes sit on the device; lines are what getline gives
// (split at '\n', a '\r' stays in the line).
//  1. k_obj_nl_count: newlines per 4 KB chunk.
//  2. (scan of the chunk counts)
//  3. k_obj_line_starts: starts[k + 1] = (position of newline k) + 1, starts[0] = 0.
//  4. k_obj_classify: per line a vertex / face / special (o, g, usemtl,
//     mtllib) flag, skipping what the reference skips: empty lines, '#'
//     lines, lines shorter than 3 characters, "vn", "vt", "s".
//  5. (scans of the three flags: each line's ordinal in its class)
//  6. k_obj_parse: vertices and face indices converted in parallel; the
//     special lines listed with the number of faces before them.
//  7. k_obj_gather: the triangles from the vertex indices.
// Errors keep the earliest line: atomicMin on (line << 8 | code).
// ---------------------------------------------------------------------------
constexpr int kObjThreads = 256;
constexpr int kObjBytes = 16;                           // bytes per thread
constexpr int kObjChunk = kObjThreads * kObjBytes;      // bytes per block
constexpr uint8_t kLineSkip = 0, kLineVertex = 1, kLineFace = 2, kLineSpecial = 3;
constexpr uint32_t kObjFormatError = 22;                // OBJ_IMPORT_FORMAT_ERROR

__device__ __forceinline__ uint32_t block_exclusive_sum(uint32_t v, uint32_t* scratch /* kObjThreads / 32 */,
                                                        uint32_t* total)
{
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = v;
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
    if (lane >= d)
      incl += y;
  }
  if (lane == 31)
    scratch[warp] = incl;
  __syncthreads();
  uint32_t before = 0, all = 0;
  for (int w = 0; w < kObjThreads / 32; ++w) {
    const uint32_t u = scratch[w];
    before += w < warp ? u : 0u;
    all += u;
  }
  __syncthreads();
  *total = all;
  return before + incl - v;
}

__global__ void __launch_bounds__(kObjThreads) k_obj_nl_count(const char* __restrict__ text, uint32_t n,
                                                              uint32_t* __restrict__ chunk_nl)
{
  __shared__ uint32_t scratch[kObjThreads / 32];
  const uint32_t base = blockIdx.x * kObjChunk + threadIdx.x * kObjBytes;
  uint32_t c = 0;
  for (int i = 0; i < kObjBytes; ++i)
    c += (base + i < n && text[base + i] == '\n') ? 1u : 0u;
  uint32_t total;
  block_exclusive_sum(c, scratch, &total);
  if (threadIdx.x == 0)
    chunk_nl[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kObjThreads) k_obj_line_starts(const char* __restrict__ text, uint32_t n,
                                                                 const uint32_t* __restrict__ chunk_off,
                                                                 uint32_t* __restrict__ starts)
{
  __shared__ uint32_t scratch[kObjThreads / 32];
  const uint32_t base = blockIdx.x * kObjChunk + threadIdx.x * kObjBytes;
  uint32_t c = 0;
  for (int i = 0; i < kObjBytes; ++i)
    c += (base + i < n && text[base + i] == '\n') ? 1u : 0u;
  uint32_t total;
  uint32_t k = chunk_off[blockIdx.x] + block_exclusive_sum(c, scratch, &total);
  for (int i = 0; i < kObjBytes; ++i)
    if (base + i < n && text[base + i] == '\n')
      starts[++k] = base + i + 1;
  if (blockIdx.x == 0 && threadIdx.x == 0)
    starts[0] = 0;
}

// line k is text[starts[k], starts[k + 1] - 1); the host sets the sentinel
// starts[n_newlines + 1] = n + 1 so that a last line without '\n' ends at n
__device__ __forceinline__ void line_range(const uint32_t* starts, uint32_t k, uint32_t* b, uint32_t* e)
{
  *b = starts[k];
  *e = starts[k + 1] - 1;
}

__global__ void k_obj_classify(const char* __restrict__ text, const uint32_t* __restrict__ starts, uint32_t n_lines,
                               uint32_t* __restrict__ is_vertex, uint32_t* __restrict__ is_face,
                               uint32_t* __restrict__ is_special)
{
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n_lines; k += gridDim.x * blockDim.x) {
    uint32_t b, e;
    line_range(starts, k, &b, &e);
    uint8_t cls = kLineSkip;
    // obj_import.cpp:188-196: empty, '#', shorter than 3: skipped
    if (e - b >= 3 && text[b] != '#') {
      const char c0 = text[b], c1 = text[b + 1];
      if (c0 == 'v')
        cls = (c1 == 'n' || c1 == 't') ? kLineSkip : kLineVertex;
      else if (c0 == 'f')
        cls = kLineFace;
      else if (c0 == 'o' || c0 == 'g' || c0 == 'u' || c0 == 'm')
        cls = kLineSpecial;
    }
    is_vertex[k] = cls == kLineVertex;
    is_face[k] = cls == kLineFace;
    is_special[k] = cls == kLineSpecial;
  }
}

__device__ __forceinline__ void obj_error(unsigned long long* err, uint32_t line, uint32_t code)
{
  atomicMin(err, ((unsigned long long)line << 8) | code);
}

__global__ void k_obj_parse(const char* __restrict__ text, const uint32_t* __restrict__ starts, uint32_t n_lines,
                            const uint32_t* __restrict__ is_vertex, const uint32_t* __restrict__ vord,
                            const uint32_t* __restrict__ is_face, const uint32_t* __restrict__ ford,
                            const uint32_t* __restrict__ is_special, const uint32_t* __restrict__ sord,
                            float* __restrict__ vertices, int32_t* __restrict__ face_idx,
                            uint32_t* __restrict__ face_line, uint32_t* __restrict__ special_line,
                            uint32_t* __restrict__ special_faces, unsigned long long* __restrict__ err)
{
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n_lines; k += gridDim.x * blockDim.x) {
    uint32_t b, e;
    line_range(starts, k, &b, &e);
    if (is_vertex[k]) {
      float v[3];
      // sscanf(str + 1, "%f %f %f"), obj_import.cpp:201-210
      if (scan_3f(text + b + 1, (int)(e - b - 1), v) == 3) {
        float* out = vertices + 3 * (size_t)vord[k];
        out[0] = v[0];
        out[1] = v[1];
        out[2] = v[2];
      } else {
        obj_error(err, k, kObjFormatError);
      }
    } else if (is_face[k]) {
      long long idx[3];
      if (scan_face(text + b + 1, (int)(e - b - 1), idx)) {
        int32_t* out = face_idx + 3 * (size_t)ford[k];
        for (int i = 0; i < 3; ++i)  // idx_face_t{i0 - 1, i1 - 1, i2 - 1}
          out[i] = (idx[i] - 1 >= -2147483647ll && idx[i] - 1 <= 2147483647ll) ? (int32_t)(idx[i] - 1) : -1;
        face_line[ford[k]] = k;
      } else {
        obj_error(err, k, kObjFormatError);
      }
    } else if (is_special[k]) {
      special_line[sord[k]] = k;
      special_faces[sord[k]] = ford[k];  // faces before this line
    }
  }
}

// faces9[f] = the three vertices of face f; an index outside the vertex list
// (undefined behaviour in the reference) is a format error at the face's line
__global__ void k_obj_gather(const float* __restrict__ vertices, uint32_t n_vertices,
                             const int32_t* __restrict__ face_idx, const uint32_t* __restrict__ face_line,
                             uint32_t n_faces, float* __restrict__ faces9, unsigned long long* __restrict__ err)
{
  for (uint32_t f = blockIdx.x * blockDim.x + threadIdx.x; f < n_faces; f += gridDim.x * blockDim.x) {
    for (int i = 0; i < 3; ++i) {
      const int32_t v = face_idx[3 * (size_t)f + i];
      float* out = faces9 + 9 * (size_t)f + 3 * i;
      if (v >= 0 && (uint32_t)v < n_vertices) {
        out[0] = vertices[3 * (size_t)v];
        out[1] = vertices[3 * (size_t)v + 1];
        out[2] = vertices[3 * (size_t)v + 2];
      } else {
        out[0] = out[1] = out[2] = 0.f;
        obj_error(err, face_line[f], kObjFormatError);
      }
    }
  }
}

// (start, end) of each special line, for the host to read them in its copy
__global__ void k_obj_special_ranges(const uint32_t* __restrict__ starts, const uint32_t* __restrict__ special_line,
                                     uint32_t n_special, uint32_t* __restrict__ ranges)
{
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_special; i += gridDim.x * blockDim.x) {
    uint32_t b, e;
    line_range(starts, special_line[i], &b, &e);
    ranges[2 * i] = b;
    ranges[2 * i + 1] = e;
  }
}
#endif  // __CUDACC__

}  // namespace obj
}  // namespace ffb
