// ffb_device.cuh -- device-side math of the B200 form-factor path.
//
// Everything here is compiled with --fmad=false, IEEE division and square
// root (nvcc defaults without -use_fast_math): every float operation rounds
// once, in the order written, which is what makes hit indices and hit points
// bit-identical to the reference's CPU casters.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ffb {

// Smallest float above the reference's double threshold 1e-8
// (math/operations.h:31).  For a float x, (double)x < 1e-8 holds exactly when
// x < FFB_EPS_ABOVE_1E8, because 1e-8 lies strictly between two floats.
#define FFB_EPS_ABOVE_1E8 0x1.5798f0p-27f
// (pi/4) / 2^21 rounded to float.
#define FFB_QUARTER_PI_OVER_2P21 0x1.921fb6p-22f

// ---------------------------------------------------------------------------
// Triangle record: four float4, 64 bytes, precomputed once per face from the
// three vertices with the operations of math/triangle.cpp:34-38,58-64.
//   q0 = (p0.xyz, uu)   q1 = (n.xyz, uv)   q2 = (u.xyz, vv)   q3 = (v.xyz, D)
// A degenerate face (dot(n,n) < 1e-8) gets n = 0: every test against it then
// fails the |b| < 1e-8 check, which the reference also treats as a miss.
// ---------------------------------------------------------------------------
struct TriRec {
  float4 q0, q1, q2, q3;
};

__host__ __device__ inline float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__host__ __device__ inline float3 sub3(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ inline float3 add3(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ inline float3 mul3(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
// (x*x' + y*y') + z*z', math/operations.h:44-47
__host__ __device__ inline float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ inline float3 cross3(float3 a, float3 b)
{
  return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

__device__ inline TriRec make_trirec(float3 p0, float3 p1, float3 p2)
{
  float3 u = sub3(p1, p0);
  float3 v = sub3(p2, p0);
  float3 n = cross3(u, v);
  if ((double)dot3(n, n) < 1e-8)
    n = f3(0.f, 0.f, 0.f);
  float uu = dot3(u, u);
  float uv = dot3(u, v);
  float vv = dot3(v, v);
  float D = uv * uv - uu * vv;
  TriRec t;
  t.q0 = make_float4(p0.x, p0.y, p0.z, uu);
  t.q1 = make_float4(n.x, n.y, n.z, uv);
  t.q2 = make_float4(u.x, u.y, u.z, vv);
  t.q3 = make_float4(v.x, v.y, v.z, D);
  return t;
}

// ---------------------------------------------------------------------------
// Division-free decisions that are exact for the reference's comparisons.
// For q = num / den rounded to nearest:
//  * q < 0 holds exactly when num and den have opposite signs, num != 0 and
//    the quotient does not round to -0; |num| > |den| * 2^-100 rules out the
//    underflow, so "surely negative" below implies q < 0.
//  * q > 1 holds when num and den share a sign and |num| > |den| * (1 + 2^-20):
//    the exact quotient then exceeds 1 by far more than half an ulp.
// Anything not decided this way goes through the IEEE division.  NaN inputs
// fail every comparison and always take the division path.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool surely_negative(float num, float den)
{
  return ((num < 0.f) != (den < 0.f)) && num != 0.f && fabsf(num) > fabsf(den) * 0x1p-100f;
}

__device__ __forceinline__ bool surely_above_one(float num, float den)
{
  return ((num < 0.f) == (den < 0.f)) && fabsf(num) > fabsf(den) * 0x1.000010p+0f;
}

// ---------------------------------------------------------------------------
// The ray/triangle test of math/triangle.cpp:40-78 on a precomputed record
// held in registers.  o is the ray origin, dir = end - origin.  Returns true
// for TRIANGLE_INTERSECTION_UNIQUE and writes the intersection point.  Every
// value that decides the result is computed with the reference's operations
// in the reference's order; the sign shortcuts above only skip divisions
// whose outcome is already known.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool tri_hit_regs(const float4 q0, const float4 q1, const float4 q2, const float4 q3,
                                             float3 o, float3 dir, float3& pt)
{
  // Every rejection that needs no division beyond r decided by one branch:
  // lanes of a warp that leave at different stages then run the same
  // instructions.  r, p, s and t numerators are computed as below; when
  // the plane stage rejects they are unused.
  float3 w0 = f3(o.x - q0.x, o.y - q0.y, o.z - q0.z);
  float a = -(q1.x * w0.x + q1.y * w0.y + q1.z * w0.z);
  float b = q1.x * dir.x + q1.y * dir.y + q1.z * dir.z;
  float r = a / b;
  float3 p = f3(o.x + r * dir.x, o.y + r * dir.y, o.z + r * dir.z);
  float3 w = f3(p.x - q0.x, p.y - q0.y, p.z - q0.z);
  float wu = w.x * q2.x + w.y * q2.y + w.z * q2.z;
  float wv = w.x * q3.x + w.y * q3.y + w.z * q3.z;
  const float uu = q0.w, uv = q1.w, vv = q2.w, D = q3.w;
  const float ns = uv * wv - vv * wu;
  const float nt = uv * wu - uu * wv;
  const bool out = (fabsf(b) < FFB_EPS_ABOVE_1E8) | (r < 0.f) | surely_negative(ns, D) | surely_above_one(ns, D) |
                   surely_negative(nt, D);
  if (out)
    return false;
  float s = ns / D;
  if (s < 0.f || s > 1.f)
    return false;
  float t = nt / D;
  if (t < 0.f || (s + t) > 1.f)
    return false;
  pt = p;
  return true;
}

// Same test on a record in memory (global or shared).
__device__ __forceinline__ bool tri_hit(const float4* rec, float3 o, float3 dir, float3& pt)
{
  return tri_hit_regs(rec[0], rec[1], rec[2], rec[3], o, dir, pt);
}

// Squared distance of the reference caster (naive_cpu.cpp:83-84).
__device__ __forceinline__ float dist2(float3 p, float3 o)
{
  float3 d = f3(p.x - o.x, p.y - o.y, p.z - o.z);
  return d.x * d.x + d.y * d.y + d.z * d.z;
}

// Nearest-hit update equivalent to scanning faces in index order with a
// strict '<' starting from FLT_MAX: the smallest distance wins and, among
// equal distances, the lowest index.
__device__ __forceinline__ void consider(float d, int idx, float& best, int& best_idx)
{
  if (d < best || (d == best && idx < best_idx)) {
    best = d;
    best_idx = idx;
  }
}

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), constants as published.
// ---------------------------------------------------------------------------
__host__ __device__ inline uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1)
{
#pragma unroll
  for (int round = 0; round < 10; ++round) {
#ifdef __CUDA_ARCH__
    uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
    uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
#else
    uint64_t p0 = (uint64_t)0xD2511F53u * c.x, p1 = (uint64_t)0xCD9E8D57u * c.z;
    uint32_t lo0 = (uint32_t)p0, hi0 = (uint32_t)(p0 >> 32);
    uint32_t lo1 = (uint32_t)p1, hi1 = (uint32_t)(p1 >> 32);
#endif
    c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

__host__ __device__ inline float u01(uint32_t x) { return (float)(x >> 8) * 0x1p-24f; }

// sin and cos of 2*pi*k/2^24 for k in [0, 2^24): exact octant reduction on
// the integer, then truncated Taylor series on [0, pi/4].
__host__ __device__ inline void sincos_turn24(uint32_t k, float& s_out, float& c_out)
{
  uint32_t oct = (k >> 21) & 7u;
  uint32_t j = k & 0x1FFFFFu;
  if (oct & 1u)
    j = 0x200000u - j;
  float x = (float)j * FFB_QUARTER_PI_OVER_2P21;
  float x2 = x * x;
  float sp = x + x * x2 * (-1.6666667e-1f + x2 * (8.3333333e-3f + x2 * (-1.9841270e-4f + x2 * 2.7557319e-6f)));
  float cp = 1.0f + x2 * (-0.5f + x2 * (4.1666668e-2f + x2 * (-1.3888889e-3f + x2 * (2.4801587e-5f + x2 * -2.7557319e-7f))));
  float sb = (oct & 1u) ? cp : sp;
  float cb = (oct & 1u) ? sp : cp;
  switch (oct >> 1) {
  case 0: s_out = sb; c_out = cb; break;
  case 1: s_out = cb; c_out = -sb; break;
  case 2: s_out = -sb; c_out = -cb; break;
  default: s_out = -cb; c_out = sb; break;
  }
}

// ---------------------------------------------------------------------------
// Emission frame of a face: p0, the two edges and the rotation of +z towards
// the face normal (math/mat.cpp:25-49 with the helpers of math/mat.h:54-91),
// stored row-major in m[9].  20 floats per face (p0, e1, e2, m, pad, pad).
// ---------------------------------------------------------------------------
struct FaceFrame {
  float v[20];
};

__host__ __device__ inline void rotate_towards(float3 s, float3 t, float* m)
{
  float3 v = cross3(s, t);
  float s2 = dot3(v, v);
  float c = dot3(s, t);
  float R[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  if (s2 > 0x1p-126f) {  // FLT_MIN
    float a[9] = {0.f, v.z, -v.y, -v.z, 0.f, v.x, v.y, -v.x, 0.f};
    float q[9];
    q[0] = a[1] * a[3] + a[2] * a[6];
    q[1] = a[5] * a[6];
    q[2] = a[7] * a[3];
    q[3] = a[1] * a[4] + a[2] * a[7];
    q[4] = a[3] * a[1] + a[5] * a[7];
    q[5] = a[6] * a[1];
    q[6] = a[1] * a[5];
    q[7] = a[3] * a[2];
    q[8] = a[6] * a[2] + a[7] * a[5];
    float k = (1.f - c) / s2;
#pragma unroll
    for (int e = 0; e < 9; ++e)
      R[e] = (R[e] + a[e]) + q[e] * k;
  } else {
    float3 f = add3(s, t);
    float l = dot3(f, f);
    if (l < 0x1p-23f) {  // FLT_EPSILON
      R[4] = -1.f;
      R[8] = -1.f;
    }
  }
#pragma unroll
  for (int e = 0; e < 9; ++e)
    m[e] = R[e];
}

// Ray j of a face (emission/malley_cpu.cpp:159-184) with Philox draws keyed
// by (seed, epoch, face, j).  Writes origin o and end point e.
// fr points at the face's 20-float frame in global memory.
__device__ __forceinline__ void emit_ray(const float* __restrict__ fr, uint32_t face, uint32_t j, int front,
                                         uint32_t key0, uint32_t key1, uint32_t epoch, float3& o, float3& e)
{
  uint4 x = philox4x32_10(make_uint4(j, face, epoch, 0x46464231u), key0, key1);
  float a = u01(x.x);
  float b = u01(x.y);
  if (a + b > 1.f) {
    a = 1.f - a;
    b = 1.f - b;
  }
  float3 p0 = f3(__ldg(fr + 0), __ldg(fr + 1), __ldg(fr + 2));
  float3 e1 = f3(__ldg(fr + 3), __ldg(fr + 4), __ldg(fr + 5));
  float3 e2 = f3(__ldg(fr + 6), __ldg(fr + 7), __ldg(fr + 8));
  float3 origin = add3(add3(p0, mul3(e1, a)), mul3(e2, b));
  float r = u01(x.z);
  float rad = sqrtf(r);
  float sphi, cphi;
  sincos_turn24(x.w >> 8, sphi, cphi);
  float3 mv = f3(rad * cphi, rad * sphi, sqrtf(1.f - r));
  if ((int)j >= front)
    mv.z = -mv.z;
  float m[9];
#pragma unroll
  for (int k = 0; k < 9; ++k)
    m[k] = __ldg(fr + 9 + k);
  float3 d = f3((m[0] * mv.x + m[3] * mv.y) + m[6] * mv.z,
                (m[1] * mv.x + m[4] * mv.y) + m[7] * mv.z,
                (m[2] * mv.x + m[5] * mv.y) + m[8] * mv.z);
  o = add3(origin, mul3(d, 0.0001f));
  e = add3(origin, d);
}

// ---------------------------------------------------------------------------
// Parallel rays from a disc (a distant source such as the Sun,
// emission/parallel_rays_cpu.cpp:88-106): a point uniform on the disc of
// `radius` in the plane z = -distance of the source frame, rotated by the
// rotation of +z towards `direction` and moved to `center`; the ray's end
// point is origin + direction * 0.1 (the reference's ray_t holds an end
// point).  Draws are Philox keyed by (seed, epoch, ray index).
// ---------------------------------------------------------------------------
struct DiscSource {
  float m[9];     // rotate_towards(+z, direction), row-major
  float3 center;
  float3 direction;
  float distance;
  float radius;
};

__host__ __device__ inline DiscSource make_disc_source(float3 direction, float3 center, float distance, float radius)
{
  DiscSource d;
  rotate_towards(f3(0.f, 0.f, 1.f), direction, d.m);
  d.center = center;
  d.direction = direction;
  d.distance = distance;
  d.radius = radius;
  return d;
}

constexpr uint32_t kDiscTag = 0x50415241u;  // Philox counter word distinguishing disc rays from face rays

__host__ __device__ inline void emit_disc_ray(const DiscSource& d, unsigned long long j, uint32_t key0, uint32_t key1,
                                              uint32_t epoch, float3& o, float3& e)
{
  const uint4 x = philox4x32_10(make_uint4((uint32_t)j, (uint32_t)(j >> 32), epoch, kDiscTag), key0, key1);
  const float rad = d.radius * sqrtf(u01(x.x));
  float st, ct;
  sincos_turn24(x.y >> 8, st, ct);
  const float px = rad * ct, py = rad * st, pz = -d.distance;
  // mat33 * vec3 (math/mat.h:30-37): column j of the row-major m times the vector
  const float3 v = f3((d.m[0] * px + d.m[3] * py) + d.m[6] * pz,
                      (d.m[1] * px + d.m[4] * py) + d.m[7] * pz,
                      (d.m[2] * px + d.m[5] * py) + d.m[8] * pz);
  o = add3(v, d.center);
  e = add3(o, mul3(d.direction, 0.1f));
}

}  // namespace ffb
