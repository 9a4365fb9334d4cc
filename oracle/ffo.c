/*
 * ffo.c -- CPU oracle for the Monte Carlo form-factor path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: tests, smoke() and the
 * CPU-baseline leg of bench.py load it to compare the CUDA path against.  The
 * product library never links, loads or calls it, and nothing here is a
 * fallback for the GPU path.
 *
 * It restates, in plain C, the reference algorithm of kroburg/form_factors:
 *   - ray/triangle test        math/triangle.cpp:28-79 (plane-then-parametric)
 *   - brute-force nearest hit  ray_caster/naive_cpu.cpp:65-97
 *   - per-face ray counts      emission/malley_emission.cpp:50-60
 *   - rotation towards normal  math/mat.cpp:25-49, math/mat.h:30-37,54-91
 *   - Malley ray construction  emission/malley_cpu.cpp:109-189
 *   - hit counting             cpuFactorsCalculator/cpu_system.cpp:167-196
 * with the reference's random source (std::mt19937) replaced by the
 * counter-based Philox4x32-10 stream that the CUDA path uses, so that a ray is
 * a pure function of (seed, epoch, face, index) and the whole pipeline can be
 * compared bit for bit.
 *
 * Compile with -ffp-contract=off and without -ffast-math: every float
 * operation must round exactly once, in the order written, as the reference's
 * ISO C++ build does.  Parity of this file is pinned against the reference
 * itself (oracle/_ref, built from the reference sources by oracle/Makefile)
 * and against the committed fixtures in tests/golden/.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#include <stdlib.h>
#include <float.h>
#include <pthread.h>
#include <unistd.h>

#include "ffo.h"

/* ------------------------------------------------------------------ */
/* Minimal parallel-for over [0, n) on pthreads with a shared cursor.   */
/* ------------------------------------------------------------------ */
typedef struct {
  long n, grain;
  long next;
  pthread_mutex_t mu;
  void (*body)(long i, void* ctx);
  void* ctx;
} pfor_t;

static void* pfor_worker(void* arg)
{
  pfor_t* p = (pfor_t*)arg;
  for (;;) {
    pthread_mutex_lock(&p->mu);
    long b = p->next;
    p->next += p->grain;
    pthread_mutex_unlock(&p->mu);
    if (b >= p->n)
      break;
    long e = b + p->grain < p->n ? b + p->grain : p->n;
    for (long i = b; i < e; ++i)
      p->body(i, p->ctx);
  }
  return 0;
}

static int g_threads = 0;

void ffo_set_threads(int n) { g_threads = n; }

static void parallel_for(long n, long grain, void (*body)(long, void*), void* ctx)
{
  int nt = g_threads > 0 ? g_threads : (int)sysconf(_SC_NPROCESSORS_ONLN);
  if (nt > 256) nt = 256;
  pfor_t p = {n, grain, 0, PTHREAD_MUTEX_INITIALIZER, body, ctx};
  if (nt <= 1 || n <= grain) {
    pfor_worker(&p);
    return;
  }
  pthread_t th[256];
  for (int t = 0; t < nt; ++t)
    pthread_create(&th[t], 0, pfor_worker, &p);
  for (int t = 0; t < nt; ++t)
    pthread_join(th[t], 0);
}

/* ------------------------------------------------------------------ */
/* vec3 helpers with the reference's evaluation order                  */
/* (math/operations.h:44-53: dot = (x*x' + y*y') + z*z')                */
/* ------------------------------------------------------------------ */
typedef struct { float x, y, z; } v3;

static inline v3 mk(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 sub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 add(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 scl(v3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
static inline float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 cross(v3 a, v3 b)
{
  return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline v3 ld(const float* p) { return mk(p[0], p[1], p[2]); }

/* ------------------------------------------------------------------ */
/* Ray/triangle test: math/triangle.cpp:28-79, op for op.               */
/* The two thresholds are the double constant 1e-8 (operations.h:31).  */
/* ------------------------------------------------------------------ */
int ffo_triangle_intersect(const float* ray6, const float* tri9, float* point3)
{
  v3 p0 = ld(tri9), p1 = ld(tri9 + 3), p2 = ld(tri9 + 6);
  v3 o = ld(ray6), e = ld(ray6 + 3);
  v3 u = sub(p1, p0);
  v3 v = sub(p2, p0);
  v3 n = cross(u, v);
  if ((double)dot(n, n) < 1e-8)
    return -FFO_DEGENERATE;
  v3 dir = sub(e, o);
  v3 w0 = sub(o, p0);
  float a = -dot(n, w0);
  float b = dot(n, dir);
  if (fabs((double)b) < 1e-8) {
    if (a == 0)
      return -FFO_SAME_PLANE;
    return -FFO_DISJOINT;
  }
  float r = a / b;
  if (r < 0.0)
    return -FFO_DISJOINT;
  v3 pt = add(o, scl(dir, r));
  point3[0] = pt.x; point3[1] = pt.y; point3[2] = pt.z;
  float uu = dot(u, u);
  float uv = dot(u, v);
  float vv = dot(v, v);
  v3 w = sub(pt, p0);
  float wu = dot(w, u);
  float wv = dot(w, v);
  float D = uv * uv - uu * vv;
  float s = (uv * wv - vv * wu) / D;
  if (s < 0.0 || s > 1.0)
    return -FFO_DISJOINT;
  float t = (uv * wu - uu * wv) / D;
  if (t < 0.0 || (s + t) > 1.0)
    return -FFO_DISJOINT;
  return FFO_UNIQUE;
}

/* Brute-force nearest hit: ray_caster/naive_cpu.cpp:65-97.  Faces are
 * scanned in index order with a strict '<' on the FP32 squared distance, so
 * the lowest index wins a tie.  Misses get -1 and leave hit_pt untouched. */
static void cast_one(int n_faces, const float* faces9, const float* ray6,
                     int32_t* hit, float* hit_pt)
{
  float best = FLT_MAX;
  int32_t idx = -1;
  v3 o = ld(ray6);
  for (int f = 0; f != n_faces; ++f) {
    float pt[3];
    if (ffo_triangle_intersect(ray6, faces9 + 9 * (size_t)f, pt) == FFO_UNIQUE) {
      v3 d = sub(ld(pt), o);
      float dist = dot(d, d);
      if (dist < best) {
        best = dist;
        idx = f;
        if (hit_pt) { hit_pt[0] = pt[0]; hit_pt[1] = pt[1]; hit_pt[2] = pt[2]; }
      }
    }
  }
  *hit = idx;
}

typedef struct {
  int n_faces;
  const float* faces9;
  const float* rays6;
  int32_t* hit;
  float* hit_pt;
} cast_ctx_t;

static void cast_body(long i, void* arg)
{
  cast_ctx_t* c = (cast_ctx_t*)arg;
  cast_one(c->n_faces, c->faces9, c->rays6 + 6 * i, c->hit + i, c->hit_pt ? c->hit_pt + 3 * i : 0);
}

void ffo_cast_naive(int n_faces, const float* faces9, long n_rays, const float* rays6,
                    int32_t* hit, float* hit_pt)
{
  cast_ctx_t c = {n_faces, faces9, rays6, hit, hit_pt};
  parallel_for(n_rays, 64, cast_body, &c);
}

/* ------------------------------------------------------------------ */
/* Per-face ray counts: emission/malley_emission.cpp:50-60.             */
/* n_rays * (w / total) is int*float -> float, then truncated.          */
/* ------------------------------------------------------------------ */
int ffo_emitted(int n_rays, float weight, float total_weight)
{
  if (!(weight > 0))
    return 0;
  int k = (int)(n_rays * (weight / total_weight));
  return k > 1 ? k : 1;
}

/* ------------------------------------------------------------------ */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: */
/* as easy as 1, 2, 3", SC'11), multipliers and Weyl constants as        */
/* published there.                                                      */
/* ------------------------------------------------------------------ */
void ffo_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4])
{
  uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  uint32_t k0 = key_in[0], k1 = key_in[1];
  for (int round = 0; round < 10; ++round) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    c0 = hi1 ^ c1 ^ k0;
    c1 = lo1;
    c2 = hi0 ^ c3 ^ k1;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Uniform float in [0, 1) from the top 24 bits. */
static inline float u01(uint32_t x) { return (float)(x >> 8) * 0x1p-24f; }

/* sin and cos of 2*pi*k/2^24, k in [0, 2^24).  The argument reduction is
 * exact integer arithmetic (octant from the top three bits, mirrored inside
 * odd octants), and the reduced angle in [0, pi/4] goes through truncated
 * Taylor series (sin to x^9, cos to x^10; remainder below 2e-9). */
void ffo_sincos_turn24(uint32_t k, float* s_out, float* c_out)
{
  uint32_t oct = (k >> 21) & 7u;
  uint32_t j = k & 0x1FFFFFu;
  if (oct & 1u)
    j = 0x200000u - j;
  float x = (float)j * FFO_QUARTER_PI_OVER_2P21;
  float x2 = x * x;
  float sp = x + x * x2 * (-1.6666667e-1f + x2 * (8.3333333e-3f + x2 * (-1.9841270e-4f + x2 * 2.7557319e-6f)));
  float cp = 1.0f + x2 * (-0.5f + x2 * (4.1666668e-2f + x2 * (-1.3888889e-3f + x2 * (2.4801587e-5f + x2 * -2.7557319e-7f))));
  float sb, cb; /* sin/cos of the angle inside its quadrant */
  if (oct & 1u) { sb = cp; cb = sp; } else { sb = sp; cb = cp; }
  switch (oct >> 1) {
  case 0: *s_out = sb; *c_out = cb; break;
  case 1: *s_out = cb; *c_out = -sb; break;
  case 2: *s_out = -sb; *c_out = -cb; break;
  default: *s_out = -cb; *c_out = sb; break;
  }
}

/* ------------------------------------------------------------------ */
/* Rotation of +z towards a face normal: math/mat.cpp:25-49 with the     */
/* matrix helpers of math/mat.h.  Stored row-major m[3*i+j] = p[i][j].   */
/* ------------------------------------------------------------------ */
void ffo_rotate_towards(const float* subject3, const float* to3, float* m9)
{
  v3 s = ld(subject3), t = ld(to3);
  v3 v = cross(s, t);
  float s2 = dot(v, v);
  float c = dot(s, t);
  float R[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  if (s2 > FLT_MIN) {
    /* skew-symmetric matrix, make_mat33 argument order (mat.cpp:36) */
    float a[9] = {0, v.z, -v.y, -v.z, 0, v.x, v.y, -v.x, 0};
#define A(i, j) a[3 * (i) + (j)]
    /* ssc_mul(a, a), mat.h:54-66 */
    float q[9];
    q[0] = A(0, 1) * A(1, 0) + A(0, 2) * A(2, 0);
    q[1] = A(1, 2) * A(2, 0);
    q[2] = A(2, 1) * A(1, 0);
    q[3] = A(0, 1) * A(1, 1) + A(0, 2) * A(2, 1);
    q[4] = A(1, 0) * A(0, 1) + A(1, 2) * A(2, 1);
    q[5] = A(2, 0) * A(0, 1);
    q[6] = A(0, 1) * A(1, 2);
    q[7] = A(1, 0) * A(0, 2);
    q[8] = A(2, 0) * A(0, 2) + A(2, 1) * A(1, 2);
    float k = (1 - c) / s2;
    /* (I + ssc) + ssc2*k: the transposes of mat.h's operator+ and
     * operator*(mat33, float) cancel, element (i,j) pairs with (i,j). */
    for (int e = 0; e < 9; ++e)
      R[e] = (R[e] + a[e]) + q[e] * k;
#undef A
  } else {
    v3 f = add(s, t);
    float l = dot(f, f);
    if (l < FLT_EPSILON) {
      float rev[9] = {1, 0, 0, 0, -1, 0, 0, 0, -1};
      memcpy(R, rev, sizeof R);
    }
  }
  memcpy(m9, R, sizeof R);
}

/* mat33 * vec3, math/mat.h:30-37 (columns of p[][] weight x, y, z). */
static inline v3 mat_vec(const float* m, v3 x)
{
  return mk((m[0] * x.x + m[3] * x.y) + m[6] * x.z,
            (m[1] * x.x + m[4] * x.y) + m[7] * x.z,
            (m[2] * x.x + m[5] * x.y) + m[8] * x.z);
}

/* Per-face emission frame: origin vertex, the two edges and the rotation of
 * +z towards the face normal (normalised unless FFO_EMIT_REF_NORMAL). */
void ffo_face_frame(const float* tri9, int flags, float* frame18)
{
  v3 p0 = ld(tri9), p1 = ld(tri9 + 3), p2 = ld(tri9 + 6);
  v3 e1 = sub(p1, p0), e2 = sub(p2, p0);
  v3 n = cross(e1, e2);
  if (!(flags & FFO_EMIT_REF_NORMAL)) {
    float len = sqrtf(dot(n, n));
    if (len > 0)
      n = mk(n.x / len, n.y / len, n.z / len);
  }
  float z[3] = {0, 0, 1};
  float nn[3] = {n.x, n.y, n.z};
  frame18[0] = p0.x; frame18[1] = p0.y; frame18[2] = p0.z;
  frame18[3] = e1.x; frame18[4] = e1.y; frame18[5] = e1.z;
  frame18[6] = e2.x; frame18[7] = e2.y; frame18[8] = e2.z;
  ffo_rotate_towards(z, nn, frame18 + 9);
}

/* Ray j of face f (j < front: front side, else rear side), as
 * emission/malley_cpu.cpp:159-184 builds it, with Philox draws:
 *   a, b  point on the face (reflected when a + b > 1)        :109-122
 *   r     radius^2 of the Malley disc point                   :133-139
 *   phi   angle, 2*pi*k/2^24                                  :133-139
 * ray = { origin + d * 1e-4, origin + d } (the second point is an end point). */
void ffo_emit_ray(const float* frame18, uint32_t face, uint32_t j, int front,
                  uint64_t seed, uint32_t epoch, float* ray6)
{
  uint32_t ctr[4] = {j, face, epoch, 0x46464231u};
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t x[4];
  ffo_philox4x32_10(ctr, key, x);
  float a = u01(x[0]);
  float b = u01(x[1]);
  if (a + b > 1) {
    a = 1.f - a;
    b = 1.f - b;
  }
  v3 p0 = ld(frame18), e1 = ld(frame18 + 3), e2 = ld(frame18 + 6);
  v3 origin = add(add(p0, scl(e1, a)), scl(e2, b));
  float r = u01(x[2]);
  float rad = sqrtf(r);
  float sphi, cphi;
  ffo_sincos_turn24(x[3] >> 8, &sphi, &cphi);
  v3 m = mk(rad * cphi, rad * sphi, sqrtf(1 - r));
  if ((int)j >= front)
    m.z = -m.z;
  v3 d = mat_vec(frame18 + 9, m);
  v3 o = add(origin, scl(d, 0.0001f));
  v3 e = add(origin, d);
  ray6[0] = o.x; ray6[1] = o.y; ray6[2] = o.z;
  ray6[3] = e.x; ray6[4] = e.y; ray6[5] = e.z;
}

/* All rays of a scene, packed face by face, front then rear
 * (emission/malley_cpu.cpp:142-189).  ray_offsets has n_faces + 1 entries. */
void ffo_emit(int n_faces, const float* faces9, const int32_t* front, const int32_t* rear,
              uint64_t seed, uint32_t epoch, int flags, float* rays6)
{
  long base = 0;
  for (int f = 0; f < n_faces; ++f) {
    float frame[18];
    ffo_face_frame(faces9 + 9 * (size_t)f, flags, frame);
    int nf = front[f] + rear[f];
    for (int j = 0; j < nf; ++j)
      ffo_emit_ray(frame, (uint32_t)f, (uint32_t)j, front[f], seed, epoch, rays6 + 6 * (base + j));
    base += nf;
  }
}

/* Emission + brute-force cast + per-(source face, hit face) uint32 counts,
 * the per-face form of cpuFactorsCalculator/cpu_system.cpp:167-196.
 * counts is n_faces*n_faces, zeroed here. */
typedef struct {
  int n_faces;
  const float* faces9;
  const int32_t *front, *rear;
  uint64_t seed;
  uint32_t epoch;
  int flags;
  uint32_t* counts;
} ff_ctx_t;

static void ff_body(long f, void* arg)
{
  ff_ctx_t* c = (ff_ctx_t*)arg;
  float frame[18];
  ffo_face_frame(c->faces9 + 9 * (size_t)f, c->flags, frame);
  int nf = c->front[f] + c->rear[f];
  for (int j = 0; j < nf; ++j) {
    float ray[6];
    int32_t h;
    ffo_emit_ray(frame, (uint32_t)f, (uint32_t)j, c->front[f], c->seed, c->epoch, ray);
    cast_one(c->n_faces, c->faces9, ray, &h, 0);
    if (h >= 0)
      c->counts[(size_t)f * c->n_faces + h] += 1;
  }
}

void ffo_form_factor_counts(int n_faces, const float* faces9, const int32_t* front,
                            const int32_t* rear, uint64_t seed, uint32_t epoch, int flags,
                            uint32_t* counts)
{
  memset(counts, 0, sizeof(uint32_t) * (size_t)n_faces * (size_t)n_faces);
  ff_ctx_t c = {n_faces, faces9, front, rear, seed, epoch, flags, counts};
  parallel_for(n_faces, 1, ff_body, &c);
}

/* ------------------------------------------------------------------ */
/* Parallel rays from a disc (emission/parallel_rays_cpu.cpp:88-106):     */
/* disc17 = rotation m9 (rotate_towards(+z, direction)), center3,        */
/* direction3, distance, radius.  Draws: Philox keyed by (seed, epoch,   */
/* ray index) -- u for the radius (radius * sqrt(u)), a 24-bit turn for   */
/* the angle.  origin = m * (x, y, -distance) + center, end = origin +    */
/* direction * 0.1.                                                       */
/* ------------------------------------------------------------------ */
void ffo_disc_source(const float* direction3, const float* center3, float distance, float radius, float* disc17)
{
  const float z[3] = {0, 0, 1};
  ffo_rotate_towards(z, direction3, disc17);
  memcpy(disc17 + 9, center3, 3 * sizeof(float));
  memcpy(disc17 + 12, direction3, 3 * sizeof(float));
  disc17[15] = distance;
  disc17[16] = radius;
}

void ffo_emit_disc_ray(const float* disc17, uint64_t j, uint64_t seed, uint32_t epoch, float* ray6)
{
  uint32_t ctr[4] = {(uint32_t)j, (uint32_t)(j >> 32), epoch, 0x50415241u};
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t x[4];
  ffo_philox4x32_10(ctr, key, x);
  float rad = disc17[16] * sqrtf(u01(x[0]));
  float st, ct;
  ffo_sincos_turn24(x[1] >> 8, &st, &ct);
  v3 v = mat_vec(disc17, mk(rad * ct, rad * st, -disc17[15]));
  v3 o = add(v, ld(disc17 + 9));
  v3 e = add(o, scl(ld(disc17 + 12), 0.1f));
  ray6[0] = o.x; ray6[1] = o.y; ray6[2] = o.z;
  ray6[3] = e.x; ray6[4] = e.y; ray6[5] = e.z;
}

void ffo_emit_parallel(const float* disc17, long n_rays, uint64_t seed, uint32_t epoch, float* rays6)
{
  for (long j = 0; j < n_rays; ++j)
    ffo_emit_disc_ray(disc17, (uint64_t)j, seed, epoch, rays6 + 6 * j);
}

/* Emission + brute-force cast + per-(hit face, side) tally of
 * thermal_equation/parallel_rays_cpu.cpp:110-122: side_counts[2h] counts
 * rays with dot(triangle_normal(h), direction) < 0 (the reference's front),
 * side_counts[2h + 1] the others.  Zeroed here. */
typedef struct {
  int n_faces;
  const float* faces9;
  const float* disc;
  uint64_t seed;
  uint32_t epoch;
  long n_rays;
  uint32_t* side_counts;
} par_ctx_t;

static void par_body(long chunk, void* arg)
{
  par_ctx_t* c = (par_ctx_t*)arg;
  long b = chunk * 256, e = b + 256 < c->n_rays ? b + 256 : c->n_rays;
  for (long j = b; j < e; ++j) {
    float ray[6];
    int32_t h;
    ffo_emit_disc_ray(c->disc, (uint64_t)j, c->seed, c->epoch, ray);
    cast_one(c->n_faces, c->faces9, ray, &h, 0);
    if (h < 0)
      continue;
    const float* t = c->faces9 + 9 * (size_t)h;
    v3 p0 = ld(t);
    v3 n = cross(sub(ld(t + 3), p0), sub(ld(t + 6), p0)); /* math/triangle.cpp:114-119 */
    float side = dot(n, ld(c->disc + 12));
    __atomic_fetch_add(c->side_counts + 2 * (size_t)h + (side < 0 ? 0 : 1), 1u, __ATOMIC_RELAXED);
  }
}

void ffo_parallel_rays(int n_faces, const float* faces9, const float* disc17, long n_rays, uint64_t seed,
                       uint32_t epoch, uint32_t* side_counts)
{
  memset(side_counts, 0, sizeof(uint32_t) * 2 * (size_t)n_faces);
  par_ctx_t c = {n_faces, faces9, disc17, seed, epoch, n_rays, side_counts};
  parallel_for((n_rays + 255) / 256, 1, par_body, &c);
}

/* ------------------------------------------------------------------ */
/* Radiance equation step (thermal_equation/radiance_cpu.cpp:142-180):    */
/* a ray of face f that hits face h adds the per-ray power of f's side    */
/* to absorption[face_to_mesh[h]].  The sums are integers: each power is  */
/* rounded to 2^k units per watt, k the largest that keeps the sum of all */
/* rays' |power| below 2^62 (the fixed point of the CUDA path, so the     */
/* results compare exactly).                                              */
/* ------------------------------------------------------------------ */
typedef struct {
  int n_faces;
  const float* faces9;
  const int32_t *front, *rear;
  const long long* fixed;
  const int32_t* face_to_mesh;
  uint64_t seed;
  uint32_t epoch;
  int flags;
  long long* sums;
} rad_ctx_t;

static void rad_body(long f, void* arg)
{
  rad_ctx_t* c = (rad_ctx_t*)arg;
  float frame[18];
  ffo_face_frame(c->faces9 + 9 * (size_t)f, c->flags, frame);
  int nf = c->front[f] + c->rear[f];
  for (int j = 0; j < nf; ++j) {
    float ray[6];
    int32_t h;
    ffo_emit_ray(frame, (uint32_t)f, (uint32_t)j, c->front[f], c->seed, c->epoch, ray);
    cast_one(c->n_faces, c->faces9, ray, &h, 0);
    if (h >= 0)
      __atomic_fetch_add(c->sums + c->face_to_mesh[h], c->fixed[2 * (size_t)f + (j < c->front[f] ? 0 : 1)],
                         __ATOMIC_RELAXED);
  }
}

void ffo_radiance_absorption(int n_faces, const float* faces9, const int32_t* front, const int32_t* rear,
                             const float* power_front, const float* power_rear, const int32_t* face_to_mesh,
                             int n_meshes, uint64_t seed, uint32_t epoch, int flags, double* absorption)
{
  double bound = 0.0;
  for (int f = 0; f < n_faces; ++f)
    bound += (double)front[f] * fabs((double)power_front[f]) + (double)rear[f] * fabs((double)power_rear[f]);
  int k = 0;
  if (bound > 0.0) {
    k = (int)floor(62.0 - log2(bound));
    if (k > 1000)
      k = 1000;
  }
  long long* fixed = (long long*)malloc(sizeof(long long) * 2 * (size_t)n_faces);
  long long* sums = (long long*)calloc((size_t)n_meshes, sizeof(long long));
  for (int f = 0; f < n_faces; ++f) {
    fixed[2 * (size_t)f] = llround(ldexp((double)power_front[f], k));
    fixed[2 * (size_t)f + 1] = llround(ldexp((double)power_rear[f], k));
  }
  rad_ctx_t c = {n_faces, faces9, front, rear, fixed, face_to_mesh, seed, epoch, flags, sums};
  parallel_for(n_faces, 1, rad_body, &c);
  for (int m = 0; m < n_meshes; ++m)
    absorption[m] = ldexp((double)sums[m], -k);
  free(fixed);
  free(sums);
}

/* ------------------------------------------------------------------ */
/* Analytic view factors in double (textbook, one-sided).               */
/* Equal coaxial parallel rectangles a x b at distance c and two          */
/* perpendicular rectangles sharing an edge; the same formulas the       */
/* reference evaluates in test/form_factors.cpp:192-206 (halved there    */
/* for its two-sided emission).                                          */
/* ------------------------------------------------------------------ */
double ffo_vf_parallel(double a, double b, double c)
{
  double x = a / c, y = b / c, xq = x * x, yq = y * y;
  return 2.0 / M_PI / x / y *
         (log(sqrt((1 + xq) * (1 + yq) / (1 + xq + yq))) + x * sqrt(1 + yq) * atan(x / sqrt(1 + yq)) +
          y * sqrt(1 + xq) * atan(y / sqrt(1 + xq)) - x * atan(x) - y * atan(y));
}

double ffo_vf_perpendicular(double H, double W, double L)
{
  double h = H / L, w = W / L;
  double a = (1 + h * h) * (1 + w * w) / (1 + h * h + w * w);
  double b = w * w * (1 + h * h + w * w) / (1 + w * w) / (h * h + w * w);
  double c = h * h * (1 + h * h + w * w) / (1 + h * h) / (h * h + w * w);
  return 1.0 / M_PI / w *
         (h * atan(1 / h) + w * atan(1 / w) - sqrt(h * h + w * w) * atan(1 / sqrt(h * h + w * w)) +
          0.25 * log(a * pow(b, w * w) * pow(c, h * h)));
}
