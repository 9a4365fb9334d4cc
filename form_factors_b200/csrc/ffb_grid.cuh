// ffb_grid.cuh -- uniform 3-D grid over the scene: device build (counting
// sort of triangle references into cells) and 3-D DDA nearest-hit traversal.
//
// The reference accelerates the same query with a 2-D grid over X/Y and
// infinite Z columns (math/grid.cpp, ray_caster/zgrid_cpu.cpp:57-132).  This
// grid is a different structure with the same answer: hit index and hit point
// equal to the brute-force definition (ray_caster/naive_cpu.cpp:65-97) for
// every ray.  Three rules make that hold:
//  1. Binning is conservative.  A triangle goes into every cell that its
//     bounding box, grown by a margin, overlaps and whose box its plane (grown
//     by the same margin) crosses.  The margin covers the rounding of a
//     computed hit point, including the extra error of sliver triangles.
//  2. Hits are merged as a lexicographic minimum of (squared distance, index),
//     which equals a strict '<' scan in index order.
//  3. Traversal stops only when the best squared distance is below the squared
//     distance at which the ray leaves the current cell, reduced by twice the
//     margin; nothing in an unvisited cell can then compute a smaller one.
#pragma once

#include "ffb_device.cuh"

namespace ffb {

struct GridView {
  float3 lo, hi;        // grid box
  float3 cs;            // cell size
  float3 inv_cs;        // 1 / cell size
  int nx, ny, nz;
  float slack;          // 2 * margin, world units
  const uint32_t* __restrict__ cell_start;  // ncells + 1
  const int32_t* __restrict__ ref_tri;      // triangle index per reference
  const TriRec* __restrict__ tri;           // triangle records
  const uint8_t* __restrict__ empty_dist;   // Chebyshev distance to the nearest occupied cell, or null
};

// Ordered-integer image of a float for atomicMin/atomicMax reductions.
__device__ __forceinline__ uint32_t f2ord(float f)
{
  uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__host__ __device__ inline float ord2f(uint32_t u)
{
  uint32_t b = (u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u;
#ifdef __CUDA_ARCH__
  return __uint_as_float(b);
#else
  float f;
  memcpy(&f, &b, 4);
  return f;
#endif
}

__device__ __forceinline__ bool finite3(float3 p)
{
  return isfinite(p.x) && isfinite(p.y) && isfinite(p.z);
}

// ---------------------------------------------------------------------------
// Per-face preparation: triangle record, binning box and the scene box.
// A face that can never be hit (degenerate: n = 0; or non-finite vertices,
// whose test always yields NaN) is marked with an empty box and not binned.
// ---------------------------------------------------------------------------
__global__ void k_face_prepare(const float* __restrict__ faces9, int n_faces, TriRec* __restrict__ tri,
                               float4* __restrict__ box_lo, float4* __restrict__ box_hi,
                               uint32_t* __restrict__ scene_ord /* 6: min xyz, max xyz (ordered) */)
{
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  float3 mn = f3(INFINITY, INFINITY, INFINITY), mx = f3(-INFINITY, -INFINITY, -INFINITY);
  if (f < n_faces) {
    const float* p = faces9 + 9 * (size_t)f;
    float3 p0 = f3(p[0], p[1], p[2]), p1 = f3(p[3], p[4], p[5]), p2 = f3(p[6], p[7], p[8]);
    TriRec t = make_trirec(p0, p1, p2);
    tri[f] = t;
    bool live = finite3(p0) && finite3(p1) && finite3(p2) && !(t.q1.x == 0.f && t.q1.y == 0.f && t.q1.z == 0.f);
    // Sliver factor kappa = uu*vv/|D| = 1/sin^2(angle at p0): bounds how far
    // a computed hit point can stray from the triangle in its plane.
    float kappa = 0.f;
    float diam = 0.f;
    if (live) {
      mn = f3(fminf(fminf(p0.x, p1.x), p2.x), fminf(fminf(p0.y, p1.y), p2.y), fminf(fminf(p0.z, p1.z), p2.z));
      mx = f3(fmaxf(fmaxf(p0.x, p1.x), p2.x), fmaxf(fmaxf(p0.y, p1.y), p2.y), fmaxf(fmaxf(p0.z, p1.z), p2.z));
      float3 w = sub3(p2, p1);
      diam = sqrtf(fmaxf(fmaxf(t.q0.w, t.q2.w), dot3(w, w)));
      float D = t.q3.w;
      kappa = (D < 0.f) ? (t.q0.w * t.q2.w) / (-D) : INFINITY;
      if (!(kappa < 1e5f))
        kappa = -1.f;  // ill-conditioned: widen by the full diameter
    }
    // .w carries the face's own extra margin (world units) beyond the grid
    // margin; a negative box (lo > hi) marks a face that is never binned.
    float extra = kappa < 0.f ? diam : 16.f * 1.1920929e-07f * kappa * diam;
    if (live) {
      box_lo[f] = make_float4(mn.x, mn.y, mn.z, extra);
      box_hi[f] = make_float4(mx.x, mx.y, mx.z, 0.f);
    } else {
      box_lo[f] = make_float4(1.f, 1.f, 1.f, 0.f);
      box_hi[f] = make_float4(-1.f, -1.f, -1.f, 0.f);
    }
  }
  // block reduction of the scene box (dead faces contribute +-inf)
  __shared__ float red[6][32];
  float v[6] = {mn.x, mn.y, mn.z, -mx.x, -mx.y, -mx.z};
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    float x = v[k];
    for (int o = 16; o > 0; o >>= 1)
      x = fminf(x, __shfl_xor_sync(0xffffffffu, x, o));
    if ((threadIdx.x & 31) == 0)
      red[k][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    int nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      float x = threadIdx.x < nw ? red[k][threadIdx.x] : INFINITY;
      for (int o = 16; o > 0; o >>= 1)
        x = fminf(x, __shfl_xor_sync(0xffffffffu, x, o));
      if (threadIdx.x == 0 && x < INFINITY) {
        if (k < 3)
          atomicMin(scene_ord + k, f2ord(x));
        else
          atomicMax(scene_ord + k, f2ord(-x));
      }
    }
  }
}

// Emission frame per face (see emit_ray): p0, e1, e2 and the rotation of +z
// towards the face normal, normalised unless ref_normal is set.
__global__ void k_face_frames(const float* __restrict__ faces9, int n_faces, int ref_normal,
                              float* __restrict__ frames /* 20 per face */)
{
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= n_faces)
    return;
  const float* p = faces9 + 9 * (size_t)f;
  float3 p0 = f3(p[0], p[1], p[2]), p1 = f3(p[3], p[4], p[5]), p2 = f3(p[6], p[7], p[8]);
  float3 e1 = sub3(p1, p0), e2 = sub3(p2, p0);
  float3 n = cross3(e1, e2);
  if (!ref_normal) {
    float len = sqrtf(dot3(n, n));
    if (len > 0.f)
      n = f3(n.x / len, n.y / len, n.z / len);
  }
  float* out = frames + 20 * (size_t)f;
  out[0] = p0.x; out[1] = p0.y; out[2] = p0.z;
  out[3] = e1.x; out[4] = e1.y; out[5] = e1.z;
  out[6] = e2.x; out[7] = e2.y; out[8] = e2.z;
  rotate_towards(f3(0.f, 0.f, 1.f), n, out + 9);
  out[18] = 0.f;
  out[19] = 0.f;
}

struct BinGeom {
  float3 lo, cs, inv_cs;
  int nx, ny, nz;
  float margin;
};

// Calls fn(cell) for every cell a face is binned into.
template <class Fn>
__device__ __forceinline__ void for_each_cell(const BinGeom& g, const float* __restrict__ faces9, int f, float4 blo,
                                              float4 bhi, Fn fn)
{
  if (blo.x > bhi.x)
    return;
  float m = g.margin + blo.w;
  int i0 = max(0, (int)floorf((blo.x - m - g.lo.x) * g.inv_cs.x));
  int j0 = max(0, (int)floorf((blo.y - m - g.lo.y) * g.inv_cs.y));
  int k0 = max(0, (int)floorf((blo.z - m - g.lo.z) * g.inv_cs.z));
  int i1 = min(g.nx - 1, (int)floorf((bhi.x + m - g.lo.x) * g.inv_cs.x));
  int j1 = min(g.ny - 1, (int)floorf((bhi.y + m - g.lo.y) * g.inv_cs.y));
  int k1 = min(g.nz - 1, (int)floorf((bhi.z + m - g.lo.z) * g.inv_cs.z));
  const float* p = faces9 + 9 * (size_t)f;
  float3 p0 = f3(p[0], p[1], p[2]);
  float3 n = cross3(sub3(f3(p[3], p[4], p[5]), p0), sub3(f3(p[6], p[7], p[8]), p0));
  float nl = sqrtf(dot3(n, n));
  n = f3(n.x / nl, n.y / nl, n.z / nl);
  // plane-box test: |n.(c - p0)| <= sum |n_a| h_a + margin, checked with a
  // little extra slack for the rounding of this float test itself
  float3 h = mul3(g.cs, 0.5f);
  float reach = fabsf(n.x) * h.x + fabsf(n.y) * h.y + fabsf(n.z) * h.z + m * 1.5f;
  bool flat = (i1 - i0 + 1) * (j1 - j0 + 1) * (k1 - k0 + 1) <= 2;
  for (int k = k0; k <= k1; ++k)
    for (int j = j0; j <= j1; ++j)
      for (int i = i0; i <= i1; ++i) {
        if (!flat) {
          float3 c = f3(g.lo.x + ((float)i + 0.5f) * g.cs.x, g.lo.y + ((float)j + 0.5f) * g.cs.y,
                        g.lo.z + ((float)k + 0.5f) * g.cs.z);
          float d = fabsf(dot3(n, sub3(c, p0)));
          if (d > reach)
            continue;
        }
        fn((k * g.ny + j) * g.nx + i);
      }
}

__global__ void k_grid_count(BinGeom g, const float* __restrict__ faces9, const float4* __restrict__ box_lo,
                             const float4* __restrict__ box_hi, int n_faces, uint32_t* __restrict__ cell_count)
{
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= n_faces)
    return;
  for_each_cell(g, faces9, f, box_lo[f], box_hi[f], [&](int c) { atomicAdd(cell_count + c, 1u); });
}

__global__ void k_grid_fill(BinGeom g, const float* __restrict__ faces9, const float4* __restrict__ box_lo,
                            const float4* __restrict__ box_hi, int n_faces, const uint32_t* __restrict__ cell_start,
                            uint32_t* __restrict__ cell_fill, int32_t* __restrict__ ref_tri)
{
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= n_faces)
    return;
  for_each_cell(g, faces9, f, box_lo[f], box_hi[f], [&](int c) {
    uint32_t pos = atomicAdd(cell_fill + c, 1u);
    ref_tri[cell_start[c] + pos] = f;
  });
}

// Sorts each cell's references by triangle index (insertion sort, one thread
// per cell): the grid is then a deterministic function of the scene.
__global__ void k_cell_sort(const uint32_t* __restrict__ cell_start, int n_cells, int32_t* __restrict__ ref_tri)
{
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cells)
    return;
  uint32_t b = cell_start[c], e = cell_start[c + 1];
  for (uint32_t i = b + 1; i < e; ++i) {
    int32_t x = ref_tri[i];
    uint32_t j = i;
    while (j > b && ref_tri[j - 1] > x) {
      ref_tri[j] = ref_tri[j - 1];
      --j;
    }
    ref_tri[j] = x;
  }
}

// ---------------------------------------------------------------------------
// Exclusive scan of uint32 counts (n + 1 outputs, out[n] = total) in three
// passes: per-block sums, a single-block scan of the sums, per-block scan.
// ---------------------------------------------------------------------------
constexpr int kScanBlock = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanBlock * kScanItems;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t x, uint32_t* total)
{
  __shared__ uint32_t warp_sums[kScanBlock / 32];
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t v = x;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o)
      v += y;
  }
  if (lane == 31)
    warp_sums[w] = v;
  __syncthreads();
  if (w == 0) {
    uint32_t s = lane < kScanBlock / 32 ? warp_sums[lane] : 0u;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o)
        s += y;
    }
    if (lane < kScanBlock / 32)
      warp_sums[lane] = s;
  }
  __syncthreads();
  uint32_t before = (w > 0 ? warp_sums[w - 1] : 0u) + v - x;
  *total = warp_sums[kScanBlock / 32 - 1];
  __syncthreads();
  return before;
}

__global__ void k_scan_reduce(const uint32_t* __restrict__ in, int n, uint32_t* __restrict__ block_sums)
{
  size_t base = (size_t)blockIdx.x * kScanTile;
  uint32_t s = 0;
  for (int k = 0; k < kScanItems; ++k) {
    size_t i = base + (size_t)k * kScanBlock + threadIdx.x;
    if (i < (size_t)n)
      s += in[i];
  }
  uint32_t total;
  block_exclusive_scan(s, &total);
  if (threadIdx.x == 0)
    block_sums[blockIdx.x] = total;
}

__global__ void k_scan_sums(uint32_t* __restrict__ block_sums, int n_blocks)
{
  // one block; exclusive scan in place, looping over tiles of kScanBlock
  uint32_t carry = 0;
  for (int base = 0; base < n_blocks; base += kScanBlock) {
    int i = base + threadIdx.x;
    uint32_t x = i < n_blocks ? block_sums[i] : 0u;
    uint32_t total;
    uint32_t ex = block_exclusive_scan(x, &total);
    if (i < n_blocks)
      block_sums[i] = carry + ex;
    carry += total;
  }
}

__global__ void k_scan_apply(const uint32_t* __restrict__ in, int n, const uint32_t* __restrict__ block_offsets,
                             uint32_t* __restrict__ out)
{
  __shared__ uint32_t tile[kScanTile];
  size_t base = (size_t)blockIdx.x * kScanTile;
  for (int k = 0; k < kScanItems; ++k) {
    size_t i = base + (size_t)k * kScanBlock + threadIdx.x;
    tile[k * kScanBlock + threadIdx.x] = i < (size_t)n ? in[i] : 0u;
  }
  __syncthreads();
  // each thread owns kScanItems consecutive items
  uint32_t local[kScanItems];
  uint32_t s = 0;
  for (int k = 0; k < kScanItems; ++k) {
    local[k] = tile[threadIdx.x * kScanItems + k];
    s += local[k];
  }
  uint32_t total;
  uint32_t ex = block_exclusive_scan(s, &total) + block_offsets[blockIdx.x];
  for (int k = 0; k < kScanItems; ++k) {
    size_t i = base + (size_t)threadIdx.x * kScanItems + k;
    if (i < (size_t)n)
      out[i] = ex;
    ex += local[k];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == kScanBlock - 1)
    out[n] = ex;  // grand total: the last thread's running sum covers the tail
}

// ---------------------------------------------------------------------------
// Empty-space distance: for each cell, the Chebyshev distance (in cells) to
// the nearest occupied cell, saturated at kEmptyCap.  The L-infinity distance
// transform is separable: pass a computes new[i] = min_j max(|i-j|, old[j])
// along axis a, starting from 0 (occupied) / kEmptyCap (empty).  A saturated
// value under-states the distance, which only shortens a jump.
// ---------------------------------------------------------------------------
constexpr int kEmptyCap = 32;
constexpr int kMaxDim = 256;

__global__ void k_empty_init(const uint32_t* __restrict__ cell_start, int n_cells, uint8_t* __restrict__ d)
{
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < n_cells)
    d[c] = cell_start[c + 1] > cell_start[c] ? 0 : kEmptyCap;
}

__global__ void k_empty_pass(uint8_t* __restrict__ d, int nx, int ny, int nz, int axis)
{
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int n_len, stride, base;
  if (axis == 0) {
    if (t >= ny * nz) return;
    n_len = nx; stride = 1; base = t * nx;
  } else if (axis == 1) {
    if (t >= nx * nz) return;
    int i = t % nx, k = t / nx;
    n_len = ny; stride = nx; base = k * nx * ny + i;
  } else {
    if (t >= nx * ny) return;
    n_len = nz; stride = nx * ny; base = t;
  }
  uint8_t buf[kMaxDim];
  for (int i = 0; i < n_len; ++i)
    buf[i] = d[base + i * stride];
  for (int i = 0; i < n_len; ++i) {
    int best = buf[i];
    for (int r = 1; r < best; ++r) {
      int v = kEmptyCap;
      if (i - r >= 0) v = min(v, (int)buf[i - r]);
      if (i + r < n_len) v = min(v, (int)buf[i + r]);
      best = min(best, max(r, v));
    }
    d[base + i * stride] = (uint8_t)best;
  }
}

// ---------------------------------------------------------------------------
// Nearest hit through the grid.  Returns the face index or -1 and writes the
// hit point of the reference's test for a hit.
// ---------------------------------------------------------------------------
// Parameter at which the ray reaches a cell boundary; NaN (a zero times an
// infinite inverse) becomes +inf so that a broken axis is never stepped.
__device__ __forceinline__ float boundary_t(float lo, int edge, float cs, float o, float inv)
{
  float t = (lo + (float)edge * cs - o) * inv;
  return t == t ? t : INFINITY;
}

template <bool kSkip>
__device__ __forceinline__ int trace_grid(const GridView& g, float3 o, float3 e, float3& hit_pt, uint32_t& n_tests,
                                          uint32_t& n_cells)
{
  const float3 dir = sub3(e, o);
  float t0 = 0.f, t1 = INFINITY;
  float inv[3];
  const float oo[3] = {o.x, o.y, o.z};
  const float dd[3] = {dir.x, dir.y, dir.z};
  const float lo[3] = {g.lo.x, g.lo.y, g.lo.z};
  const float hi[3] = {g.hi.x, g.hi.y, g.hi.z};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (dd[a] == 0.f) {
      inv[a] = INFINITY;
      if (!(oo[a] >= lo[a] && oo[a] <= hi[a]))
        return -1;
    } else {
      inv[a] = 1.f / dd[a];
      float ta = (lo[a] - oo[a]) * inv[a], tb = (hi[a] - oo[a]) * inv[a];
      t0 = fmaxf(t0, fminf(ta, tb));
      t1 = fminf(t1, fmaxf(ta, tb));
    }
  }
  if (!(t0 <= t1))
    return -1;
  const float cs[3] = {g.cs.x, g.cs.y, g.cs.z};
  const float ics[3] = {g.inv_cs.x, g.inv_cs.y, g.inv_cs.z};
  const int nn[3] = {g.nx, g.ny, g.nz};
  int c[3], st[3];
  float tn[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float p = oo[a] + t0 * dd[a];
    int ci = (int)floorf((p - lo[a]) * ics[a]);
    c[a] = min(max(ci, 0), nn[a] - 1);
    st[a] = dd[a] > 0.f ? 1 : (dd[a] < 0.f ? -1 : 0);
    tn[a] = st[a] == 0 ? INFINITY : boundary_t(lo[a], c[a] + (st[a] > 0), cs[a], oo[a], inv[a]);
  }
  const float dlen = sqrtf(dot3(dir, dir));
  float best = 3.40282347e+38f;  // FLT_MAX, the reference's starting distance
  int best_idx = -1;
  float3 best_pt = f3(0.f, 0.f, 0.f);
  const int max_iter = g.nx + g.ny + g.nz + 4;
  for (int it = 0; it < max_iter; ++it) {
    const int cell = (c[2] * g.ny + c[1]) * g.nx + c[0];
    ++n_cells;
    int jump = 0;
    if (kSkip)
      jump = g.empty_dist[cell];
    if (!kSkip || jump == 0) {
      const uint32_t b = g.cell_start[cell], en = g.cell_start[cell + 1];
      for (uint32_t i = b; i < en; ++i) {
        const int f = g.ref_tri[i];
        float3 pt;
        ++n_tests;
        if (tri_hit(reinterpret_cast<const float4*>(g.tri + f), o, dir, pt)) {
          const float d = dist2(pt, o);
          if (d < best || (d == best && f < best_idx)) {
            best = d;
            best_idx = f;
            best_pt = pt;
          }
        }
      }
    }
    const float tx = fminf(fminf(tn[0], tn[1]), tn[2]);
    if (best_idx >= 0) {
      const float L = fminf(tx, t1) * dlen - g.slack;
      if (L > 0.f && best < L * L)
        break;
    }
    if (!(tx < t1))
      break;
    if (kSkip && jump >= 2) {
      // every cell within Chebyshev distance jump-1 is empty: leave that cube
      float tj = INFINITY;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        if (st[a] != 0) {
          int edge = st[a] > 0 ? c[a] + jump : c[a] - jump + 1;
          tj = fminf(tj, boundary_t(lo[a], edge, cs[a], oo[a], inv[a]));
        }
      }
      if (!(tj < t1))
        break;
      int nc[3];
      bool moved = false;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        float p = oo[a] + tj * dd[a];
        int ci = (int)floorf((p - lo[a]) * ics[a]);
        // never move against the ray or beyond the cube
        if (st[a] > 0) ci = min(max(ci, c[a]), c[a] + jump);
        else if (st[a] < 0) ci = max(min(ci, c[a]), c[a] - jump);
        else ci = c[a];
        nc[a] = ci;
        moved |= ci != c[a];
      }
      if (moved) {
        bool out = false;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          c[a] = nc[a];
          out |= c[a] < 0 || c[a] >= nn[a];
          tn[a] = st[a] == 0 ? INFINITY : boundary_t(lo[a], c[a] + (st[a] > 0), cs[a], oo[a], inv[a]);
        }
        if (out)
          break;
        continue;
      }
    }
    // one DDA step along the axis whose boundary comes first
    int a = (tn[0] <= tn[1] && tn[0] <= tn[2]) ? 0 : (tn[1] <= tn[2] ? 1 : 2);
    if (st[a] == 0)
      break;
    c[a] += st[a];
    if (c[a] < 0 || c[a] >= nn[a])
      break;
    tn[a] = boundary_t(lo[a], c[a] + (st[a] > 0), cs[a], oo[a], inv[a]);
  }
  if (best_idx >= 0)
    hit_pt = best_pt;
  return best_idx;
}

}  // namespace ffb
