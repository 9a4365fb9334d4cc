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
//     distance at which the ray leaves the current cell (or the empty cube
//     it jumps across), reduced by twice the margin; nothing in an unvisited
//     cell can then compute a smaller one.
#pragma once

#include "ffb_device.cuh"

namespace ffb {

struct GridView {
  float3 lo, hi;        // grid box
  float3 cs;            // cell size
  float3 inv_cs;        // 1 / cell size
  int nx, ny, nz;
  float slack;          // 2 * margin, world units
  const int32_t* __restrict__ ref_tri;      // triangle index per reference
  const TriRec* __restrict__ ref_rec;       // triangle record per reference (a copy of tri[ref_tri[i]])
  const uint2* __restrict__ cell_rec;       // per cell: {start, end} of its references, or {0, kCellEmpty | jump}
};

// Packed cell record: an occupied cell holds {first reference, end}; an
// empty one {0, kCellEmpty | d} with d its empty-space distance (1 when the
// grid has no distance map).  One 8-byte load replaces the distance byte and
// the two offsets.
constexpr uint32_t kCellEmpty = 0x80000000u;

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
  // Edge axes of the separating-axis test: edge x unit axis, for the three
  // edges.  Each axis is an exact float vector (a permutation of an edge's
  // components), so only the projections round.  The cell grown by the
  // margin on every axis, as the box range above grows it, reaches
  // r = sum (h_a + m) |A_a| along axis A; a further 0.5 m per axis covers
  // the rounding of the projections (coordinates relative to p0).  An axis
  // that separates the triangle from the grown cell proves that no hit point
  // computed on the triangle can land in the cell.
  const float3 ed[3] = {sub3(f3(p[3], p[4], p[5]), p0), sub3(f3(p[6], p[7], p[8]), f3(p[3], p[4], p[5])),
                        sub3(p0, f3(p[6], p[7], p[8]))};
  const float3 q1 = ed[0], q2 = sub3(f3(p[6], p[7], p[8]), p0);  // vertices relative to p0 (q0 = 0)
  const float3 hm = f3(h.x + 1.5f * m, h.y + 1.5f * m, h.z + 1.5f * m);
  float ax_lo[9], ax_hi[9], ax_r[9];
#pragma unroll
  for (int e = 0; e < 3; ++e) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float3 A = a == 0 ? f3(0.f, ed[e].z, -ed[e].y) : (a == 1 ? f3(-ed[e].z, 0.f, ed[e].x)
                                                                     : f3(ed[e].y, -ed[e].x, 0.f));
      const float v1 = dot3(q1, A), v2 = dot3(q2, A);
      ax_lo[3 * e + a] = fminf(0.f, fminf(v1, v2));
      ax_hi[3 * e + a] = fmaxf(0.f, fmaxf(v1, v2));
      ax_r[3 * e + a] = fabsf(A.x) * hm.x + fabsf(A.y) * hm.y + fabsf(A.z) * hm.z;
    }
  }
  for (int k = k0; k <= k1; ++k)
    for (int j = j0; j <= j1; ++j)
      for (int i = i0; i <= i1; ++i) {
        if (!flat) {
          float3 c = f3(g.lo.x + ((float)i + 0.5f) * g.cs.x, g.lo.y + ((float)j + 0.5f) * g.cs.y,
                        g.lo.z + ((float)k + 0.5f) * g.cs.z);
          const float3 dc = sub3(c, p0);
          float d = fabsf(dot3(n, dc));
          if (d > reach)
            continue;
          bool sep = false;
#pragma unroll
          for (int e = 0; e < 3; ++e) {
#pragma unroll
            for (int a = 0; a < 3; ++a) {
              const float3 A = a == 0 ? f3(0.f, ed[e].z, -ed[e].y) : (a == 1 ? f3(-ed[e].z, 0.f, ed[e].x)
                                                                             : f3(ed[e].y, -ed[e].x, 0.f));
              const float pc = dot3(dc, A);
              sep |= (ax_lo[3 * e + a] > pc + ax_r[3 * e + a]) | (ax_hi[3 * e + a] < pc - ax_r[3 * e + a]);
            }
          }
          if (sep)
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

// Counts the faces with a non-empty binning box (the grid's live faces):
// one atomic per warp.
__global__ void k_count_live(const float4* __restrict__ box_lo, const float4* __restrict__ box_hi, int n_faces,
                             uint32_t* __restrict__ live)
{
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  const bool ok = f < n_faces && box_lo[f].x <= box_hi[f].x;
  const unsigned m = __ballot_sync(0xFFFFFFFFu, ok);
  if ((threadIdx.x & 31) == 0 && m)
    atomicAdd(live, (uint32_t)__popc(m));
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

// Per-reference copy of the triangle records: a cell's candidates are
// contiguous and a test needs no index load before its record.
__global__ void k_ref_gather(const int32_t* __restrict__ ref_tri, uint32_t n_refs, const TriRec* __restrict__ tri,
                             TriRec* __restrict__ ref_rec)
{
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_refs; i += gridDim.x * blockDim.x)
    ref_rec[i] = tri[ref_tri[i]];
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
// Empty-space distance per octant.  For each empty cell and each of the 8
// octants of ray directions, the largest k such that the cube of k x k x k
// cells with the cell at its corner, extending from it in the octant's
// directions, holds no reference: the L-infinity distance to the nearest
// occupied cell lying in that octant of the cell.  A ray whose direction
// lies in the octant leaves the cube only through its far faces, so it jumps
// to them (tracer_advance); occupied cells behind the ray do not shorten the
// jump.  The transform is separable: pass a computes, along axis a and in
// each direction, new[i] = min_{r >= 0} max(r, old[i + r*s]), starting from
// 0 (occupied) / kEmptyCap (empty), in one linear scan per line.  Octant o has bit a set when it points
// down axis a.  A saturated value under-states the distance, which only
// shortens a jump.
// ---------------------------------------------------------------------------
#ifndef FFB_EMPTY_CAP
#define FFB_EMPTY_CAP 127
#endif
constexpr int kEmptyCap = FFB_EMPTY_CAP;  // at most 127: 7 bits per octant in the cell record
static_assert(kEmptyCap >= 1 && kEmptyCap <= 127, "octant distances are 7-bit fields");
constexpr int kOctants = 8;
constexpr int kMaxDim = 256;

__global__ void k_empty_init(const uint32_t* __restrict__ cell_start, int n_cells, uint8_t* __restrict__ d)
{
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < n_cells)
    d[c] = cell_start[c + 1] > cell_start[c] ? 0 : kEmptyCap;
}

// One pass along `axis`: octant slot blockIdx.y (< 2^axis, the octants of
// the axes before) holds the input; the positive direction is written back
// in place and the negative one to slot blockIdx.y | 2^axis.  One thread per
// line of cells; slots are n_cells bytes apart.
__global__ void k_empty_pass(uint8_t* __restrict__ d, long long n_cells, int nx, int ny, int nz, int axis)
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
  uint8_t* in = d + (size_t)blockIdx.y * n_cells;
  uint8_t* neg = d + (size_t)(blockIdx.y | (1u << axis)) * n_cells;
  uint8_t buf[kMaxDim];
  for (int i = 0; i < n_len; ++i)
    buf[i] = in[base + i * stride];
  // Linear scan against the direction.  With G the value one step ahead,
  // the new value is min(w, G) when a position within G steps ahead holds
  // G, else min(w, G + 1): the positions within G steps all hold at least
  // G.  last[v] is the scan index of the nearest position seen holding v.
  int16_t last[kEmptyCap + 1];
  for (int dir = 0; dir < 2; ++dir) {  // 0: positive direction (in place), 1: negative
    uint8_t* out = dir ? neg : in;
    for (int v = 0; v <= kEmptyCap; ++v)
      last[v] = -32768;
    int G = kEmptyCap;
    for (int k = 0; k < n_len; ++k) {
      const int i = dir ? k : n_len - 1 - k;
      const int w = buf[i];
      int h = kEmptyCap;
      if (k > 0)
        h = (G < kEmptyCap && k - last[G] <= G) ? G : min(G + 1, kEmptyCap);
      const int g = min(w, h);
      out[base + i * stride] = (uint8_t)g;
      last[w] = (int16_t)k;
      G = g;
    }
  }
}

// Packs the cell records: occupied {start, end}; empty {octants 0-3, flag |
// octants 4-7}, one byte per octant (octant o in byte o & 3).  Without a
// distance map every octant distance is 1 (single DDA steps).
__global__ void k_cell_rec(const uint32_t* __restrict__ cell_start, const uint8_t* __restrict__ empty_dist,
                           long long n_cells, uint2* __restrict__ rec)
{
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n_cells;
       c += (long long)gridDim.x * blockDim.x) {
    const uint32_t b = cell_start[c], e = cell_start[c + 1];
    if (e > b) {
      rec[c] = make_uint2(b, e);
      continue;
    }
    uint32_t w[2] = {0x01010101u, 0x01010101u};
    if (empty_dist) {
      w[0] = w[1] = 0;
#pragma unroll
      for (int o = 0; o < kOctants; ++o)
        w[o >> 2] |= (uint32_t)empty_dist[(size_t)o * n_cells + c] << (8 * (o & 3));
    }
    rec[c] = make_uint2(w[0], kCellEmpty | w[1]);
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

// Slab clip of the ray o + t*d, t >= 0, against [lo, hi] on one axis.
__device__ __forceinline__ bool slab(float d, float o, float lo, float hi, float& inv, float& t0, float& t1)
{
  if (d == 0.f) {
    inv = INFINITY;
    return o >= lo && o <= hi;
  }
  inv = 1.f / d;
  const float ta = (lo - o) * inv, tb = (hi - o) * inv;
  t0 = fmaxf(t0, fminf(ta, tb));
  t1 = fminf(t1, fmaxf(ta, tb));
  return true;
}

__device__ __forceinline__ int cell_of(float p, float lo, float ics, int n)
{
  return min(max((int)floorf((p - lo) * ics), 0), n - 1);
}

__device__ __forceinline__ int sgn(float d) { return d > 0.f ? 1 : (d < 0.f ? -1 : 0); }

// Next boundary parameter on an axis for cell c and step s (inf when s == 0).
__device__ __forceinline__ float next_t(int s, int c, float lo, float cs, float o, float inv)
{
  return s == 0 ? INFINITY : boundary_t(lo, c + (s > 0), cs, o, inv);
}

// Landing cell on one axis after a jump to parameter tj: never against the
// ray, never beyond the far face of the empty cube of `jump` cells per side.
__device__ __forceinline__ int land(int s, int c, int jump, float o, float d, float tj, float lo, float ics)
{
  if (s == 0)
    return c;
  const int ci = (int)floorf(((o + tj * d) - lo) * ics);
  return s > 0 ? min(max(ci, c), c + jump) : max(min(ci, c), c - jump);
}

// ---------------------------------------------------------------------------
// Nearest hit through the grid as a per-lane state machine.  One call does
// one unit of work: test one triangle reference of the current cell, or (when
// the cell is exhausted) decide termination and move to the next cell or jump
// over empty space.  Lanes of a warp stay in step whatever the cell
// occupancy, and a lane whose ray finishes can start another ray at once
// (persistent refill).
//
// Stopping rule: after a cell, stop when the best squared distance is below
// the squared distance at which the ray leaves that cell (or the empty cube
// it is about to cross), reduced by twice the binning margin; any triangle
// not yet tested lies in unvisited cells and cannot compute a smaller
// distance.
// ---------------------------------------------------------------------------
struct Tracer {
  float3 o, dir, inv;
  float dlen, best;
  float3 best_pt;
  int cx, cy, cz;
  int best_ref;      // reference (position in ref_tri) of the best hit, -1 if none
  int jump;          // empty-space distance of the current cell
  uint32_t i, en;    // pending references of the current cell
  int sx, sy, sz;    // signs of the direction
};

template <bool kSkip>
__device__ __forceinline__ void tracer_enter(Tracer& T, const GridView& g)
{
  const int cell = (T.cz * g.ny + T.cy) * g.nx + T.cx;
  const uint2 r = __ldg(g.cell_rec + cell);
  const bool empty = (r.y & kCellEmpty) != 0;
  if (kSkip) {
    // the distance of the octant of the ray's direction
    const uint32_t w = T.dir.z < 0.f ? r.y : r.x;
    const int sh = (T.dir.x < 0.f ? 8 : 0) + (T.dir.y < 0.f ? 16 : 0);
    T.jump = empty ? (int)((w >> sh) & 0x7Fu) : 0;
  } else {
    T.jump = 0;
  }
  T.i = r.x;
  T.en = empty ? 0u : r.y;
}

// Sets up a ray; false when it misses the grid box (no hit possible).
template <bool kSkip>
__device__ __forceinline__ bool tracer_begin(Tracer& T, const GridView& g, float3 o, float3 e, uint32_t& n_cells)
{
  T.o = o;
  T.dir = sub3(e, o);
  float t0 = 0.f;
  float t1 = INFINITY;
  T.sx = sgn(T.dir.x);
  T.sy = sgn(T.dir.y);
  T.sz = sgn(T.dir.z);
  if (!slab(T.dir.x, o.x, g.lo.x, g.hi.x, T.inv.x, t0, t1) || !slab(T.dir.y, o.y, g.lo.y, g.hi.y, T.inv.y, t0, t1) ||
      !slab(T.dir.z, o.z, g.lo.z, g.hi.z, T.inv.z, t0, t1) || !(t0 <= t1))
    return false;
  T.cx = cell_of(o.x + t0 * T.dir.x, g.lo.x, g.inv_cs.x, g.nx);
  T.cy = cell_of(o.y + t0 * T.dir.y, g.lo.y, g.inv_cs.y, g.ny);
  T.cz = cell_of(o.z + t0 * T.dir.z, g.lo.z, g.inv_cs.z, g.nz);
  T.dlen = sqrtf(dot3(T.dir, T.dir));
  T.best = 3.40282347e+38f;  // FLT_MAX, the reference's starting distance
  T.best_ref = -1;
  ++n_cells;
  tracer_enter<kSkip>(T, g);
  return true;
}

// Tests the next pending reference of the current cell and merges a hit
// into (best, best_ref, best_pt): the smallest squared distance wins and,
// among equal distances, the lowest face index, which equals the reference's
// strict '<' scan in index order.
__device__ __forceinline__ void tracer_test(Tracer& T, const GridView& g, uint32_t& n_tests)
{
  const uint32_t i = T.i++;
  ++n_tests;
  const float4* rec = reinterpret_cast<const float4*>(g.ref_rec + i);
  float3 pt;
  if (tri_hit_regs(__ldg(rec), __ldg(rec + 1), __ldg(rec + 2), __ldg(rec + 3), T.o, T.dir, pt)) {
    const float d = dist2(pt, T.o);
    if (d < T.best) {
      T.best = d;
      T.best_ref = (int)i;
      T.best_pt = pt;
    } else if (d == T.best && T.best_ref >= 0) {
      // equal distance: the lower face index wins (a repeated reference of
      // the same face compares equal and changes nothing)
      if (__ldg(g.ref_tri + i) < __ldg(g.ref_tri + T.best_ref)) {
        T.best_ref = (int)i;
        T.best_pt = pt;
      }
    }
  }
}

// Face index of the finished ray's nearest hit, or -1.
__device__ __forceinline__ int tracer_result(const Tracer& T, const GridView& g)
{
  return T.best_ref >= 0 ? __ldg(g.ref_tri + T.best_ref) : -1;
}

// The current cell is exhausted: stop, or move to the next cell.  Returns
// false when the ray is finished.
//
// Every move leaves the empty cube of `jump` cells per side that extends
// from the cell in the octant of the ray's direction (the cell itself when
// jump <= 1: an occupied cell, or a plain DDA step).  The ray starts inside
// the cube and moves monotonically, so it leaves through a far face, at tj,
// and lands in the cell where it crosses that face.  A diagonal landing skips
// only cells that the ray touches within rounding of the landing cell, whose
// triangles the binning margin puts into the landing cell as well.  Lanes
// that step and lanes that jump run the same instructions.  Every move
// advances at least one cell coordinate in the ray's direction (landings are
// clamped monotone, and a landing that rounds back becomes a step), so a ray
// leaves the grid after at most nx + ny + nz moves.
//
// Stopping rule, checked before the move: every reference whose computed
// hit lies before tj, less twice the margin, is in a visited cell (the cube
// holds none, and nothing lies outside the grid), so a best hit closer than
// that is final.  A ray that leaves the grid lands outside it and stops at
// the bounds check.
template <bool kSkip>
__device__ __forceinline__ bool tracer_advance(Tracer& T, const GridView& g, uint32_t& n_cells, uint32_t& n_jumps)
{
  const int sx = T.sx, sy = T.sy, sz = T.sz;
  const int jump = max(T.jump, 1);
  float ex = sx ? boundary_t(g.lo.x, sx > 0 ? T.cx + jump : T.cx - jump + 1, g.cs.x, T.o.x, T.inv.x) : INFINITY;
  float ey = sy ? boundary_t(g.lo.y, sy > 0 ? T.cy + jump : T.cy - jump + 1, g.cs.y, T.o.y, T.inv.y) : INFINITY;
  float ez = sz ? boundary_t(g.lo.z, sz > 0 ? T.cz + jump : T.cz - jump + 1, g.cs.z, T.o.z, T.inv.z) : INFINITY;
  const float tj = fminf(fminf(ex, ey), ez);
  if (T.best_ref >= 0) {
    const float L = tj * T.dlen - g.slack;
    if (L > 0.f && T.best < L * L)
      return false;
  }
  if (!(tj < INFINITY))
    return false;
  int nx = land(sx, T.cx, jump, T.o.x, T.dir.x, tj, g.lo.x, g.inv_cs.x);
  int ny = land(sy, T.cy, jump, T.o.y, T.dir.y, tj, g.lo.y, g.inv_cs.y);
  int nz = land(sz, T.cz, jump, T.o.z, T.dir.z, tj, g.lo.z, g.inv_cs.z);
  if (nx == T.cx && ny == T.cy && nz == T.cz) {
    // The landing point rounded back into the cell: one DDA step along the
    // axis whose cell boundary the ray reaches first.  With jump 1 the cube
    // exits are those boundaries; a longer jump lands in another cell unless
    // rounding exceeds a cell, and then the cell's own boundaries decide.
    if (jump > 1) {
      ex = next_t(sx, T.cx, g.lo.x, g.cs.x, T.o.x, T.inv.x);
      ey = next_t(sy, T.cy, g.lo.y, g.cs.y, T.o.y, T.inv.y);
      ez = next_t(sz, T.cz, g.lo.z, g.cs.z, T.o.z, T.inv.z);
    }
    const bool ax = ex <= ey && ex <= ez;
    const bool ay = !ax && ey <= ez;
    nx += ax ? sx : 0;
    ny += ay ? sy : 0;
    nz += (ax || ay) ? 0 : sz;
  }
  if ((unsigned)nx >= (unsigned)g.nx || (unsigned)ny >= (unsigned)g.ny || (unsigned)nz >= (unsigned)g.nz)
    return false;
  n_jumps += jump >= 2;
  T.cx = nx;
  T.cy = ny;
  T.cz = nz;
  ++n_cells;
  tracer_enter<kSkip>(T, g);
  return true;
}

}  // namespace ffb
