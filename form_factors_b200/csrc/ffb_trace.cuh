// ffb_trace.cuh -- the hot kernels: fused emission + nearest-hit trace +
// per-source histogram (form-factor counts), ray-batch casts (grid and brute
// force) and ray materialisation.
#pragma once

#include "ffb_grid.cuh"

namespace ffb {

// A unit of work of the fused kernel: `count` consecutive rays [j0, j0+count)
// of one face.  Rays j < front leave the front side, the others the rear.
struct Chunk {
  int32_t face;
  int32_t j0;
  int32_t count;
  int32_t front;
};

// Statistics slots (uint64 each), accumulated once per block.
enum { kStatTests = 0, kStatCells = 1, kStatRays = 2, kStatHits = 3, kStatSlots = 4 };

struct TraceParams {
  GridView g;
  const float* __restrict__ frames;          // 20 floats per face
  const Chunk* __restrict__ chunks;
  int n_chunks;
  const int32_t* __restrict__ face_to_row;   // face -> matrix row/column (mesh), or null for identity
  int n_cols;                                 // matrix side
  uint32_t* __restrict__ counts;              // n_cols * n_cols
  uint32_t key0, key1, epoch;
  uint32_t* __restrict__ chunk_cursor;        // work counter, zero before the launch
  unsigned long long* __restrict__ stats;     // kStatSlots, or null
  int hash_cap;                               // hash mode: slots (power of two)
};

constexpr int kTraceThreads = 128;

__device__ __forceinline__ void block_stats(unsigned long long* stats, uint32_t tests, uint32_t cells,
                                            uint32_t rays, uint32_t hits)
{
  if (!stats)
    return;
  unsigned long long v[4] = {tests, cells, rays, hits};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    unsigned long long x = v[k];
    for (int o = 16; o > 0; o >>= 1)
      x += __shfl_xor_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0 && x)
      atomicAdd(stats + k, x);
  }
}

__device__ __forceinline__ uint32_t hash_slot(int key, int cap)
{
  return ((uint32_t)key * 2654435761u) & (uint32_t)(cap - 1);
}

// ---------------------------------------------------------------------------
// Fused form-factor kernel.  Persistent blocks take chunks from a global
// cursor.  For each chunk the block generates its rays (Philox, keyed by
// seed/epoch/face/j), traces them through the grid and counts hit columns in
// a shared-memory histogram of the chunk's source row, then flushes the
// non-zero bins to the global uint32 matrix with atomic adds (several chunks
// may share a row).  kHash selects an open-addressing table (keys = column)
// for matrices too wide for a dense shared-memory row.
// ---------------------------------------------------------------------------
template <bool kHash, bool kSkip>
__global__ void __launch_bounds__(kTraceThreads) k_form_factors(TraceParams p)
{
  extern __shared__ uint32_t smem[];
  __shared__ int s_chunk;
  uint32_t* hist = smem;                                  // dense: n_cols bins
  int* keys = reinterpret_cast<int*>(smem);               // hash: hash_cap keys
  uint32_t* vals = smem + (kHash ? p.hash_cap : 0);       // hash: hash_cap values
  const int bins = kHash ? p.hash_cap : p.n_cols;
  for (int i = threadIdx.x; i < bins; i += blockDim.x) {
    if (kHash) {
      keys[i] = -1;
      vals[i] = 0;
    } else {
      hist[i] = 0;
    }
  }
  uint32_t n_tests = 0, n_cells = 0, n_rays = 0, n_hits = 0;
  for (;;) {
    if (threadIdx.x == 0)
      s_chunk = (int)atomicAdd(p.chunk_cursor, 1u);
    __syncthreads();
    const int k = s_chunk;
    if (k >= p.n_chunks)
      break;
    const Chunk ch = p.chunks[k];
    const float* fr = p.frames + 20 * (size_t)ch.face;
    float frame[18];
#pragma unroll
    for (int e = 0; e < 18; ++e)
      frame[e] = __ldg(fr + e);
    const int row = p.face_to_row ? __ldg(p.face_to_row + ch.face) : ch.face;
    for (int j = ch.j0 + threadIdx.x; j < ch.j0 + ch.count; j += blockDim.x) {
      float3 o, e;
      emit_ray(frame, (uint32_t)ch.face, (uint32_t)j, ch.front, p.key0, p.key1, p.epoch, o, e);
      float3 pt;
      const int h = trace_grid<kSkip>(p.g, o, e, pt, n_tests, n_cells);
      ++n_rays;
      if (h >= 0) {
        ++n_hits;
        const int col = p.face_to_row ? __ldg(p.face_to_row + h) : h;
        if (!kHash) {
          atomicAdd(hist + col, 1u);
        } else {
          uint32_t s = hash_slot(col, p.hash_cap);
          bool done = false;
          for (int probe = 0; probe < p.hash_cap; ++probe) {
            int cur = keys[s];
            if (cur == -1)
              cur = atomicCAS(keys + s, -1, col);
            if (cur == -1 || cur == col) {
              atomicAdd(vals + s, 1u);
              done = true;
              break;
            }
            s = (s + 1) & (uint32_t)(p.hash_cap - 1);
          }
          if (!done)  // table full (not reachable with cap >= 2 * chunk rays)
            atomicAdd(p.counts + (size_t)row * p.n_cols + col, 1u);
        }
      }
    }
    __syncthreads();
    uint32_t* out_row = p.counts + (size_t)row * p.n_cols;
    for (int i = threadIdx.x; i < bins; i += blockDim.x) {
      if (kHash) {
        const int key = keys[i];
        if (key >= 0) {
          atomicAdd(out_row + key, vals[i]);
          keys[i] = -1;
          vals[i] = 0;
        }
      } else {
        const uint32_t v = hist[i];
        if (v) {
          atomicAdd(out_row + i, v);
          hist[i] = 0;
        }
      }
    }
    __syncthreads();
  }
  block_stats(p.stats, n_tests, n_cells, n_rays, n_hits);
}

// ---------------------------------------------------------------------------
// Ray-batch cast through the grid (the ray_caster interface): rays are
// {origin, end point} as in math::ray_t.  hit_face gets the face index or -1;
// hit_point (optional) gets the point, NaN for a miss.
// ---------------------------------------------------------------------------
template <bool kSkip>
__global__ void __launch_bounds__(kTraceThreads) k_cast(GridView g, const float* __restrict__ rays6, long n_rays,
                                                         int32_t* __restrict__ hit_face, float* __restrict__ hit_point,
                                                         unsigned long long* __restrict__ stats)
{
  uint32_t n_tests = 0, n_cells = 0, n_done = 0, n_hits = 0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n_rays; i += (long)gridDim.x * blockDim.x) {
    const float* r = rays6 + 6 * i;
    const float3 o = f3(__ldg(r + 0), __ldg(r + 1), __ldg(r + 2));
    const float3 e = f3(__ldg(r + 3), __ldg(r + 4), __ldg(r + 5));
    float3 pt = f3(NAN, NAN, NAN);
    const int h = trace_grid<kSkip>(g, o, e, pt, n_tests, n_cells);
    hit_face[i] = h;
    if (hit_point) {
      if (h < 0)
        pt = f3(NAN, NAN, NAN);
      hit_point[3 * i + 0] = pt.x;
      hit_point[3 * i + 1] = pt.y;
      hit_point[3 * i + 2] = pt.z;
    }
    ++n_done;
    n_hits += h >= 0;
  }
  block_stats(stats, n_tests, n_cells, n_done, n_hits);
}

// Brute force: every ray against every face (the naive_cpu definition),
// faces staged through shared memory in tiles.
constexpr int kBruteTile = 128;

__global__ void __launch_bounds__(kTraceThreads) k_cast_brute(const TriRec* __restrict__ tri, int n_faces,
                                                               const float* __restrict__ rays6, long n_rays,
                                                               int32_t* __restrict__ hit_face,
                                                               float* __restrict__ hit_point)
{
  __shared__ TriRec tile[kBruteTile];
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = i < n_rays;
  float3 o = f3(0.f, 0.f, 0.f), e = f3(0.f, 0.f, 0.f);
  if (live) {
    const float* r = rays6 + 6 * i;
    o = f3(r[0], r[1], r[2]);
    e = f3(r[3], r[4], r[5]);
  }
  const float3 dir = sub3(e, o);
  float best = 3.40282347e+38f;
  int best_idx = -1;
  float3 best_pt = f3(NAN, NAN, NAN);
  for (int base = 0; base < n_faces; base += kBruteTile) {
    __syncthreads();
    for (int k = threadIdx.x; k < kBruteTile && base + k < n_faces; k += blockDim.x)
      tile[k] = tri[base + k];
    __syncthreads();
    const int m = min(kBruteTile, n_faces - base);
    if (live) {
      for (int k = 0; k < m; ++k) {
        float3 pt;
        const float4* rec = reinterpret_cast<const float4*>(tile + k);
        // shared-memory copy of tri_hit (no __ldg on shared memory)
        const float4 q0 = rec[0], q1 = rec[1];
        float3 w0 = f3(o.x - q0.x, o.y - q0.y, o.z - q0.z);
        float a = -(q1.x * w0.x + q1.y * w0.y + q1.z * w0.z);
        float b = q1.x * dir.x + q1.y * dir.y + q1.z * dir.z;
        if (fabsf(b) < FFB_EPS_ABOVE_1E8)
          continue;
        float r = a / b;
        if (r < 0.f)
          continue;
        pt = f3(o.x + r * dir.x, o.y + r * dir.y, o.z + r * dir.z);
        const float4 q2 = rec[2], q3 = rec[3];
        float3 w = f3(pt.x - q0.x, pt.y - q0.y, pt.z - q0.z);
        float wu = w.x * q2.x + w.y * q2.y + w.z * q2.z;
        float wv = w.x * q3.x + w.y * q3.y + w.z * q3.z;
        float s = (q1.w * wv - q2.w * wu) / q3.w;
        if (s < 0.f || s > 1.f)
          continue;
        float t = (q1.w * wu - q0.w * wv) / q3.w;
        if (t < 0.f || (s + t) > 1.f)
          continue;
        const float d = dist2(pt, o);
        if (d < best) {  // faces arrive in index order: strict '<' as the reference
          best = d;
          best_idx = base + k;
          best_pt = pt;
        }
      }
    }
  }
  if (live) {
    hit_face[i] = best_idx;
    if (hit_point) {
      hit_point[3 * i + 0] = best_pt.x;
      hit_point[3 * i + 1] = best_pt.y;
      hit_point[3 * i + 2] = best_pt.z;
    }
  }
}

// Materialises the emission rays (packed face by face, front then rear, as
// emission/malley_cpu.cpp:142-189 packs them).  ray_offsets[f] is the first
// ray of face f (n_faces + 1 entries).
__global__ void k_emit(const float* __restrict__ frames, const long long* __restrict__ ray_offsets,
                       const int32_t* __restrict__ front, int n_faces, long n_rays, uint32_t key0, uint32_t key1,
                       uint32_t epoch, float* __restrict__ rays6)
{
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n_rays; i += (long)gridDim.x * blockDim.x) {
    int lo = 0, hi = n_faces;  // largest f with ray_offsets[f] <= i
    while (hi - lo > 1) {
      int mid = (lo + hi) >> 1;
      if (ray_offsets[mid] <= i)
        lo = mid;
      else
        hi = mid;
    }
    const int f = lo;
    const uint32_t j = (uint32_t)(i - ray_offsets[f]);
    float frame[18];
#pragma unroll
    for (int e = 0; e < 18; ++e)
      frame[e] = __ldg(frames + 20 * (size_t)f + e);
    float3 o, e;
    emit_ray(frame, (uint32_t)f, j, front[f], key0, key1, epoch, o, e);
    float* r = rays6 + 6 * i;
    r[0] = o.x; r[1] = o.y; r[2] = o.z;
    r[3] = e.x; r[4] = e.y; r[5] = e.z;
  }
}

// Per-mesh normalisation of the counts (cpuFactorsCalculator/cpu_system.cpp
// :193-195): ff[m][j] = (float)count[m][j] * (1.f / (float)outgoing[m]).
__global__ void k_normalise(const uint32_t* __restrict__ counts, const int32_t* __restrict__ outgoing, int n_rows,
                            float* __restrict__ ff)
{
  const size_t n = (size_t)n_rows * n_rows;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int m = (int)(i / n_rows);
    const float ratio = 1.f / (float)outgoing[m];
    ff[i] = (float)counts[i] * ratio;
  }
}

}  // namespace ffb
