// ffb_trace.cuh -- the hot kernels: fused emission + nearest-hit trace +
// per-(source, hit) histogram (form-factor counts), ray-batch casts (grid and
// brute force) and ray materialisation.
#pragma once

#include "ffb_grid.cuh"

namespace ffb {

// A unit of work of the fused kernel: `count` consecutive rays [j0, j0+count)
// of face `face` (index within its scene).  Rays j < front leave the front
// side, the others the rear.
struct Chunk {
  int32_t face;
  int32_t j0;
  int32_t count;
  int32_t front;
};

// Writes the work chunks of the emitting faces: src[i] = {face, front rays,
// front + rear rays, first chunk}; the face's rays [0, nf) become chunks of
// kRays consecutive rays (the last one shorter), one warp per face.
template <int kRays>
__global__ void k_chunk_fill(const int4* __restrict__ src, int n, Chunk* __restrict__ chunks)
{
  const int lane = threadIdx.x & 31;
  const int warps = (int)((gridDim.x * blockDim.x) >> 5);
  for (int i = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); i < n; i += warps) {
    const int4 f = src[i];
    const int nc = (f.z + kRays - 1) / kRays;
    for (int j = lane; j < nc; j += 32)
      chunks[(uint32_t)f.w + (uint32_t)j] = Chunk{f.x, j * kRays, min(kRays, f.z - j * kRays), f.y};
  }
}

// Statistics slots (uint64 each), accumulated once per warp.
enum { kStatTests = 0, kStatCells = 1, kStatRays = 2, kStatHits = 3, kStatJumps = 4, kStatSlots = 5 };

// The scene of a fused launch: its grid, its count matrix and where its
// faces start in the launch's frame table.
struct SceneSlot {
  GridView g;
  uint32_t* __restrict__ counts;              // n_cols * n_cols
  const int32_t* __restrict__ face_to_row;   // face -> matrix row/column (mesh), or null for identity
  int face_base;                              // first frame of the scene
  int n_cols;                                 // matrix side
};

// Scenes of one batch (ffb_batch_set); each is traced by its own launch.
constexpr int kMaxBatchScenes = 4096;

struct TraceParams {
  const float* __restrict__ frames;          // 20 floats per face, scenes concatenated
  const Chunk* __restrict__ chunks;
  int n_chunks;
  uint32_t key0, key1, epoch;
  const uint32_t* __restrict__ epoch_ptr;    // when set, the epoch is read from device memory
  const uint2* __restrict__ scene_keys;      // device Philox key of the scene, or null for (key0, key1)
  uint32_t* __restrict__ chunk_cursor;        // work counter, zero before the launch
  unsigned long long* __restrict__ stats;     // kStatSlots, or null
  // radiance sink (kPower): per-ray power of each (face, side) as 64-bit
  // fixed point, and the per-mesh absorbed power it adds to (mesh = the
  // scene's face_to_row of the hit face)
  const unsigned long long* __restrict__ power;
  unsigned long long* __restrict__ absorb;
  // when set: [0] gets the earliest block start and [1] the latest warp end
  // of the launch, in %globaltimer nanoseconds (atomicMin / atomicMax, so
  // several launches may share one pair)
  unsigned long long* __restrict__ span;
  SceneSlot scene;
};

__device__ __forceinline__ unsigned long long global_ns()
{
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

constexpr int kTraceThreads = 128;
constexpr int kWarpsPerBlock = kTraceThreads / 32;
// Blocks per SM the trace kernels are compiled for: 8 blocks of 128 threads
// cap registers at 64 per thread (32 warps per SM to hide L1/L2 latency).
#ifndef FFB_MIN_BLOCKS
#define FFB_MIN_BLOCKS 8
#endif
constexpr int kWarpHashLog2 = 9;
constexpr int kWarpHash = 1 << kWarpHashLog2;  // histogram slots per warp
constexpr uint32_t kEmptyKey = 0xFFFFFFFFu;
constexpr size_t kHashSmem = sizeof(uint32_t) * 2 * kWarpHash * kWarpsPerBlock;  // dynamic shared bytes with kHash
constexpr unsigned kFull = 0xFFFFFFFFu;

__device__ __forceinline__ void warp_stats(unsigned long long* stats, uint32_t tests, uint32_t cells, uint32_t rays,
                                           uint32_t hits, uint32_t jumps)
{
  if (!stats)
    return;
  unsigned long long v[kStatSlots] = {tests, cells, rays, hits, jumps};
#pragma unroll
  for (int k = 0; k < kStatSlots; ++k) {
    unsigned long long x = v[k];
    for (int o = 16; o > 0; o >>= 1)
      x += __shfl_xor_sync(kFull, x, o);
    if ((threadIdx.x & 31) == 0 && x)
      atomicAdd(stats + k, x);
  }
}

// Adds 1 to the bin of `key` in a warp's open-addressing table.  Returns true
// when the key took a new slot.  Keys are matrix indices row * n_cols + col.
__device__ __forceinline__ bool warp_hash_add(uint32_t* keys, uint32_t* vals, uint32_t key, uint32_t* counts)
{
  uint32_t s = (key * 2654435761u) >> (32 - kWarpHashLog2);
  volatile uint32_t* vk = keys;
  for (int probe = 0; probe < kWarpHash; ++probe) {
    uint32_t cur = vk[s];
    if (cur == kEmptyKey) {
      cur = atomicCAS(keys + s, kEmptyKey, key);
      if (cur == kEmptyKey) {
        atomicAdd(vals + s, 1u);
        return true;
      }
    }
    if (cur == key) {
      atomicAdd(vals + s, 1u);
      return false;
    }
    s = (s + 1) & (kWarpHash - 1);
  }
  atomicAdd(counts + key, 1u);  // full table; unreachable: flushed at half load
  return false;
}

// Adds every occupied bin of a warp's table to the global matrix and clears it.
__device__ __forceinline__ void warp_hash_flush(uint32_t* keys, uint32_t* vals, uint32_t* counts, int lane)
{
  __syncwarp();
  for (int i = lane; i < kWarpHash; i += 32) {
    const uint32_t k = keys[i];
    if (k != kEmptyKey) {
      atomicAdd(counts + k, vals[i]);
      keys[i] = kEmptyKey;
      vals[i] = 0;
    }
  }
  __syncwarp();
}

// ---------------------------------------------------------------------------
// Fused form-factor kernel.  Persistent warps, no block barriers.  Each warp
// keeps a current chunk (consecutive rays of one face) and hands its rays to
// lanes as they fall idle (one ballot per refill, one global atomic per
// chunk), so a warp may hold rays of several faces at once.  Idle lanes are
// refilled together once at least the shape's `refill` of them wait (or the
// whole warp is idle): emission and ray setup then run with several lanes at
// once instead of one lane at a time.  Each iteration a lane whose cell is
// exhausted moves on (stop, DDA step or empty-space jump; up to the shape's
// `adv` moves while it lands in empty cells) and then tests up to its `test`
// references of its cell.  Doing both kinds of work in one
// iteration keeps lanes of a warp in the same code more of the time than
// one kind per iteration does.  A finished hit adds one to the
// warp's shared-memory hash histogram keyed by the matrix index
// row(f) * n_cols + row(h); the warp flushes the table to the global uint32
// matrix with atomic adds when it is half full and at the end.
//
// kPower (the radiance equation, thermal_equation/radiance_cpu.cpp:142-180)
// replaces the matrix: a hit adds the per-ray power of the ray's (source
// face, side) to the absorbed power of the hit face's mesh, in 64-bit fixed
// point (integer sums: the same result whatever the order of the hits).
// kStats adds the test / cell / ray / hit counters (four live registers per
// lane); without it p.stats is ignored.  kHash selects the warp histogram;
// without it each hit is one global reduction (red.global.add) into the
// matrix, which suits large, sparse matrices (distinct keys per warp, so the
// histogram merges little) and leaves the shared memory to the L1 cache.
// ---------------------------------------------------------------------------
#ifndef FFB_REFILL_MIN
#define FFB_REFILL_MIN 6
#endif
constexpr int kRefillMin = FFB_REFILL_MIN;
// cell advances and triangle tests a lane may do per iteration
#ifndef FFB_ADV_PER_ITER
#define FFB_ADV_PER_ITER 2
#endif
#ifndef FFB_TEST_PER_ITER
#define FFB_TEST_PER_ITER 2
#endif

// Launch shapes of the fused kernel, the choices of the autotuner
// (ffb_autotune): cell advances and triangle tests a lane may do per
// iteration, the idle lanes a warp waits for before it refills them, and the
// resident blocks of 128 threads per SM the kernel is compiled for (which
// caps its registers at 65536 / (128 * blocks)).  Shape 0 is the default.
// The shape changes only the order in which lanes do their work, never a
// ray's result or the counts.
// With `coherent` set, a warp hands out the rays of each chunk it takes in
// the order of their directions (bins of an 8 x 8 Morton order on the Malley
// disk) instead of in index order, so that lanes refilled together trace
// rays of similar direction from the same face.
// With `lanes` = K > 0, each lane keeps K rays in shared memory instead of
// one in registers, and each iteration the warp runs ONE body -- the cell
// advances or the triangle tests -- chosen by a vote of its lanes, each lane
// working on one of its rays in that phase; `refill` is then the number of
// lanes with a free ray slot that triggers a refill.
struct TraceShape {
  int adv, test, refill, blocks, coherent, lanes;
};
constexpr int kNumShapes = 14;
__host__ __device__ constexpr TraceShape trace_shape(int v)
{
  return v == 1 ? TraceShape{1, 1, 4, 8, 0, 0}
       : v == 2 ? TraceShape{2, 1, 6, 8, 0, 0}
       : v == 3 ? TraceShape{1, 2, 6, 8, 0, 0}
       : v == 4 ? TraceShape{3, 3, 6, 8, 0, 0}
       : v == 5 ? TraceShape{2, 2, 10, 8, 0, 0}
       : v == 6 ? TraceShape{2, 2, 6, 6, 0, 0}
       : v == 7 ? TraceShape{2, 2, 6, 8, 1, 0}
       : v == 8 ? TraceShape{2, 2, 10, 8, 1, 0}
       : v == 9 ? TraceShape{2, 2, 8, 8, 0, 2}
       : v == 10 ? TraceShape{2, 2, 8, 8, 1, 2}
       : v == 11 ? TraceShape{2, 2, 8, 8, 0, 3}
       : v == 12 ? TraceShape{2, 3, 8, 8, 0, 2}
       : v == 13 ? TraceShape{2, 3, 8, 8, 0, 3}
                 : TraceShape{FFB_ADV_PER_ITER, FFB_TEST_PER_ITER, FFB_REFILL_MIN, FFB_MIN_BLOCKS, 0, 0};
}

constexpr int kChunkRaysMax = 256;  // rays per chunk (the host's chunk size)
constexpr int kDirBins = 64;        // direction bins of the coherent hand-out

// Direction bin of ray j of a face (the draws of emit_ray): the Malley disk
// point (sqrt(r) cos phi, sqrt(r) sin phi) on an 8 x 8 grid, in Morton order.
__device__ __forceinline__ int direction_bin(uint32_t face, uint32_t j, uint32_t key0, uint32_t key1, uint32_t epoch)
{
  const uint4 x = philox4x32_10(make_uint4(j, face, epoch, 0x46464231u), key0, key1);
  const float rad = sqrtf(u01(x.z));
  float sphi, cphi;
  sincos_turn24(x.w >> 8, sphi, cphi);
  const int qx = min(7, max(0, (int)((rad * cphi + 1.f) * 4.f)));
  const int qy = min(7, max(0, (int)((rad * sphi + 1.f) * 4.f)));
  int code = 0;
#pragma unroll
  for (int b = 0; b < 3; ++b)
    code |= (((qx >> b) & 1) << (2 * b)) | (((qy >> b) & 1) << (2 * b + 1));
  return code;
}

// Order of the chunk's rays [0, count) by direction bin (a counting sort in
// the warp's shared memory: `cnt` kDirBins counters, `perm` the order).
__device__ __forceinline__ void direction_order(uint32_t face, uint32_t j0, int count, uint32_t key0, uint32_t key1,
                                                uint32_t epoch, uint32_t* cnt, uint8_t* perm, int lane)
{
  cnt[lane] = 0;
  cnt[lane + 32] = 0;
  __syncwarp();
  uint32_t code[kChunkRaysMax / 32];
#pragma unroll
  for (int m = 0; m < kChunkRaysMax / 32; ++m) {
    const int idx = m * 32 + lane;
    code[m] = 0;
    if (idx < count) {
      const int bin = direction_bin(face, j0 + (uint32_t)idx, key0, key1, epoch);
      code[m] = (uint32_t)bin | (atomicAdd(cnt + bin, 1u) << 8);
    }
  }
  __syncwarp();
  // exclusive scan of the counters, two per lane
  const uint32_t a = cnt[2 * lane], b = cnt[2 * lane + 1];
  uint32_t incl = a + b;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(kFull, incl, o);
    if (lane >= o)
      incl += y;
  }
  __syncwarp();
  cnt[2 * lane] = incl - a - b;
  cnt[2 * lane + 1] = incl - b;
  __syncwarp();
#pragma unroll
  for (int m = 0; m < kChunkRaysMax / 32; ++m) {
    const int idx = m * 32 + lane;
    if (idx < count)
      perm[cnt[code[m] & 0xFFu] + (code[m] >> 8)] = (uint8_t)idx;
  }
  __syncwarp();
}

// Ray state of the shared-memory lanes (TraceShape::lanes): field f of the
// ray in column c at R[f * kCols + c], 32-bit words, kCols = K * 128.  The cell
// coordinates (each below 256) and the empty-space distance (below 128) share
// one word; the direction signs are recomputed from the direction.
enum {
  kRayOx, kRayOy, kRayOz, kRayDx, kRayDy, kRayDz, kRayIx, kRayIy, kRayIz, kRayDlen, kRayBest, kRayBestRef, kRayI,
  kRayEn, kRayCell, kRayRow, kRayFields
};
template <int kCols>
__device__ __forceinline__ void lane_ray_load(const uint32_t* R, int c, Tracer& T)
{
  T.o = f3(__uint_as_float(R[kRayOx * kCols + c]), __uint_as_float(R[kRayOy * kCols + c]),
           __uint_as_float(R[kRayOz * kCols + c]));
  T.dir = f3(__uint_as_float(R[kRayDx * kCols + c]), __uint_as_float(R[kRayDy * kCols + c]),
             __uint_as_float(R[kRayDz * kCols + c]));
  T.inv = f3(__uint_as_float(R[kRayIx * kCols + c]), __uint_as_float(R[kRayIy * kCols + c]),
             __uint_as_float(R[kRayIz * kCols + c]));
  T.dlen = __uint_as_float(R[kRayDlen * kCols + c]);
  T.best = __uint_as_float(R[kRayBest * kCols + c]);
  T.best_ref = (int)R[kRayBestRef * kCols + c];
  T.i = R[kRayI * kCols + c];
  T.en = R[kRayEn * kCols + c];
  const uint32_t cell = R[kRayCell * kCols + c];
  T.cx = (int)(cell & 0xFFu);
  T.cy = (int)((cell >> 8) & 0xFFu);
  T.cz = (int)((cell >> 16) & 0xFFu);
  T.jump = (int)(cell >> 24);
  T.sx = sgn(T.dir.x);
  T.sy = sgn(T.dir.y);
  T.sz = sgn(T.dir.z);
}

template <int kCols>
__device__ __forceinline__ void lane_ray_store_cell(uint32_t* R, int c, const Tracer& T)
{
  R[kRayI * kCols + c] = T.i;
  R[kRayEn * kCols + c] = T.en;
  R[kRayCell * kCols + c] =
      (uint32_t)T.cx | ((uint32_t)T.cy << 8) | ((uint32_t)T.cz << 16) | ((uint32_t)T.jump << 24);
}

template <int kCols>
__device__ __forceinline__ void lane_ray_store_test(uint32_t* R, int c, const Tracer& T)
{
  R[kRayBest * kCols + c] = __float_as_uint(T.best);
  R[kRayBestRef * kCols + c] = (uint32_t)T.best_ref;
  R[kRayI * kCols + c] = T.i;
}

template <int kCols>
__device__ __forceinline__ void lane_ray_store(uint32_t* R, int c, const Tracer& T)
{
  R[kRayOx * kCols + c] = __float_as_uint(T.o.x);
  R[kRayOy * kCols + c] = __float_as_uint(T.o.y);
  R[kRayOz * kCols + c] = __float_as_uint(T.o.z);
  R[kRayDx * kCols + c] = __float_as_uint(T.dir.x);
  R[kRayDy * kCols + c] = __float_as_uint(T.dir.y);
  R[kRayDz * kCols + c] = __float_as_uint(T.dir.z);
  R[kRayIx * kCols + c] = __float_as_uint(T.inv.x);
  R[kRayIy * kCols + c] = __float_as_uint(T.inv.y);
  R[kRayIz * kCols + c] = __float_as_uint(T.inv.z);
  R[kRayDlen * kCols + c] = __float_as_uint(T.dlen);
  lane_ray_store_test<kCols>(R, c, T);
  lane_ray_store_cell<kCols>(R, c, T);
}

template <bool kSkip, bool kStats, bool kHash, bool kPower = false, int kShape = 0>
__global__ void __launch_bounds__(kTraceThreads, trace_shape(kShape).blocks)
    k_form_factors(const __grid_constant__ TraceParams p)
{
  constexpr TraceShape kS = trace_shape(kShape);
  extern __shared__ uint32_t s_hash[];  // kWarpsPerBlock x (keys, values) when kHash
  // coherent hand-out: per warp, direction-bin counters and the chunk's ray order
  __shared__ uint32_t s_bins[kS.coherent ? kWarpsPerBlock * kDirBins : 1];
  __shared__ uint8_t s_perm[kS.coherent ? kWarpsPerBlock * kChunkRaysMax : 1];
  // K rays per lane: kRayFields fields of kTraceThreads * K slots
  __shared__ uint32_t s_rays[kS.lanes ? kRayFields * kTraceThreads * kS.lanes : 1];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (p.span && threadIdx.x == 0)
    atomicMin(p.span, global_ns());
  uint32_t* keys = s_hash + warp * 2 * kWarpHash;
  uint32_t* vals = keys + kWarpHash;
  if (kHash) {
    for (int i = lane; i < kWarpHash; i += 32) {
      keys[i] = kEmptyKey;
      vals[i] = 0;
    }
    __syncwarp();
  }
  const uint32_t epoch = p.epoch_ptr ? *p.epoch_ptr : p.epoch;
  const unsigned lane_below = (1u << lane) - 1u;
  int fill = 0;  // occupied slots (warp-uniform)
  // current chunk (warp-uniform); c_pos: its rays handed out so far
  int c_face = 0, c_j = 0, c_left = 0, c_front = 0, c_row = 0, c_pos = 0;
  const SceneSlot& S = p.scene;
  uint32_t key0 = p.key0, key1 = p.key1;
  if (p.scene_keys) {
    const uint2 k = p.scene_keys[0];
    key0 = k.x;
    key1 = k.y;
  }
  bool exhausted = false;
  uint32_t n_tests = 0, n_cells = 0, n_rays = 0, n_hits = 0, n_jumps = 0;
  if constexpr (kS.lanes > 0) {
    // ---- K rays per lane in shared memory, one body per iteration ----
    constexpr int K = kS.lanes;
    constexpr int kCols = K * kTraceThreads;
    uint32_t* const R = s_rays;
    // the fields of slot k of this lane: column (warp * K + k) * 32 + lane,
    // so that the 32 lanes of a warp always hit 32 different banks
    const int col0 = warp * K * 32 + lane;
    uint32_t ph = 0;  // 2 bits per slot: 0 free, 1 cell exhausted (advance), 2 references pending (test)
    for (;;) {
      bool has_free = false, has_adv = false, has_test = false;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const uint32_t s = (ph >> (2 * k)) & 3u;
        has_free |= s == 0u;
        has_adv |= s == 1u;
        has_test |= s == 2u;
      }
      unsigned need = __ballot_sync(kFull, has_free);
      const unsigned busy = __ballot_sync(kFull, has_adv || has_test);
      if (__popc(need) < kS.refill && busy)
        need = 0;
      while (need && !exhausted) {
        if (c_left == 0) {
          int k = 0;
          if (lane == 0)
            k = (int)atomicAdd(p.chunk_cursor, 1u);
          k = __shfl_sync(kFull, k, 0);
          if (k >= p.n_chunks) {
            exhausted = true;
            break;
          }
          const Chunk ch = p.chunks[k];
          c_face = ch.face;
          c_j = ch.j0;
          c_left = ch.count;
          c_front = ch.front;
          c_row = S.face_to_row ? __ldg(S.face_to_row + ch.face) : ch.face;
          c_pos = 0;
          if (kS.coherent)
            direction_order((uint32_t)c_face, (uint32_t)c_j, c_left, key0, key1, epoch, s_bins + warp * kDirBins,
                            s_perm + warp * kChunkRaysMax, lane);
        }
        const int take = min(__popc(need), c_left);
        const int rank = __popc(need & lane_below);
        const bool mine = ((need >> lane) & 1u) && rank < take;
        if (mine) {
          const int j = c_j + (kS.coherent ? (int)s_perm[warp * kChunkRaysMax + c_pos + rank] : c_pos + rank);
          float3 o, e;
          emit_ray(p.frames + 20 * ((size_t)S.face_base + c_face), (uint32_t)c_face, (uint32_t)j, c_front, key0,
                   key1, epoch, o, e);
          ++n_rays;
          Tracer T;
          if (tracer_begin<kSkip>(T, S.g, o, e, n_cells)) {
            int k = 0;
            while (k < K - 1 && ((ph >> (2 * k)) & 3u) != 0u)
              ++k;
            const int c = col0 + 32 * k;
            lane_ray_store<kCols>(R, c, T);
            R[kRayRow * kCols + c] = (uint32_t)(kPower ? 2 * c_face + (j >= c_front ? 1 : 0) : c_row);
            ph |= (T.i < T.en ? 2u : 1u) << (2 * k);
          }
        }
        need &= ~__ballot_sync(kFull, mine);
        c_pos += take;
        c_left -= take;
      }
      has_adv = has_test = false;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const uint32_t s = (ph >> (2 * k)) & 3u;
        has_adv |= s == 1u;
        has_test |= s == 2u;
      }
      const unsigned va = __ballot_sync(kFull, has_adv), vt = __ballot_sync(kFull, has_test);
      if (exhausted && !(va | vt))
        break;
      const bool do_test = __popc(vt) >= __popc(va);
      int hit = -1, row = 0;
      if (do_test ? has_test : has_adv) {
        const uint32_t want = do_test ? 2u : 1u;
        int k = 0;
        while (k < K - 1 && ((ph >> (2 * k)) & 3u) != want)
          ++k;
        const int c = col0 + 32 * k;
        Tracer T;
        lane_ray_load<kCols>(R, c, T);
        uint32_t s;
        if (do_test) {
#pragma unroll
          for (int t = 0; t < kS.test; ++t)
            if (T.i < T.en)
              tracer_test(T, S.g, n_tests);
          lane_ray_store_test<kCols>(R, c, T);
          s = T.i < T.en ? 2u : 1u;
        } else {
          bool live = true;
#pragma unroll
          for (int a = 0; a < kS.adv; ++a)
            if (live && T.i >= T.en)
              live = tracer_advance<kSkip>(T, S.g, n_cells, n_jumps);
          if (!live) {
            hit = tracer_result(T, S.g);
            row = (int)R[kRayRow * kCols + c];
            s = 0u;
          } else {
            lane_ray_store_cell<kCols>(R, c, T);
            s = T.i < T.en ? 2u : 1u;
          }
        }
        ph = (ph & ~(3u << (2 * k))) | (s << (2 * k));
      }
      bool fresh = false;
      if (hit >= 0) {
        ++n_hits;
        const int hcol = S.face_to_row ? __ldg(S.face_to_row + hit) : hit;
        if (kPower) {
          atomicAdd(p.absorb + hcol, __ldg(p.power + row));
        } else {
          const uint32_t key = (uint32_t)row * (uint32_t)S.n_cols + (uint32_t)hcol;
          if (kHash)
            fresh = warp_hash_add(keys, vals, key, S.counts);
          else
            atomicAdd(S.counts + key, 1u);
        }
      }
      if (kHash) {
        fill += __popc(__ballot_sync(kFull, fresh));
        if (fill > kWarpHash / 2) {
          warp_hash_flush(keys, vals, S.counts, lane);
          fill = 0;
        }
      }
    }
  } else {
  // lane state
  Tracer T;
  bool active = false;
  int my_row = 0;
  for (;;) {
    unsigned need = __ballot_sync(kFull, !active);

    if (__popc(need) < kS.refill && need != kFull)
      need = 0;
    while (need && !exhausted) {
      if (c_left == 0) {
        int k = 0;
        if (lane == 0)
          k = (int)atomicAdd(p.chunk_cursor, 1u);
        k = __shfl_sync(kFull, k, 0);
        if (k >= p.n_chunks) {
          exhausted = true;
          break;
        }
        const Chunk ch = p.chunks[k];
        c_face = ch.face;
        c_j = ch.j0;
        c_left = ch.count;
        c_front = ch.front;
        c_row = S.face_to_row ? __ldg(S.face_to_row + ch.face) : ch.face;
        c_pos = 0;
        if (kS.coherent)
          direction_order((uint32_t)c_face, (uint32_t)c_j, c_left, key0, key1, epoch, s_bins + warp * kDirBins,
                          s_perm + warp * kChunkRaysMax, lane);
      }
      const int take = min(__popc(need), c_left);
      const int rank = __popc(need & lane_below);
      const bool mine = ((need >> lane) & 1u) && rank < take;
      if (mine) {
        const int j = c_j + (kS.coherent ? (int)s_perm[warp * kChunkRaysMax + c_pos + rank] : c_pos + rank);
        float3 o, e;
        emit_ray(p.frames + 20 * ((size_t)S.face_base + c_face), (uint32_t)c_face, (uint32_t)j, c_front, key0, key1,
                 epoch, o, e);
        ++n_rays;
        my_row = kPower ? 2 * c_face + (j >= c_front ? 1 : 0) : c_row;
        active = tracer_begin<kSkip>(T, S.g, o, e, n_cells);
      }
      need &= ~__ballot_sync(kFull, mine);
      c_pos += take;
      c_left -= take;
    }
    if (exhausted && !__any_sync(kFull, active))
      break;
    int hit = -1;
    if (active) {
      bool live = true;
#pragma unroll
      for (int k = 0; k < kS.adv; ++k)
        if (live && T.i >= T.en)
          live = tracer_advance<kSkip>(T, S.g, n_cells, n_jumps);
      if (!live) {
        active = false;
        hit = tracer_result(T, S.g);
      } else {
#pragma unroll
        for (int k = 0; k < kS.test; ++k)
          if (T.i < T.en)
            tracer_test(T, S.g, n_tests);
      }
    }
    bool fresh = false;
    if (hit >= 0) {
      ++n_hits;
      const int col = S.face_to_row ? __ldg(S.face_to_row + hit) : hit;
      if (kPower) {
        atomicAdd(p.absorb + col, __ldg(p.power + my_row));
      } else {
        const uint32_t key = (uint32_t)my_row * (uint32_t)S.n_cols + (uint32_t)col;
        if (kHash)
          fresh = warp_hash_add(keys, vals, key, S.counts);
        else
          atomicAdd(S.counts + key, 1u);
      }
    }
    if (kHash) {
      fill += __popc(__ballot_sync(kFull, fresh));
      if (fill > kWarpHash / 2) {
        warp_hash_flush(keys, vals, S.counts, lane);
        fill = 0;
      }
    }
  }
  }  // one ray per lane in registers
  if (kHash)
    warp_hash_flush(keys, vals, S.counts, lane);
  if (kStats)
    warp_stats(p.stats, n_tests, n_cells, n_rays, n_hits, n_jumps);
  if (p.span && lane == 0)
    atomicMax(p.span + 1, global_ns());
}

// ---------------------------------------------------------------------------
// Parallel rays from a disc (a distant source): the thermal_equation
// parallel_rays_cpu path (thermal_equation/parallel_rays_cpu.cpp:92-131)
// with emission, trace and the per-face tally fused.  Persistent warps take
// ray indices from a global cursor (one atomic per refill of at least
// kRefillMin idle lanes); a hit on face h adds one to side_counts[2h] when
// the ray meets its front (dot(triangle_normal(h), direction) < 0, as the
// reference chooses the front absorbance) and to side_counts[2h + 1]
// otherwise.
// ---------------------------------------------------------------------------
template <bool kSkip, bool kStats>
__global__ void __launch_bounds__(kTraceThreads, FFB_MIN_BLOCKS)
    k_parallel_rays(GridView g, const __grid_constant__ DiscSource src, const float* __restrict__ faces9,
                    unsigned long long n_rays, uint32_t key0, uint32_t key1, uint32_t epoch,
                    uint32_t* __restrict__ side_counts, unsigned long long* __restrict__ cursor,
                    unsigned long long* __restrict__ stats)
{
  const int lane = threadIdx.x & 31;
  const unsigned lane_below = (1u << lane) - 1u;
  uint32_t n_tests = 0, n_cells = 0, n_done = 0, n_hits = 0, n_jumps = 0;
  Tracer T;
  bool active = false;
  bool exhausted = false;
  for (;;) {
    const unsigned need = __ballot_sync(kFull, !active);
    if ((__popc(need) >= kRefillMin || need == kFull) && !exhausted) {
      unsigned long long base = 0;
      if (lane == 0)
        base = atomicAdd(cursor, (unsigned long long)__popc(need));
      base = __shfl_sync(kFull, base, 0);
      if (base >= n_rays)
        exhausted = true;
      if ((need >> lane) & 1u) {
        const unsigned long long j = base + __popc(need & lane_below);
        if (j < n_rays) {
          float3 o, e;
          emit_disc_ray(src, j, key0, key1, epoch, o, e);
          ++n_done;
          active = tracer_begin<kSkip>(T, g, o, e, n_cells);
        }
      }
    }
    if (exhausted && !__any_sync(kFull, active))
      break;
    if (active) {
      bool live = true;
#pragma unroll
      for (int k = 0; k < FFB_ADV_PER_ITER; ++k)
        if (live && T.i >= T.en)
          live = tracer_advance<kSkip>(T, g, n_cells, n_jumps);
      if (!live) {
        active = false;
        const int h = tracer_result(T, g);
        if (h >= 0) {
          ++n_hits;
          // triangle_normal (math/triangle.cpp:114-119), dot with the direction
          const float* q = faces9 + 9 * (size_t)h;
          const float3 p0 = f3(__ldg(q + 0), __ldg(q + 1), __ldg(q + 2));
          const float3 nrm = cross3(sub3(f3(__ldg(q + 3), __ldg(q + 4), __ldg(q + 5)), p0),
                                    sub3(f3(__ldg(q + 6), __ldg(q + 7), __ldg(q + 8)), p0));
          const float side = dot3(nrm, src.direction);
          atomicAdd(side_counts + 2 * (size_t)h + (side < 0.f ? 0 : 1), 1u);
        }
      } else {
#pragma unroll
        for (int k = 0; k < FFB_TEST_PER_ITER; ++k)
          if (T.i < T.en)
            tracer_test(T, g, n_tests);
      }
    }
  }
  if (kStats)
    warp_stats(stats, n_tests, n_cells, n_done, n_hits, n_jumps);
}

// Materialises rays [0, n_rays) of a disc source (parallel_rays_cpu.cpp:88-106).
__global__ void k_emit_disc(const __grid_constant__ DiscSource src, unsigned long long n_rays, uint32_t key0,
                            uint32_t key1, uint32_t epoch, float* __restrict__ rays6)
{
  for (unsigned long long j = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; j < n_rays;
       j += (unsigned long long)gridDim.x * blockDim.x) {
    float3 o, e;
    emit_disc_ray(src, j, key0, key1, epoch, o, e);
    float* r = rays6 + 6 * j;
    r[0] = o.x; r[1] = o.y; r[2] = o.z;
    r[3] = e.x; r[4] = e.y; r[5] = e.z;
  }
}

// Advances the device-resident Philox epoch of a captured launch, so that every
// replay of a CUDA graph draws fresh rays.
__global__ void k_epoch_bump(uint32_t* epoch)
{
  if (threadIdx.x == 0 && blockIdx.x == 0)
    *epoch += 1;
}

// ---------------------------------------------------------------------------
// Ray-batch cast through the grid (the ray_caster interface): rays are
// {origin, end point} as in math::ray_t.  hit_face gets the face index or -1;
// hit_point (optional) gets the point, NaN for a miss.  Persistent warps take
// rays from a global cursor (one atomic per refill) as lanes fall idle.
// ---------------------------------------------------------------------------
template <bool kSkip>
__global__ void __launch_bounds__(kTraceThreads, FFB_MIN_BLOCKS)
    k_cast(GridView g, const float* __restrict__ rays6, long n_rays, int32_t* __restrict__ hit_face,
           float* __restrict__ hit_point, unsigned long long* __restrict__ stats,
           unsigned long long* __restrict__ cursor)
{
  const int lane = threadIdx.x & 31;
  const unsigned lane_below = (1u << lane) - 1u;
  uint32_t n_tests = 0, n_cells = 0, n_done = 0, n_hits = 0, n_jumps = 0;
  Tracer T;
  bool active = false;
  long id = -1;
  bool exhausted = false;
  auto finish = [&](long i, int h, float3 pt) {
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
  };
  for (;;) {
    const unsigned need = __ballot_sync(kFull, !active);
    if ((__popc(need) >= kRefillMin || need == kFull) && !exhausted) {
      unsigned long long base = 0;
      if (lane == 0)
        base = atomicAdd(cursor, (unsigned long long)__popc(need));
      base = __shfl_sync(kFull, base, 0);
      if (base >= (unsigned long long)n_rays)
        exhausted = true;
      if ((need >> lane) & 1u) {
        const unsigned long long r = base + __popc(need & lane_below);
        if (r < (unsigned long long)n_rays) {
          id = (long)r;
          const float* q = rays6 + 6 * r;
          const float3 o = f3(__ldg(q + 0), __ldg(q + 1), __ldg(q + 2));
          const float3 e = f3(__ldg(q + 3), __ldg(q + 4), __ldg(q + 5));
          active = tracer_begin<kSkip>(T, g, o, e, n_cells);
          if (!active)
            finish(id, -1, o);
        }
      }
    }
    if (exhausted && !__any_sync(kFull, active))
      break;
    if (active) {
      bool live = true;
#pragma unroll
      for (int k = 0; k < FFB_ADV_PER_ITER; ++k)
        if (live && T.i >= T.en)
          live = tracer_advance<kSkip>(T, g, n_cells, n_jumps);
      if (!live) {
        active = false;
        finish(id, tracer_result(T, g), T.best_pt);
      } else {
#pragma unroll
        for (int k = 0; k < FFB_TEST_PER_ITER; ++k)
          if (T.i < T.en)
            tracer_test(T, g, n_tests);
      }
    }
  }
  warp_stats(stats, n_tests, n_cells, n_done, n_hits, n_jumps);
}

// Brute force: every ray against every face (the naive_cpu definition),
// faces staged through shared memory in tiles, in index order with a strict
// '<' as the reference scans them.
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
        if (tri_hit(reinterpret_cast<const float4*>(tile + k), o, dir, pt)) {
          const float d = dist2(pt, o);
          if (d < best) {
            best = d;
            best_idx = base + k;
            best_pt = pt;
          }
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
      const int mid = (lo + hi) >> 1;
      if (ray_offsets[mid] <= i)
        lo = mid;
      else
        hi = mid;
    }
    const int f = lo;
    const uint32_t j = (uint32_t)(i - ray_offsets[f]);
    float3 o, e;
    emit_ray(frames + 20 * (size_t)f, (uint32_t)f, j, front[f], key0, key1, epoch, o, e);
    float* r = rays6 + 6 * i;
    r[0] = o.x; r[1] = o.y; r[2] = o.z;
    r[3] = e.x; r[4] = e.y; r[5] = e.z;
  }
}

// Per-mesh normalisation of the counts (cpuFactorsCalculator/cpu_system.cpp
// :193-195): ff[m][j] = (float)count[m][j] * (1.f / (float)outgoing[m]) for
// `rows` rows of n_cols entries (outgoing indexed from the first of them).
__global__ void k_normalise(const uint32_t* __restrict__ counts, const int32_t* __restrict__ outgoing, int rows,
                            int n_cols, float* __restrict__ ff)
{
  const size_t n = (size_t)rows * n_cols;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int m = (int)(i / n_cols);
    const float ratio = 1.f / (float)outgoing[m];
    ff[i] = (float)counts[i] * ratio;
  }
}

}  // namespace ffb
