// ffb_api.cu -- the C ABI of libffb200.so (declared in include/ffb.h).
//
// Host orchestration of the B200 form-factor path: resident scenes and grids
// per context (one main scene, or a batch of scenes for one fused launch),
// one CUDA stream per context, grow-only device scratch, pinned staging for
// host arguments.  No CPU fallback: every result is computed by the kernels of
// ffb_grid.cuh / ffb_trace.cuh.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include <map>
#include <mutex>
#include <tuple>
#include <utility>

#include <cuda_runtime.h>

#include "ffb.h"
#include "ffb_csv.cuh"
#include "ffb_internal.h"
#include "ffb_obj.cuh"
#include "ffb_pack.cuh"
#include "ffb_trace.cuh"

using namespace ffb;

namespace {

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...)
{
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

#define FFB_CUDA(call)                                                                                   \
  do {                                                                                                   \
    cudaError_t e_ = (call);                                                                             \
    if (e_ != cudaSuccess)                                                                               \
      return fail(e_ == cudaErrorMemoryAllocation ? FFB_ERR_NO_MEMORY : FFB_ERR_CUDA, "%s: %s (%s:%d)", \
                  #call, cudaGetErrorString(e_), __FILE__, __LINE__);                                    \
  } while (0)

#define FFB_TRY(expr)   \
  do {                  \
    int r_ = (expr);    \
    if (r_ < 0)         \
      return r_;        \
  } while (0)

// Grow-only device buffer.
struct DevBuf {
  void* ptr = nullptr;
  size_t cap = 0;
};

constexpr int kChunkRays = 256;  // rays per work chunk of the fused kernel
static_assert(kChunkRays == kChunkRaysMax, "the coherent hand-out orders whole chunks");
constexpr int kMaxRows = 65535;  // matrix index row * n + col stays below 0xFFFFFFFF
constexpr int kMaxPipeBlocks = 16;  // row blocks of a pipelined host output

// Host outputs of the count matrix of at least FFB_PIPELINE_MIN_BYTES are
// traced in row blocks of about FFB_PIPELINE_BLOCK_BYTES (2 to
// kMaxPipeBlocks) whose copies overlap the next block's trace.
#ifndef FFB_PIPELINE_MIN_BYTES
#define FFB_PIPELINE_MIN_BYTES (64ull << 20)
#endif
#ifndef FFB_PIPELINE_BLOCK_BYTES
#define FFB_PIPELINE_BLOCK_BYTES (160ull << 20)
#endif

// One resident scene: faces, triangle records and its grid.
struct SceneData {
  int n_faces = -1;  // -1: no scene
  DevBuf faces, tri, box_lo, box_hi, scene_ord;
  bool grid_ok = false;
  ffb_grid_info info{};
  DevBuf cell_start, cell_fill, ref_tri, ref_rec, empty_dist, cell_rec;
};

}  // namespace

// Records an error for ffb_last_error (shared with the other translation
// units of the library) and returns `code`.
int ffb_set_error(int code, const char* msg)
{
  g_last_error = msg ? msg : "";
  return code;
}

struct ffb_ctx {
  int device = 0;
  int n_sm = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  unsigned long long budget = 0;  // 0 = unlimited
  unsigned long long bytes = 0;   // device bytes held in DevBufs
  bool stats_on = true;           // fused kernel with counters
  int trace_shape = 0;            // launch shape of the fused kernel (trace_shape(), chosen by ffb_autotune)

  SceneData main;                 // the scene of the single-scene calls
  DevBuf frames;                  // emission frames of the main scene
  int frames_mode = -1;           // emission flags the frames were built for

  std::vector<SceneData> batch;   // the scenes of the batched calls
  std::vector<long long> batch_offsets;
  DevBuf batch_frames, batch_chunks, batch_keys, batch_epoch;
  int batch_frames_mode = -1;
  int batch_n_chunks = 0;
  std::vector<int> batch_chunk_first;  // first chunk of each scene (scene-major), plus the total
  std::vector<int> batch_shape;        // launch shape of each scene (ffb_batch_autotune), default 0
  // side streams of the batched launch: one launch per scene, spread over
  // them so that a scene's launch tail overlaps the next scenes
  cudaStream_t batch_streams[4] = {};
  cudaEvent_t batch_fork = nullptr, batch_join[4] = {};

  // per-call scratch
  DevBuf scan_sums, chunks, chunk_src, rows, cursor, stats, tmp_in, tmp_out, tmp_out2, offsets, front_dev, ray_cursor, ff_counts;
  DevBuf csv_tile_len, csv_tile_off, csv_text;  // CSV formatting
  DevBuf power_tab, absorb;                     // radiance sink
  DevBuf span;                                  // sliced traces: earliest start / latest end (globaltimer ns)
  DevBuf live_count;                            // grid build: faces with a non-empty binning box
  TraceParams slice_params{};                   // sliced traces: the prepared launch
  bool slice_ready = false;
  long long slice_chunks = 0;
  // OBJ import: the text and its line tables, the parsed geometry
  DevBuf obj_text, obj_chunk, obj_chunk_off, obj_starts, obj_flags, obj_ords, obj_vertices, obj_face_idx,
      obj_face_line, obj_special, obj_ranges, obj_faces, obj_err;
  std::vector<ffb_mesh> obj_meshes;
  std::vector<ffb_material> obj_materials;
  long long obj_n_faces = -1;  // faces of the last successful parse
  void* csv_pinned[2] = {nullptr, nullptr};     // double-buffered text on its way to a file
  size_t csv_pinned_cap[2] = {0, 0};
  void* pinned = nullptr;
  size_t pinned_cap = 0;
  cudaEvent_t pinned_free = nullptr;  // recorded after the last copy out of `pinned`
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  bool timed = false;
  // pipelined host output of the count matrix: a copy stream fed by one
  // event per row block (created on first use)
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t block_done[kMaxPipeBlocks] = {};
  cudaEvent_t block_copied[kMaxPipeBlocks] = {};
  cudaEvent_t copies_done = nullptr;
  // the same output moved as (column, count) pairs: device packs of the row
  // blocks and their headers, pinned copies of them, and the host threads
  // that expand them into the caller's rows
  DevBuf pack_hdr, pack_pairs;
  uint32_t* pack_hdr_host = nullptr;
  size_t pack_hdr_host_cap = 0;
  uint32_t* pack_stage[2] = {nullptr, nullptr};
  size_t pack_stage_cap = 0;
  int host_threads = -1;  // -1: the default, min(12, hardware threads)
  ffb_host_pool* host_pool = nullptr;
  unsigned long long last_d2h = 0;  // device->host bytes of the last counts call
};

namespace {

int ensure(ffb_ctx* c, DevBuf& b, size_t need)
{
  if (need <= b.cap)
    return FFB_OK;
  size_t want = std::max(need, b.cap + b.cap / 2);
  if (c->budget && c->bytes - b.cap + want > c->budget) {
    want = need;
    if (c->bytes - b.cap + want > c->budget)
      return fail(FFB_ERR_NO_MEMORY, "device budget of %llu bytes exceeded (need %zu more)", c->budget, want);
  }
  if (b.ptr) {
    cudaFreeAsync(b.ptr, c->stream);
    c->bytes -= b.cap;
    b.ptr = nullptr;
    b.cap = 0;
  }
  cudaError_t e = cudaMallocAsync(&b.ptr, want, c->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(FFB_ERR_NO_MEMORY, "cudaMallocAsync(%zu): %s", want, cudaGetErrorString(e));
  }
  b.cap = want;
  c->bytes += want;
  return FFB_OK;
}

void release(ffb_ctx* c, DevBuf& b)
{
  if (b.ptr) {
    cudaFreeAsync(b.ptr, c->stream);
    c->bytes -= b.cap;
  }
  b.ptr = nullptr;
  b.cap = 0;
}

void release_scene(ffb_ctx* c, SceneData& s)
{
  DevBuf* bufs[] = {&s.faces,      &s.tri,     &s.box_lo,  &s.box_hi,  &s.scene_ord,
                    &s.cell_start, &s.cell_fill, &s.ref_tri, &s.ref_rec, &s.empty_dist, &s.cell_rec};
  for (DevBuf* b : bufs)
    release(c, *b);
  s.n_faces = -1;
  s.grid_ok = false;
}

template <class T>
T* dptr(DevBuf& b) { return reinterpret_cast<T*>(b.ptr); }

// Where `p` lives: *dev is true for memory the context's device takes as a
// kernel operand (device memory of that device, or managed memory) and false
// for host memory (pageable or pinned).  Device memory of another device is
// an argument error: a kernel would reach it only through peer access, and
// fault without it.
int ptr_kind(ffb_ctx* c, const void* p, bool* dev)
{
  *dev = false;
  if (!p)
    return FFB_OK;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return FFB_OK;
  }
  if (a.type == cudaMemoryTypeManaged) {
    *dev = true;
  } else if (a.type == cudaMemoryTypeDevice) {
    if (a.device != c->device)
      return fail(FFB_ERR_ARG, "device pointer %p belongs to device %d; the context runs on device %d", p, a.device,
                  c->device);
    *dev = true;
  }
  return FFB_OK;
}

// Pinned staging buffer; waits for the previous copy out of it first.
int stage(ffb_ctx* c, size_t bytes, void** out)
{
  if (c->pinned_free)
    FFB_CUDA(cudaEventSynchronize(c->pinned_free));
  if (bytes > c->pinned_cap) {
    if (c->pinned)
      cudaFreeHost(c->pinned);
    c->pinned = nullptr;
    // at least 8 MiB, doubling: page-locked allocations synchronise the
    // device, so the staging buffer grows rarely
    size_t want = std::max(std::max(bytes, c->pinned_cap * 2), (size_t)8 << 20);
    FFB_CUDA(cudaMallocHost(&c->pinned, want));
    c->pinned_cap = want;
  }
  *out = c->pinned;
  return FFB_OK;
}

// Copies host data into device buffer `b` through the pinned stage.
int upload(ffb_ctx* c, DevBuf& b, const void* host, size_t bytes)
{
  FFB_TRY(ensure(c, b, std::max<size_t>(bytes, 16)));
  if (!bytes)
    return FFB_OK;
  void* st;
  FFB_TRY(stage(c, bytes, &st));
  memcpy(st, host, bytes);
  FFB_CUDA(cudaMemcpyAsync(b.ptr, st, bytes, cudaMemcpyHostToDevice, c->stream));
  FFB_CUDA(cudaEventRecord(c->pinned_free, c->stream));
  return FFB_OK;
}

int grid_blocks(long long n, int threads, int max_blocks = 1 << 20)
{
  long long b = (n + threads - 1) / threads;
  return (int)std::max<long long>(1, std::min<long long>(b, max_blocks));
}

GridView make_view(SceneData& s)
{
  GridView g;
  const ffb_grid_info& I = s.info;
  g.lo = make_float3(I.lo[0], I.lo[1], I.lo[2]);
  g.hi = make_float3(I.hi[0], I.hi[1], I.hi[2]);
  g.cs = make_float3(I.cell[0], I.cell[1], I.cell[2]);
  g.inv_cs = make_float3(1.f / I.cell[0], 1.f / I.cell[1], 1.f / I.cell[2]);
  g.nx = I.nx;
  g.ny = I.ny;
  g.nz = I.nz;
  g.slack = 2.f * I.margin;
  g.ref_tri = dptr<int32_t>(s.ref_tri);
  g.ref_rec = dptr<TriRec>(s.ref_rec);
  g.cell_rec = dptr<uint2>(s.cell_rec);
  return g;
}

int check_ctx(ffb_ctx* c)
{
  if (!c)
    return fail(FFB_ERR_ARG, "null context");
  FFB_CUDA(cudaSetDevice(c->device));
  return FFB_OK;
}

// Emission frames for n_faces faces starting at `faces9` into `frames`.
int build_frames(ffb_ctx* c, const float* faces9, int n_faces, int mode, float* frames)
{
  if (n_faces > 0)
    k_face_frames<<<grid_blocks(n_faces, 256), 256, 0, c->stream>>>(faces9, n_faces, mode, frames);
  FFB_CUDA(cudaGetLastError());
  return FFB_OK;
}

int ensure_frames(ffb_ctx* c, int flags)
{
  const int mode = flags & FFB_EMIT_REF_NORMAL;
  if (c->frames_mode == mode)
    return FFB_OK;
  FFB_TRY(ensure(c, c->frames, sizeof(float) * 20 * (size_t)std::max(c->main.n_faces, 1)));
  FFB_TRY(build_frames(c, dptr<float>(c->main.faces), c->main.n_faces, mode, dptr<float>(c->frames)));
  c->frames_mode = mode;
  return FFB_OK;
}

// Exclusive scan of n uint32 counts into out[0..n] (out[n] = total).
int scan(ffb_ctx* c, const uint32_t* in, int n, uint32_t* out)
{
  int nb = (n + kScanTile - 1) / kScanTile;
  FFB_TRY(ensure(c, c->scan_sums, sizeof(uint32_t) * (size_t)std::max(nb, 1)));
  uint32_t* sums = dptr<uint32_t>(c->scan_sums);
  k_scan_reduce<<<nb, kScanBlock, 0, c->stream>>>(in, n, sums);
  k_scan_sums<<<1, kScanBlock, 0, c->stream>>>(sums, nb);
  k_scan_apply<<<nb, kScanBlock, 0, c->stream>>>(in, n, sums, out);
  FFB_CUDA(cudaGetLastError());
  return FFB_OK;
}

int ensure_pipeline(ffb_ctx* c)
{
  if (c->copy_stream)
    return FFB_OK;
  cudaError_t e = cudaEventCreateWithFlags(&c->copies_done, cudaEventDisableTiming);
  for (int b = 0; b < kMaxPipeBlocks && e == cudaSuccess; ++b) {
    e = cudaEventCreateWithFlags(&c->block_done[b], cudaEventDisableTiming);
    if (e == cudaSuccess)
      e = cudaEventCreateWithFlags(&c->block_copied[b], cudaEventDisableTiming);
  }
  if (e == cudaSuccess)
    e = cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess)
    return fail(FFB_ERR_CUDA, "copy stream/event creation: %s", cudaGetErrorString(e));
  return FFB_OK;
}

// Host threads that expand packed host outputs (0: dense copies only).
int host_threads(const ffb_ctx* c)
{
  if (c->host_threads >= 0)
    return c->host_threads;
  const unsigned hw = std::thread::hardware_concurrency();
  return (int)std::min(12u, std::max(hw, 1u));
}

int ensure_batch_streams(ffb_ctx* c)
{
  if (c->batch_fork)
    return FFB_OK;
  cudaError_t e = cudaSuccess;
  for (cudaStream_t& st : c->batch_streams)
    if (e == cudaSuccess)
      e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  for (cudaEvent_t& ev : c->batch_join)
    if (e == cudaSuccess)
      e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
  if (e == cudaSuccess)
    e = cudaEventCreateWithFlags(&c->batch_fork, cudaEventDisableTiming);
  if (e != cudaSuccess)
    return fail(FFB_ERR_CUDA, "batch stream/event creation: %s", cudaGetErrorString(e));
  return FFB_OK;
}

void timing_begin(ffb_ctx* c)
{
  cudaEventRecord(c->ev0, c->stream);
}

void timing_end(ffb_ctx* c)
{
  cudaEventRecord(c->ev1, c->stream);
  c->timed = true;
}

// ---------------------------------------------------------------------------
// Scene upload and grid build on a SceneData
// ---------------------------------------------------------------------------
int scene_upload(ffb_ctx* c, SceneData& s, const float* faces9, int n_faces)
{
  s.grid_ok = false;
  s.n_faces = n_faces;
  if (n_faces == 0)
    return FFB_OK;
  const size_t bytes = sizeof(float) * 9 * (size_t)n_faces;
  bool dev = false;
  FFB_TRY(ptr_kind(c, faces9, &dev));
  if (dev) {
    FFB_TRY(ensure(c, s.faces, bytes));
    FFB_CUDA(cudaMemcpyAsync(s.faces.ptr, faces9, bytes, cudaMemcpyDeviceToDevice, c->stream));
  } else {
    FFB_TRY(upload(c, s.faces, faces9, bytes));
  }
  FFB_TRY(ensure(c, s.tri, sizeof(TriRec) * (size_t)n_faces));
  FFB_TRY(ensure(c, s.box_lo, sizeof(float4) * (size_t)n_faces));
  FFB_TRY(ensure(c, s.box_hi, sizeof(float4) * (size_t)n_faces));
  FFB_TRY(ensure(c, s.scene_ord, sizeof(uint32_t) * 6));
  uint32_t init[6] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u, 0u};
  FFB_TRY(upload(c, s.scene_ord, init, sizeof init));
  k_face_prepare<<<grid_blocks(n_faces, 256), 256, 0, c->stream>>>(
      dptr<float>(s.faces), n_faces, dptr<TriRec>(s.tri), dptr<float4>(s.box_lo), dptr<float4>(s.box_hi),
      dptr<uint32_t>(s.scene_ord));
  FFB_CUDA(cudaGetLastError());
  return FFB_OK;
}

int grid_build(ffb_ctx* c, SceneData& s, const ffb_grid_params* params)
{
  s.grid_ok = false;
  if (s.n_faces <= 0)
    return fail(FFB_ERR_NO_SCENE, "grid build without a scene (or with an empty scene)");
  ffb_grid_params P = {0, 0, 0, 2.f, 1};
  if (params)
    P = *params;
  if (P.cells_per_face <= 0.f)
    P.cells_per_face = 32.f;
  if (P.nx < 0 || P.ny < 0 || P.nz < 0 || P.nx > kMaxDim || P.ny > kMaxDim || P.nz > kMaxDim)
    return fail(FFB_ERR_TOO_LARGE, "grid dims %dx%dx%d outside [0, %d]", P.nx, P.ny, P.nz, kMaxDim);

  uint32_t ord[6];
  FFB_CUDA(cudaMemcpyAsync(ord, s.scene_ord.ptr, sizeof ord, cudaMemcpyDeviceToHost, c->stream));
  FFB_CUDA(cudaStreamSynchronize(c->stream));
  float smin[3], smax[3];
  for (int a = 0; a < 3; ++a) {
    smin[a] = ord2f(ord[a]);
    smax[a] = ord2f(ord[3 + a]);
  }
  ffb_grid_info I{};
  bool any = ord[0] != 0xFFFFFFFFu && smin[0] <= smax[0];
  if (!any) {  // nothing can be hit: a single empty cell
    for (int a = 0; a < 3; ++a) {
      smin[a] = 0.f;
      smax[a] = 1.f;
    }
  }
  float max_ext = 0.f, max_abs = 0.f;
  for (int a = 0; a < 3; ++a) {
    max_ext = std::max(max_ext, smax[a] - smin[a]);
    max_abs = std::max(max_abs, std::max(std::fabs(smin[a]), std::fabs(smax[a])));
  }
  // margin: far above the rounding of a computed hit point (a few ulps of the
  // coordinates) and far below a cell
  const float margin = max_ext * 0x1p-12f + max_abs * 0x1p-17f + 1e-30f;
  double ext[3];
  for (int a = 0; a < 3; ++a) {
    I.lo[a] = smin[a] - 2.f * margin;
    I.hi[a] = smax[a] + 2.f * margin;
    ext[a] = (double)I.hi[a] - (double)I.lo[a];
  }
  int dims[3] = {P.nx, P.ny, P.nz};
  if (!any) {
    dims[0] = dims[1] = dims[2] = 1;
  } else if (!P.nx || !P.ny || !P.nz) {
    double mx = std::max(ext[0], std::max(ext[1], ext[2]));
    double vol = 1.0;
    for (int a = 0; a < 3; ++a)
      vol *= std::max(ext[a], mx / 32.0);
    double target = (double)P.cells_per_face * s.n_faces;
    double sc = std::cbrt(target / vol);
    for (int a = 0; a < 3; ++a) {
      if (!dims[a])
        dims[a] = (int)std::min<double>(kMaxDim, std::max(1.0, std::round(ext[a] * sc)));
    }
  }
  I.nx = dims[0];
  I.ny = dims[1];
  I.nz = dims[2];
  for (int a = 0; a < 3; ++a)
    I.cell[a] = (float)(ext[a] / dims[a]);
  // the last boundary lo + n*cs must reach hi: nudge the cell size up if the
  // float product falls short
  for (int a = 0; a < 3; ++a) {
    while (I.lo[a] + (float)dims[a] * I.cell[a] < I.hi[a])
      I.cell[a] = std::nextafter(I.cell[a], INFINITY);
    I.hi[a] = I.lo[a] + (float)dims[a] * I.cell[a];
  }
  I.margin = margin;
  I.skip_empty = P.skip_empty ? 1 : 0;
  const long long n_cells = (long long)I.nx * I.ny * I.nz;

  FFB_TRY(ensure(c, s.cell_start, sizeof(uint32_t) * (size_t)(n_cells + 1)));
  FFB_TRY(ensure(c, s.cell_fill, sizeof(uint32_t) * (size_t)n_cells));
  FFB_CUDA(cudaMemsetAsync(s.cell_fill.ptr, 0, sizeof(uint32_t) * (size_t)n_cells, c->stream));
  BinGeom bg;
  bg.lo = make_float3(I.lo[0], I.lo[1], I.lo[2]);
  bg.cs = make_float3(I.cell[0], I.cell[1], I.cell[2]);
  bg.inv_cs = make_float3(1.f / I.cell[0], 1.f / I.cell[1], 1.f / I.cell[2]);
  bg.nx = I.nx;
  bg.ny = I.ny;
  bg.nz = I.nz;
  bg.margin = margin;
  const int nb = grid_blocks(s.n_faces, 128);
  k_grid_count<<<nb, 128, 0, c->stream>>>(bg, dptr<float>(s.faces), dptr<float4>(s.box_lo), dptr<float4>(s.box_hi),
                                          s.n_faces, dptr<uint32_t>(s.cell_fill));
  FFB_CUDA(cudaGetLastError());
  FFB_TRY(scan(c, dptr<uint32_t>(s.cell_fill), (int)n_cells, dptr<uint32_t>(s.cell_start)));
  // the live faces (non-empty binning boxes), counted on the device and read
  // with the reference total
  FFB_TRY(ensure(c, c->live_count, sizeof(uint32_t)));
  FFB_CUDA(cudaMemsetAsync(c->live_count.ptr, 0, sizeof(uint32_t), c->stream));
  k_count_live<<<grid_blocks(s.n_faces, 256), 256, 0, c->stream>>>(dptr<float4>(s.box_lo), dptr<float4>(s.box_hi),
                                                                  s.n_faces, dptr<uint32_t>(c->live_count));
  FFB_CUDA(cudaGetLastError());
  uint32_t total = 0, live = 0;
  FFB_CUDA(cudaMemcpyAsync(&total, dptr<uint32_t>(s.cell_start) + n_cells, sizeof total, cudaMemcpyDeviceToHost,
                           c->stream));
  FFB_CUDA(cudaMemcpyAsync(&live, c->live_count.ptr, sizeof live, cudaMemcpyDeviceToHost, c->stream));
  FFB_CUDA(cudaStreamSynchronize(c->stream));
  if (total >= kCellEmpty)  // reference offsets must stay below the empty-cell flag
    return fail(FFB_ERR_TOO_LARGE, "%u grid references; at most %u", total, kCellEmpty - 1);
  FFB_TRY(ensure(c, s.ref_tri, sizeof(int32_t) * (size_t)std::max<uint32_t>(total, 1)));
  FFB_CUDA(cudaMemsetAsync(s.cell_fill.ptr, 0, sizeof(uint32_t) * (size_t)n_cells, c->stream));
  k_grid_fill<<<nb, 128, 0, c->stream>>>(bg, dptr<float>(s.faces), dptr<float4>(s.box_lo), dptr<float4>(s.box_hi),
                                         s.n_faces, dptr<uint32_t>(s.cell_start), dptr<uint32_t>(s.cell_fill),
                                         dptr<int32_t>(s.ref_tri));
  k_cell_sort<<<grid_blocks(n_cells, 128), 128, 0, c->stream>>>(dptr<uint32_t>(s.cell_start), (int)n_cells,
                                                                dptr<int32_t>(s.ref_tri));
  FFB_TRY(ensure(c, s.ref_rec, sizeof(TriRec) * (size_t)std::max<uint32_t>(total, 1)));
  k_ref_gather<<<grid_blocks(total, 256, c->n_sm * 8), 256, 0, c->stream>>>(
      dptr<int32_t>(s.ref_tri), total, dptr<TriRec>(s.tri), dptr<TriRec>(s.ref_rec));
  FFB_CUDA(cudaGetLastError());
  if (I.skip_empty) {
    // one byte per cell and octant; passes along x, y, z double the octants
    FFB_TRY(ensure(c, s.empty_dist, (size_t)kOctants * n_cells));
    uint8_t* d = dptr<uint8_t>(s.empty_dist);
    k_empty_init<<<grid_blocks(n_cells, 256), 256, 0, c->stream>>>(dptr<uint32_t>(s.cell_start), (int)n_cells, d);
    const long long lines[3] = {(long long)I.ny * I.nz, (long long)I.nx * I.nz, (long long)I.nx * I.ny};
    for (int axis = 0; axis < 3; ++axis)
      k_empty_pass<<<dim3(grid_blocks(lines[axis], 128), 1u << axis), 128, 0, c->stream>>>(d, n_cells, I.nx, I.ny,
                                                                                         I.nz, axis);
    FFB_CUDA(cudaGetLastError());
  }
  FFB_TRY(ensure(c, s.cell_rec, sizeof(uint2) * (size_t)n_cells));
  k_cell_rec<<<grid_blocks(n_cells, 256, c->n_sm * 8), 256, 0, c->stream>>>(
      dptr<uint32_t>(s.cell_start), I.skip_empty ? dptr<uint8_t>(s.empty_dist) : nullptr, n_cells,
      dptr<uint2>(s.cell_rec));
  FFB_CUDA(cudaGetLastError());
  I.n_refs = total;
  I.n_live_faces = (int)live;
  s.info = I;
  s.grid_ok = true;
  return FFB_OK;
}

// Chunk table of the emitting faces `faces` (in launch order) built on the
// device: the host computes each face's first chunk (work linear in faces,
// not in rays) and uploads 16 bytes per face; k_chunk_fill writes the
// chunks.  first[i] gets the first chunk of faces[i], *n_chunks the total.
int device_chunks(ffb_ctx* c, const std::vector<int32_t>& faces, const int32_t* front, const int32_t* rear,
                  std::vector<long long>& first, long long* n_chunks, bool short_tail = false)
{
  // With short_tail, the faces that hold the last sixteenth of the rays get
  // chunks of kTailRays: the launch's last chunks are short, so its warps
  // run out of work closer together (a 256-ray chunk takes a warp about as
  // long as 1/18 of a full-GPU launch).
  constexpr int kTailRays = 64;
  long long tail_from = LLONG_MAX;
  if (short_tail) {
    long long all = 0;
    for (const int f : faces)
      all += (long long)front[f] + rear[f];
    tail_from = all - all / 16;
  }
  std::vector<int4> head, tail;
  head.reserve(faces.size());
  first.resize(faces.size());
  long long next = 0, rays = 0;
  for (size_t i = 0; i < faces.size(); ++i) {
    const int f = faces[i];
    const long long nf = (long long)front[f] + rear[f];
    if (nf > INT_MAX - kChunkRays)
      return fail(FFB_ERR_TOO_LARGE, "face %d emits %lld rays; at most %d", f, nf, INT_MAX - kChunkRays);
    const int size = rays >= tail_from ? kTailRays : kChunkRays;
    first[i] = next;
    (size == kChunkRays ? head : tail).push_back(make_int4(f, front[f], (int)nf, (int)next));
    next += (nf + size - 1) / size;
    rays += nf;
    if (next > INT_MAX)
      return fail(FFB_ERR_TOO_LARGE, "more than %d work chunks", INT_MAX);
  }
  *n_chunks = next;
  if (next > 0) {
    FFB_TRY(ensure(c, c->chunks, sizeof(Chunk) * (size_t)next));
    // one staged upload: the head's records, then the tail's
    const size_t nh = head.size();
    head.insert(head.end(), tail.begin(), tail.end());
    FFB_TRY(upload(c, c->chunk_src, head.data(), sizeof(int4) * head.size()));
    if (nh)
      k_chunk_fill<kChunkRays><<<grid_blocks((long long)nh * 32, 256, c->n_sm * 8), 256, 0, c->stream>>>(
          dptr<int4>(c->chunk_src), (int)nh, dptr<Chunk>(c->chunks));
    if (!tail.empty())
      k_chunk_fill<kTailRays><<<grid_blocks((long long)tail.size() * 32, 256, c->n_sm * 8), 256, 0, c->stream>>>(
          dptr<int4>(c->chunk_src) + nh, (int)tail.size(), dptr<Chunk>(c->chunks));
    FFB_CUDA(cudaGetLastError());
  }
  return FFB_OK;
}

int check_counts(int n_faces, const int32_t* front, const int32_t* rear, long long* total)
{
  if (!front || !rear)
    return fail(FFB_ERR_ARG, "null ray counts");
  long long t = 0;
  for (int f = 0; f < n_faces; ++f) {
    if (front[f] < 0 || rear[f] < 0)
      return fail(FFB_ERR_ARG, "negative ray count at face %d", f);
    t += (long long)front[f] + rear[f];
  }
  *total = t;
  return FFB_OK;
}

// Matrices of at least this many entries take one global reduction per hit
// instead of the warp histogram (keys rarely repeat within a warp there).
#ifndef FFB_DIRECT_MIN_WORDS
#define FFB_DIRECT_MIN_WORDS (1ull << 22)
#endif

// The timed kernel variant (no counters, matrix sink) for each launch shape.
template <bool kSkip, bool kHash, int... S>
void (*shaped_kernel(int shape, std::integer_sequence<int, S...>))(TraceParams)
{
  static void (*const table[])(TraceParams) = {k_form_factors<kSkip, false, kHash, false, S>...};
  return table[shape];
}

// Occupancy-sized persistent launch of the fused kernel for p.n_chunks
// chunks, in the context's launch shape (the counter and radiance variants
// always take shape 0).
template <bool kSkip>
int launch_fused(ffb_ctx* c, const TraceParams& p, bool timed, cudaStream_t stream = nullptr, int shape = -1)
{
  if (!stream)
    stream = c->stream;
  if (shape < 0)
    shape = c->trace_shape;
  bool hash = (unsigned long long)p.scene.n_cols * (unsigned long long)p.scene.n_cols < FFB_DIRECT_MIN_WORDS;
  void (*kern)(TraceParams);
  if (p.stats)
    kern = hash ? k_form_factors<kSkip, true, true> : k_form_factors<kSkip, true, false>;
  else if (hash)
    kern = shaped_kernel<kSkip, true>(shape, std::make_integer_sequence<int, kNumShapes>{});
  else
    kern = shaped_kernel<kSkip, false>(shape, std::make_integer_sequence<int, kNumShapes>{});
  if (p.power) {  // radiance sink: no matrix, no histogram
    kern = p.stats ? k_form_factors<kSkip, true, false, true> : k_form_factors<kSkip, false, false, true>;
    hash = false;
  }
  const size_t smem = hash ? kHashSmem : 0;
  int per_sm = 0;
  FFB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kTraceThreads, smem));
  // persistent blocks: a full wave, fewer when there are fewer chunks than warps
  const long long wave = (long long)std::max(per_sm, 1) * c->n_sm;
  const long long by_work = ((long long)p.n_chunks + kWarpsPerBlock - 1) / kWarpsPerBlock;
  const int blocks = (int)std::max<long long>(1, std::min(wave, by_work));
  if (timed)
    timing_begin(c);
  kern<<<blocks, kTraceThreads, smem, stream>>>(p);
  if (timed)
    timing_end(c);
  FFB_CUDA(cudaGetLastError());
  return FFB_OK;
}

}  // namespace

// ===========================================================================
// Context
// ===========================================================================
extern "C" int ffb_ctx_create(int device, ffb_ctx** out)
{
  if (!out)
    return fail(FFB_ERR_ARG, "null output pointer");
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return fail(FFB_ERR_NO_DEVICE, "no CUDA device");
  }
  if (device < 0 || device >= n)
    return fail(FFB_ERR_ARG, "device %d out of range (%d devices)", device, n);
  cudaDeviceProp prop;
  FFB_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10)
    return fail(FFB_ERR_NO_DEVICE, "device %d is sm_%d%d; this library is built for sm_100a", device, prop.major,
                prop.minor);
  FFB_CUDA(cudaSetDevice(device));
  ffb_ctx* c = new ffb_ctx;
  c->device = device;
  c->n_sm = prop.multiProcessorCount;
  cudaError_t e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->pinned_free, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreate(&c->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&c->ev1);
  if (e != cudaSuccess) {
    delete c;
    return fail(FFB_ERR_CUDA, "stream/event creation: %s", cudaGetErrorString(e));
  }
  c->stream = c->own_stream;
  // Keep freed blocks in this process's default memory pool instead of
  // returning them at every synchronisation: contexts grow and release
  // multi-GB buffers (count matrices), and mapping them again on the next
  // allocation costs more than the trace of a small request.  Trimmed when
  // a context is destroyed.
  {
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      uint64_t keep = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
  }
  *out = c;
  return FFB_OK;
}

extern "C" void ffb_ctx_destroy(ffb_ctx* c)
{
  if (!c)
    return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  release_scene(c, c->main);
  for (SceneData& s : c->batch)
    release_scene(c, s);
  DevBuf* bufs[] = {&c->frames,   &c->batch_frames, &c->batch_chunks, &c->batch_keys, &c->batch_epoch,
                    &c->scan_sums, &c->chunks,      &c->chunk_src,    &c->rows,         &c->cursor,     &c->stats,
                    &c->tmp_in,   &c->tmp_out,      &c->tmp_out2,     &c->offsets,    &c->front_dev,
                    &c->ray_cursor, &c->ff_counts, &c->csv_tile_len, &c->csv_tile_off, &c->csv_text,
                    &c->power_tab, &c->absorb, &c->span, &c->live_count, &c->pack_hdr, &c->pack_pairs, &c->obj_text,
                    &c->obj_chunk, &c->obj_chunk_off,
                    &c->obj_starts, &c->obj_flags, &c->obj_ords, &c->obj_vertices, &c->obj_face_idx,
                    &c->obj_face_line, &c->obj_special, &c->obj_ranges, &c->obj_faces, &c->obj_err};
  for (DevBuf* b : bufs)
    release(c, *b);
  cudaStreamSynchronize(c->stream);
  if (c->pinned)
    cudaFreeHost(c->pinned);
  for (void* p : c->csv_pinned)
    if (p)
      cudaFreeHost(p);
  for (cudaStream_t st : c->batch_streams)
    if (st) cudaStreamDestroy(st);
  for (cudaEvent_t e : c->batch_join)
    if (e) cudaEventDestroy(e);
  if (c->batch_fork) cudaEventDestroy(c->batch_fork);
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  if (c->copies_done) cudaEventDestroy(c->copies_done);
  for (cudaEvent_t e : c->block_done)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : c->block_copied)
    if (e) cudaEventDestroy(e);
  ffb_host_pool_destroy(c->host_pool);
  if (c->pack_hdr_host) cudaFreeHost(c->pack_hdr_host);
  for (uint32_t* p : c->pack_stage)
    if (p) cudaFreeHost(p);
  if (c->pinned_free) cudaEventDestroy(c->pinned_free);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  {
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, c->device) == cudaSuccess)
      cudaMemPoolTrimTo(pool, 0);
    cudaGetLastError();
  }
  delete c;
}

extern "C" int ffb_ctx_set_stream(ffb_ctx* c, void* stream)
{
  FFB_TRY(check_ctx(c));
  // finish work on the old stream before switching (buffers are shared)
  FFB_CUDA(cudaStreamSynchronize(c->stream));
  c->stream = stream ? (cudaStream_t)stream : c->own_stream;
  return FFB_OK;
}

extern "C" void* ffb_ctx_stream(ffb_ctx* c) { return c ? (void*)c->stream : nullptr; }

extern "C" int ffb_ctx_synchronize(ffb_ctx* c)
{
  FFB_TRY(check_ctx(c));
  FFB_CUDA(cudaStreamSynchronize(c->stream));
  return FFB_OK;
}

extern "C" int ffb_ctx_set_budget(ffb_ctx* c, unsigned long long bytes)
{
  if (!c)
    return fail(FFB_ERR_ARG, "null context");
  c->budget = bytes;
  return FFB_OK;
}

extern "C" unsigned long long ffb_ctx_bytes(ffb_ctx* c) { return c ? c->bytes : 0; }

extern "C" int ffb_ctx_set_host_threads(ffb_ctx* c, int n)
{
  if (!c)
    return fail(FFB_ERR_ARG, "null context");
  if (n < -1 || n > 256)
    return fail(FFB_ERR_ARG, "host threads %d outside [-1, 256]", n);
  c->host_threads = n;
  return FFB_OK;
}

extern "C" int ffb_ctx_host_threads(ffb_ctx* c) { return c ? host_threads(c) : 0; }

extern "C" int ffb_ctx_set_stats(ffb_ctx* c, int on)
{
  if (!c)
    return fail(FFB_ERR_ARG, "null context");
  c->stats_on = on != 0;
  return FFB_OK;
}

extern "C" const char* ffb_last_error(void) { return g_last_error.c_str(); }

// ===========================================================================
// Scene and grid
// ===========================================================================
extern "C" int ffb_scene_set(ffb_ctx* c, const float* faces9, int n_faces)
{
  FFB_TRY(check_ctx(c));
  if (n_faces < 0 || (n_faces > 0 && !faces9))
    return fail(FFB_ERR_ARG, "bad scene (n_faces=%d)", n_faces);
  c->frames_mode = -1;
  return scene_upload(c, c->main, faces9, n_faces);
}

extern "C" int ffb_grid_build(ffb_ctx* c, const ffb_grid_params* params)
{
  FFB_TRY(check_ctx(c));
  return grid_build(c, c->main, params);
}

extern "C" int ffb_grid_info_get(ffb_ctx* c, ffb_grid_info* out)
{
  if (!c || !out)
    return fail(FFB_ERR_ARG, "null argument");
  if (!c->main.grid_ok)
    return fail(FFB_ERR_NO_GRID, "no grid built");
  *out = c->main.info;
  return FFB_OK;
}

extern "C" int ffb_grid_export(ffb_ctx* c, uint32_t* cell_rec, int32_t* ref_tri)
{
  FFB_TRY(check_ctx(c));
  SceneData& s = c->main;
  if (!s.grid_ok)
    return fail(FFB_ERR_NO_GRID, "no grid built");
  const size_t n_cells = (size_t)s.info.nx * s.info.ny * s.info.nz;
  if (cell_rec)
    FFB_CUDA(cudaMemcpyAsync(cell_rec, s.cell_rec.ptr, sizeof(uint2) * n_cells, cudaMemcpyDefault, c->stream));
  if (ref_tri && s.info.n_refs > 0)
    FFB_CUDA(cudaMemcpyAsync(ref_tri, s.ref_tri.ptr, sizeof(int32_t) * (size_t)s.info.n_refs, cudaMemcpyDefault,
                             c->stream));
  FFB_CUDA(cudaStreamSynchronize(c->stream));
  return FFB_OK;
}

// ===========================================================================
// Casts
// ===========================================================================
namespace {

// Resolves an input array: device pointers pass through, host data is copied
// into `tmp`.
int input_ptr(ffb_ctx* c, const void* p, size_t bytes, DevBuf& tmp, const void** out)
{
  bool dev = false;
  FFB_TRY(ptr_kind(c, p, &dev));
  if (dev) {
    *out = p;
    return FFB_OK;
  }
  FFB_TRY(ensure(c, tmp, std::max<size_t>(bytes, 16)));
  if (bytes)
    FFB_CUDA(cudaMemcpyAsync(tmp.ptr, p, bytes, cudaMemcpyHostToDevice, c->stream));
  *out = tmp.ptr;
  return FFB_OK;
}

// Resolves an output array: device pointers pass through, host outputs get a
// device temporary copied back by finish_output.
int output_ptr(ffb_ctx* c, void* p, size_t bytes, DevBuf& tmp, void** out, bool* host)
{
  bool dev = false;
  FFB_TRY(ptr_kind(c, p, &dev));
  *host = p && !dev;
  if (!p || !*host) {
    *out = p;
    return FFB_OK;
  }
  FFB_TRY(ensure(c, tmp, std::max<size_t>(bytes, 16)));
  *out = tmp.ptr;
  return FFB_OK;
}

int finish_output(ffb_ctx* c, void* host, const void* dev, size_t bytes)
{
  if (bytes)
    FFB_CUDA(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, c->stream));
  return FFB_OK;
}

int cast_impl(ffb_ctx* c, const float* rays6, long long n_rays, int32_t* hit_face, float* hit_point, bool brute)
{
  FFB_TRY(check_ctx(c));
  if (n_rays < 0 || (n_rays > 0 && (!rays6 || !hit_face)))
    return fail(FFB_ERR_ARG, "bad cast arguments");
  SceneData& s = c->main;
  if (s.n_faces < 0)
    return fail(FFB_ERR_NO_SCENE, "cast without a scene");
  if (!brute && !s.grid_ok)
    return fail(FFB_ERR_NO_GRID, "cast before ffb_grid_build");
  if (n_rays == 0)
    return FFB_OK;
  const void* d_rays;
  void *d_hit, *d_pt;
  bool host_hit, host_pt, rays_dev = false;
  FFB_TRY(ptr_kind(c, rays6, &rays_dev));
  FFB_TRY(input_ptr(c, rays6, sizeof(float) * 6 * (size_t)n_rays, c->tmp_in, &d_rays));
  FFB_TRY(output_ptr(c, hit_face, sizeof(int32_t) * (size_t)n_rays, c->tmp_out, &d_hit, &host_hit));
  FFB_TRY(output_ptr(c, hit_point, sizeof(float) * 3 * (size_t)n_rays, c->tmp_out2, &d_pt, &host_pt));
  FFB_TRY(ensure(c, c->stats, sizeof(unsigned long long) * kStatSlots));
  FFB_CUDA(cudaMemsetAsync(c->stats.ptr, 0, sizeof(unsigned long long) * kStatSlots, c->stream));
  timing_begin(c);
  if (brute || s.n_faces == 0) {
    k_cast_brute<<<grid_blocks(n_rays, kTraceThreads), kTraceThreads, 0, c->stream>>>(
        dptr<TriRec>(s.tri), s.n_faces, (const float*)d_rays, (long)n_rays, (int32_t*)d_hit, (float*)d_pt);
  } else {
    GridView g = make_view(s);
    FFB_TRY(ensure(c, c->ray_cursor, sizeof(unsigned long long)));
    FFB_CUDA(cudaMemsetAsync(c->ray_cursor.ptr, 0, sizeof(unsigned long long), c->stream));
    auto kern = s.info.skip_empty ? k_cast<true> : k_cast<false>;
    int per_sm = 0;
    FFB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kTraceThreads, 0));
    const int blocks = grid_blocks(n_rays, kTraceThreads, std::max(1, per_sm) * c->n_sm);
    kern<<<blocks, kTraceThreads, 0, c->stream>>>(g, (const float*)d_rays, (long)n_rays, (int32_t*)d_hit,
                                                  (float*)d_pt, dptr<unsigned long long>(c->stats),
                                                  dptr<unsigned long long>(c->ray_cursor));
  }
  timing_end(c);
  FFB_CUDA(cudaGetLastError());
  if (host_hit)
    FFB_TRY(finish_output(c, hit_face, d_hit, sizeof(int32_t) * (size_t)n_rays));
  if (host_pt)
    FFB_TRY(finish_output(c, hit_point, d_pt, sizeof(float) * 3 * (size_t)n_rays));
  if (host_hit || host_pt || !rays_dev)
    FFB_CUDA(cudaStreamSynchronize(c->stream));
  return FFB_OK;
}

}  // namespace

extern "C" int ffb_cast(ffb_ctx* c, const float* rays6, long long n_rays, int32_t* hit_face, float* hit_point)
{
  return cast_impl(c, rays6, n_rays, hit_face, hit_point, false);
}

extern "C" int ffb_cast_bruteforce(ffb_ctx* c, const float* rays6, long long n_rays, int32_t* hit_face,
                                   float* hit_point)
{
  return cast_impl(c, rays6, n_rays, hit_face, hit_point, true);
}

// ===========================================================================
// Emission and form factors
// ===========================================================================
extern "C" int ffb_emit(ffb_ctx* c, const int32_t* front, const int32_t* rear, uint64_t seed, uint32_t epoch,
                        int flags, float* rays6)
{
  FFB_TRY(check_ctx(c));
  if (c->main.n_faces <= 0)
    return fail(FFB_ERR_NO_SCENE, "no scene");
  const int n_faces = c->main.n_faces;
  long long total = 0;
  FFB_TRY(check_counts(n_faces, front, rear, &total));
  if (total == 0)
    return FFB_OK;
  if (!rays6)
    return fail(FFB_ERR_ARG, "null ray output");
  FFB_TRY(ensure_frames(c, flags));
  std::vector<long long> offs((size_t)n_faces + 1);
  offs[0] = 0;
  for (int f = 0; f < n_faces; ++f)
    offs[f + 1] = offs[f] + front[f] + rear[f];
  FFB_TRY(upload(c, c->offsets, offs.data(), sizeof(long long) * offs.size()));
  FFB_TRY(upload(c, c->front_dev, front, sizeof(int32_t) * (size_t)n_faces));
  void* d_rays;
  bool host_out;
  FFB_TRY(output_ptr(c, rays6, sizeof(float) * 6 * (size_t)total, c->tmp_out, &d_rays, &host_out));
  k_emit<<<grid_blocks(total, 256, c->n_sm * 32), 256, 0, c->stream>>>(
      dptr<float>(c->frames), dptr<long long>(c->offsets), dptr<int32_t>(c->front_dev), n_faces, (long)total,
      (uint32_t)seed, (uint32_t)(seed >> 32), epoch, (float*)d_rays);
  FFB_CUDA(cudaGetLastError());
  if (host_out) {
    FFB_TRY(finish_output(c, rays6, d_rays, sizeof(float) * 6 * (size_t)total));
    FFB_CUDA(cudaStreamSynchronize(c->stream));
  }
  return FFB_OK;
}

namespace {

// Whether rows [row_begin, row_end) of the count matrix are sparse enough
// for the packed transfer: a row holds at most min(its rays, n_rows)
// nonzero entries, and the bound summed over the rows must fit the pair
// caps (a quarter of the entries).  Denser matrices go dense as a whole.
// The context's host threads, started (or restarted with a new count) on
// first use; false when they cannot be started.
bool ensure_host_pool(ffb_ctx* c)
{
  if (c->host_pool && ffb_host_pool_threads(c->host_pool) == host_threads(c))
    return true;
  ffb_host_pool_destroy(c->host_pool);
  c->host_pool = ffb_host_pool_create(host_threads(c));
  return c->host_pool != nullptr;
}

bool face_rows_ok(int n_faces, const int32_t* face_to_row, int n_rows)
{
  for (int f = 0; f < n_faces; ++f)
    if (face_to_row[f] < 0 || face_to_row[f] >= n_rows)
      return false;
  return true;
}

bool sparse_enough(int n_faces, const int32_t* front, const int32_t* rear, const int32_t* face_to_row, int n_rows,
                   int row_begin, int row_end)
{
  std::vector<long long> rays((size_t)n_rows, 0);
  for (int f = 0; f < n_faces; ++f)
    rays[(size_t)(face_to_row ? face_to_row[f] : f)] += (long long)front[f] + rear[f];
  long long bound = 0;
  for (int r = row_begin; r < row_end; ++r)
    bound += std::min<long long>(rays[(size_t)r], n_rows);
  return bound <= (long long)(row_end - row_begin) * n_rows / 4;
}

// Pinned host memory of at least `bytes` in *p (capacity *cap), kept and
// grown by doubling (page-locking costs tens of ms per hundred MB, so a
// run of growing requests must not pay it each time).
int ensure_pinned(uint32_t** p, size_t* cap, size_t bytes)
{
  if (bytes <= *cap)
    return FFB_OK;
  const size_t want = std::max(std::max(bytes, 2 * *cap), (size_t)8 << 20);
  if (*p)
    cudaFreeHost(*p);
  *p = nullptr;
  *cap = 0;
  FFB_CUDA(cudaMallocHost((void**)p, want));
  *cap = want;
  return FFB_OK;
}

// A host output of several row blocks moved as (column, count) pairs: called
// after every block's trace and pack are queued on the context stream
// (block_done[b] recorded after block b's pack).  Every device-to-host copy
// goes on the copy stream, issued once its block is done: block b's header,
// then its pairs (or, when they would not fit its cap of a quarter of its
// entries, its dense rows).  A copy queued early on the context stream would
// hold the copy engine's queue until that stream reached it.  Host threads
// expand block b while block b + 1's copies run.
// A host output written as the normalised form factors instead of the
// counts (ffb_form_factors): ff the host matrix, inv[m] = 1.f /
// (float)outgoing[m] for every row, outgoing the same on the device and
// scratch a device float block (dense blocks are normalised there first).
struct FloatSink {
  float* ff;
  const float* inv;
  const int32_t* outgoing;
  float* scratch;
};

int fetch_packed(ffb_ctx* c, const std::vector<int>& bounds, int row_begin, int n_rows, const uint32_t* d_counts,
                 uint32_t* counts, const std::vector<size_t>& hdr_off, const std::vector<size_t>& pair_off,
                 const std::vector<uint32_t>& cap, bool narrow, const FloatSink* fs)
{
  const size_t pair_bytes = narrow ? sizeof(uint32_t) : sizeof(uint2);
  const int n_blocks = (int)bounds.size() - 1;
  std::vector<char> dense((size_t)n_blocks, 0);
  auto fetch = [&](int b) -> int {
    const int rows = bounds[b + 1] - bounds[b];
    FFB_CUDA(cudaStreamWaitEvent(c->copy_stream, c->block_done[b], 0));
    FFB_CUDA(cudaMemcpyAsync(c->pack_hdr_host + hdr_off[b], dptr<uint32_t>(c->pack_hdr) + hdr_off[b],
                             sizeof(uint32_t) * pack_header_words(rows), cudaMemcpyDeviceToHost, c->copy_stream));
    FFB_CUDA(cudaStreamSynchronize(c->copy_stream));
    const uint32_t total = c->pack_hdr_host[hdr_off[b]];
    const size_t off = (size_t)(bounds[b] - row_begin) * n_rows;
    const size_t n_words = (size_t)rows * n_rows;
    c->last_d2h += sizeof(uint32_t) * pack_header_words(rows);
    if (total > cap[b] && fs) {
      dense[b] = 1;
      k_normalise<<<grid_blocks((long long)n_words, 256, c->n_sm * 16), 256, 0, c->copy_stream>>>(
          d_counts + off, fs->outgoing + bounds[b], rows, n_rows, fs->scratch);
      FFB_CUDA(cudaGetLastError());
      FFB_CUDA(cudaMemcpyAsync(fs->ff + off, fs->scratch, sizeof(float) * n_words, cudaMemcpyDeviceToHost,
                               c->copy_stream));
      c->last_d2h += sizeof(float) * n_words;
    } else if (total > cap[b]) {
      dense[b] = 1;
      FFB_CUDA(cudaMemcpyAsync(counts + off, d_counts + off, sizeof(uint32_t) * n_words, cudaMemcpyDeviceToHost,
                               c->copy_stream));
      c->last_d2h += sizeof(uint32_t) * n_words;
    } else if (total > 0) {
      FFB_CUDA(cudaMemcpyAsync(c->pack_stage[b & 1], dptr<unsigned char>(c->pack_pairs) + pair_bytes * pair_off[b],
                               pair_bytes * (size_t)total, cudaMemcpyDeviceToHost, c->copy_stream));
      c->last_d2h += pair_bytes * (size_t)total;
    }
    FFB_CUDA(cudaEventRecord(c->block_copied[b], c->copy_stream));
    return FFB_OK;
  };
  FFB_TRY(fetch(0));
  for (int b = 0; b < n_blocks; ++b) {
    FFB_CUDA(cudaEventSynchronize(c->block_copied[b]));
    const int rows = bounds[b + 1] - bounds[b];
    const uint32_t* h = c->pack_hdr_host + hdr_off[b];
    const size_t off = (size_t)(bounds[b] - row_begin) * n_rows;
    if (!dense[b] && fs)
      ffb_host_expand_norm_start(c->host_pool, fs->ff + off, rows, n_rows, h + 2, h + 2 + rows, c->pack_stage[b & 1],
                                 narrow, fs->inv + bounds[b]);
    else if (!dense[b])
      ffb_host_expand_start(c->host_pool, counts + off, rows, n_rows, h + 2, h + 2 + rows, c->pack_stage[b & 1],
                            narrow);
    // the next block's pairs go to the other stage, which block b - 1 used
    const int rc = b + 1 < n_blocks ? fetch(b + 1) : FFB_OK;
    if (!dense[b])
      ffb_host_expand_join(c->host_pool);
    FFB_TRY(rc);
  }
  return FFB_OK;
}

}  // namespace

namespace {

// ffb_form_factor_counts_rows; with fs, the output is fs's host float
// matrix of normalised form factors instead of `counts` (a packed host
// output: the caller checks that it is one).
int counts_rows_impl(ffb_ctx* c, const int32_t* front, const int32_t* rear, uint64_t seed, uint32_t epoch, int flags,
                     const int32_t* face_to_row, int n_rows, int row_begin, int row_end, uint32_t* counts,
                     const FloatSink* fs)
{
  FFB_TRY(check_ctx(c));
  SceneData& s = c->main;
  if (s.n_faces <= 0)
    return fail(FFB_ERR_NO_SCENE, "no scene");
  if (!s.grid_ok)
    return fail(FFB_ERR_NO_GRID, "form factors before ffb_grid_build");
  long long total = 0;
  FFB_TRY(check_counts(s.n_faces, front, rear, &total));
  if (!counts && !fs)
    return fail(FFB_ERR_ARG, "null counts");
  if (!face_to_row && n_rows != s.n_faces)
    return fail(FFB_ERR_ARG, "identity rows need n_rows == n_faces (%d != %d)", n_rows, s.n_faces);
  if (n_rows <= 0)
    return fail(FFB_ERR_ARG, "n_rows must be positive");
  if (n_rows > kMaxRows)
    return fail(FFB_ERR_TOO_LARGE, "n_rows %d above %d", n_rows, kMaxRows);
  if (row_begin < 0 || row_end > n_rows || row_begin >= row_end)
    return fail(FFB_ERR_ARG, "row range [%d, %d) outside [0, %d)", row_begin, row_end, n_rows);
  if (face_to_row) {
    for (int f = 0; f < s.n_faces; ++f)
      if (face_to_row[f] < 0 || face_to_row[f] >= n_rows)
        return fail(FFB_ERR_ARG, "face_to_row[%d] = %d outside [0, %d)", f, face_to_row[f], n_rows);
  }
  FFB_TRY(ensure_frames(c, flags));
  const size_t words = (size_t)(row_end - row_begin) * n_rows;
  void* d_counts;
  bool host_out = true;
  if (fs) {
    FFB_TRY(ensure(c, c->tmp_out, sizeof(uint32_t) * words));
    d_counts = c->tmp_out.ptr;
  } else {
    FFB_TRY(output_ptr(c, counts, sizeof(uint32_t) * words, c->tmp_out, &d_counts, &host_out));
  }
  // Row blocks: one launch each.  A host output of FFB_PIPELINE_MIN_BYTES or
  // more is split so that each finished block goes to the host on the copy
  // stream while the next block traces.
  const int span = row_end - row_begin;
  int n_blocks = 1;
  if (host_out && sizeof(uint32_t) * words >= FFB_PIPELINE_MIN_BYTES) {
    const size_t want = (sizeof(uint32_t) * words + FFB_PIPELINE_BLOCK_BYTES - 1) / FFB_PIPELINE_BLOCK_BYTES;
    n_blocks = (int)std::min<size_t>(std::max<size_t>(want, 2), (size_t)std::min(kMaxPipeBlocks, span));
  }
  // Equal blocks, except that the first of several has half the rows (when
  // every block keeps one): the host's side of a pipelined output starts
  // once it is done.
  std::vector<int> bounds(n_blocks + 1);
  const bool half_first = n_blocks > 1 && span >= 2 * n_blocks;
  for (int b = 0; b <= n_blocks; ++b)
    bounds[b] = b == 0 ? row_begin
                : half_first ? row_begin + (int)((long long)span * (2 * b - 1) / (2 * n_blocks - 1))
                             : row_begin + (int)((long long)span * b / n_blocks);
  // the chunks of each block, block after block; faces outside
  // [row_begin, row_end) do not emit
  std::vector<int> face_block(s.n_faces, -1);
  for (int f = 0; f < s.n_faces; ++f) {
    const int row = face_to_row ? face_to_row[f] : f;
    if (row >= row_begin && row < row_end)
      face_block[f] = (int)(std::upper_bound(bounds.begin(), bounds.end(), row) - bounds.begin()) - 1;
  }
  // emitting faces block after block (ascending within a block)
  std::vector<std::vector<int32_t>> by_block(n_blocks);
  for (int f = 0; f < s.n_faces; ++f)
    if (face_block[f] >= 0 && front[f] + (long long)rear[f] > 0)
      by_block[face_block[f]].push_back(f);
  std::vector<int32_t> order;
  order.reserve((size_t)s.n_faces);
  std::vector<size_t> block_pos(n_blocks + 1, 0);
  for (int b = 0; b < n_blocks; ++b) {
    block_pos[b] = order.size();
    order.insert(order.end(), by_block[b].begin(), by_block[b].end());
  }
  block_pos[n_blocks] = order.size();
  std::vector<long long> face_first;
  long long n_chunks = 0;
  FFB_TRY(device_chunks(c, order, front, rear, face_first, &n_chunks, n_blocks == 1));
  std::vector<int> first(n_blocks + 1, 0);
  for (int b = 0; b <= n_blocks; ++b)
    first[b] = (int)(block_pos[b] < order.size() ? face_first[block_pos[b]] : n_chunks);
  FFB_TRY(ensure(c, c->stats, sizeof(unsigned long long) * kStatSlots));
  FFB_CUDA(cudaMemsetAsync(c->stats.ptr, 0, sizeof(unsigned long long) * kStatSlots, c->stream));
  if (n_chunks > 0 && face_to_row)
    FFB_TRY(upload(c, c->rows, face_to_row, sizeof(int32_t) * (size_t)s.n_faces));
  FFB_TRY(ensure(c, c->cursor, sizeof(uint32_t) * kMaxPipeBlocks));
  if (n_blocks > 1)
    FFB_TRY(ensure_pipeline(c));
  // A pipelined host output moves as (column, count) pairs when host threads
  // are enabled and the rows are sparse enough: per block a header
  // (pack_header_words) and at most a quarter of its entries as pairs (at
  // most 1 or 2 bytes per entry with one- or two-word pairs, against 4).
  bool packed = host_out && n_blocks > 1 && host_threads(c) > 0 &&
                sparse_enough(s.n_faces, front, rear, face_to_row, n_rows, row_begin, row_end);
  packed = packed && ensure_host_pool(c);  // without host threads the blocks are copied dense
  if (fs && !packed)
    return fail(FFB_ERR_ARG, "normalised host output without a packed transfer");
  // One word per pair (column | count << 16) when no column and no count
  // reaches 2^16: a count is at most its row's rays.
  bool narrow = false;
  if (packed && n_rows <= 65536) {
    std::vector<long long> row_rays(face_to_row ? (size_t)n_rows : 0, 0);
    long long most = 0;
    for (int f = 0; f < s.n_faces; ++f) {
      const long long r = (long long)front[f] + rear[f];
      if (face_to_row)
        most = std::max(most, row_rays[(size_t)face_to_row[f]] += r);
      else
        most = std::max(most, r);
    }
    narrow = most < 65536;
  }
  const size_t pair_bytes = narrow ? sizeof(uint32_t) : sizeof(uint2);
  std::vector<size_t> hdr_off, pair_off;
  std::vector<uint32_t> cap;
  size_t hdr_words = 0;
  c->last_d2h = 0;
  if (packed) {
    size_t& hw = hdr_words;
    size_t pw = 0, max_cap = 0;
    for (int b = 0; b < n_blocks; ++b) {
      const int rows = bounds[b + 1] - bounds[b];
      hdr_off.push_back(hw);
      pair_off.push_back(pw);
      cap.push_back((uint32_t)std::min<size_t>((size_t)rows * n_rows / 4, UINT32_MAX));
      hw += pack_header_words(rows);
      pw += cap.back();
      max_cap = std::max<size_t>(max_cap, cap.back());
    }
    FFB_TRY(ensure(c, c->pack_hdr, sizeof(uint32_t) * hw));
    FFB_TRY(ensure(c, c->pack_pairs, pair_bytes * std::max<size_t>(pw, 1)));
    FFB_TRY(ensure_pinned(&c->pack_hdr_host, &c->pack_hdr_host_cap, sizeof(uint32_t) * hw));
    // both stages hold a block's pairs; sized at once for blocks of up to
    // FFB_PIPELINE_BLOCK_BYTES (the blocks of every matrix below 16 of them)
    const size_t stage_bytes = std::max(pair_bytes * std::max<size_t>(max_cap, 1),
                                        (size_t)FFB_PIPELINE_BLOCK_BYTES / 2);
    size_t stage_cap = c->pack_stage_cap;
    for (uint32_t*& st : c->pack_stage) {
      stage_cap = c->pack_stage_cap;  // both stages have the same capacity
      FFB_TRY(ensure_pinned(&st, &stage_cap, stage_bytes));
    }
    c->pack_stage_cap = stage_cap;
  }
  TraceParams p;
  p.frames = dptr<float>(c->frames);
  p.key0 = (uint32_t)seed;
  p.key1 = (uint32_t)(seed >> 32);
  p.epoch = epoch;
  p.epoch_ptr = nullptr;
  p.scene_keys = nullptr;
  p.stats = c->stats_on ? dptr<unsigned long long>(c->stats) : nullptr;
  p.power = nullptr;
  p.absorb = nullptr;
  p.span = nullptr;
  p.scene.g = make_view(s);
  // the kernel adds at row * n_rows + col; the output holds rows from
  // row_begin, so its base is moved back by row_begin rows (only rows of the
  // range are ever written)
  p.scene.counts = (uint32_t*)((uintptr_t)d_counts - sizeof(uint32_t) * (size_t)row_begin * n_rows);
  p.scene.face_to_row = face_to_row ? dptr<int32_t>(c->rows) : nullptr;
  p.scene.face_base = 0;
  p.scene.n_cols = n_rows;
  FFB_CUDA(cudaMemsetAsync(c->cursor.ptr, 0, sizeof(uint32_t) * n_blocks, c->stream));
  if (packed)  // the blocks' pair cursors (header word 0) start at zero
    FFB_CUDA(cudaMemsetAsync(c->pack_hdr.ptr, 0, sizeof(uint32_t) * hdr_words, c->stream));
  timing_begin(c);
  // Row blocks alternate between two side streams, so that one block's
  // launch tail (a block holds a few chunks per warp) overlaps the next
  // block's launch; blocks share nothing they write (rows, cursor, pairs).
  constexpr int kBlockStreams = 2;
  if (n_blocks > 1) {
    FFB_TRY(ensure_batch_streams(c));
    FFB_CUDA(cudaEventRecord(c->batch_fork, c->stream));
    for (int k = 0; k < kBlockStreams; ++k)
      FFB_CUDA(cudaStreamWaitEvent(c->batch_streams[k], c->batch_fork, 0));
  }
  for (int b = 0; b < n_blocks; ++b) {
    cudaStream_t st = n_blocks > 1 ? c->batch_streams[b % kBlockStreams] : c->stream;
    const size_t off = (size_t)(bounds[b] - row_begin) * n_rows;
    const size_t n_words = (size_t)(bounds[b + 1] - bounds[b]) * n_rows;
    FFB_CUDA(cudaMemsetAsync((uint32_t*)d_counts + off, 0, sizeof(uint32_t) * n_words, st));
    if (first[b + 1] > first[b]) {
      p.chunks = dptr<Chunk>(c->chunks) + first[b];
      p.n_chunks = first[b + 1] - first[b];
      p.chunk_cursor = dptr<uint32_t>(c->cursor) + b;
      if (s.info.skip_empty)
        FFB_TRY((launch_fused<true>(c, p, false, st)));
      else
        FFB_TRY((launch_fused<false>(c, p, false, st)));
    }
    if (packed && bounds[b + 1] > bounds[b]) {
      const int rows = bounds[b + 1] - bounds[b];
      (narrow ? k_rows_pack<true> : k_rows_pack<false>)<<<std::min(rows, c->n_sm * 8), kPackThreads, 0, st>>>(
          (const uint32_t*)d_counts + off, rows, n_rows, dptr<uint32_t>(c->pack_hdr) + hdr_off[b], cap[b],
          dptr<unsigned char>(c->pack_pairs) + pair_bytes * pair_off[b]);
      FFB_CUDA(cudaGetLastError());
    }
    if (n_blocks > 1)
      FFB_CUDA(cudaEventRecord(c->block_done[b], st));
  }
  if (n_blocks > 1)  // the context stream continues after every block
    for (int k = 0; k < kBlockStreams; ++k) {
      FFB_CUDA(cudaEventRecord(c->batch_join[k], c->batch_streams[k]));
      FFB_CUDA(cudaStreamWaitEvent(c->stream, c->batch_join[k], 0));
    }
  timing_end(c);
  if (!host_out)
    return FFB_OK;
  if (packed) {
    FloatSink sink;
    if (fs) {  // dense blocks are normalised into a device block before their copy
      size_t max_words = 0;
      for (int b = 0; b < n_blocks; ++b)
        max_words = std::max(max_words, (size_t)(bounds[b + 1] - bounds[b]) * n_rows);
      FFB_TRY(ensure(c, c->tmp_out2, sizeof(float) * max_words));
      sink = *fs;
      sink.scratch = dptr<float>(c->tmp_out2);
    }
    const int rc = fetch_packed(c, bounds, row_begin, n_rows, (const uint32_t*)d_counts, counts, hdr_off, pair_off,
                                cap, narrow, fs ? &sink : nullptr);
    if (rc != FFB_OK) {  // nothing may still write into the caller's buffer once the call returns
      cudaStreamSynchronize(c->copy_stream);
      cudaStreamSynchronize(c->stream);
      cudaGetLastError();
      return rc;
    }
  } else if (n_blocks == 1) {
    c->last_d2h = sizeof(uint32_t) * words;
    FFB_TRY(finish_output(c, counts, d_counts, sizeof(uint32_t) * words));
  } else {
    c->last_d2h = sizeof(uint32_t) * words;
    // all launches are queued before the first copy: a copy to pageable
    // memory holds the host until it ends
    for (int b = 0; b < n_blocks; ++b) {
      const size_t off = (size_t)(bounds[b] - row_begin) * n_rows;
      const size_t n_words = (size_t)(bounds[b + 1] - bounds[b]) * n_rows;
      FFB_CUDA(cudaStreamWaitEvent(c->copy_stream, c->block_done[b], 0));
      FFB_CUDA(cudaMemcpyAsync(counts + off, (const uint32_t*)d_counts + off, sizeof(uint32_t) * n_words,
                               cudaMemcpyDeviceToHost, c->copy_stream));
    }
    // later work on the context stream (a reuse of the device output) waits
    // for the copies
    FFB_CUDA(cudaEventRecord(c->copies_done, c->copy_stream));
    FFB_CUDA(cudaStreamWaitEvent(c->stream, c->copies_done, 0));
  }
  FFB_CUDA(cudaStreamSynchronize(c->stream));
  return FFB_OK;
}

}  // namespace

extern "C" int ffb_form_factor_counts_rows(ffb_ctx* c, const int32_t* front, const int32_t* rear, uint64_t seed,
                                           uint32_t epoch, int flags, const int32_t* face_to_row, int n_rows,
                                           int row_begin, int row_end, uint32_t* counts)
{
  return counts_rows_impl(c, front, rear, seed, epoch, flags, face_to_row, n_rows, row_begin, row_end, counts,
                          nullptr);
}

// ===========================================================================
// Sliced traces (the serving loop of ffb_server.cpp): one prepared launch
// whose chunk table is traced in consecutive slices, each its own launch on
// the context stream, all adding into the same device count matrix.
// ===========================================================================
int ffb_trace_prepare(ffb_ctx* c, const int32_t* front, const int32_t* rear, uint64_t seed, uint32_t epoch, int flags,
                      uint32_t* counts, long long* n_chunks)
{
  FFB_TRY(check_ctx(c));
  c->slice_ready = false;
  SceneData& s = c->main;
  if (s.n_faces <= 0)
    return fail(FFB_ERR_NO_SCENE, "no scene");
  if (!s.grid_ok)
    return fail(FFB_ERR_NO_GRID, "sliced trace before ffb_grid_build");
  if (s.n_faces > kMaxRows)
    return fail(FFB_ERR_TOO_LARGE, "%d faces; at most %d", s.n_faces, kMaxRows);
  long long total = 0;
  FFB_TRY(check_counts(s.n_faces, front, rear, &total));
  bool dev = false;
  FFB_TRY(ptr_kind(c, counts, &dev));
  if (!counts || !dev || !n_chunks)
    return fail(FFB_ERR_ARG, "sliced traces need a device count matrix and a chunk-count output");
  FFB_TRY(ensure_frames(c, flags));
  std::vector<int32_t> order;
  order.reserve((size_t)s.n_faces);
  for (int f = 0; f < s.n_faces; ++f)
    if (front[f] + (long long)rear[f] > 0)
      order.push_back(f);
  std::vector<long long> first;
  long long nch = 0;
  FFB_TRY(device_chunks(c, order, front, rear, first, &nch));
  FFB_TRY(ensure(c, c->cursor, sizeof(uint32_t) * kMaxPipeBlocks));
  FFB_TRY(ensure(c, c->span, 2 * sizeof(unsigned long long)));
  const unsigned long long span0[2] = {~0ull, 0ull};
  FFB_TRY(upload(c, c->span, span0, sizeof span0));
  FFB_CUDA(cudaMemsetAsync(counts, 0, sizeof(uint32_t) * (size_t)s.n_faces * s.n_faces, c->stream));
  TraceParams& p = c->slice_params;
  p.frames = dptr<float>(c->frames);
  p.chunks = dptr<Chunk>(c->chunks);
  p.n_chunks = 0;
  p.key0 = (uint32_t)seed;
  p.key1 = (uint32_t)(seed >> 32);
  p.epoch = epoch;
  p.epoch_ptr = nullptr;
  p.scene_keys = nullptr;
  p.chunk_cursor = dptr<uint32_t>(c->cursor);
  p.stats = nullptr;
  p.power = nullptr;
  p.absorb = nullptr;
  p.span = dptr<unsigned long long>(c->span);
  p.scene.g = make_view(s);
  p.scene.counts = counts;
  p.scene.face_to_row = nullptr;
  p.scene.face_base = 0;
  p.scene.n_cols = s.n_faces;
  c->slice_chunks = nch;
  c->slice_ready = true;
  *n_chunks = nch;
  return FFB_OK;
}

int ffb_trace_slice(ffb_ctx* c, long long first, long long count, void* stream)
{
  FFB_TRY(check_ctx(c));
  if (!c->slice_ready)
    return fail(FFB_ERR_ARG, "ffb_trace_slice before ffb_trace_prepare");
  if (first < 0 || count <= 0 || first + count > c->slice_chunks || count > INT_MAX)
    return fail(FFB_ERR_ARG, "slice [%lld, %lld) outside the %lld prepared chunks", first, first + count,
                c->slice_chunks);
  TraceParams p = c->slice_params;
  p.chunks = dptr<Chunk>(c->chunks) + first;
  p.n_chunks = (int)count;
  // slices of one prepared trace run in stream order, so one cursor serves them all
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  FFB_CUDA(cudaMemsetAsync(p.chunk_cursor, 0, sizeof(uint32_t), st));
  if (c->main.info.skip_empty)
    return launch_fused<true>(c, p, false, st);
  return launch_fused<false>(c, p, false, st);
}

int ffb_trace_span(ffb_ctx* c, unsigned long long* start_ns, unsigned long long* end_ns)
{
  FFB_TRY(check_ctx(c));
  unsigned long long v[2] = {0, 0};
  if (c->span.ptr) {
    FFB_CUDA(cudaMemcpyAsync(v, c->span.ptr, sizeof v, cudaMemcpyDeviceToHost, c->stream));
    FFB_CUDA(cudaStreamSynchronize(c->stream));
  }
  *start_ns = v[0] == ~0ull ? 0 : v[0];
  *end_ns = v[1];
  return FFB_OK;
}

extern "C" int ffb_form_factor_counts(ffb_ctx* c, const int32_t* front, const int32_t* rear, uint64_t seed,
                                      uint32_t epoch, int flags, const int32_t* face_to_row, int n_rows,
                                      uint32_t* counts)
{
  return ffb_form_factor_counts_rows(c, front, rear, seed, epoch, flags, face_to_row, n_rows, 0, n_rows, counts);
}

extern "C" int ffb_normalise(ffb_ctx* c, const uint32_t* counts, const int32_t* outgoing, int n_rows, float* ff)
{
  FFB_TRY(check_ctx(c));
  if (n_rows <= 0 || !counts || !outgoing || !ff)
    return fail(FFB_ERR_ARG, "bad normalise arguments");
  const size_t mat = (size_t)n_rows * n_rows;
  const void* d_counts;
  void* d_ff;
  bool host_out;
  FFB_TRY(input_ptr(c, counts, sizeof(uint32_t) * mat, c->tmp_in, &d_counts));
  FFB_TRY(upload(c, c->front_dev, outgoing, sizeof(int32_t) * (size_t)n_rows));
  FFB_TRY(output_ptr(c, ff, sizeof(float) * mat, c->tmp_out2, &d_ff, &host_out));
  k_normalise<<<grid_blocks((long long)mat, 256, c->n_sm * 16), 256, 0, c->stream>>>(
      (const uint32_t*)d_counts, dptr<int32_t>(c->front_dev), n_rows, n_rows, (float*)d_ff);
  FFB_CUDA(cudaGetLastError());
  if (host_out) {
    FFB_TRY(finish_output(c, ff, d_ff, sizeof(float) * mat));
    FFB_CUDA(cudaStreamSynchronize(c->stream));
  }
  return FFB_OK;
}

extern "C" int ffb_form_factors(ffb_ctx* c, const int32_t* front, const int32_t* rear, uint64_t seed, uint32_t epoch,
                                int flags, const int32_t* face_to_row, int n_rows, const int32_t* outgoing, float* ff)
{
  FFB_TRY(check_ctx(c));
  if (n_rows <= 0 || !outgoing || !ff)
    return fail(FFB_ERR_ARG, "bad form-factor arguments");
  if (n_rows > kMaxRows)
    return fail(FFB_ERR_TOO_LARGE, "n_rows %d above %d", n_rows, kMaxRows);
  const size_t mat = (size_t)n_rows * n_rows;
  bool ff_dev = false;
  FFB_TRY(ptr_kind(c, ff, &ff_dev));
  if (!ff_dev && sizeof(float) * mat >= FFB_PIPELINE_MIN_BYTES && host_threads(c) > 0 && c->main.n_faces > 0 &&
      front && rear && (!face_to_row || face_rows_ok(c->main.n_faces, face_to_row, n_rows)) &&
      sparse_enough(c->main.n_faces, front, rear, face_to_row, n_rows, 0, n_rows) && ensure_host_pool(c)) {
    // a large host matrix: traced in row blocks whose nonzero counts cross
    // PCIe packed and are normalised into the rows by the host threads, with
    // the device's operations: (float)count * (1.f / (float)outgoing[m])
    std::vector<float> inv((size_t)n_rows);
    for (int m = 0; m < n_rows; ++m)
      inv[(size_t)m] = 1.f / (float)outgoing[m];
    FFB_TRY(upload(c, c->front_dev, outgoing, sizeof(int32_t) * (size_t)n_rows));
    FloatSink fs{ff, inv.data(), dptr<int32_t>(c->front_dev), nullptr};
    return counts_rows_impl(c, front, rear, seed, epoch, flags, face_to_row, n_rows, 0, n_rows, nullptr, &fs);
  }
  FFB_TRY(ensure(c, c->ff_counts, sizeof(uint32_t) * mat));
  FFB_TRY(ffb_form_factor_counts(c, front, rear, seed, epoch, flags, face_to_row, n_rows,
                                 dptr<uint32_t>(c->ff_counts)));
  return ffb_normalise(c, dptr<uint32_t>(c->ff_counts), outgoing, n_rows, ff);
}

// ===========================================================================
// Radiance equation step (thermal_equation/radiance_cpu.cpp:96-190)
// ===========================================================================
extern "C" int ffb_radiance_absorption(ffb_ctx* c, const int32_t* front, const int32_t* rear, const float* power_front,
                                       const float* power_rear, const int32_t* face_to_mesh, int n_meshes,
                                       uint64_t seed, uint32_t epoch, int flags, double* absorption)
{
  FFB_TRY(check_ctx(c));
  SceneData& s = c->main;
  if (s.n_faces <= 0)
    return fail(FFB_ERR_NO_SCENE, "no scene");
  if (!s.grid_ok)
    return fail(FFB_ERR_NO_GRID, "radiance before ffb_grid_build");
  long long total = 0;
  FFB_TRY(check_counts(s.n_faces, front, rear, &total));
  if (!power_front || !power_rear || !face_to_mesh || !absorption || n_meshes <= 0)
    return fail(FFB_ERR_ARG, "bad radiance arguments");
  for (int f = 0; f < s.n_faces; ++f)
    if (face_to_mesh[f] < 0 || face_to_mesh[f] >= n_meshes)
      return fail(FFB_ERR_ARG, "face_to_mesh[%d] = %d outside [0, %d)", f, face_to_mesh[f], n_meshes);
  // 64-bit fixed point with 2^scale_exp units per watt, the largest power of
  // two that keeps the sum of all rays' powers below 2^62
  double bound = 0.0;
  for (int f = 0; f < s.n_faces; ++f) {
    if (!std::isfinite(power_front[f]) || !std::isfinite(power_rear[f]))
      return fail(FFB_ERR_ARG, "non-finite ray power at face %d", f);
    bound += (double)front[f] * std::fabs((double)power_front[f]) + (double)rear[f] * std::fabs((double)power_rear[f]);
  }
  int scale_exp = 0;
  if (bound > 0.0)
    scale_exp = std::min(1000, (int)std::floor(62.0 - std::log2(bound)));
  std::vector<long long> fixed(2 * (size_t)s.n_faces);
  for (int f = 0; f < s.n_faces; ++f) {
    fixed[2 * (size_t)f] = std::llround(std::ldexp((double)power_front[f], scale_exp));
    fixed[2 * (size_t)f + 1] = std::llround(std::ldexp((double)power_rear[f], scale_exp));
  }
  FFB_TRY(ensure_frames(c, flags));
  std::vector<int32_t> order;
  order.reserve((size_t)s.n_faces);
  for (int f = 0; f < s.n_faces; ++f)
    if (front[f] + (long long)rear[f] > 0)
      order.push_back(f);
  std::vector<long long> face_first;
  long long n_chunks = 0;
  FFB_TRY(device_chunks(c, order, front, rear, face_first, &n_chunks, true));
  FFB_TRY(ensure(c, c->absorb, sizeof(unsigned long long) * (size_t)n_meshes));
  FFB_CUDA(cudaMemsetAsync(c->absorb.ptr, 0, sizeof(unsigned long long) * (size_t)n_meshes, c->stream));
  FFB_TRY(ensure(c, c->stats, sizeof(unsigned long long) * kStatSlots));
  FFB_CUDA(cudaMemsetAsync(c->stats.ptr, 0, sizeof(unsigned long long) * kStatSlots, c->stream));
  if (n_chunks > 0) {
    FFB_TRY(upload(c, c->power_tab, fixed.data(), sizeof(long long) * fixed.size()));
    FFB_TRY(upload(c, c->rows, face_to_mesh, sizeof(int32_t) * (size_t)s.n_faces));
    FFB_TRY(ensure(c, c->cursor, sizeof(uint32_t)));
    FFB_CUDA(cudaMemsetAsync(c->cursor.ptr, 0, sizeof(uint32_t), c->stream));
    TraceParams p;
    p.frames = dptr<float>(c->frames);
    p.chunks = dptr<Chunk>(c->chunks);
    p.n_chunks = (int)n_chunks;
    p.key0 = (uint32_t)seed;
    p.key1 = (uint32_t)(seed >> 32);
    p.epoch = epoch;
    p.epoch_ptr = nullptr;
    p.scene_keys = nullptr;
    p.chunk_cursor = dptr<uint32_t>(c->cursor);
    p.stats = c->stats_on ? dptr<unsigned long long>(c->stats) : nullptr;
    p.power = dptr<unsigned long long>(c->power_tab);
    p.absorb = dptr<unsigned long long>(c->absorb);
    p.span = nullptr;
    p.scene.g = make_view(s);
    p.scene.counts = nullptr;
    p.scene.face_to_row = dptr<int32_t>(c->rows);
    p.scene.face_base = 0;
    p.scene.n_cols = n_meshes;
    if (s.info.skip_empty)
      FFB_TRY((launch_fused<true>(c, p, true)));
    else
      FFB_TRY((launch_fused<false>(c, p, true)));
  }
  std::vector<long long> sums((size_t)n_meshes);
  FFB_CUDA(cudaMemcpyAsync(sums.data(), c->absorb.ptr, sizeof(long long) * sums.size(), cudaMemcpyDeviceToHost,
                           c->stream));
  FFB_CUDA(cudaStreamSynchronize(c->stream));
  for (int m = 0; m < n_meshes; ++m)
    absorption[m] = std::ldexp((double)sums[(size_t)m], -scale_exp);
  return FFB_OK;
}

// ===========================================================================
// Parallel rays from a disc (emission/parallel_rays_cpu.cpp:88-106,
// thermal_equation/parallel_rays_cpu.cpp:92-131)
// ===========================================================================
namespace {

int disc_source(const ffb_disc_source* src, DiscSource* out)
{
  if (!src)
    return fail(FFB_ERR_ARG, "null source");
  *out = make_disc_source(f3(src->direction[0], src->direction[1], src->direction[2]),
                          f3(src->center[0], src->center[1], src->center[2]), src->distance, src->radius);
  return FFB_OK;
}

}  // namespace

extern "C" int ffb_emit_parallel(ffb_ctx* c, const ffb_disc_source* src, long long n_rays, uint64_t seed,
                                 uint32_t epoch, float* rays6)
{
  FFB_TRY(check_ctx(c));
  if (n_rays < 0 || (n_rays && !rays6))
    return fail(FFB_ERR_ARG, "bad parallel emission arguments");
  DiscSource d;
  FFB_TRY(disc_source(src, &d));
  void* d_rays;
  bool host_out;
  FFB_TRY(output_ptr(c, rays6, sizeof(float) * 6 * (size_t)n_rays, c->tmp_out, &d_rays, &host_out));
  if (n_rays) {
    k_emit_disc<<<grid_blocks(n_rays, 256, c->n_sm * 16), 256, 0, c->stream>>>(
        d, (unsigned long long)n_rays, (uint32_t)seed, (uint32_t)(seed >> 32), epoch, (float*)d_rays);
    FFB_CUDA(cudaGetLastError());
  }
  if (host_out) {
    FFB_TRY(finish_output(c, rays6, d_rays, sizeof(float) * 6 * (size_t)n_rays));
    FFB_CUDA(cudaStreamSynchronize(c->stream));
  }
  return FFB_OK;
}

extern "C" int ffb_parallel_rays(ffb_ctx* c, const ffb_disc_source* src, long long n_rays, uint64_t seed,
                                 uint32_t epoch, uint32_t* side_counts)
{
  FFB_TRY(check_ctx(c));
  SceneData& s = c->main;
  if (s.n_faces <= 0)
    return fail(FFB_ERR_NO_SCENE, "no scene");
  if (!s.grid_ok)
    return fail(FFB_ERR_NO_GRID, "parallel rays before ffb_grid_build");
  if (n_rays < 0 || !side_counts)
    return fail(FFB_ERR_ARG, "bad parallel-ray arguments");
  DiscSource d;
  FFB_TRY(disc_source(src, &d));
  const size_t bytes = sizeof(uint32_t) * 2 * (size_t)s.n_faces;
  void* d_counts;
  bool host_out;
  FFB_TRY(output_ptr(c, side_counts, bytes, c->tmp_out, &d_counts, &host_out));
  FFB_CUDA(cudaMemsetAsync(d_counts, 0, bytes, c->stream));
  FFB_TRY(ensure(c, c->stats, sizeof(unsigned long long) * kStatSlots));
  FFB_CUDA(cudaMemsetAsync(c->stats.ptr, 0, sizeof(unsigned long long) * kStatSlots, c->stream));
  FFB_TRY(ensure(c, c->ray_cursor, sizeof(unsigned long long)));
  FFB_CUDA(cudaMemsetAsync(c->ray_cursor.ptr, 0, sizeof(unsigned long long), c->stream));
  if (n_rays) {
    const GridView g = make_view(s);
    const bool stats = c->stats_on;
    auto kern = s.info.skip_empty ? (stats ? k_parallel_rays<true, true> : k_parallel_rays<true, false>)
                                  : (stats ? k_parallel_rays<false, true> : k_parallel_rays<false, false>);
    int per_sm = 0;
    FFB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kTraceThreads, 0));
    const long long wave = (long long)std::max(per_sm, 1) * c->n_sm;
    const long long by_work = (n_rays + kTraceThreads - 1) / kTraceThreads;
    const int blocks = (int)std::max<long long>(1, std::min(wave, by_work));
    timing_begin(c);
    kern<<<blocks, kTraceThreads, 0, c->stream>>>(g, d, dptr<float>(s.faces), (unsigned long long)n_rays,
                                                  (uint32_t)seed, (uint32_t)(seed >> 32), epoch, (uint32_t*)d_counts,
                                                  dptr<unsigned long long>(c->ray_cursor),
                                                  dptr<unsigned long long>(c->stats));
    timing_end(c);
    FFB_CUDA(cudaGetLastError());
  }
  if (host_out) {
    FFB_TRY(finish_output(c, side_counts, d_counts, bytes));
    FFB_CUDA(cudaStreamSynchronize(c->stream));
  }
  return FFB_OK;
}

// ===========================================================================
// Wavefront OBJ import (import_export/obj_import.cpp:44-340)
// ===========================================================================
namespace {

constexpr int kObjFileError = 21, kObjFormatError = 22, kObjMaterialNotDefined = 23,
              kObjMaterialNotEnough = 24, kObjMaterialInvalidValue = 25;

// subject::black_body (subject/objects.cpp:157-188)
ffb_material black_body()
{
  ffb_material m;
  memset(&m, 0, sizeof m);
  m.shell_density = m.shell_heat_capacity = m.shell_thermal_conductivity = m.shell_thickness = 1.f;
  m.front_absorbance = m.front_emissivity = 1.f;
  m.rear_absorbance = m.rear_emissivity = 1.f;
  strcpy(m.name, "black_body");
  return m;
}

bool getline_str(FILE* f, std::string& out)
{
  out.clear();
  int ch;
  bool any = false;
  while ((ch = fgetc(f)) != EOF) {
    any = true;
    if (ch == '\n')
      return true;
    out.push_back((char)ch);
  }
  return any;
}

// obj_import::material_lib (obj_import.cpp:44-164), host side: a material
// library is a handful of lines.  Returns 0 or the reference's negative code.
int material_lib(const char* filename, std::vector<ffb_material>& materials, std::map<std::string, int>& library)
{
  FILE* file = fopen(filename, "rb");
  if (!file)
    return -kObjFileError;
  static const char* kNames[14] = {"shell.density", "shell.heat_capacity", "shell.thermal_conductivity",
                                   "shell.thickness", "front.specular_reflectance", "front.diffuse_reflectance",
                                   "front.absorbance", "front.transmittance", "front.emissivity",
                                   "rear.specular_reflectance", "rear.diffuse_reflectance", "rear.absorbance",
                                   "rear.transmittance", "rear.emissivity"};
  std::string str;
  int rc = 0;
  while (rc == 0 && getline_str(file, str)) {
    if (str.empty() || str[0] == '#')
      continue;
    if (str[0] != 'n')
      continue;
    if (strncmp("newmtl", str.c_str(), 6) != 0) {
      rc = -kObjFormatError;
      break;
    }
    const std::string name = str.size() > 7 ? str.substr(7) : std::string();
    ffb_material m;
    memset(&m, 0, sizeof m);
    if (name.length() >= sizeof(m.name)) {
      rc = -kObjFormatError;
      break;
    }
    memcpy(m.name, name.c_str(), name.length());
    float* fields[14] = {&m.shell_density, &m.shell_heat_capacity, &m.shell_thermal_conductivity,
                         &m.shell_thickness, &m.front_specular_reflectance, &m.front_diffuse_reflectance,
                         &m.front_absorbance, &m.front_transmittance, &m.front_emissivity,
                         &m.rear_specular_reflectance, &m.rear_diffuse_reflectance, &m.rear_absorbance,
                         &m.rear_transmittance, &m.rear_emissivity};
    bool parsed[14] = {false};
    int n_parsed = 0;
    // as the reference: getline first, then the count test (the line after
    // the fourteenth property is consumed)
    while (getline_str(file, str) && n_parsed != 14) {
      if (str.empty())
        break;
      if (str[0] == '#')
        continue;
      const std::string::size_type pos = str.find_first_of(" \t");
      if (pos == std::string::npos || pos + 1 >= str.length()) {
        rc = -kObjFormatError;
        break;
      }
      const std::string prop = str.substr(0, pos), value = str.substr(pos + 1);
      int k = 0;
      while (k < 14 && prop != kNames[k])
        ++k;
      if (k == 14)
        continue;  // unknown property: skipped
      if (sscanf(value.c_str(), "%f", fields[k]) != 1) {
        rc = -kObjMaterialInvalidValue;
        break;
      }
      if (!parsed[k]) {
        parsed[k] = true;
        ++n_parsed;
      }
    }
    if (rc)
      break;
    if (n_parsed != 14) {
      rc = -kObjMaterialNotEnough;
      break;
    }
    materials.push_back(m);
    library[name] = (int)materials.size() - 1;
  }
  fclose(file);
  return rc;
}

}  // namespace

extern "C" int ffb_obj_parse(ffb_ctx* c, const char* text, unsigned long long n_bytes, const char* filename,
                             ffb_obj_info* info)
{
  FFB_TRY(check_ctx(c));
  if (!info || (n_bytes && !text))
    return fail(FFB_ERR_ARG, "bad OBJ arguments");
  if (n_bytes >= 0xFFFFFFF0ull)
    return fail(FFB_ERR_TOO_LARGE, "OBJ text of %llu bytes; at most 4 GiB", n_bytes);
  memset(info, 0, sizeof *info);
  c->obj_n_faces = -1;
  c->obj_meshes.clear();
  c->obj_materials.clear();
  const uint32_t n = (uint32_t)n_bytes;
  // the text, and its newlines per chunk
  FFB_TRY(upload(c, c->obj_text, text, n));
  const uint32_t chunks = (n + obj::kObjChunk - 1) / obj::kObjChunk;
  FFB_TRY(ensure(c, c->obj_chunk, sizeof(uint32_t) * (size_t)std::max(chunks, 1u)));
  FFB_TRY(ensure(c, c->obj_chunk_off, sizeof(uint32_t) * (size_t)(chunks + 1)));
  uint32_t n_nl = 0;
  if (chunks) {
    obj::k_obj_nl_count<<<chunks, obj::kObjThreads, 0, c->stream>>>(dptr<char>(c->obj_text), n,
                                                                      dptr<uint32_t>(c->obj_chunk));
    FFB_CUDA(cudaGetLastError());
    FFB_TRY(scan(c, dptr<uint32_t>(c->obj_chunk), (int)chunks, dptr<uint32_t>(c->obj_chunk_off)));
    FFB_CUDA(cudaMemcpyAsync(&n_nl, dptr<uint32_t>(c->obj_chunk_off) + chunks, sizeof n_nl,
                             cudaMemcpyDeviceToHost, c->stream));
    FFB_CUDA(cudaStreamSynchronize(c->stream));
  }
  const uint32_t n_lines = n_nl + ((n > 0 && text[n - 1] != '\n') ? 1u : 0u);
  FFB_TRY(ensure(c, c->obj_starts, sizeof(uint32_t) * ((size_t)n_nl + 2)));
  if (chunks) {
    obj::k_obj_line_starts<<<chunks, obj::kObjThreads, 0, c->stream>>>(
        dptr<char>(c->obj_text), n, dptr<uint32_t>(c->obj_chunk_off), dptr<uint32_t>(c->obj_starts));
    FFB_CUDA(cudaGetLastError());
  }
  const uint32_t sentinel = n + 1;  // the last line ends at n
  FFB_CUDA(cudaMemcpyAsync(dptr<uint32_t>(c->obj_starts) + n_nl + 1, &sentinel, sizeof sentinel,
                           cudaMemcpyHostToDevice, c->stream));
  // classes and ordinals
  const size_t L = std::max<size_t>(n_lines, 1);
  FFB_TRY(ensure(c, c->obj_flags, sizeof(uint32_t) * 3 * L));
  FFB_TRY(ensure(c, c->obj_ords, sizeof(uint32_t) * 3 * (L + 1)));
  uint32_t* is_v = dptr<uint32_t>(c->obj_flags);
  uint32_t* is_f = is_v + L;
  uint32_t* is_s = is_f + L;
  uint32_t* vord = dptr<uint32_t>(c->obj_ords);
  uint32_t* ford = vord + (L + 1);
  uint32_t* sord = ford + (L + 1);
  uint32_t counts[3] = {0, 0, 0};
  if (n_lines) {
    obj::k_obj_classify<<<grid_blocks(n_lines, 256, c->n_sm * 16), 256, 0, c->stream>>>(
        dptr<char>(c->obj_text), dptr<uint32_t>(c->obj_starts), n_lines, is_v, is_f, is_s);
    FFB_CUDA(cudaGetLastError());
    FFB_TRY(scan(c, is_v, (int)n_lines, vord));
    FFB_TRY(scan(c, is_f, (int)n_lines, ford));
    FFB_TRY(scan(c, is_s, (int)n_lines, sord));
    FFB_CUDA(cudaMemcpyAsync(&counts[0], vord + n_lines, 4, cudaMemcpyDeviceToHost, c->stream));
    FFB_CUDA(cudaMemcpyAsync(&counts[1], ford + n_lines, 4, cudaMemcpyDeviceToHost, c->stream));
    FFB_CUDA(cudaMemcpyAsync(&counts[2], sord + n_lines, 4, cudaMemcpyDeviceToHost, c->stream));
    FFB_CUDA(cudaStreamSynchronize(c->stream));
  }
  const uint32_t n_vertices = counts[0], n_faces = counts[1], n_special = counts[2];
  // parse
  FFB_TRY(ensure(c, c->obj_vertices, sizeof(float) * 3 * std::max<size_t>(n_vertices, 1)));
  FFB_TRY(ensure(c, c->obj_face_idx, sizeof(int32_t) * 3 * std::max<size_t>(n_faces, 1)));
  FFB_TRY(ensure(c, c->obj_face_line, sizeof(uint32_t) * std::max<size_t>(n_faces, 1)));
  FFB_TRY(ensure(c, c->obj_special, sizeof(uint32_t) * 2 * std::max<size_t>(n_special, 1)));
  FFB_TRY(ensure(c, c->obj_ranges, sizeof(uint32_t) * 2 * std::max<size_t>(n_special, 1)));
  FFB_TRY(ensure(c, c->obj_faces, sizeof(float) * 9 * std::max<size_t>(n_faces, 1)));
  FFB_TRY(ensure(c, c->obj_err, sizeof(unsigned long long)));
  FFB_CUDA(cudaMemsetAsync(c->obj_err.ptr, 0xFF, sizeof(unsigned long long), c->stream));
  uint32_t* sp_line = dptr<uint32_t>(c->obj_special);
  uint32_t* sp_faces = sp_line + std::max<uint32_t>(n_special, 1);
  if (n_lines) {
    obj::k_obj_parse<<<grid_blocks(n_lines, 256, c->n_sm * 16), 256, 0, c->stream>>>(
        dptr<char>(c->obj_text), dptr<uint32_t>(c->obj_starts), n_lines, is_v, vord, is_f, ford, is_s, sord,
        dptr<float>(c->obj_vertices), dptr<int32_t>(c->obj_face_idx), dptr<uint32_t>(c->obj_face_line), sp_line,
        sp_faces, dptr<unsigned long long>(c->obj_err));
    FFB_CUDA(cudaGetLastError());
  }
  if (n_faces) {
    obj::k_obj_gather<<<grid_blocks(n_faces, 256, c->n_sm * 16), 256, 0, c->stream>>>(
        dptr<float>(c->obj_vertices), n_vertices, dptr<int32_t>(c->obj_face_idx), dptr<uint32_t>(c->obj_face_line),
        n_faces, dptr<float>(c->obj_faces), dptr<unsigned long long>(c->obj_err));
    FFB_CUDA(cudaGetLastError());
  }
  std::vector<uint32_t> ranges(2 * (size_t)n_special), sp_count((size_t)n_special), sp_lines((size_t)n_special);
  if (n_special) {
    obj::k_obj_special_ranges<<<grid_blocks(n_special, 256, c->n_sm * 4), 256, 0, c->stream>>>(
        dptr<uint32_t>(c->obj_starts), sp_line, n_special, dptr<uint32_t>(c->obj_ranges));
    FFB_CUDA(cudaGetLastError());
    FFB_CUDA(cudaMemcpyAsync(ranges.data(), c->obj_ranges.ptr, sizeof(uint32_t) * ranges.size(),
                             cudaMemcpyDeviceToHost, c->stream));
    FFB_CUDA(cudaMemcpyAsync(sp_count.data(), sp_faces, sizeof(uint32_t) * n_special, cudaMemcpyDeviceToHost,
                             c->stream));
    FFB_CUDA(cudaMemcpyAsync(sp_lines.data(), sp_line, sizeof(uint32_t) * n_special, cudaMemcpyDeviceToHost,
                             c->stream));
  }
  unsigned long long dev_err = 0;
  FFB_CUDA(cudaMemcpyAsync(&dev_err, c->obj_err.ptr, sizeof dev_err, cudaMemcpyDeviceToHost, c->stream));
  FFB_CUDA(cudaStreamSynchronize(c->stream));
  // special lines in file order (obj_import.cpp:228-300), stopping at the
  // first error; a geometry error on an earlier line wins
  const unsigned long long dev_line = dev_err >> 8;
  int status = 0;
  unsigned long long err_line = ~0ull;
  std::vector<ffb_mesh> meshes;
  std::vector<ffb_material> materials;
  std::map<std::string, int> library;
  for (uint32_t i = 0; i < n_special && status == 0; ++i) {
    if (sp_lines[i] > dev_line)
      break;
    const std::string str(text + ranges[2 * i], text + ranges[2 * i + 1]);
    int r = 0;
    switch (str[0]) {
    case 'o':
    case 'g': {
      ffb_mesh m = {(int)sp_count[i], 0, 0};
      if (!meshes.empty())
        meshes.back().n_faces = (int)sp_count[i] - meshes.back().first_idx;
      meshes.push_back(m);
    } break;
    case 'u': {
      const std::string::size_type pos = str.find_first_of(" \t");
      if (pos == std::string::npos || str.substr(0, pos) != "usemtl") {
        r = -kObjFormatError;
        break;
      }
      const auto found = library.find(str.substr(pos + 1));
      if (found == library.end())
        r = -kObjMaterialNotDefined;
      else if (meshes.empty())
        r = -kObjFormatError;  // usemtl before any object (undefined in the reference)
      else
        meshes.back().material_idx = found->second;
    } break;
    case 'm': {
      if (strncmp("mtllib", str.c_str(), 6) != 0) {
        r = -kObjFormatError;
        break;
      }
      // the library path as obj_import.cpp:263-277 builds it
      const std::string library_name = str.size() > 7 ? str.substr(7) : std::string();
      std::string library_path = library_name;
      if (library_name.find("/\\") > library_name.length()) {
        std::string base_name(filename ? filename : "");
        const size_t dir_pos = base_name.find_last_of("/\\");
        base_name = dir_pos < base_name.length() ? base_name.substr(0, dir_pos + 1) : std::string();
        library_path = base_name + library_name;
      }
      r = material_lib(library_path.c_str(), materials, library);
    } break;
    }
    if (r < 0) {
      status = r;
      err_line = sp_lines[i];
    }
  }
  if (dev_err != ~0ull && dev_line < err_line) {
    status = -(int)(dev_err & 0xFF);
    err_line = dev_line;
  }
  info->n_vertices = (int)n_vertices;
  info->n_faces = (int)n_faces;
  info->status = status;
  info->error_line = status ? (int)(err_line + 1) : 0;
  if (status)
    return fail(FFB_ERR_FORMAT, "OBJ import failed with status %d at line %d", status, info->error_line);
  // meshes and materials as obj_import.cpp:320-340 finish them
  if (meshes.empty())
    meshes.push_back(ffb_mesh{0, (int)n_faces, 0});
  else
    meshes.back().n_faces = (int)n_faces - meshes.back().first_idx;
  if (materials.empty())
    materials.push_back(black_body());
  info->n_meshes = (int)meshes.size();
  info->n_materials = (int)materials.size();
  c->obj_meshes = meshes;
  c->obj_materials = materials;
  c->obj_n_faces = n_faces;
  return FFB_OK;
}

extern "C" int ffb_obj_load(ffb_ctx* c, const char* filename, ffb_obj_info* info)
{
  FFB_TRY(check_ctx(c));
  if (!filename || !info)
    return fail(FFB_ERR_ARG, "bad OBJ arguments");
  memset(info, 0, sizeof *info);
  FILE* f = fopen(filename, "rb");
  if (!f) {
    info->status = -kObjFileError;
    return fail(FFB_ERR_FILE, "cannot open %s", filename);
  }
  std::vector<char> text;
  char buf[1 << 16];
  size_t k;
  while ((k = fread(buf, 1, sizeof buf, f)) > 0)
    text.insert(text.end(), buf, buf + k);
  fclose(f);
  return ffb_obj_parse(c, text.data(), text.size(), filename, info);
}

extern "C" int ffb_obj_result(ffb_ctx* c, float* faces9, ffb_mesh* meshes, ffb_material* materials)
{
  FFB_TRY(check_ctx(c));
  if (c->obj_n_faces < 0)
    return fail(FFB_ERR_NO_SCENE, "no parsed OBJ scene");
  if (faces9 && c->obj_n_faces) {
    FFB_CUDA(cudaMemcpyAsync(faces9, c->obj_faces.ptr, sizeof(float) * 9 * (size_t)c->obj_n_faces, cudaMemcpyDefault,
                             c->stream));
    FFB_CUDA(cudaStreamSynchronize(c->stream));
  }
  if (meshes)
    memcpy(meshes, c->obj_meshes.data(), sizeof(ffb_mesh) * c->obj_meshes.size());
  if (materials)
    memcpy(materials, c->obj_materials.data(), sizeof(ffb_material) * c->obj_materials.size());
  return FFB_OK;
}

extern "C" int ffb_obj_scene_set(ffb_ctx* c)
{
  FFB_TRY(check_ctx(c));
  if (c->obj_n_faces < 0)
    return fail(FFB_ERR_NO_SCENE, "no parsed OBJ scene");
  return ffb_scene_set(c, dptr<float>(c->obj_faces), (int)c->obj_n_faces);
}

// ===========================================================================
// CSV text of the matrix (csv_export::export_csv, import_export/csv_export.cpp:26-46)
// ===========================================================================
namespace {

constexpr int kCsvSegmentTiles = 4096;  // tiles per staged segment (16.8 M entries, <= 218 MB of text)

// Formats the n x n matrix of `src`.  A device buffer gets the text from one
// single-pass launch (k_csv_fused).  Otherwise one length pass and one scan
// cover the whole matrix; then the text goes, for a host buffer or a file,
// segment by segment through a device staging buffer (a file gets pinned
// double buffers: the host writes one segment while the GPU formats the
// next).  Exactly one sink is used: text (device or host, cap bytes), file,
// or neither (length only).  *total gets the text length.
int csv_run(ffb_ctx* c, csv::Source src, char* text, unsigned long long cap, FILE* file, unsigned long long* total)
{
  // per device (the attribute belongs to the current device); cheap to repeat
  FFB_CUDA(cudaFuncSetAttribute(csv::k_csv_write, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)csv::write_smem(csv::kTileBytes)));
  src.n_entries = (long long)src.n * src.n;
  const long long n_tiles = (src.n_entries + csv::kTile - 1) / csv::kTile;
  const long long n_fused = (src.n_entries + csv::kFusedTile - 1) / csv::kFusedTile;
  FFB_TRY(ensure(c, c->csv_tile_len, sizeof(unsigned long long) * (size_t)std::max(n_tiles, n_fused)));
  FFB_TRY(ensure(c, c->csv_tile_off, sizeof(unsigned long long) * (size_t)(n_tiles + 2)));
  auto* tile_len = dptr<unsigned long long>(c->csv_tile_len);
  auto* tile_off = dptr<unsigned long long>(c->csv_tile_off);
  bool text_dev = false;
  FFB_TRY(ptr_kind(c, text, &text_dev));
  if (text_dev) {
    // one pass: the tile-length buffer holds the look-back status words; the
    // first two words of the offset buffer the ticket and error bits, then
    // the total
    FFB_CUDA(cudaFuncSetAttribute(csv::k_csv_fused, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)csv::kFusedSmem));
    FFB_CUDA(cudaMemsetAsync(tile_len, 0, sizeof(unsigned long long) * (size_t)n_fused, c->stream));
    FFB_CUDA(cudaMemsetAsync(tile_off, 0, 2 * sizeof(unsigned long long), c->stream));
    csv::FusedSink sink;
    sink.text = text;
    sink.cap = cap;
    sink.status = tile_len;
    sink.ticket = reinterpret_cast<unsigned int*>(tile_off);
    sink.err = reinterpret_cast<unsigned int*>(tile_off) + 1;
    sink.total = tile_off + 1;
    sink.n_tiles = n_fused;
    csv::k_csv_fused<<<(unsigned)n_fused, csv::kFusedThreads, csv::kFusedSmem, c->stream>>>(src, sink);
    FFB_CUDA(cudaGetLastError());
    unsigned long long aux[2] = {0, 0};  // {ticket | err << 32, total}
    FFB_CUDA(cudaMemcpyAsync(aux, tile_off, sizeof aux, cudaMemcpyDeviceToHost, c->stream));
    FFB_CUDA(cudaStreamSynchronize(c->stream));
    *total = aux[1];
    const unsigned err = (unsigned)(aux[0] >> 32);
    if (err & csv::kFusedTimeout)
      return fail(FFB_ERR_TIMEOUT, "CSV formatting: a tile's offset never arrived");
    if (err & csv::kFusedOverflow)
      return fail(FFB_ERR_ARG, "CSV text of %llu bytes does not fit the %llu-byte buffer", aux[1], cap);
    return FFB_OK;
  }
  csv::k_csv_len<<<(unsigned)n_tiles, csv::kThreads, 0, c->stream>>>(src, tile_len);
  csv::k_csv_scan<<<1, csv::kScanThreads, 0, c->stream>>>(tile_len, (int)n_tiles, tile_off);
  FFB_CUDA(cudaGetLastError());
  unsigned long long tail[2] = {0, 0};  // total, longest tile
  FFB_CUDA(cudaMemcpyAsync(tail, tile_off + n_tiles, sizeof tail, cudaMemcpyDeviceToHost, c->stream));
  FFB_CUDA(cudaStreamSynchronize(c->stream));
  const unsigned long long all = tail[0];
  *total = all;
  // shared text region sized for the longest tile (sparse matrices: a few KB)
  const size_t smem = csv::write_smem(tail[1]);
  const uint32_t region = (uint32_t)(smem - csv::kIndexSmem);
  if (!text && !file)
    return FFB_OK;
  if (text && all > cap)
    return fail(FFB_ERR_ARG, "CSV text of %llu bytes does not fit the %llu-byte buffer", all, cap);
  // staged: segment byte ranges from the tile offsets
  std::vector<unsigned long long> off((size_t)n_tiles + 1);
  FFB_CUDA(cudaMemcpy(off.data(), tile_off, sizeof(unsigned long long) * off.size(), cudaMemcpyDeviceToHost));

  unsigned long long seg_max = 0;
  for (long long t = 0; t < n_tiles; t += kCsvSegmentTiles)
    seg_max = std::max(seg_max, off[(size_t)std::min(n_tiles, t + kCsvSegmentTiles)] - off[(size_t)t]);
  FFB_TRY(ensure(c, c->csv_text, std::max<size_t>(seg_max, 16)));
  char* stage = dptr<char>(c->csv_text);
  if (file) {
    for (int k = 0; k < 2; ++k) {
      if (seg_max > c->csv_pinned_cap[k]) {
        if (c->csv_pinned[k])
          cudaFreeHost(c->csv_pinned[k]);
        c->csv_pinned[k] = nullptr;
        c->csv_pinned_cap[k] = 0;
        FFB_CUDA(cudaMallocHost(&c->csv_pinned[k], seg_max));
        c->csv_pinned_cap[k] = seg_max;
      }
    }
  }
  int prev = -1, cur = 0;
  unsigned long long prev_len = 0;
  for (long long t = 0; t < n_tiles; t += kCsvSegmentTiles) {
    const long long te = std::min(n_tiles, t + kCsvSegmentTiles);
    const unsigned long long b0 = off[(size_t)t], len = off[(size_t)te] - b0;
    csv::k_csv_write<<<(unsigned)(te - t), csv::kThreads, smem, c->stream>>>(src, tile_off, t, b0, region, stage);
    FFB_CUDA(cudaGetLastError());
    if (text) {
      FFB_CUDA(cudaMemcpyAsync(text + b0, stage, len, cudaMemcpyDeviceToHost, c->stream));
      continue;
    }
    FFB_CUDA(cudaMemcpyAsync(c->csv_pinned[cur], stage, len, cudaMemcpyDeviceToHost, c->stream));
    // the host writes the previous segment while the GPU formats this one
    if (prev >= 0 && fwrite(c->csv_pinned[prev], 1, prev_len, file) != prev_len)
      return fail(FFB_ERR_FILE, "CSV write failed");
    FFB_CUDA(cudaStreamSynchronize(c->stream));  // this segment is in pinned[cur]; stage is free again
    prev = cur;
    prev_len = len;
    cur ^= 1;
  }
  FFB_CUDA(cudaStreamSynchronize(c->stream));
  if (file && prev >= 0 && fwrite(c->csv_pinned[prev], 1, prev_len, file) != prev_len)
    return fail(FFB_ERR_FILE, "CSV write failed");
  return FFB_OK;
}

int csv_source(ffb_ctx* c, const float* ff, const uint32_t* counts, const int32_t* outgoing, int n, csv::Source* src)
{
  FFB_TRY(check_ctx(c));
  if (n < 0 || (!ff && (!counts || !outgoing)))
    return fail(FFB_ERR_ARG, "bad CSV arguments");
  if (n > kMaxRows)
    return fail(FFB_ERR_TOO_LARGE, "n %d above %d", n, kMaxRows);
  const size_t mat = (size_t)n * n;
  memset(src, 0, sizeof *src);
  src->n = n;
  if (!n)
    return FFB_OK;
  if (ff) {
    const void* d;
    FFB_TRY(input_ptr(c, ff, sizeof(float) * mat, c->tmp_in, &d));
    src->ff = (const float*)d;
  } else {
    const void* d;
    FFB_TRY(input_ptr(c, counts, sizeof(uint32_t) * mat, c->tmp_in, &d));
    src->counts = (const uint32_t*)d;
    const void* o;
    FFB_TRY(input_ptr(c, outgoing, sizeof(int32_t) * (size_t)n, c->front_dev, &o));
    src->outgoing = (const int32_t*)o;
  }
  return FFB_OK;
}

int csv_format(ffb_ctx* c, const float* ff, const uint32_t* counts, const int32_t* outgoing, int n, char* text,
               unsigned long long text_cap, unsigned long long* text_len)
{
  if (!text_len)
    return fail(FFB_ERR_ARG, "null text_len");
  csv::Source src;
  FFB_TRY(csv_source(c, ff, counts, outgoing, n, &src));
  unsigned long long total = 0;
  if (n)
    FFB_TRY(csv_run(c, src, text, text_cap, nullptr, &total));
  *text_len = total;
  return FFB_OK;
}

int csv_export(ffb_ctx* c, const char* filename, const float* ff, const uint32_t* counts, const int32_t* outgoing,
               int n)
{
  if (!filename)
    return fail(FFB_ERR_ARG, "null file name");
  csv::Source src;
  FFB_TRY(csv_source(c, ff, counts, outgoing, n, &src));
  FILE* f = fopen(filename, "wb");
  if (!f)
    return fail(FFB_ERR_FILE, "cannot open %s for writing", filename);
  unsigned long long total = 0;
  const int rc = n ? csv_run(c, src, nullptr, 0, f, &total) : FFB_OK;
  if (fclose(f) != 0 && rc == FFB_OK)
    return fail(FFB_ERR_FILE, "closing %s failed", filename);
  return rc;
}

}  // namespace

extern "C" int ffb_csv_format(ffb_ctx* c, const float* ff, int n, char* text, unsigned long long text_cap,
                              unsigned long long* text_len)
{
  if (!ff && n)
    return fail(FFB_ERR_ARG, "null matrix");
  return csv_format(c, ff, nullptr, nullptr, n, text, text_cap, text_len);
}

extern "C" int ffb_csv_format_counts(ffb_ctx* c, const uint32_t* counts, const int32_t* outgoing, int n, char* text,
                                     unsigned long long text_cap, unsigned long long* text_len)
{
  if ((!counts || !outgoing) && n)
    return fail(FFB_ERR_ARG, "null counts or outgoing");
  return csv_format(c, nullptr, counts, outgoing, n, text, text_cap, text_len);
}

extern "C" int ffb_csv_export(ffb_ctx* c, const char* filename, const float* ff, int n)
{
  if (!ff && n)
    return fail(FFB_ERR_ARG, "null matrix");
  return csv_export(c, filename, ff, nullptr, nullptr, n);
}

extern "C" int ffb_csv_export_counts(ffb_ctx* c, const char* filename, const uint32_t* counts, const int32_t* outgoing,
                                     int n)
{
  if ((!counts || !outgoing) && n)
    return fail(FFB_ERR_ARG, "null counts or outgoing");
  return csv_export(c, filename, nullptr, counts, outgoing, n);
}

// ===========================================================================
// Batched scenes: one fused launch over many independent scenes
// ===========================================================================
extern "C" int ffb_batch_set(ffb_ctx* c, int n_scenes, const long long* face_offsets, const float* faces9,
                             const ffb_grid_params* params)
{
  FFB_TRY(check_ctx(c));
  if (n_scenes <= 0 || n_scenes > kMaxBatchScenes || !face_offsets || !faces9)
    return fail(FFB_ERR_ARG, "batch of %d scenes (1..%d) without offsets or faces", n_scenes, kMaxBatchScenes);
  for (int s = 0; s < n_scenes; ++s) {
    const long long n = face_offsets[s + 1] - face_offsets[s];
    if (face_offsets[s] < 0 || n <= 0 || n > 0x7FFFFFFF)
      return fail(FFB_ERR_ARG, "scene %d has %lld faces", s, n);
  }
  for (SceneData& s : c->batch)
    release_scene(c, s);
  c->batch.clear();
  c->batch.resize((size_t)n_scenes);
  c->batch_offsets.assign(face_offsets, face_offsets + n_scenes + 1);
  c->batch_frames_mode = -1;
  c->batch_n_chunks = 0;
  c->batch_shape.assign((size_t)n_scenes, 0);
  for (int s = 0; s < n_scenes; ++s) {
    const long long f0 = face_offsets[s];
    const int n = (int)(face_offsets[s + 1] - f0);
    FFB_TRY(scene_upload(c, c->batch[s], faces9 + 9 * f0, n));
    FFB_TRY(grid_build(c, c->batch[s], params ? params + s : nullptr));
  }
  return FFB_OK;
}

extern "C" int ffb_batch_grid_info(ffb_ctx* c, int scene, ffb_grid_info* out)
{
  if (!c || !out || scene < 0 || scene >= (int)c->batch.size())
    return fail(FFB_ERR_ARG, "bad batch scene %d", scene);
  *out = c->batch[scene].info;
  return FFB_OK;
}

extern "C" int ffb_batch_prepare(ffb_ctx* c, const int32_t* front, const int32_t* rear, const uint64_t* seeds,
                                 int flags)
{
  FFB_TRY(check_ctx(c));
  const int n_scenes = (int)c->batch.size();
  if (!n_scenes)
    return fail(FFB_ERR_NO_SCENE, "no batch set");
  const long long n_all = c->batch_offsets[n_scenes];
  long long total = 0;
  FFB_TRY(check_counts((int)n_all, front, rear, &total));
  // The chunk table, scene after scene, written on the device from one
  // 16-byte record per emitting face (scene-local face, front rays, rays,
  // first chunk): the host's work and upload are linear in faces, not rays.
  // As in a single-scene launch, the faces holding the last sixteenth of a
  // scene's rays get 64-ray chunks (its launch's tail is shorter).
  constexpr int kTailRays = 64;
  std::vector<int4> src, tail;
  src.reserve((size_t)n_all);
  c->batch_chunk_first.assign(n_scenes + 1, 0);
  long long next = 0;
  for (int s = 0; s < n_scenes; ++s) {
    const long long f0 = c->batch_offsets[s];
    c->batch_chunk_first[s] = (int)next;
    long long all = 0, rays = 0;
    for (int f = 0; f < c->batch[s].n_faces; ++f)
      all += (long long)front[f0 + f] + rear[f0 + f];
    const long long tail_from = all - all / 16;
    for (int f = 0; f < c->batch[s].n_faces; ++f) {
      const long long nf = (long long)front[f0 + f] + rear[f0 + f];
      if (nf == 0)
        continue;
      if (nf > INT_MAX - kChunkRays)
        return fail(FFB_ERR_TOO_LARGE, "scene %d face %d emits %lld rays; at most %d", s, f, nf,
                    INT_MAX - kChunkRays);
      const int size = rays >= tail_from ? kTailRays : kChunkRays;
      (size == kChunkRays ? src : tail).push_back(make_int4(f, front[f0 + f], (int)nf, (int)next));
      next += (nf + size - 1) / size;
      rays += nf;
      if (next > INT_MAX)
        return fail(FFB_ERR_TOO_LARGE, "more than %d work chunks", INT_MAX);
    }
  }
  c->batch_chunk_first[n_scenes] = (int)next;
  c->batch_n_chunks = (int)next;
  if (next > 0) {
    FFB_TRY(ensure(c, c->batch_chunks, sizeof(Chunk) * (size_t)next));
    const size_t nh = src.size();
    src.insert(src.end(), tail.begin(), tail.end());  // one staged upload
    FFB_TRY(upload(c, c->chunk_src, src.data(), sizeof(int4) * src.size()));
    if (nh)
      k_chunk_fill<kChunkRays><<<grid_blocks((long long)nh * 32, 256, c->n_sm * 8), 256, 0, c->stream>>>(
          dptr<int4>(c->chunk_src), (int)nh, dptr<Chunk>(c->batch_chunks));
    if (!tail.empty())
      k_chunk_fill<kTailRays><<<grid_blocks((long long)tail.size() * 32, 256, c->n_sm * 8), 256, 0, c->stream>>>(
          dptr<int4>(c->chunk_src) + nh, (int)tail.size(), dptr<Chunk>(c->batch_chunks));
    FFB_CUDA(cudaGetLastError());
  }
  std::vector<uint2> keys((size_t)n_scenes);
  for (int s = 0; s < n_scenes; ++s) {
    const uint64_t k = seeds ? seeds[s] : 1;
    keys[s] = make_uint2((uint32_t)k, (uint32_t)(k >> 32));
  }
  FFB_TRY(upload(c, c->batch_keys, keys.data(), sizeof(uint2) * keys.size()));
  const int mode = flags & FFB_EMIT_REF_NORMAL;
  if (c->batch_frames_mode != mode) {
    FFB_TRY(ensure(c, c->batch_frames, sizeof(float) * 20 * (size_t)n_all));
    for (int s = 0; s < n_scenes; ++s)
      FFB_TRY(build_frames(c, dptr<float>(c->batch[s].faces), c->batch[s].n_faces, mode,
                           dptr<float>(c->batch_frames) + 20 * c->batch_offsets[s]));
    c->batch_frames_mode = mode;
  }
  FFB_TRY(ensure(c, c->cursor, sizeof(uint32_t) * (size_t)std::max(n_scenes, kMaxPipeBlocks)));
  FFB_TRY(ensure(c, c->batch_epoch, sizeof(uint32_t)));
  FFB_TRY(ensure(c, c->stats, sizeof(unsigned long long) * kStatSlots));
  FFB_CUDA(cudaMemsetAsync(c->batch_epoch.ptr, 0, sizeof(uint32_t), c->stream));
  FFB_CUDA(cudaStreamSynchronize(c->stream));
  return FFB_OK;
}

extern "C" int ffb_batch_launch(ffb_ctx* c, uint32_t* counts, const unsigned long long* counts_offsets,
                                unsigned long long counts_words, int advance_epoch)
{
  FFB_TRY(check_ctx(c));
  const int n_scenes = (int)c->batch.size();
  if (!n_scenes || !c->batch_keys.ptr)
    return fail(FFB_ERR_NO_SCENE, "batch not set and prepared");
  if (!counts || !counts_offsets)
    return fail(FFB_ERR_ARG, "null counts");
  for (int s = 0; s < n_scenes; ++s) {
    const unsigned long long n = (unsigned long long)c->batch[s].n_faces;
    if (counts_offsets[s] + n * n > counts_words)
      return fail(FFB_ERR_ARG, "scene %d matrix beyond the counts buffer", s);
    if (c->batch[s].n_faces > kMaxRows)
      return fail(FFB_ERR_TOO_LARGE, "scene %d has more than %d faces", s, kMaxRows);
  }
  bool counts_dev = false;
  FFB_TRY(ptr_kind(c, counts, &counts_dev));
  if (!counts_dev)
    return fail(FFB_ERR_ARG, "batched counts must be device memory");
  FFB_CUDA(cudaMemsetAsync(counts, 0, sizeof(uint32_t) * counts_words, c->stream));
  FFB_CUDA(cudaMemsetAsync(c->stats.ptr, 0, sizeof(unsigned long long) * kStatSlots, c->stream));
  FFB_CUDA(cudaMemsetAsync(c->cursor.ptr, 0, sizeof(uint32_t) * (size_t)n_scenes, c->stream));
  if (advance_epoch) {
    k_epoch_bump<<<1, 32, 0, c->stream>>>(dptr<uint32_t>(c->batch_epoch));
    FFB_CUDA(cudaGetLastError());
  }
  if (c->batch_n_chunks == 0)
    return FFB_OK;
  FFB_TRY(ensure_batch_streams(c));
  constexpr int kSide = (int)(sizeof(c->batch_streams) / sizeof(c->batch_streams[0]));
  FFB_CUDA(cudaEventRecord(c->batch_fork, c->stream));
  for (int k = 0; k < kSide; ++k)
    FFB_CUDA(cudaStreamWaitEvent(c->batch_streams[k], c->batch_fork, 0));
  // largest scenes first, dealt round-robin over the side streams
  std::vector<int> order(n_scenes);
  for (int s = 0; s < n_scenes; ++s)
    order[s] = s;
  const std::vector<int>& first = c->batch_chunk_first;
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return first[a + 1] - first[a] > first[b + 1] - first[b]; });
  int k = 0;
  for (int s : order) {
    if (first[s + 1] == first[s])
      continue;
    TraceParams p;
    p.frames = dptr<float>(c->batch_frames);
    p.chunks = dptr<Chunk>(c->batch_chunks) + first[s];
    p.n_chunks = first[s + 1] - first[s];
    p.key0 = p.key1 = p.epoch = 0;
    p.epoch_ptr = dptr<uint32_t>(c->batch_epoch);
    p.scene_keys = dptr<uint2>(c->batch_keys) + s;
    p.chunk_cursor = dptr<uint32_t>(c->cursor) + s;
    p.stats = c->stats_on ? dptr<unsigned long long>(c->stats) : nullptr;
    p.power = nullptr;
    p.absorb = nullptr;
    p.span = nullptr;
    SceneSlot& slot = p.scene;
    slot.g = make_view(c->batch[s]);
    slot.counts = counts + counts_offsets[s];
    slot.face_to_row = nullptr;
    slot.face_base = (int)c->batch_offsets[s];
    slot.n_cols = c->batch[s].n_faces;
    cudaStream_t st = c->batch_streams[k++ % kSide];
    const int shape = s < (int)c->batch_shape.size() ? c->batch_shape[(size_t)s] : 0;
    if (c->batch[s].info.skip_empty)
      FFB_TRY((launch_fused<true>(c, p, false, st, shape)));
    else
      FFB_TRY((launch_fused<false>(c, p, false, st, shape)));
  }
  for (int j = 0; j < kSide; ++j) {
    FFB_CUDA(cudaEventRecord(c->batch_join[j], c->batch_streams[j]));
    FFB_CUDA(cudaStreamWaitEvent(c->stream, c->batch_join[j], 0));
  }
  return FFB_OK;
}

// ===========================================================================
// Autotuning: grid and launch shape
// ===========================================================================
namespace {

// Process-wide cache of tuning choices: (faces in half-octaves, scene-box
// aspect in octaves, rays per emitting face in octaves, jumps on/off).
typedef std::tuple<int, int, int, int> TuneKey;
struct TuneChoice {
  ffb_grid_params grid;
  int shape;
};
std::mutex g_tune_mu;
std::map<TuneKey, TuneChoice> g_tune_cache;

int tune_key(ffb_ctx* c, SceneData& s, const int32_t* front, const int32_t* rear, int skip, TuneKey* key)
{
  uint32_t ord[6];
  FFB_CUDA(cudaMemcpyAsync(ord, s.scene_ord.ptr, sizeof ord, cudaMemcpyDeviceToHost, c->stream));
  FFB_CUDA(cudaStreamSynchronize(c->stream));
  double lo = INFINITY, hi = 0.0;
  for (int a = 0; a < 3; ++a) {
    const double e = (double)ord2f(ord[3 + a]) - (double)ord2f(ord[a]);
    if (e > 0.0 && std::isfinite(e)) {
      lo = std::min(lo, e);
      hi = std::max(hi, e);
    }
  }
  const int aspect = hi > 0.0 ? (int)std::lround(std::log2(hi / std::max(lo, hi * 1e-3))) : 0;
  long long rays = 0, emitting = 0;
  for (int f = 0; f < s.n_faces; ++f) {
    const long long nf = (long long)front[f] + rear[f];
    rays += nf;
    emitting += nf > 0;
  }
  const int per_face = emitting ? (int)std::lround(std::log2(std::max(1.0, (double)rays / emitting))) : 0;
  *key = TuneKey((int)std::lround(2.0 * std::log2((double)std::max(s.n_faces, 1))), aspect, per_face, skip);
  return FFB_OK;
}

// Kernel time (ms, best of two runs: the first warms the grid into L2) of
// the sample trace in launch shape `shape`, counts into device `counts`.
int time_sample(ffb_ctx* c, const int32_t* fr, const int32_t* re, uint64_t seed, uint32_t* counts, int shape,
                float* ms)
{
  const int saved_shape = c->trace_shape;
  const bool saved_stats = c->stats_on;
  c->trace_shape = shape;
  c->stats_on = false;
  float best = INFINITY;
  int rc = FFB_OK;
  for (int rep = 0; rep < 2 && rc == FFB_OK; ++rep) {
    rc = ffb_form_factor_counts(c, fr, re, seed, 0, 0, nullptr, c->main.n_faces, counts);
    float t = 0;
    if (rc == FFB_OK && cudaStreamSynchronize(c->stream) == cudaSuccess &&
        cudaEventElapsedTime(&t, c->ev0, c->ev1) == cudaSuccess)
      best = std::min(best, t);
    else if (rc == FFB_OK)
      rc = fail(FFB_ERR_CUDA, "timing of a tuning sample failed: %s", cudaGetErrorString(cudaGetLastError()));
  }
  c->trace_shape = saved_shape;
  c->stats_on = saved_stats;
  *ms = best;
  return rc;
}

}  // namespace

extern "C" int ffb_trace_shape_count(void) { return kNumShapes; }

extern "C" int ffb_trace_shape_get(int shape, ffb_trace_shape* out)
{
  if (shape < 0 || shape >= kNumShapes || !out)
    return fail(FFB_ERR_ARG, "shape %d outside [0, %d)", shape, kNumShapes);
  const TraceShape t = trace_shape(shape);
  *out = ffb_trace_shape{t.adv, t.test, t.refill, t.blocks, t.coherent, t.lanes};
  return FFB_OK;
}

extern "C" int ffb_ctx_set_trace_shape(ffb_ctx* c, int shape)
{
  if (!c)
    return fail(FFB_ERR_ARG, "null context");
  if (shape < 0 || shape >= kNumShapes)
    return fail(FFB_ERR_ARG, "shape %d outside [0, %d)", shape, kNumShapes);
  c->trace_shape = shape;
  return FFB_OK;
}

extern "C" int ffb_ctx_trace_shape(ffb_ctx* c) { return c ? c->trace_shape : FFB_ERR_ARG; }

extern "C" int ffb_autotune(ffb_ctx* c, const int32_t* front, const int32_t* rear, uint64_t seed,
                            const ffb_grid_params* candidates, int n_candidates, int sample_every, int flags,
                            uint32_t* scratch, ffb_tune_result* out)
{
  FFB_TRY(check_ctx(c));
  SceneData& s = c->main;
  if (s.n_faces <= 0)
    return fail(FFB_ERR_NO_SCENE, "no scene");
  if (s.n_faces > kMaxRows)
    return fail(FFB_ERR_TOO_LARGE, "scene of %d faces; at most %d", s.n_faces, kMaxRows);
  if (candidates && n_candidates <= 0)
    return fail(FFB_ERR_ARG, "no candidates");
  long long total = 0;
  FFB_TRY(check_counts(s.n_faces, front, rear, &total));
  std::vector<ffb_grid_params> cands;
  if (candidates) {
    cands.assign(candidates, candidates + n_candidates);
  } else {
    for (float cpf : {32.f, 64.f, 128.f, 192.f, 256.f})
      cands.push_back(ffb_grid_params{0, 0, 0, cpf, 1});
  }
  int skip_key = 0;
  for (const ffb_grid_params& g : cands)
    skip_key |= g.skip_empty ? 1 : 2;
  ffb_tune_result res{};
  TuneKey key;
  FFB_TRY(tune_key(c, s, front, rear, skip_key, &key));
  if (!(flags & FFB_TUNE_FORCE)) {
    TuneChoice hit{};
    bool found = false;
    {
      std::lock_guard<std::mutex> lock(g_tune_mu);
      auto it = g_tune_cache.find(key);
      if (it != g_tune_cache.end()) {
        hit = it->second;
        found = true;
      }
    }
    if (found) {
      FFB_TRY(grid_build(c, s, &hit.grid));
      c->trace_shape = hit.shape;
      res.grid = hit.grid;
      res.shape = hit.shape;
      res.from_cache = 1;
      if (out)
        *out = res;
      return FFB_OK;
    }
  }
  // the sample: every k-th face emits its rays (the same rays as in the full solve)
  if (sample_every <= 0)
    sample_every = (int)std::max<long long>(1, (total + (2ll << 20)) / (4ll << 20));
  std::vector<int32_t> fr((size_t)s.n_faces, 0), re((size_t)s.n_faces, 0);
  long long sample_rays = 0;
  for (int f = 0; f < s.n_faces; f += sample_every) {
    fr[f] = front[f];
    re[f] = rear[f];
    sample_rays += (long long)front[f] + rear[f];
  }
  res.sample_rays = sample_rays;
  uint32_t* counts = scratch;
  if (counts) {
    bool dev = false;
    FFB_TRY(ptr_kind(c, counts, &dev));
    if (!dev)
      return fail(FFB_ERR_ARG, "tuning scratch must be device memory");
  } else {
    FFB_TRY(ensure(c, c->ff_counts, sizeof(uint32_t) * (size_t)s.n_faces * s.n_faces));
    counts = dptr<uint32_t>(c->ff_counts);
  }
  int best_g = 0, best_shape = 0;
  float best_t = INFINITY;
  if (sample_rays > 0) {
    for (size_t i = 0; i < cands.size(); ++i) {
      FFB_TRY(grid_build(c, s, &cands[i]));
      float t;
      FFB_TRY(time_sample(c, fr.data(), re.data(), seed, counts, 0, &t));
      ++res.timed;
      if (t < best_t) {
        best_t = t;
        best_g = (int)i;
      }
    }
    FFB_TRY(grid_build(c, s, &cands[(size_t)best_g]));
    for (int shape = 1; shape < kNumShapes; ++shape) {
      float t;
      FFB_TRY(time_sample(c, fr.data(), re.data(), seed, counts, shape, &t));
      ++res.timed;
      if (t < best_t) {
        best_t = t;
        best_shape = shape;
      }
    }
  } else {
    FFB_TRY(grid_build(c, s, &cands[0]));
    best_t = 0.f;
  }
  c->trace_shape = best_shape;
  res.grid = cands[(size_t)best_g];
  res.shape = best_shape;
  res.sample_ms = best_t;
  if (sample_rays > 0) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune_cache[key] = TuneChoice{res.grid, res.shape};
  }
  if (out)
    *out = res;
  return FFB_OK;
}

extern "C" int ffb_autotune_grid(ffb_ctx* c, const int32_t* front, const int32_t* rear, uint64_t seed,
                                 const ffb_grid_params* candidates, int n_candidates, int sample_every,
                                 ffb_grid_params* best, float* best_ms)
{
  FFB_TRY(check_ctx(c));
  if (!candidates || n_candidates <= 0 || !best)
    return fail(FFB_ERR_ARG, "no candidates");
  SceneData& s = c->main;
  if (s.n_faces <= 0)
    return fail(FFB_ERR_NO_SCENE, "no scene");
  if (s.n_faces > kMaxRows)
    return fail(FFB_ERR_TOO_LARGE, "scene too large");
  long long total = 0;
  FFB_TRY(check_counts(s.n_faces, front, rear, &total));
  if (sample_every < 1)
    sample_every = 1;
  std::vector<int32_t> fr((size_t)s.n_faces, 0), re((size_t)s.n_faces, 0);
  for (int f = 0; f < s.n_faces; f += sample_every) {
    fr[f] = front[f];
    re[f] = rear[f];
  }
  FFB_TRY(ensure(c, c->ff_counts, sizeof(uint32_t) * (size_t)s.n_faces * s.n_faces));
  float best_t = INFINITY;
  int best_i = 0;
  for (int i = 0; i < n_candidates; ++i) {
    FFB_TRY(grid_build(c, s, candidates + i));
    float t;
    FFB_TRY(time_sample(c, fr.data(), re.data(), seed, dptr<uint32_t>(c->ff_counts), c->trace_shape, &t));
    if (t < best_t) {
      best_t = t;
      best_i = i;
    }
  }
  *best = candidates[best_i];
  if (best_ms)
    *best_ms = best_t;
  return grid_build(c, s, best);
}

extern "C" int ffb_batch_autotune(ffb_ctx* c, const int32_t* front, const int32_t* rear, int* shapes)
{
  FFB_TRY(check_ctx(c));
  const int n_scenes = (int)c->batch.size();
  if (!n_scenes)
    return fail(FFB_ERR_NO_SCENE, "no batch set");
  long long total = 0;
  FFB_TRY(check_counts((int)c->batch_offsets[n_scenes], front, rear, &total));
  c->batch_shape.assign((size_t)n_scenes, 0);
  for (int i = 0; i < n_scenes; ++i) {
    SceneData& b = c->batch[i];
    const long long f0 = c->batch_offsets[i];
    TuneKey key;
    FFB_TRY(tune_key(c, b, front + f0, rear + f0, 1, &key));
    TuneChoice choice{};
    bool found = false;
    {
      std::lock_guard<std::mutex> lock(g_tune_mu);
      auto it = g_tune_cache.find(key);
      if (it != g_tune_cache.end()) {
        choice = it->second;
        found = true;
      }
    }
    if (!found) {
      // tune on this scene through the main scene (the faces copy on the device)
      c->frames_mode = -1;
      FFB_TRY(scene_upload(c, c->main, dptr<float>(b.faces), b.n_faces));
      ffb_tune_result r;
      FFB_TRY(ffb_autotune(c, front + f0, rear + f0, 1, nullptr, 0, 0, FFB_TUNE_FORCE, nullptr, &r));
      choice = TuneChoice{r.grid, r.shape};
    }
    FFB_TRY(grid_build(c, b, &choice.grid));
    c->batch_shape[(size_t)i] = choice.shape;
    if (shapes)
      shapes[i] = choice.shape;
  }
  return FFB_OK;
}

extern "C" int ffb_stats_get(ffb_ctx* c, ffb_stats* out)
{
  FFB_TRY(check_ctx(c));
  if (!out)
    return fail(FFB_ERR_ARG, "null output");
  memset(out, 0, sizeof *out);
  FFB_CUDA(cudaStreamSynchronize(c->stream));
  if (c->stats.ptr) {
    unsigned long long s[kStatSlots];
    FFB_CUDA(cudaMemcpy(s, c->stats.ptr, sizeof s, cudaMemcpyDeviceToHost));
    out->tests = s[kStatTests];
    out->cells = s[kStatCells];
    out->rays = s[kStatRays];
    out->hits = s[kStatHits];
    out->jumps = s[kStatJumps];
  }
  out->d2h_bytes = c->last_d2h;
  if (c->timed)
    cudaEventElapsedTime(&out->kernel_ms, c->ev0, c->ev1);
  return FFB_OK;
}
