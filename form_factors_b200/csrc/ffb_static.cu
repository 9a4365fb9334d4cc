// ffb_static.cu -- ffb_cast_bruteforce_static: the brute-force ray cast for
// callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: a process whose device memory is
// entirely pre-reserved by its own allocator, or a plugin host that forbids
// device allocations after start-up.  For them this entry point keeps its
// only scratch -- the precomputed 64-byte triangle records that
// ffb_cast_bruteforce keeps in context memory -- in the file-scope array
// below.  The caller passes the faces, the rays and both outputs in device
// memory; nothing is allocated or freed on any call.
//
// Limits and sharing:
//  * at most kStaticMaxFaces faces per call (1 MiB of records); larger
//    scenes are rejected with FFB_ERR_TOO_LARGE;
//  * every GPU that loads the library holds the array until the process
//    exits;
//  * all calls share the array and it keeps the last call's records; calls
//    that overlap on the GPU (on different streams, or from several host
//    threads) race on it and must be serialised by the caller;
//  * the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress) with that device current; make that first call
//    before any stream capture.
#include <mutex>

#include <cuda_runtime.h>

#include "ffb.h"
#include "ffb_device.cuh"

namespace {

constexpr int kStaticMaxFaces = 16384;
constexpr int kThreads = 128;
constexpr int kTile = 128;
constexpr int kMaxDevices = 64;
constexpr long long kMaxGridX = 0x7FFFFFFFLL;  // largest grid x dimension of a launch

// The static scratch: one triangle record per face.
__device__ __align__(256) ffb::TriRec g_static_records[kStaticMaxFaces];

std::mutex g_setup_mutex;
ffb::TriRec* g_records_ptr[kMaxDevices] = {};

// Triangle records (math/triangle.cpp:34-38,58-64 precomputed per face).
__global__ void k_static_records(const float* __restrict__ faces9, int n_faces, ffb::TriRec* __restrict__ rec)
{
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= n_faces)
    return;
  const float* p = faces9 + 9 * (size_t)f;
  rec[f] = ffb::make_trirec(ffb::f3(p[0], p[1], p[2]), ffb::f3(p[3], p[4], p[5]), ffb::f3(p[6], p[7], p[8]));
}

// Every ray against every face in index order with a strict '<' on the
// squared distance (ray_caster/naive_cpu.cpp:65-97), records staged through
// shared memory.
__global__ void __launch_bounds__(kThreads) k_static_brute(const ffb::TriRec* __restrict__ rec, int n_faces,
                                                           const float* __restrict__ rays6, long long n_rays,
                                                           int32_t* __restrict__ hit_face,
                                                           float* __restrict__ hit_point)
{
  __shared__ ffb::TriRec tile[kTile];
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = i < n_rays;
  float3 o = ffb::f3(0.f, 0.f, 0.f), e = ffb::f3(0.f, 0.f, 0.f);
  if (live) {
    const float* r = rays6 + 6 * i;
    o = ffb::f3(r[0], r[1], r[2]);
    e = ffb::f3(r[3], r[4], r[5]);
  }
  const float3 dir = ffb::sub3(e, o);
  float best = 3.40282347e+38f;
  int best_idx = -1;
  float3 best_pt = ffb::f3(NAN, NAN, NAN);
  for (int base = 0; base < n_faces; base += kTile) {
    __syncthreads();
    for (int k = threadIdx.x; k < kTile && base + k < n_faces; k += blockDim.x)
      tile[k] = rec[base + k];
    __syncthreads();
    const int m = min(kTile, n_faces - base);
    if (live) {
      for (int k = 0; k < m; ++k) {
        float3 pt;
        if (ffb::tri_hit(reinterpret_cast<const float4*>(tile + k), o, dir, pt)) {
          const float d = ffb::dist2(pt, o);
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

// True for memory that device `dev` takes as a kernel operand: its own device
// memory, or managed memory.  Host memory and another device's memory are
// refused (the kernels would fault on them, or reach them only through peer
// access).
bool on_device(const void* p, int dev)
{
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeManaged || (a.type == cudaMemoryTypeDevice && a.device == dev);
}

}  // namespace

// Error reporting shared with the rest of the C ABI (ffb_api.cu).
int ffb_set_error(int code, const char* msg);

extern "C" int ffb_cast_bruteforce_static(const float* faces9, int n_faces, const float* rays6, long long n_rays,
                                          int32_t* hit_face, float* hit_point, void* stream)
{
  if (n_faces < 0 || n_rays < 0)
    return ffb_set_error(FFB_ERR_ARG, "ffb_cast_bruteforce_static: negative size");
  if (n_faces > kStaticMaxFaces)
    return ffb_set_error(FFB_ERR_TOO_LARGE,
                         "ffb_cast_bruteforce_static: n_faces above the static scratch limit of 16384 faces");
  if (n_rays == 0)
    return FFB_OK;
  if (!rays6 || !hit_face || (n_faces > 0 && !faces9))
    return ffb_set_error(FFB_ERR_ARG, "ffb_cast_bruteforce_static: null pointer");
  // one thread per ray: the grid's x dimension bounds the rays of one call
  if ((n_rays + kThreads - 1) / kThreads > (long long)kMaxGridX)
    return ffb_set_error(FFB_ERR_TOO_LARGE, "ffb_cast_bruteforce_static: n_rays above 2^31 - 1 blocks of 128 rays");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return ffb_set_error(FFB_ERR_NO_DEVICE, "ffb_cast_bruteforce_static: no usable current device");
  }
  if ((n_faces > 0 && !on_device(faces9, dev)) || !on_device(rays6, dev) || !on_device(hit_face, dev) ||
      (hit_point && !on_device(hit_point, dev)))
    return ffb_set_error(FFB_ERR_ARG,
                         "ffb_cast_bruteforce_static: every buffer must be device memory of the current device");
  ffb::TriRec* rec = nullptr;
  {
    // set-up, once per device, with that device current
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_records_ptr[dev]) {
      cudaError_t e = cudaGetSymbolAddress((void**)&g_records_ptr[dev], g_static_records);
      if (e != cudaSuccess) {
        g_records_ptr[dev] = nullptr;
        cudaGetLastError();
        return ffb_set_error(FFB_ERR_CUDA, cudaGetErrorString(e));
      }
    }
    rec = g_records_ptr[dev];
  }
  cudaStream_t s = (cudaStream_t)stream;
  if (n_faces > 0)
    k_static_records<<<(n_faces + 255) / 256, 256, 0, s>>>(faces9, n_faces, rec);
  k_static_brute<<<(unsigned)((n_rays + kThreads - 1) / kThreads), kThreads, 0, s>>>(rec, n_faces, rays6, n_rays,
                                                                                   hit_face, hit_point);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return ffb_set_error(FFB_ERR_CUDA, cudaGetErrorString(e));
  return FFB_OK;
}
