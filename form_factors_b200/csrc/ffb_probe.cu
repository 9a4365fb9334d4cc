// ffb_probe.cu -- measurement helper for bench.py (libffb200_probe.so): the
// FP32 issue rate of this device for separate multiply and add instructions
// (the trace kernels are compiled with --fmad=false, so their arithmetic is
// FMUL/FADD, never FFMA).  Not part of the form-factor C ABI.
#include <cuda_runtime.h>

namespace {

constexpr int kChains = 8;
constexpr int kIters = 4096;

__global__ void k_fp32_issue(float* out, float a, float b)
{
  float x[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k)
    x[k] = threadIdx.x * 1e-3f + k;
  for (int i = 0; i < kIters; ++i) {
#pragma unroll
    for (int k = 0; k < kChains; ++k)
      x[k] = x[k] * a + b;  // one FMUL and one FADD under --fmad=false
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < kChains; ++k)
    s += x[k];
  if (s == 12345.678f)
    out[blockIdx.x] = s;
}

}  // namespace

// Returns FP32 operations per second (multiplies and adds counted separately)
// measured with CUDA events over `reps` launches filling every SM.
extern "C" int ffb_probe_fp32_ops(int device, int reps, double* ops_per_s)
{
  if (cudaSetDevice(device) != cudaSuccess)
    return -1;
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, device);
  const int threads = 256;
  const int blocks = prop.multiProcessorCount * (prop.maxThreadsPerMultiProcessor / threads) * 4;
  float* out = nullptr;
  if (cudaMalloc(&out, sizeof(float) * blocks) != cudaSuccess)
    return -2;
  cudaStream_t s;
  cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  k_fp32_issue<<<blocks, threads, 0, s>>>(out, 0.999f, 1e-4f);  // warm-up
  cudaEventRecord(e0, s);
  for (int r = 0; r < reps; ++r)
    k_fp32_issue<<<blocks, threads, 0, s>>>(out, 0.999f, 1e-4f);
  cudaEventRecord(e1, s);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  const double ops = 2.0 * kChains * (double)kIters * threads * (double)blocks * reps;
  *ops_per_s = ops / (ms * 1e-3);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(s);
  cudaFree(out);
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}
