// ffb_server.cpp -- a serving loop for form-factor solves (include/ffb.h,
// ffb_server_*): requests of different sizes are admitted by a device-memory
// budget into a fixed number of slots, each slot a context with its own CUDA
// stream and worker thread, so that the device work of admitted requests
// overlaps (grid builds, zeroing, traces and result copies of different
// requests run concurrently).  Each request's scene, grid and count matrix
// stay resident on the device until the client releases the result.
//
// A request's counts depend only on its scene, ray budget, seed and flags
// (Philox keyed by seed, epoch 0, face, ray), never on what else runs: the
// result is bit-identical alone and in the mix.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "ffb.h"

int ffb_set_error(int code, const char* msg);

namespace {

using Clock = std::chrono::steady_clock;

double secs(Clock::time_point t0, Clock::time_point t1) { return std::chrono::duration<double>(t1 - t0).count(); }

struct Request {
  long long id = 0;
  std::vector<float> faces;
  int n_faces = 0;
  int rays_per_face = 0;
  uint64_t seed = 0;
  int flags = 0;
  float cells_per_face = 32.f;
  unsigned long long reserve = 0;  // bytes reserved in the budget
  int state = FFB_REQ_QUEUED;
  int error = 0;
  std::string message;
  uint32_t* counts = nullptr;      // device, n_faces^2, until released
  int readers = 0;                 // ffb_server_result copies in progress (release waits for them)
  int device = 0;
  Clock::time_point t_submit, t_admit, t_done;
  double gpu_ms = 0;               // events around the request's device work
};

}  // namespace

struct ffb_server {
  int device = 0;
  unsigned long long budget = 0;
  unsigned long long reserved = 0;
  int n_slots = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<Request>> queue;
  std::map<long long, std::shared_ptr<Request>> all;
  long long next_id = 1;
  bool stopping = false;
  std::vector<std::thread> workers;
  int running = 0;
  int peak_running = 0;
  // Held around each request's trace: the fused kernel fills the whole GPU,
  // so two traces at once only share it (and mix their grids in L2); the
  // other slots meanwhile upload scenes and build grids.
  std::mutex trace_mu;
};

namespace {

// Device bytes a request may hold: its count matrix plus a generous bound on
// the scene, records, grid and per-reference copies of a 32-cells-per-face
// grid (about 1.3 KB per face).
unsigned long long estimate_bytes(int n_faces)
{
  const unsigned long long n = (unsigned long long)n_faces;
  return 4ull * n * n + 1536ull * n + (8ull << 20);
}

int run_request(ffb_server* s, ffb_ctx* ctx, cudaStream_t stream, Request& r)
{
  int rc = ffb_scene_set(ctx, r.faces.data(), r.n_faces);
  ffb_grid_params gp = {0, 0, 0, r.cells_per_face, 1};
  if (rc >= 0)
    rc = ffb_grid_build(ctx, &gp);
  if (rc < 0)
    return rc;
  const size_t mat = (size_t)r.n_faces * r.n_faces;
  cudaError_t e = cudaMallocAsync((void**)&r.counts, sizeof(uint32_t) * mat, stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    r.counts = nullptr;
    return ffb_set_error(FFB_ERR_NO_MEMORY, "request matrix allocation failed");
  }
  std::vector<int32_t> front((size_t)r.n_faces, r.rays_per_face), rear((size_t)r.n_faces, 0);
  if ((e = cudaStreamSynchronize(stream)) != cudaSuccess)  // preparation done before taking the GPU
    return ffb_set_error(FFB_ERR_CUDA, cudaGetErrorString(e));
  std::lock_guard<std::mutex> trace(s->trace_mu);
  rc = ffb_form_factor_counts(ctx, front.data(), rear.data(), r.seed, 0, r.flags, nullptr, r.n_faces, r.counts);
  if (rc < 0)
    return rc;
  if ((e = cudaStreamSynchronize(stream)) != cudaSuccess)
    return ffb_set_error(FFB_ERR_CUDA, cudaGetErrorString(e));
  return FFB_OK;
}

void worker_main(ffb_server* s, int slot)
{
  cudaSetDevice(s->device);
  ffb_ctx* ctx = nullptr;
  int rc = ffb_ctx_create(s->device, &ctx);
  if (ctx)
    ffb_ctx_set_stats(ctx, 0);  // requests return counts only
  cudaStream_t stream = ctx ? (cudaStream_t)ffb_ctx_stream(ctx) : nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  (void)slot;
  for (;;) {
    std::shared_ptr<Request> r;
    {
      std::unique_lock<std::mutex> lock(s->mu);
      // admission in arrival order: the oldest queued request enters as soon
      // as its reservation fits the budget (no overtaking, so a large request
      // cannot be starved by a stream of small ones)
      s->cv_work.wait(lock, [&] {
        return s->stopping ||
               (!s->queue.empty() && (s->budget == 0 || s->reserved + s->queue.front()->reserve <= s->budget));
      });
      if (s->stopping)
        break;
      r = s->queue.front();
      s->queue.pop_front();
      s->reserved += r->reserve;
      r->state = FFB_REQ_RUNNING;
      r->t_admit = Clock::now();
      ++s->running;
      s->peak_running = std::max(s->peak_running, s->running);
    }
    int err = rc;
    if (err >= 0) {
      cudaEventRecord(e0, stream);
      err = run_request(s, ctx, stream, *r);
      cudaEventRecord(e1, stream);
      cudaEventSynchronize(e1);
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      r->gpu_ms = ms;
    }
    std::string msg = err < 0 ? ffb_last_error() : "";
    {
      std::lock_guard<std::mutex> lock(s->mu);
      r->t_done = Clock::now();
      --s->running;
      r->faces.clear();
      r->faces.shrink_to_fit();
      if (err < 0) {
        r->state = FFB_REQ_FAILED;
        r->error = err;
        r->message = msg;
        if (r->counts) {
          cudaFree(r->counts);
          r->counts = nullptr;
        }
        s->reserved -= r->reserve;
        r->reserve = 0;
      } else {
        r->state = FFB_REQ_DONE;
      }
    }
    s->cv_done.notify_all();
    s->cv_work.notify_all();
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ffb_ctx_destroy(ctx);
}

}  // namespace

extern "C" int ffb_server_create(int device, unsigned long long budget_bytes, int n_slots, ffb_server** out)
{
  if (!out || n_slots <= 0 || n_slots > 64)
    return ffb_set_error(FFB_ERR_ARG, "ffb_server_create: bad arguments (1..64 slots)");
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
    cudaGetLastError();
    return ffb_set_error(FFB_ERR_NO_DEVICE, "ffb_server_create: no such device");
  }
  ffb_server* s = new ffb_server;
  s->device = device;
  s->budget = budget_bytes;
  s->n_slots = n_slots;
  for (int i = 0; i < n_slots; ++i)
    s->workers.emplace_back(worker_main, s, i);
  *out = s;
  return FFB_OK;
}

extern "C" void ffb_server_destroy(ffb_server* s)
{
  if (!s)
    return;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    s->stopping = true;
  }
  s->cv_work.notify_all();
  for (auto& t : s->workers)
    t.join();
  cudaSetDevice(s->device);
  for (auto& kv : s->all)
    if (kv.second->counts)
      cudaFree(kv.second->counts);
  delete s;
}

extern "C" int ffb_server_submit(ffb_server* s, const float* faces9, int n_faces, int rays_per_face, uint64_t seed,
                                 int flags, float cells_per_face, long long* request_id)
{
  if (!s || !faces9 || n_faces <= 0 || rays_per_face < 0 || !request_id)
    return ffb_set_error(FFB_ERR_ARG, "ffb_server_submit: bad arguments");
  if (n_faces > 65535)
    return ffb_set_error(FFB_ERR_TOO_LARGE, "ffb_server_submit: more than 65535 faces");
  auto r = std::make_shared<Request>();
  r->faces.assign(faces9, faces9 + 9 * (size_t)n_faces);
  r->n_faces = n_faces;
  r->rays_per_face = rays_per_face;
  r->seed = seed;
  r->flags = flags;
  r->cells_per_face = cells_per_face > 0 ? cells_per_face : 32.f;
  r->reserve = estimate_bytes(n_faces);
  r->device = s->device;
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->budget && r->reserve > s->budget)
      return ffb_set_error(FFB_ERR_NO_MEMORY, "ffb_server_submit: request larger than the whole budget");
    r->id = s->next_id++;
    s->all[r->id] = r;
    s->queue.push_back(r);
    *request_id = r->id;
  }
  s->cv_work.notify_all();
  return FFB_OK;
}

extern "C" int ffb_server_wait(ffb_server* s, long long id, double timeout_s, ffb_request_info* info)
{
  if (!s)
    return ffb_set_error(FFB_ERR_ARG, "null server");
  std::unique_lock<std::mutex> lock(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end())
    return ffb_set_error(FFB_ERR_ARG, "unknown request");
  std::shared_ptr<Request> r = it->second;
  auto done = [&] { return r->state == FFB_REQ_DONE || r->state == FFB_REQ_FAILED; };
  if (timeout_s < 0)
    s->cv_done.wait(lock, done);
  else
    s->cv_done.wait_for(lock, std::chrono::duration<double>(timeout_s), done);
  if (info) {
    memset(info, 0, sizeof *info);
    info->state = r->state;
    info->error = r->error;
    info->n_faces = r->n_faces;
    info->queue_s = r->state >= FFB_REQ_RUNNING ? secs(r->t_submit, r->t_admit) : secs(r->t_submit, Clock::now());
    info->latency_s = done() ? secs(r->t_submit, r->t_done) : 0.0;
    info->gpu_ms = r->gpu_ms;
  }
  if (r->state == FFB_REQ_FAILED)
    return ffb_set_error(r->error, r->message.c_str());
  return done() ? FFB_OK : ffb_set_error(FFB_ERR_TIMEOUT, "request not finished before the timeout");
}

extern "C" int ffb_server_result(ffb_server* s, long long id, uint32_t* counts)
{
  std::shared_ptr<Request> r;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end() || it->second->state != FFB_REQ_DONE || !it->second->counts)
      return ffb_set_error(FFB_ERR_ARG, "no finished result for this request");
    r = it->second;
    ++r->readers;  // a concurrent release waits until this copy is done
  }
  cudaSetDevice(s->device);
  const size_t bytes = sizeof(uint32_t) * (size_t)r->n_faces * r->n_faces;
  cudaError_t e = cudaMemcpy(counts, r->counts, bytes, cudaMemcpyDefault);
  {
    std::lock_guard<std::mutex> lock(s->mu);
    --r->readers;
  }
  s->cv_done.notify_all();
  if (e != cudaSuccess)
    return ffb_set_error(FFB_ERR_CUDA, cudaGetErrorString(e));
  return FFB_OK;
}

extern "C" int ffb_server_release(ffb_server* s, long long id)
{
  std::shared_ptr<Request> r;
  {
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end())
      return ffb_set_error(FFB_ERR_ARG, "unknown request");
    r = it->second;
    if (r->state != FFB_REQ_DONE && r->state != FFB_REQ_FAILED)
      return ffb_set_error(FFB_ERR_ARG, "request still queued or running");
    // the matrix is freed below: wait for result copies still reading it
    s->cv_done.wait(lock, [&] { return r->readers == 0; });
    it = s->all.find(id);
    if (it == s->all.end())
      return ffb_set_error(FFB_ERR_ARG, "request released concurrently");
    s->all.erase(it);
    s->reserved -= r->reserve;
    r->reserve = 0;
  }
  if (r->counts) {
    cudaSetDevice(s->device);
    cudaFree(r->counts);
    r->counts = nullptr;
  }
  s->cv_work.notify_all();
  return FFB_OK;
}

extern "C" int ffb_server_stats(ffb_server* s, ffb_server_info* out)
{
  if (!s || !out)
    return ffb_set_error(FFB_ERR_ARG, "null argument");
  std::lock_guard<std::mutex> lock(s->mu);
  memset(out, 0, sizeof *out);
  out->queued = (int)s->queue.size();
  out->running = s->running;
  out->peak_running = s->peak_running;
  out->reserved_bytes = s->reserved;
  out->budget_bytes = s->budget;
  return FFB_OK;
}
