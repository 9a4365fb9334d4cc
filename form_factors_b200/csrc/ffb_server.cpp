// ffb_server.cpp -- a serving loop for form-factor solves (include/ffb.h,
// ffb_server_*) with continuous batching on the device.
//
// Requests of different sizes are admitted in arrival order while a slot is
// free and the device-memory budget allows.  Each slot is a context (its own
// CUDA stream and resident scene) with a worker thread that prepares its
// request: uploads the scene, builds the grid, allocates and zeroes the
// count matrix and builds the chunk table.  A prepared request joins the
// trace rotation of one scheduler thread, which launches the requests'
// traces in slices of at most `slice_rays` rays (ffb_server_set_slicing),
// round-robin over the prepared requests, with `window` slices in flight:
// the next slice is
// queued while the current one runs, and slices of different requests run
// on different streams, so a request admitted while others trace starts at
// the next slice boundary and its kernels overlap theirs on the device (a
// small request's launch shares the SMs; a large one's blocks take over SMs
// as the previous slice's blocks retire).  Round-robin over slices is
// processor sharing: a small request finishes within its first turn
// instead of waiting behind a large one.  Each request's scene, grid and
// count matrix stay resident until the client releases the result.
//
// A request's counts depend only on its scene, ray budget, seed and flags
// (Philox keyed by seed, epoch 0, face, ray) and are integer sums, so the
// result is bit-identical alone and in the mix, whatever the slicing.
//
// The consumer this stands in for is the per-scene form-factor solve of the
// reference's thermal model (thermal_equation/form_factors.cpp:88-98), one
// scene after another.
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
#include "ffb_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

double secs(Clock::time_point t0, Clock::time_point t1) { return std::chrono::duration<double>(t1 - t0).count(); }

// Default rays per trace slice: about 25 ms of trace on a B200, long
// against a launch and its tail, short against the large requests that
// small ones would otherwise wait behind.
constexpr long long kSliceRays = 64ll << 20;
constexpr long long kChunkRays = 256;  // rays per chunk of the fused kernel
constexpr int kWindow = 2;             // default slices in flight
constexpr int kMaxWindow = 8;

struct Request {
  long long id = 0;
  std::vector<float> faces;
  int n_faces = 0;
  int rays_per_face = 0;
  uint64_t seed = 0;
  int flags = 0;
  float cells_per_face = 32.f;     // 0: grid and launch shape autotuned
  int tuned_shape = 0;
  float tuned_cells_per_face = 0.f;
  unsigned long long reserve = 0;  // bytes reserved in the budget
  int state = FFB_REQ_QUEUED;
  int error = 0;
  std::string message;
  uint32_t* counts = nullptr;      // device, n_faces^2, until released
  int readers = 0;                 // ffb_server_result copies in progress (release waits for them)
  Clock::time_point t_submit, t_admit, t_done;
  unsigned long long start_ns = 0, end_ns = 0;  // trace span on the device (%globaltimer)
  int slices = 0;
};

// A slot: one context and its worker.  `phase` is guarded by the server
// mutex: the worker prepares (kPreparing), the scheduler traces
// (kTracing: chunks handed out up to `next`), then the worker finishes.
enum Phase { kIdle, kPreparing, kTracing, kTraced };

struct Slot {
  ffb_ctx* ctx = nullptr;       // on `prep`: the preparation
  cudaStream_t prep = nullptr;  // low priority
  cudaStream_t trace = nullptr; // high priority: the trace slices
  std::shared_ptr<Request> req;
  Phase phase = kIdle;
  long long n_chunks = 0, next = 0;
  int in_flight = 0;  // launched slices not yet retired
  int error = 0;      // a failed slice launch
  std::string message;
};

struct Inflight {
  int slot;
  cudaEvent_t done;
};

}  // namespace

struct ffb_server {
  int device = 0;
  unsigned long long budget = 0;
  unsigned long long reserved = 0;
  int n_slots = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done, cv_sched, cv_slot;
  std::deque<std::shared_ptr<Request>> queue;
  std::map<long long, std::shared_ptr<Request>> all;
  long long next_id = 1;
  bool stopping = false;
  std::vector<Slot> slots;
  std::vector<std::thread> workers;
  std::thread scheduler;
  int running = 0;
  int peak_running = 0;
  int peak_tracing = 0;  // most requests in the trace rotation at once
  long long slice_chunks = kSliceRays / kChunkRays;
  int window = kWindow;
  int policy = FFB_ADMIT_FIFO;  // admission order (ffb_server_set_admission)
  double max_wait_s = 0.0;      // FFB_ADMIT_SHORTEST: age past which the oldest request goes first
  // frees of released matrices, off every slot's stream: a synchronous
  // cudaFree would wait for the whole device and drain the slice pipeline
  cudaStream_t free_stream = nullptr;
};

namespace {

// Device bytes a request may hold: its count matrix plus a generous bound on
// the scene, records, grid and per-reference copies: about 1.3 KB per face
// for a grid of cells_per_face 32, and 10 KB per face for an autotuned one
// (its grid candidates go up to 256 cells per face).
unsigned long long estimate_bytes(int n_faces, bool tuned)
{
  const unsigned long long n = (unsigned long long)n_faces;
  return 4ull * n * n + (tuned ? 10240ull : 1536ull) * n + (8ull << 20);
}

// Position in the queue of the request to admit next, or -1 when none may
// enter yet.  FIFO: the oldest, once its reservation fits the budget (no
// overtaking, so a large request cannot be starved by a stream of small
// ones).  Shortest first: the request with the least work (faces x rays per
// face), unless the oldest has waited longer than max_wait_s, which then
// goes first: starvation is bounded by the age limit.
long admission_pick(const ffb_server* s)
{
  if (s->queue.empty())
    return -1;
  size_t idx = 0;
  if (s->policy == FFB_ADMIT_SHORTEST && secs(s->queue.front()->t_submit, Clock::now()) <= s->max_wait_s) {
    unsigned long long best = ~0ull;
    for (size_t i = 0; i < s->queue.size(); ++i) {
      const Request& q = *s->queue[i];
      const unsigned long long work = (unsigned long long)q.n_faces * (unsigned long long)q.rays_per_face;
      if (work < best) {
        best = work;
        idx = i;
      }
    }
  }
  const Request& r = *s->queue[idx];
  if (s->budget && s->reserved + r.reserve > s->budget)
    return -1;
  return (long)idx;
}

// The worker's part of a request before its trace: scene, grid, matrix,
// chunk table.
int prepare(Slot& sl, Request& r, long long* n_chunks)
{
  ffb_ctx* ctx = sl.ctx;
  int rc = ffb_scene_set(ctx, r.faces.data(), r.n_faces);
  if (rc < 0)
    return rc;
  cudaStream_t stream = (cudaStream_t)ffb_ctx_stream(ctx);
  const size_t mat = (size_t)r.n_faces * r.n_faces;
  cudaError_t e = cudaMallocAsync((void**)&r.counts, sizeof(uint32_t) * mat, stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    r.counts = nullptr;
    return ffb_set_error(FFB_ERR_NO_MEMORY, "request matrix allocation failed");
  }
  std::vector<int32_t> front((size_t)r.n_faces, r.rays_per_face), rear((size_t)r.n_faces, 0);
  if (r.cells_per_face > 0) {
    ffb_grid_params gp = {0, 0, 0, r.cells_per_face, 1};
    rc = ffb_ctx_set_trace_shape(ctx, 0);
    if (rc >= 0)
      rc = ffb_grid_build(ctx, &gp);
  } else {
    // grid and launch shape from the tuning cache (a tuning run on a miss,
    // with the request's own matrix as the sample's scratch)
    ffb_tune_result tr{};
    rc = ffb_autotune(ctx, front.data(), rear.data(), r.seed, nullptr, 0, 0, 0, r.counts, &tr);
    r.tuned_shape = tr.shape;
    r.tuned_cells_per_face = tr.grid.cells_per_face;
  }
  if (rc < 0)
    return rc;
  rc = ffb_trace_prepare(ctx, front.data(), rear.data(), r.seed, 0, r.flags, r.counts, n_chunks);
  if (rc < 0)
    return rc;
  if ((e = cudaStreamSynchronize(stream)) != cudaSuccess)
    return ffb_set_error(FFB_ERR_CUDA, cudaGetErrorString(e));
  return FFB_OK;
}

void finish(ffb_server* s, Slot& sl, const std::shared_ptr<Request>& r, int err, const std::string& msg)
{
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
        // after whatever the failed preparation left queued on the slot's stream
        cudaFreeAsync(r->counts, (cudaStream_t)ffb_ctx_stream(sl.ctx));
        r->counts = nullptr;
      }
      s->reserved -= r->reserve;
      r->reserve = 0;
    } else {
      r->state = FFB_REQ_DONE;
    }
    sl.req.reset();
    sl.phase = kIdle;
  }
  s->cv_done.notify_all();
  s->cv_work.notify_all();
}

void worker_main(ffb_server* s, int slot)
{
  cudaSetDevice(s->device);
  Slot& sl = s->slots[(size_t)slot];
  for (;;) {
    std::shared_ptr<Request> r;
    {
      std::unique_lock<std::mutex> lock(s->mu);
      long pick = -1;
      s->cv_work.wait(lock, [&] { return s->stopping || (pick = admission_pick(s)) >= 0; });
      if (s->stopping)
        break;
      r = s->queue[(size_t)pick];
      s->queue.erase(s->queue.begin() + pick);
      s->reserved += r->reserve;
      r->state = FFB_REQ_RUNNING;
      r->t_admit = Clock::now();
      ++s->running;
      s->peak_running = std::max(s->peak_running, s->running);
      sl.req = r;
      sl.phase = kPreparing;
    }
    long long n_chunks = 0;
    int err = prepare(sl, *r, &n_chunks);
    std::string msg = err < 0 ? ffb_last_error() : "";
    if (err >= 0 && n_chunks > 0) {
      // hand the trace to the scheduler and wait for its last slice
      std::unique_lock<std::mutex> lock(s->mu);
      sl.n_chunks = n_chunks;
      sl.next = 0;
      sl.in_flight = 0;
      sl.error = 0;
      sl.phase = kTracing;
      int tracing = 0;
      for (const Slot& o : s->slots)
        tracing += o.phase == kTracing;
      s->peak_tracing = std::max(s->peak_tracing, tracing);
      s->cv_sched.notify_all();
      s->cv_slot.wait(lock, [&] { return sl.phase == kTraced; });
      err = sl.error;
      msg = sl.message;
    }
    if (err >= 0) {
      unsigned long long t0 = 0, t1 = 0;
      err = ffb_trace_span(sl.ctx, &t0, &t1);
      r->start_ns = t0;
      r->end_ns = t1;
      if (err < 0)
        msg = ffb_last_error();
    }
    finish(s, sl, r, err, msg);
  }
}

// Launches slices round-robin over the slots in kTracing, keeping kWindow
// in flight, and retires them in launch order.  A slot leaves the rotation
// (kTraced) when its last slice has retired.
void scheduler_main(ffb_server* s)
{
  cudaSetDevice(s->device);
  std::vector<cudaEvent_t> pool;
  for (int k = 0; k < kMaxWindow; ++k) {
    cudaEvent_t e = nullptr;
    cudaEventCreateWithFlags(&e, cudaEventDisableTiming | cudaEventBlockingSync);
    pool.push_back(e);
  }
  std::deque<Inflight> inflight;
  size_t rr = 0;
  for (;;) {
    {
      std::unique_lock<std::mutex> lock(s->mu);
      // fill the window: the next slot in round-robin order with chunks left
      while ((int)inflight.size() < s->window) {
        int pick = -1;
        for (size_t k = 0; k < s->slots.size(); ++k) {
          const size_t i = (rr + k) % s->slots.size();
          const Slot& sl = s->slots[i];
          if (sl.phase == kTracing && sl.error == 0 && sl.next < sl.n_chunks) {
            pick = (int)i;
            break;
          }
        }
        if (pick < 0)
          break;
        rr = (size_t)pick + 1;
        Slot& sl = s->slots[(size_t)pick];
        const long long first = sl.next, count = std::min(s->slice_chunks, sl.n_chunks - sl.next);
        sl.next += count;
        int rc = ffb_trace_slice(sl.ctx, first, count, sl.trace);
        cudaEvent_t ev = pool.back();
        if (rc >= 0 && cudaEventRecord(ev, sl.trace) != cudaSuccess) {
          cudaGetLastError();
          rc = ffb_set_error(FFB_ERR_CUDA, "event record after a trace slice failed");
        }
        if (rc < 0) {
          sl.error = rc;
          sl.message = ffb_last_error();
          sl.next = sl.n_chunks;  // no more slices for this request
          if (sl.in_flight == 0) {
            sl.phase = kTraced;
            s->cv_slot.notify_all();
          }
          continue;
        }
        pool.pop_back();
        ++sl.in_flight;
        ++sl.req->slices;
        inflight.push_back(Inflight{pick, ev});
      }
      if (inflight.empty()) {
        if (s->stopping)
          break;
        s->cv_sched.wait(lock);
        continue;
      }
    }
    // retire the oldest slice (no lock held while the device runs)
    Inflight f = inflight.front();
    inflight.pop_front();
    cudaError_t e = cudaEventSynchronize(f.done);
    pool.push_back(f.done);
    std::lock_guard<std::mutex> lock(s->mu);
    Slot& sl = s->slots[(size_t)f.slot];
    --sl.in_flight;
    if (e != cudaSuccess && sl.error == 0) {
      sl.error = ffb_set_error(FFB_ERR_CUDA, cudaGetErrorString(e));
      sl.message = cudaGetErrorString(e);
      sl.next = sl.n_chunks;
    }
    if (sl.next >= sl.n_chunks && sl.in_flight == 0) {
      sl.phase = kTraced;
      s->cv_slot.notify_all();
    }
  }
  for (cudaEvent_t e : pool)
    cudaEventDestroy(e);
}

}  // namespace

extern "C" int ffb_server_create(int device, unsigned long long budget_bytes, int n_slots, ffb_server** out)
{
  if (!out || n_slots <= 0 || n_slots > 64)
    return ffb_set_error(FFB_ERR_ARG, "ffb_server_create: bad arguments (1..64 slots)");
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
    cudaGetLastError();
    return ffb_set_error(FFB_ERR_NO_DEVICE, "ffb_server_create: no such device");
  }
  ffb_server* s = new ffb_server;
  s->device = device;
  s->budget = budget_bytes;
  s->n_slots = n_slots;
  s->slots.resize((size_t)n_slots);
  cudaSetDevice(device);
  if (cudaStreamCreateWithFlags(&s->free_stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    delete s;
    return ffb_set_error(FFB_ERR_CUDA, "ffb_server_create: stream creation failed");
  }

  // Traces at the device's highest stream priority, preparation at its
  // lowest: when a slice's blocks retire, the block scheduler gives the SMs
  // to the next slice before another request's grid build or zeroing.
  int prio_low = 0, prio_high = 0;
  cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
  for (Slot& sl : s->slots) {
    int rc = ffb_ctx_create(device, &sl.ctx);
    cudaStream_t prep = nullptr;
    if (rc >= 0 && (cudaStreamCreateWithPriority(&prep, cudaStreamNonBlocking, prio_low) != cudaSuccess ||
                    cudaStreamCreateWithPriority(&sl.trace, cudaStreamNonBlocking, prio_high) != cudaSuccess)) {
      cudaGetLastError();
      rc = ffb_set_error(FFB_ERR_CUDA, "ffb_server_create: stream creation failed");
    }
    if (rc >= 0)
      rc = ffb_ctx_set_stream(sl.ctx, prep);
    sl.prep = prep;
    if (rc < 0) {
      for (Slot& o : s->slots) {
        ffb_ctx_destroy(o.ctx);
        if (o.prep)
          cudaStreamDestroy(o.prep);
        if (o.trace)
          cudaStreamDestroy(o.trace);
      }
      cudaStreamDestroy(s->free_stream);
      delete s;
      return rc;
    }
    ffb_ctx_set_stats(sl.ctx, 0);  // requests return counts only
  }
  if (budget_bytes > 0) {
    // Map the budget into the device's stream-ordered pool once (the contexts set it to keep
    // freed memory): the requests' matrices are then
    // carved out of memory that is already mapped, instead of growing the
    // pool -- new mappings while other requests' kernels run -- on the way.
    void* p = nullptr;
    if (cudaMallocAsync(&p, (size_t)budget_bytes, s->free_stream) == cudaSuccess) {
      cudaFreeAsync(p, s->free_stream);
      cudaStreamSynchronize(s->free_stream);
    }
    cudaGetLastError();  // a budget beyond the free memory is not an error here
  }
  s->scheduler = std::thread(scheduler_main, s);
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
  // workers stop between requests: a request being traced finishes first
  s->cv_work.notify_all();
  for (auto& t : s->workers)
    t.join();
  {
    std::lock_guard<std::mutex> lock(s->mu);
    s->cv_sched.notify_all();
  }
  s->scheduler.join();
  cudaSetDevice(s->device);
  for (auto& kv : s->all)
    if (kv.second->counts)
      cudaFreeAsync(kv.second->counts, s->free_stream);
  cudaStreamSynchronize(s->free_stream);
  cudaStreamDestroy(s->free_stream);
  for (Slot& sl : s->slots) {
    ffb_ctx_destroy(sl.ctx);
    cudaStreamDestroy(sl.prep);
    cudaStreamDestroy(sl.trace);
  }
  delete s;
}

extern "C" int ffb_server_submit(ffb_server* s, const float* faces9, int n_faces, int rays_per_face, uint64_t seed,
                                 int flags, float cells_per_face, long long* request_id)
{
  if (!s || !faces9 || n_faces <= 0 || rays_per_face < 0 || !request_id || !(cells_per_face >= 0.f))
    return ffb_set_error(FFB_ERR_ARG, "ffb_server_submit: bad arguments");
  if (n_faces > 65535)
    return ffb_set_error(FFB_ERR_TOO_LARGE, "ffb_server_submit: more than 65535 faces");
  auto r = std::make_shared<Request>();
  r->faces.assign(faces9, faces9 + 9 * (size_t)n_faces);
  r->n_faces = n_faces;
  r->rays_per_face = rays_per_face;
  r->seed = seed;
  r->flags = flags;
  r->cells_per_face = cells_per_face > 0 ? cells_per_face : 0.f;
  r->reserve = estimate_bytes(n_faces, r->cells_per_face == 0.f);
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
    info->gpu_ms = r->end_ns > r->start_ns ? 1e-6 * (double)(r->end_ns - r->start_ns) : 0.0;
    info->trace_start_ns = r->start_ns;
    info->trace_end_ns = r->end_ns;
    info->slices = r->slices;
    info->shape = r->tuned_shape;
    info->cells_per_face = r->cells_per_face > 0 ? r->cells_per_face : r->tuned_cells_per_face;
  }
  if (r->state == FFB_REQ_FAILED)
    return ffb_set_error(r->error, r->message.c_str());
  return done() ? FFB_OK : ffb_set_error(FFB_ERR_TIMEOUT, "request not finished before the timeout");
}

extern "C" int ffb_server_wait_any(ffb_server* s, const long long* ids, int n, double timeout_s, long long* done_id,
                                   ffb_request_info* info)
{
  if (!s || !ids || n <= 0 || !done_id)
    return ffb_set_error(FFB_ERR_ARG, "ffb_server_wait_any: bad arguments");
  long long found = -1;
  {
    std::unique_lock<std::mutex> lock(s->mu);
    for (int k = 0; k < n; ++k)
      if (s->all.find(ids[k]) == s->all.end())
        return ffb_set_error(FFB_ERR_ARG, "ffb_server_wait_any: unknown request");
    auto any_done = [&] {
      for (int k = 0; k < n; ++k) {
        auto it = s->all.find(ids[k]);
        // a request released meanwhile ends the wait (ffb_server_wait then reports it unknown)
        if (it == s->all.end() || it->second->state == FFB_REQ_DONE || it->second->state == FFB_REQ_FAILED) {
          found = ids[k];
          return true;
        }
      }
      return false;
    };
    if (timeout_s < 0)
      s->cv_done.wait(lock, any_done);
    else
      s->cv_done.wait_for(lock, std::chrono::duration<double>(timeout_s), any_done);
  }
  if (found < 0)
    return ffb_set_error(FFB_ERR_TIMEOUT, "no request finished before the timeout");
  *done_id = found;
  return ffb_server_wait(s, found, 0.0, info);
}

extern "C" int ffb_server_result(ffb_server* s, long long id, uint32_t* counts)
{
  if (!s || !counts)
    return ffb_set_error(FFB_ERR_ARG, "null argument");
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
  if (!s)
    return ffb_set_error(FFB_ERR_ARG, "null server");
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
    // the request's trace has retired and no result copy is in progress
    cudaSetDevice(s->device);
    cudaFreeAsync(r->counts, s->free_stream);
    r->counts = nullptr;
  }
  s->cv_work.notify_all();
  return FFB_OK;
}

extern "C" int ffb_server_set_slicing(ffb_server* s, long long slice_rays, int window)
{
  if (!s || slice_rays < kChunkRays || window < 1 || window > kMaxWindow)
    return ffb_set_error(FFB_ERR_ARG, "ffb_server_set_slicing: slice_rays >= 256 and 1 <= window <= 8");
  std::lock_guard<std::mutex> lock(s->mu);
  s->slice_chunks = slice_rays / kChunkRays;
  s->window = window;
  return FFB_OK;
}

extern "C" int ffb_server_set_admission(ffb_server* s, int policy, double max_wait_s)
{
  if (!s || (policy != FFB_ADMIT_FIFO && policy != FFB_ADMIT_SHORTEST) || !(max_wait_s >= 0.0))
    return ffb_set_error(FFB_ERR_ARG, "ffb_server_set_admission: FFB_ADMIT_FIFO or FFB_ADMIT_SHORTEST, max_wait_s >= 0");
  {
    std::lock_guard<std::mutex> lock(s->mu);
    s->policy = policy;
    s->max_wait_s = max_wait_s;
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
  out->peak_tracing = s->peak_tracing;
  return FFB_OK;
}
