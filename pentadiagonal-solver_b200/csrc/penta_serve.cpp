// penta_serve.cpp -- the request loop's native core: a serving handle.
//
// Requests (one FP64 grid and a solve direction each, with the forward-error
// tolerance the caller needs) are submitted from the host as they arrive.
// pentadsolver_server_progress then
//
//   * completes the batches whose work has finished on the GPU (an event per
//     batch), reading each batch's own status word, freeing its memory and
//     reporting its requests with those status bits;
//   * launches, while fewer than `max_in_flight` batches are on the GPU, the
//     group of queued requests that shares the oldest request's key -- its
//     solve direction and precision class -- as one plan (one persistent
//     launch for all its grids) on the next of several streams, so batches
//     overlap on the device and requests that arrive while others run join
//     the next batch as soon as memory frees.
//
// Memory: every batch's plan memory (job table, scratch; for refined batches
// the FP32 copies, residual and saved right-hand side) is carved out of one
// device arena the caller hands over at creation -- the HBM budget.  A batch
// that does not fit is shortened; a request that alone exceeds the whole
// arena is completed at once with SERVER_REJECTED_BIT.  Nothing is allocated
// on the device after creation.
//
// Precision classes: requests with tol >= 1e-10 may use FP32 sweeps with FP64
// refinement under the mixed policy -- along a solve direction where the
// server measured the refined form faster than plain FP64
// (pentadsolver_server_calibrate), or everywhere when it was not measured.
// Tighter requests always run in plain FP64.  The sequential policy solves
// one request at a time, in arrival order, with the plain call (the baseline).
//
// Coefficients and right-hand sides stay where the caller keeps them (device
// memory); x is solved in place.  The server's streams are non-blocking: work
// that writes a request's arrays must have completed before the
// pentadsolver_server_progress call that launches it.  Each batch runs on a
// stream of its own (at most one batch per stream in flight).  The handle is
// not thread-safe: submit, progress and poll from one thread, or serialise
// them.
#include <cuda_runtime_api.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <deque>
#include <map>
#include <vector>

#include "pentad_common.hpp"
#include "pentadsolver_ext.h"

namespace {

constexpr size_t kAlign = 256;
size_t round_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

// First-fit suballocator over [0, size) with coalescing of freed blocks.
class Arena {
 public:
  explicit Arena(size_t size) : size_(size) { free_[0] = size; }
  // offset of a block of `bytes` (rounded to 256), or SIZE_MAX
  size_t alloc(size_t bytes) {
    bytes = round_up(std::max<size_t>(bytes, 1));
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < bytes) continue;
      const size_t off = it->first, len = it->second;
      free_.erase(it);
      if (len > bytes) free_[off + bytes] = len - bytes;
      used_ += bytes;
      peak_ = std::max(peak_, used_);
      return off;
    }
    return SIZE_MAX;
  }
  void release(size_t off, size_t bytes) {
    bytes = round_up(std::max<size_t>(bytes, 1));
    used_ -= bytes;
    auto it = free_.emplace(off, bytes).first;
    auto next = std::next(it);
    if (next != free_.end() && it->first + it->second == next->first) {
      it->second += next->second;
      free_.erase(next);
    }
    if (it != free_.begin()) {
      auto prev = std::prev(it);
      if (prev->first + prev->second == it->first) {
        prev->second += it->second;
        free_.erase(it);
      }
    }
  }
  size_t used() const { return used_; }
  size_t peak() const { return peak_; }
  size_t size() const { return size_; }

 private:
  size_t size_, used_ = 0, peak_ = 0;
  std::map<size_t, size_t> free_;  // offset -> length
};

struct Req {
  unsigned long long id;
  pentadsolver_grid_t grid;
  int solvedim;
  bool loose;  // tol >= 1e-10: may be refined
};

struct Batch {
  std::vector<Req> reqs;
  pentadsolver_plan_t plan = nullptr;
  size_t off = 0, bytes = 0;
  size_t stream_index = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
};

}  // namespace

struct pentadsolver_server_s {
  pentadsolver_handle_t handle = nullptr;
  unsigned char *base = nullptr;
  Arena arena{0};
  std::vector<cudaStream_t> streams;
  std::vector<char> stream_busy;  // a batch in flight on it
  size_t next_stream = 0;
  int max_batch = 64, max_in_flight = 3, refine_steps = 1, policy = 0;
  bool refine_pays[3] = {true, true, true};
  std::deque<Req> queue;
  std::vector<Batch> in_flight;
  std::vector<std::pair<unsigned long long, int>> completed;
  unsigned long long next_id = 0, batches = 0;

  // (solve direction, refined) of a request under the policy
  std::pair<int, bool> key_of(const Req &r) const {
    const bool refined = policy == PENTADSOLVER_SERVE_MIXED && r.loose && refine_pays[r.solvedim];
    return {r.solvedim, refined};
  }
};

namespace {

// The sequential baseline solves each request alone with the plain call (the
// reference-sized buffer from the arena), not as a one-grid plan.
bool direct(pentadsolver_server_t s) { return s->policy == PENTADSOLVER_SERVE_SEQUENTIAL; }

pentadStatus_t plan_bytes(pentadsolver_server_t s, const std::vector<Req> &reqs, bool refined,
                          size_t *bytes) {
  if (direct(s))
    return pentadsolver_buffer_size_ex(s->handle, 8, reqs[0].grid.dims, reqs[0].grid.ndim,
                                       reqs[0].solvedim, bytes);
  std::vector<pentadsolver_grid_t> g;
  for (const Req &r : reqs) g.push_back(r.grid);
  return refined ? pentadsolver_refine_plan_buffer_size(s->handle, (int)g.size(), g.data(),
                                                        reqs[0].solvedim, bytes)
                 : pentadsolver_plan_buffer_size(s->handle, 8, (int)g.size(), g.data(),
                                                 reqs[0].solvedim, bytes);
}

pentadStatus_t make_plan(pentadsolver_server_t s, const std::vector<Req> &reqs, bool refined,
                         void *buf, size_t bytes, pentadsolver_plan_t *plan) {
  std::vector<pentadsolver_grid_t> g;
  for (const Req &r : reqs) g.push_back(r.grid);
  return refined ? pentadsolver_refine_plan_create(s->handle, (int)g.size(), g.data(),
                                                   reqs[0].solvedim, s->refine_steps, buf,
                                                   bytes, 0, plan)
                 : pentadsolver_plan_create(s->handle, 8, (int)g.size(), g.data(),
                                            reqs[0].solvedim, buf, bytes, 0, plan);
}

// Finish the batches whose event has completed.
pentadStatus_t complete_ready(pentadsolver_server_t s, bool wait) {
  for (size_t i = 0; i < s->in_flight.size();) {
    Batch &b = s->in_flight[i];
    const cudaError_t q = wait ? cudaEventSynchronize(b.done) : cudaEventQuery(b.done);
    if (q == cudaErrorNotReady) {
      ++i;
      continue;
    }
    if (q != cudaSuccess) {
      cudaGetLastError();
      return PENTAD_STATUS_EXECUTION_FAILED;
    }
    int bits = 0;
    pentadStatus_t st = b.plan ? pentadsolver_plan_status_check(b.plan, b.stream, &bits)
                               : pentadsolver_status_check(s->handle, b.stream, &bits);
    if (st != PENTAD_STATUS_SUCCESS && st != PENTAD_STATUS_ZERO_PIVOT) return st;
    if (b.plan) pentadsolver_plan_destroy(b.plan);
    cudaEventDestroy(b.done);
    s->arena.release(b.off, b.bytes);
    s->stream_busy[b.stream_index] = 0;
    for (const Req &r : b.reqs) s->completed.emplace_back(r.id, bits);
    s->in_flight.erase(s->in_flight.begin() + (long)i);
  }
  return PENTAD_STATUS_SUCCESS;
}

// Launch batches while there is room on the device and in the arena.
pentadStatus_t launch_ready(pentadsolver_server_t s) {
  while (!s->queue.empty() && (int)s->in_flight.size() < s->max_in_flight) {
    // a stream with nothing in flight: a batch never queues behind another,
    // and its completion (event, status read) waits for itself only
    size_t si = s->streams.size();
    for (size_t k = 0; k < s->streams.size(); ++k) {
      const size_t c = (s->next_stream + k) % s->streams.size();
      if (!s->stream_busy[c]) {
        si = c;
        break;
      }
    }
    if (si == s->streams.size()) break;
    const auto key = s->key_of(s->queue.front());
    const int cap = s->policy == PENTADSOLVER_SERVE_SEQUENTIAL ? 1 : s->max_batch;
    std::vector<size_t> idx;
    for (size_t i = 0; i < s->queue.size() && (int)idx.size() < cap; ++i)
      if (s->key_of(s->queue[i]) == key) idx.push_back(i);
    std::vector<Req> reqs;
    for (size_t i : idx) reqs.push_back(s->queue[i]);
    size_t off = SIZE_MAX, bytes = 0;
    while (!reqs.empty()) {  // shorten the batch until its memory fits
      pentadStatus_t st = plan_bytes(s, reqs, key.second, &bytes);
      if (st != PENTAD_STATUS_SUCCESS) return st;
      off = s->arena.alloc(bytes);
      if (off != SIZE_MAX) break;
      reqs.pop_back();
      idx.pop_back();
    }
    if (reqs.empty()) {
      // not even the oldest request fits now: wait for memory, unless nothing
      // is in flight -- then it can never fit
      if (!s->in_flight.empty()) break;
      s->completed.emplace_back(s->queue.front().id, PENTADSOLVER_SERVER_REJECTED_BIT);
      s->queue.pop_front();
      continue;
    }
    Batch b;
    b.reqs = reqs;
    b.off = off;
    b.bytes = bytes;
    b.stream_index = si;
    b.stream = s->streams[si];
    s->next_stream = (si + 1) % s->streams.size();
    pentadStatus_t st;
    if (direct(s)) {  // one request, the plain call
      const pentadsolver_grid_t &g = reqs[0].grid;
      st = pentadsolver_D_gpsv_batch_ex(
          s->handle, static_cast<const double *>(g.ds), static_cast<const double *>(g.dl),
          static_cast<const double *>(g.d), static_cast<const double *>(g.du),
          static_cast<const double *>(g.dw), static_cast<double *>(g.x), g.dims, g.ndim,
          reqs[0].solvedim, s->base + off, bytes, b.stream);
    } else {
      st = make_plan(s, reqs, key.second, s->base + off, bytes, &b.plan);
      if (st == PENTAD_STATUS_SUCCESS) st = pentadsolver_plan_execute(b.plan, b.stream);
    }
    if (st == PENTAD_STATUS_SUCCESS &&
        (cudaEventCreateWithFlags(&b.done, cudaEventDisableTiming) != cudaSuccess ||
         cudaEventRecord(b.done, b.stream) != cudaSuccess)) {
      cudaGetLastError();
      st = PENTAD_STATUS_EXECUTION_FAILED;
    }
    if (st != PENTAD_STATUS_SUCCESS) {
      if (b.plan) pentadsolver_plan_destroy(b.plan);
      if (b.done) cudaEventDestroy(b.done);
      s->arena.release(off, bytes);
      return st;
    }
    for (size_t k = idx.size(); k-- > 0;) s->queue.erase(s->queue.begin() + (long)idx[k]);
    s->stream_busy[si] = 1;
    s->in_flight.push_back(b);
    ++s->batches;
  }
  return PENTAD_STATUS_SUCCESS;
}

}  // namespace

extern "C" PENTAD_API pentadStatus_t pentadsolver_server_create(
    pentadsolver_handle_t handle, void *arena, size_t arena_bytes, int policy, int n_streams,
    int max_batch, int max_in_flight, int refine_steps, pentadsolver_server_t *server) {
  if (server == nullptr) return PENTAD_STATUS_INVALID_VALUE;
  *server = nullptr;
  if (arena == nullptr || arena_bytes < kAlign ||
      reinterpret_cast<uintptr_t>(arena) % kAlign != 0 || policy < PENTADSOLVER_SERVE_FP64 ||
      policy > PENTADSOLVER_SERVE_SEQUENTIAL || n_streams < 1 || n_streams > 64 ||
      max_batch < 1 || max_in_flight < 1 || refine_steps < 0 || refine_steps > 8)
    return PENTAD_STATUS_INVALID_VALUE;
  auto *s = new pentadsolver_server_s();
  s->handle = handle;
  s->base = static_cast<unsigned char *>(arena);
  s->arena = Arena(arena_bytes / kAlign * kAlign);
  s->policy = policy;
  s->max_batch = max_batch;
  s->max_in_flight = policy == PENTADSOLVER_SERVE_SEQUENTIAL ? 1 : max_in_flight;
  s->refine_steps = refine_steps;
  for (int i = 0; i < n_streams; ++i) {
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      for (cudaStream_t t : s->streams) cudaStreamDestroy(t);
      delete s;
      return PENTAD_STATUS_NOT_INITIALIZED;
    }
    s->streams.push_back(st);
  }
  s->stream_busy.assign(s->streams.size(), 0);
  s->max_in_flight = std::min<int>(s->max_in_flight, (int)s->streams.size());
  *server = s;
  return PENTAD_STATUS_SUCCESS;
}

extern "C" PENTAD_API pentadStatus_t pentadsolver_server_submit(pentadsolver_server_t s,
                                                                const pentadsolver_grid_t *grid,
                                                                int solvedim, double tol,
                                                                unsigned long long *id) {
  if (s == nullptr || grid == nullptr || !(tol > 0)) return PENTAD_STATUS_INVALID_VALUE;
  size_t bytes = 0;  // the shape rules of every solve
  pentadStatus_t st = pentadsolver_plan_buffer_size(s->handle, 8, 1, grid, solvedim, &bytes);
  if (st != PENTAD_STATUS_SUCCESS) return st;
  Req r;
  r.id = s->next_id++;
  r.grid = *grid;
  r.solvedim = solvedim;
  r.loose = tol >= 1e-10;
  s->queue.push_back(r);
  if (id) *id = r.id;
  return PENTAD_STATUS_SUCCESS;
}

extern "C" PENTAD_API pentadStatus_t pentadsolver_server_progress(pentadsolver_server_t s,
                                                                  int wait) {
  if (s == nullptr) return PENTAD_STATUS_INVALID_VALUE;
  pentadStatus_t st = complete_ready(s, false);
  if (st == PENTAD_STATUS_SUCCESS) st = launch_ready(s);
  if (st == PENTAD_STATUS_SUCCESS && wait) {
    // run until every submitted request has completed
    while (st == PENTAD_STATUS_SUCCESS && (!s->queue.empty() || !s->in_flight.empty())) {
      st = complete_ready(s, true);
      if (st == PENTAD_STATUS_SUCCESS) st = launch_ready(s);
    }
  }
  return st;
}

extern "C" PENTAD_API pentadStatus_t pentadsolver_server_poll(pentadsolver_server_t s,
                                                              unsigned long long *ids,
                                                              int *bits, int capacity, int *n) {
  if (s == nullptr || n == nullptr || capacity < 0 || (capacity > 0 && ids == nullptr))
    return PENTAD_STATUS_INVALID_VALUE;
  const int k = std::min<int>(capacity, (int)s->completed.size());
  for (int i = 0; i < k; ++i) {
    ids[i] = s->completed[(size_t)i].first;
    if (bits) bits[i] = s->completed[(size_t)i].second;
  }
  s->completed.erase(s->completed.begin(), s->completed.begin() + k);
  *n = k;
  return PENTAD_STATUS_SUCCESS;
}

extern "C" PENTAD_API pentadStatus_t pentadsolver_server_stats(pentadsolver_server_t s,
                                                               size_t *out, int count) {
  if (s == nullptr || out == nullptr || count < 1) return PENTAD_STATUS_INVALID_VALUE;
  const size_t v[6] = {s->queue.size(), s->in_flight.size(), s->arena.used(), s->arena.peak(),
                       s->arena.size(), (size_t)s->batches};
  for (int i = 0; i < count && i < 6; ++i) out[i] = v[i];
  return PENTAD_STATUS_SUCCESS;
}

extern "C" PENTAD_API pentadStatus_t pentadsolver_server_calibrate(
    pentadsolver_server_t s, const pentadsolver_grid_t *sample, int reps, double *ms) {
  if (s == nullptr || sample == nullptr || reps < 1 || reps > 100 || !s->in_flight.empty())
    return PENTAD_STATUS_INVALID_VALUE;
  cudaStream_t stream = s->streams[0];
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    cudaGetLastError();
    if (e0) cudaEventDestroy(e0);
    return PENTAD_STATUS_EXECUTION_FAILED;
  }
  pentadStatus_t st = PENTAD_STATUS_SUCCESS;
  for (int d = 0; d < 3 && st == PENTAD_STATUS_SUCCESS; ++d) {
    float t[2] = {0.f, 0.f};
    for (int refined = 0; refined < 2 && st == PENTAD_STATUS_SUCCESS; ++refined) {
      Req r;
      r.id = 0;
      r.grid = *sample;
      r.solvedim = d;
      r.loose = true;
      size_t bytes = 0;
      if ((st = plan_bytes(s, {r}, refined != 0, &bytes)) != PENTAD_STATUS_SUCCESS) break;
      const size_t off = s->arena.alloc(bytes);
      if (off == SIZE_MAX) {
        st = PENTAD_STATUS_ALLOC_FAILED;
        break;
      }
      pentadsolver_plan_t plan = nullptr;
      st = make_plan(s, {r}, refined != 0, s->base + off, bytes, &plan);
      if (st == PENTAD_STATUS_SUCCESS) st = pentadsolver_plan_execute(plan, stream);  // warm-up
      if (st == PENTAD_STATUS_SUCCESS) {
        bool ok = cudaEventRecord(e0, stream) == cudaSuccess;
        for (int k = 0; ok && k < reps; ++k)
          ok = pentadsolver_plan_execute(plan, stream) == PENTAD_STATUS_SUCCESS;
        ok = ok && cudaEventRecord(e1, stream) == cudaSuccess &&
             cudaEventSynchronize(e1) == cudaSuccess &&
             cudaEventElapsedTime(&t[refined], e0, e1) == cudaSuccess;
        if (!ok) {
          cudaGetLastError();
          st = PENTAD_STATUS_EXECUTION_FAILED;
        }
      }
      if (plan) pentadsolver_plan_destroy(plan);
      s->arena.release(off, bytes);
    }
    if (st == PENTAD_STATUS_SUCCESS) {
      s->refine_pays[d] = t[1] < t[0];
      if (ms) {
        ms[2 * d] = t[0] / reps;
        ms[2 * d + 1] = t[1] / reps;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return st;
}

extern "C" PENTAD_API pentadStatus_t pentadsolver_server_destroy(pentadsolver_server_t s) {
  if (s == nullptr) return PENTAD_STATUS_INVALID_VALUE;
  complete_ready(s, true);
  for (Batch &b : s->in_flight) {  // only left when completing failed
    cudaEventSynchronize(b.done);
    pentadsolver_plan_destroy(b.plan);
    cudaEventDestroy(b.done);
  }
  for (cudaStream_t t : s->streams) cudaStreamDestroy(t);
  cudaGetLastError();
  delete s;
  return PENTAD_STATUS_SUCCESS;
}
