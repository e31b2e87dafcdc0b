// smac_async.cu -- projections with host buffers, copies overlapped with the
// solves of neighbouring projections.
//
// A stream of independent projections (smac_project) whose inputs and
// outputs live in host memory.  Per projection the input u* is copied in
// (3 face arrays) and u and p_delta are copied out (3 face arrays and one
// cell array), 0.97 GB at 256^3, against about 7 ms of solve: over PCIe the
// copies, not the solve, set the pace.  PCIe carries both directions at
// once, so the queue keeps three things in flight on three streams:
//
//   copy-in stream   H2D of projection i+1      (enqueued by smac_async_submit)
//   compute stream   projection i               (the handle's stream, worker thread)
//   copy-out stream  D2H of projection i-1      (enqueued by the worker)
//
// Two device staging slots alternate between projections.  Events order the
// reuse of a slot: projection i+2 copies its input in only after projection i
// has read it (compute_done), and writes its outputs only after projection
// i's outputs have been copied out (out_done).  The solve loop of
// smac_project waits on the device's convergence flag, so it runs in a
// worker thread, which keeps smac_async_submit from blocking on it.
//
// Host buffers should be page-locked (cudaHostAlloc / cudaHostRegister) for
// the copies to overlap; the caller keeps them valid until smac_async_wait
// returns for the projection.  While a queue is open, the handle must not be
// used from any other thread.
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>

#include <cuda_runtime.h>

#include "smac_b200.h"

namespace smac {
cudaStream_t handle_stream(const smac_handle* h);
void handle_shape(const smac_handle* h, int* nx, int* ny, int* nz);
void set_error_text(const char* fmt, ...);
}  // namespace smac

namespace {

struct AsyncJob {
  unsigned long long id;
  const double* in[3];
  double* out[4];  // vx, vy, vz, p_delta
  double dt;
};

struct AsyncSlot {
  double* u_in[3] = {nullptr, nullptr, nullptr};
  double* u_out[3] = {nullptr, nullptr, nullptr};
  double* pd = nullptr;
  cudaEvent_t in_ready = nullptr, compute_done = nullptr, out_done = nullptr;
};

struct AsyncResult {
  smac_status status;
  smac_stats stats;
};

}  // namespace

struct smac_async {
  smac_handle* h = nullptr;
  int device = 0;
  size_t n_face[3] = {0, 0, 0};  // elements of the x-, y-, z-face arrays
  size_t n_cell = 0;
  cudaStream_t s_in = nullptr, s_out = nullptr, s_comp = nullptr;
  AsyncSlot slot[2];
  std::thread worker;
  std::mutex mu;
  std::condition_variable cv;     // queue and progress changes
  std::deque<AsyncJob> queue;
  bool stop = false;
  unsigned long long next_id = 0;      // ids handed out so far
  unsigned long long started = 0;      // jobs whose compute_done is recorded
  unsigned long long finished = 0;     // jobs whose results are stored
  std::unordered_map<unsigned long long, AsyncResult> results;
};

namespace {

void worker_main(smac_async* a) {
  cudaSetDevice(a->device);
  for (;;) {
    AsyncJob job;
    {
      std::unique_lock<std::mutex> lk(a->mu);
      a->cv.wait(lk, [&] { return a->stop || !a->queue.empty(); });
      if (a->queue.empty()) return;  // stop requested and nothing left
      job = a->queue.front();
      a->queue.pop_front();
    }
    AsyncSlot& sl = a->slot[job.id & 1];
    AsyncResult res{};
    // the input is on the device; the slot's outputs of two projections ago
    // have left it
    cudaStreamWaitEvent(a->s_comp, sl.in_ready, 0);
    cudaStreamWaitEvent(a->s_comp, sl.out_done, 0);
    res.status = smac_project(a->h, sl.u_in[0], sl.u_in[1], sl.u_in[2], job.dt, sl.pd, sl.u_out[0], sl.u_out[1],
                              sl.u_out[2], &res.stats);
    cudaEventRecord(sl.compute_done, a->s_comp);
    {
      std::lock_guard<std::mutex> lk(a->mu);
      a->started = job.id + 1;
    }
    a->cv.notify_all();
    cudaStreamWaitEvent(a->s_out, sl.compute_done, 0);
    for (int d = 0; d < 3; ++d)
      cudaMemcpyAsync(job.out[d], sl.u_out[d], a->n_face[d] * sizeof(double), cudaMemcpyDeviceToHost, a->s_out);
    cudaMemcpyAsync(job.out[3], sl.pd, a->n_cell * sizeof(double), cudaMemcpyDeviceToHost, a->s_out);
    cudaEventRecord(sl.out_done, a->s_out);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess && res.status == SMAC_OK) {
      smac::set_error_text("smac_async: %s", cudaGetErrorString(e));
      res.status = SMAC_CUDA_ERROR;
    }
    {
      std::lock_guard<std::mutex> lk(a->mu);
      a->results[job.id] = res;
      a->finished = job.id + 1;
    }
    a->cv.notify_all();
  }
}

void release(smac_async* a) {
  for (AsyncSlot& sl : a->slot) {
    for (int d = 0; d < 3; ++d) {
      if (sl.u_in[d]) cudaFree(sl.u_in[d]);
      if (sl.u_out[d]) cudaFree(sl.u_out[d]);
    }
    if (sl.pd) cudaFree(sl.pd);
    if (sl.in_ready) cudaEventDestroy(sl.in_ready);
    if (sl.compute_done) cudaEventDestroy(sl.compute_done);
    if (sl.out_done) cudaEventDestroy(sl.out_done);
  }
  if (a->s_in) cudaStreamDestroy(a->s_in);
  if (a->s_out) cudaStreamDestroy(a->s_out);
  delete a;
}

}  // namespace

extern "C" {

smac_status smac_async_create(smac_handle* h, smac_async** out) {
  if (!h || !out) {
    smac::set_error_text("smac_async_create: null argument");
    return SMAC_BAD_ARG;
  }
  *out = nullptr;
  smac_async* a = new (std::nothrow) smac_async;
  if (!a) {
    smac::set_error_text("smac_async_create: out of host memory");
    return SMAC_CUDA_ERROR;
  }
  a->h = h;
  cudaGetDevice(&a->device);
  int nx, ny, nz;
  smac::handle_shape(h, &nx, &ny, &nz);
  const size_t X = nx, Y = ny, Z = nz;
  a->n_face[0] = (X + 3) * (Y + 2) * (Z + 2);
  a->n_face[1] = (X + 2) * (Y + 3) * (Z + 2);
  a->n_face[2] = (X + 2) * (Y + 2) * (Z + 3);
  a->n_cell = (X + 2) * (Y + 2) * (Z + 2);
  a->s_comp = smac::handle_stream(h);
  cudaError_t e = cudaStreamCreateWithFlags(&a->s_in, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&a->s_out, cudaStreamNonBlocking);
  for (AsyncSlot& sl : a->slot) {
    for (int d = 0; d < 3 && e == cudaSuccess; ++d) {
      e = cudaMalloc(&sl.u_in[d], a->n_face[d] * sizeof(double));
      if (e == cudaSuccess) e = cudaMalloc(&sl.u_out[d], a->n_face[d] * sizeof(double));
    }
    if (e == cudaSuccess) e = cudaMalloc(&sl.pd, a->n_cell * sizeof(double));
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.in_ready, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.compute_done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.out_done, cudaEventDisableTiming);
  }
  if (e != cudaSuccess) {
    smac::set_error_text("smac_async_create: %s", cudaGetErrorString(e));
    cudaGetLastError();
    release(a);
    return SMAC_CUDA_ERROR;
  }
  a->worker = std::thread(worker_main, a);
  *out = a;
  return SMAC_OK;
}

smac_status smac_async_submit(smac_async* a, const double* vxs, const double* vys, const double* vzs, double dt,
                              double* p_delta, double* vx, double* vy, double* vz, unsigned long long* ticket) {
  if (!a || !vxs || !vys || !vzs || !p_delta || !vx || !vy || !vz || !ticket) {
    smac::set_error_text("smac_async_submit: null argument");
    return SMAC_BAD_ARG;
  }
  AsyncJob job{};
  {
    std::unique_lock<std::mutex> lk(a->mu);
    job.id = a->next_id++;
    // the slot's previous projection (two back) must have read its input:
    // its compute_done event is recorded once the worker has started it
    const unsigned long long need = job.id >= 2 ? job.id - 1 : 0;
    a->cv.wait(lk, [&] { return a->started >= need; });
  }
  AsyncSlot& sl = a->slot[job.id & 1];
  job.in[0] = vxs;
  job.in[1] = vys;
  job.in[2] = vzs;
  job.out[0] = vx;
  job.out[1] = vy;
  job.out[2] = vz;
  job.out[3] = p_delta;
  job.dt = dt;
  cudaStreamWaitEvent(a->s_in, sl.compute_done, 0);
  for (int d = 0; d < 3; ++d)
    cudaMemcpyAsync(sl.u_in[d], job.in[d], a->n_face[d] * sizeof(double), cudaMemcpyHostToDevice, a->s_in);
  cudaEventRecord(sl.in_ready, a->s_in);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    smac::set_error_text("smac_async_submit: %s", cudaGetErrorString(e));
    return SMAC_CUDA_ERROR;
  }
  {
    std::lock_guard<std::mutex> lk(a->mu);
    a->queue.push_back(job);
  }
  a->cv.notify_all();
  *ticket = job.id;
  return SMAC_OK;
}

smac_status smac_async_wait(smac_async* a, unsigned long long ticket, smac_stats* stats) {
  if (!a) {
    smac::set_error_text("smac_async_wait: null argument");
    return SMAC_BAD_ARG;
  }
  AsyncResult res{};
  {
    std::unique_lock<std::mutex> lk(a->mu);
    if (ticket >= a->next_id) {
      smac::set_error_text("smac_async_wait: ticket %llu was not issued", ticket);
      return SMAC_BAD_ARG;
    }
    a->cv.wait(lk, [&] { return a->finished > ticket; });
    auto it = a->results.find(ticket);
    if (it == a->results.end()) {
      smac::set_error_text("smac_async_wait: ticket %llu was already collected", ticket);
      return SMAC_BAD_ARG;
    }
    res = it->second;
    a->results.erase(it);
  }
  // copies leave in order on one stream: the slot's latest copy-out covers this one
  const cudaError_t e = cudaEventSynchronize(a->slot[ticket & 1].out_done);
  if (e != cudaSuccess) {
    smac::set_error_text("smac_async_wait: %s", cudaGetErrorString(e));
    return SMAC_CUDA_ERROR;
  }
  if (stats) *stats = res.stats;
  return res.status;
}

void smac_async_destroy(smac_async* a) {
  if (!a) return;
  {
    std::lock_guard<std::mutex> lk(a->mu);
    a->stop = true;
  }
  a->cv.notify_all();
  if (a->worker.joinable()) a->worker.join();
  cudaStreamSynchronize(a->s_in);
  cudaStreamSynchronize(a->s_out);
  cudaStreamSynchronize(a->s_comp);
  release(a);
}

}  // extern "C"
