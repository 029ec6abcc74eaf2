// Serving layer of the B200 Fourier-reconstruction engine: the C-ABI declared in
// include/umpalumpa_fr_server.h.  Many reconstruction jobs share one GPU: a dispatcher
// thread gathers the pending projection batches of every admitted job into one batched
// insertion launch per step (fr_batch_execute), a completion thread retires finished steps,
// and jobs are admitted first come first served within an HBM budget.  The reference runs
// one volume per operation instance and feeds it batch by batch
// (examples/fourier_reconstruction/fr.cpp:205-228); a served job is that loop, with the
// batches of concurrently open jobs sharing each launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "fr_device_guard.h"
#include "fr_engine.h"
#include "fr_kernels.h"
#include "umpalumpa_fr.h"
#include "umpalumpa_fr_server.h"

namespace {

using frb::DeviceGuard;
using Clock = std::chrono::steady_clock;

int fail(int code, const std::string &msg) { return frb::set_last_error(code, msg.c_str()); }

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

bool host_memory(const void *p)
{
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return true;
  }
  return a.type == cudaMemoryTypeHost || a.type == cudaMemoryTypeUnregistered;
}

// One submitted batch and how much of it has been handed to steps.
struct Batch {
  fr_server_batch b{};
  bool host = false;         // fft (and scales) in host memory
  bool rot_host = false;     // rotations in host memory
  bool spaces_host = false;  // spaces in host memory
  uint64_t total = 0;        // traverse spaces to insert
  uint64_t dispatched = 0;   // traverse spaces handed to steps
  int inflight = 0;          // steps in flight holding a slice of it
};

struct Job {
  uint64_t id = 0;
  fr_server_job_desc d{};
  int state = FR_JOB_QUEUED;
  bool closed = false;
  bool admitting = false;  // its volume is being allocated (lock released): not yet active
  size_t footprint = 0;
  void *volume = nullptr;
  float *weight = nullptr;
  std::deque<Batch> batches;  // not yet done, oldest first
  uint64_t submitted = 0, done = 0, spaces_done = 0;
  double t_open = 0, t_admit = -1, t_done = -1;
};

// A slice [off, off + take) of one batch, with everything the launch needs copied out of
// the shared state so the dispatcher can stage and launch without holding the lock.
struct Slice {
  uint64_t job = 0;
  Batch *batch = nullptr;  // only dereferenced under the lock after the job is looked up
  fr_server_batch b{};
  bool host = false, rot_host = false, spaces_host = false;
  uint64_t off = 0, take = 0;
  fr_server_job_desc d{};
  void *volume = nullptr;
  float *weight = nullptr;
};

// Staging of one in-flight step: traverse spaces, plus host-resident inputs copied over.
struct Slot {
  fr_traverse_space *spaces = nullptr;  // max_step_projections spaces
  unsigned char *stage = nullptr;       // staging_bytes
  cudaEvent_t ready = nullptr;          // staging finished (copy stream)
  cudaEvent_t free = nullptr;           // the step that read the slot finished (compute stream)
};

struct Step {
  int slot = 0;
  cudaEvent_t start = nullptr, done = nullptr;
  std::vector<Slice> slices;
  uint64_t spaces = 0;
  double t_formed = 0, t_enqueued = 0, t_launched = 0;
};

constexpr size_t kStepLog = 4096;  // retired steps kept for fr_server_step_log

}// namespace

struct fr_server {
  int device = 0;
  fr_server_config cfg{};
  fr_settings settings{};
  Clock::time_point t0;
  size_t elem = 8;  // bytes per stored complex value
  fr_handle *engine = nullptr;
  cudaStream_t compute = nullptr, copy = nullptr, readback = nullptr;
  cudaMemPool_t pool = nullptr;
  float *table = nullptr;
  Slot slots[2];
  // start/done events of the steps, a ring of three: with at most two steps in flight the
  // previous step's done event is intact when a step completes
  cudaEvent_t step_events[3][2] = {};
  uint64_t step_seq = 0;
  int next_slot = 0;

  std::mutex mu;
  std::condition_variable cv_dispatch, cv_complete, cv_wait;
  bool stop = false, stop_complete = false;
  bool failed = false;
  std::string failure;
  std::map<uint64_t, Job> jobs;
  std::deque<uint64_t> queued;   // waiting for admission, first come first served
  std::vector<uint64_t> active;  // admitted and not yet done
  uint32_t admitting = 0;        // jobs between admission and activation (hold slot and budget)
  uint64_t next_id = 1;
  std::deque<Step> inflight;
  fr_server_stats stats{};
  std::deque<fr_server_step_record> step_log;
  std::thread dispatcher, completer;

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

namespace {

// Bytes of slot staging a slice of `take` spaces needs (each allocation 256-byte aligned).
size_t stage_bytes(const fr_server &S, const Slice &s, uint64_t take)
{
  const size_t pb = size_t(s.d.fft_x) * s.d.fft_y * S.elem;
  const bool scaled = S.settings.storage != FR_STORAGE_FP32;
  size_t n = 0;
  if (s.b.rotations) {
    if (s.rot_host) n += align256(take * 9 * sizeof(float));
    if (s.host) n += align256(take * pb) + (scaled ? align256(take * sizeof(float)) : 0);
  } else if (s.host) {
    n += align256(s.b.n_projections * pb) + (scaled ? align256(s.b.n_projections * sizeof(float)) : 0);
  }
  return n;
}

void fail_all(fr_server &S, const std::string &msg)
{
  if (!S.failed) {
    S.failed = true;
    S.failure = msg;
  }
  for (auto &kv : S.jobs)
    if (kv.second.state == FR_JOB_ACTIVE || kv.second.state == FR_JOB_QUEUED) kv.second.state = FR_JOB_FAILED;
  S.active.clear();
  S.queued.clear();
  S.cv_wait.notify_all();
  S.cv_dispatch.notify_all();
}

void finish_if_complete(fr_server &S, Job &J)
{
  if (J.state != FR_JOB_ACTIVE || !J.closed || !J.batches.empty()) return;
  J.state = FR_JOB_DONE;
  J.t_done = S.now();
  S.stats.jobs_done += 1;
  S.active.erase(std::remove(S.active.begin(), S.active.end(), J.id), S.active.end());
  S.cv_wait.notify_all();
}

// Admits queued jobs, oldest first, while they fit.  The caller holds the lock; it is released
// around each admitted job's allocation and zeroing (a memory-pool call can take tens of
// milliseconds, which under the lock would stall the dispatcher and the completion thread).
// Meanwhile the job holds its budget and slot and stays queued to clients.
void admit(fr_server &S, std::unique_lock<std::mutex> &lk)
{
  while (!S.failed && !S.queued.empty()) {
    auto it = S.jobs.find(S.queued.front());
    if (it == S.jobs.end() || it->second.state != FR_JOB_QUEUED) {
      S.queued.pop_front();
      continue;
    }
    Job &J = it->second;
    if (S.active.size() + S.admitting >= S.cfg.max_jobs || S.stats.bytes_admitted + J.footprint > S.cfg.hbm_budget)
      return;
    S.queued.pop_front();
    J.admitting = true;
    S.admitting += 1;
    S.stats.bytes_admitted += J.footprint;
    S.stats.peak_bytes_admitted = std::max(S.stats.peak_bytes_admitted, S.stats.bytes_admitted);
    const uint64_t id = J.id;
    const size_t voxels = size_t(J.d.volume_x) * J.d.volume_y * J.d.volume_z;
    const double ta = S.now();
    lk.unlock();
    void *vol = nullptr;
    float *w = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&vol, voxels * 8, S.pool, S.compute);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync(reinterpret_cast<void **>(&w), voxels * 4, S.pool, S.compute);
    if (e == cudaSuccess) e = cudaMemsetAsync(vol, 0, voxels * 8, S.compute);
    if (e == cudaSuccess) e = cudaMemsetAsync(w, 0, voxels * 4, S.compute);
    if (e != cudaSuccess) cudaGetLastError();
    const double tb = S.now();
    lk.lock();
    S.admitting -= 1;
    Job &K = S.jobs.at(id);  // release waits while a job is being admitted: it is still there
    K.admitting = false;
    S.cv_wait.notify_all();
    S.stats.max_admit_ms = std::max(S.stats.max_admit_ms, (tb - ta) * 1e3);
    if (e != cudaSuccess || K.state != FR_JOB_QUEUED) {  // allocation failed, or the server failed
      if (vol) cudaFreeAsync(vol, S.compute);
      if (w) cudaFreeAsync(w, S.compute);
      S.stats.bytes_admitted -= K.footprint;
      K.state = FR_JOB_FAILED;
      S.cv_wait.notify_all();
      continue;
    }
    K.volume = vol;
    K.weight = w;
    K.state = FR_JOB_ACTIVE;
    K.t_admit = tb;
    S.active.push_back(K.id);
    S.stats.peak_jobs_active = std::max<uint32_t>(S.stats.peak_jobs_active, uint32_t(S.active.size()));
    finish_if_complete(S, K);
    S.cv_dispatch.notify_all();
  }
}

bool has_work(const fr_server &S)
{
  for (uint64_t id : S.active) {
    const Job &J = S.jobs.at(id);
    for (const Batch &B : J.batches)
      if (B.dispatched < B.total) return true;
  }
  return false;
}

// Picks the slices of the next step (caller holds the lock).  Jobs are served closed ones
// first -- every batch of a closed job has arrived, so its remaining work is all that stands
// between it and completion -- then open ones, each group oldest first; a job hands over its
// pending batches oldest first until the step's space, slice or staging limits are reached.
// Open jobs cannot starve: every job is eventually closed and then served ahead of later ones.
void select(fr_server &S, Step &st)
{
  uint64_t room = S.cfg.max_step_projections;
  size_t stage_left = S.cfg.staging_bytes;
  std::vector<Job *> order;
  order.reserve(S.active.size());
  for (uint64_t id : S.active) order.push_back(&S.jobs.at(id));
  std::stable_sort(order.begin(), order.end(), [](const Job *a, const Job *b) {
    if (a->closed != b->closed) return a->closed;
    return a->id < b->id;  // ids grow with open time
  });
  for (Job *Jp : order) {
    if (room == 0) break;
    Job &J = *Jp;
    for (Batch &B : J.batches) {
      if (room == 0 || st.slices.size() >= S.cfg.max_step_entries) break;
      if (B.dispatched >= B.total) continue;
      Slice s;
      s.job = J.id;
      s.batch = &B;
      s.b = B.b;
      s.host = B.host;
      s.rot_host = B.rot_host;
      s.spaces_host = B.spaces_host;
      s.off = B.dispatched;
      s.d = J.d;
      s.volume = J.volume;
      s.weight = J.weight;
      uint64_t take = std::min<uint64_t>(B.total - B.dispatched, room);
      if (B.b.rotations && (B.host || B.rot_host)) {
        // staging grows with the slice: shrink it to what is left
        while (take > 0 && stage_bytes(S, s, take) > stage_left) {
          const size_t per = std::max<size_t>(1, stage_bytes(S, s, take) / take);
          take = std::min<uint64_t>(take - 1, stage_left / per);
        }
      } else if (stage_bytes(S, s, take) > stage_left) {
        take = 0;
      }
      if (take == 0) break;  // this job's next batch waits for the next step
      s.take = take;
      stage_left -= stage_bytes(S, s, take);
      B.dispatched += take;
      B.inflight += 1;
      room -= take;
      st.spaces += take;
      st.slices.push_back(s);
    }
  }
}

// Stages the slices' inputs and traverse spaces on the copy stream and enqueues the batched
// insertion on the compute stream (dispatcher thread, lock not held).
int launch(fr_server &S, Step &st, std::vector<fr_job> &jobs)
{
  Slot &sl = S.slots[st.slot];
  const bool scaled = S.settings.storage != FR_STORAGE_FP32;
  if (cudaStreamWaitEvent(S.copy, sl.free, 0) != cudaSuccess) return fail(FR_E_CUDA, "cudaStreamWaitEvent failed");
  if (cudaEventRecord(st.start, S.copy) != cudaSuccess) return fail(FR_E_CUDA, "cudaEventRecord failed");
  size_t so = 0;
  uint64_t sp = 0;
  auto stage = [&](const void *src, size_t bytes) -> void * {
    void *dst = sl.stage + so;
    so += align256(bytes);
    if (cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, S.copy) != cudaSuccess) return nullptr;
    return dst;
  };
  jobs.resize(st.slices.size());
  for (size_t k = 0; k < st.slices.size(); ++k) {
    const Slice &s = st.slices[k];
    const size_t pb = size_t(s.d.fft_x) * s.d.fft_y * S.elem;
    fr_job &J = jobs[k];
    std::memset(&J, 0, sizeof(J));
    J.volume = s.volume;
    J.weight = s.weight;
    J.fft_x = s.d.fft_x;
    J.fft_y = s.d.fft_y;
    J.volume_x = s.d.volume_x;
    J.volume_y = s.d.volume_y;
    J.volume_z = s.d.volume_z;
    J.n_spaces = s.take;
    if (s.b.rotations) {
      const float *rot = s.b.rotations + s.off * 9;
      if (s.rot_host && !(rot = static_cast<const float *>(stage(rot, s.take * 9 * sizeof(float)))))
        return fail(FR_E_CUDA, "staging the rotations failed");
      if (s.host) {
        J.fft = stage(static_cast<const unsigned char *>(s.b.fft) + s.off * pb, s.take * pb);
        if (scaled) J.scales = static_cast<const float *>(stage(s.b.scales + s.off, s.take * sizeof(float)));
        if (!J.fft || (scaled && !J.scales)) return fail(FR_E_CUDA, "staging the projections failed");
        J.n_projections = s.take;
      } else {  // only this slice's projections (the batch copies them into bands)
        J.fft = static_cast<const unsigned char *>(s.b.fft) + s.off * pb;
        J.scales = scaled ? s.b.scales + s.off : nullptr;
        J.n_projections = s.take;
      }
      fr_traverse_space *out = sl.spaces + sp;
      sp += s.take;
      if (frb::launch_traverse_spaces(rot, int64_t(s.take), s.d.image_x, s.d.image_y, s.d.volume_x - 1,
            s.d.volume_y - 1, S.settings.type == FR_TYPE_FAST, S.settings.blob_radius, s.d.space_weight, 0, out,
            S.copy) != cudaSuccess)
        return fail(FR_E_CUDA, "traverse-space kernel launch failed");
      J.spaces = out;
    } else {
      if (s.spaces_host) {
        fr_traverse_space *out = sl.spaces + sp;
        sp += s.take;
        if (cudaMemcpyAsync(out, s.b.spaces + s.off, s.take * sizeof(fr_traverse_space), cudaMemcpyHostToDevice,
              S.copy) != cudaSuccess)
          return fail(FR_E_CUDA, "staging the traverse spaces failed");
        J.spaces = out;
      } else {
        J.spaces = s.b.spaces + s.off;
      }
      if (s.host) {
        J.fft = stage(s.b.fft, s.b.n_projections * pb);
        if (scaled) J.scales = static_cast<const float *>(stage(s.b.scales, s.b.n_projections * sizeof(float)));
        if (!J.fft || (scaled && !J.scales)) return fail(FR_E_CUDA, "staging the projections failed");
      } else {
        J.fft = s.b.fft;
        J.scales = s.b.scales;
      }
      J.n_projections = s.b.n_projections;
    }
  }
  if (cudaEventRecord(sl.ready, S.copy) != cudaSuccess || cudaStreamWaitEvent(S.compute, sl.ready, 0) != cudaSuccess)
    return fail(FR_E_CUDA, "ordering the step after its staging failed");
  const int rc = fr_batch_execute(S.engine, jobs.data(), jobs.size(), S.table, 0);
  if (rc) return rc;
  if (cudaEventRecord(sl.free, S.compute) != cudaSuccess || cudaEventRecord(st.done, S.compute) != cudaSuccess)
    return fail(FR_E_CUDA, "cudaEventRecord failed");
  return FR_OK;
}

void dispatch_loop(fr_server *Sp)
{
  fr_server &S = *Sp;
  cudaSetDevice(S.device);
  std::vector<fr_job> jobs;
  std::unique_lock<std::mutex> lk(S.mu);
  for (;;) {
    S.cv_dispatch.wait(lk, [&] {
      return S.stop || (!S.failed && S.inflight.size() < S.cfg.pipeline_depth && has_work(S));
    });
    if (S.stop) break;
    Step st;
    st.slot = S.next_slot;
    st.start = S.step_events[S.step_seq % 3][0];
    st.done = S.step_events[S.step_seq % 3][1];
    select(S, st);
    st.t_formed = S.now();
    if (st.slices.empty()) {  // nothing fits this step's limits yet
      S.cv_dispatch.wait_for(lk, std::chrono::milliseconds(1));
      continue;
    }
    S.next_slot ^= 1;
    S.step_seq += 1;
    lk.unlock();
    const int rc = launch(S, st, jobs);
    st.t_enqueued = S.now();
    const std::string msg = rc ? std::string(fr_last_error()) : std::string();
    lk.lock();
    if (rc) {
      fail_all(S, "step launch failed: " + msg);
      continue;
    }
    st.t_launched = S.now();
    S.inflight.push_back(std::move(st));
    S.cv_complete.notify_one();
  }
}

void complete_loop(fr_server *Sp)
{
  fr_server &S = *Sp;
  cudaSetDevice(S.device);
  std::unique_lock<std::mutex> lk(S.mu);
  cudaEvent_t prev_done = nullptr;  // the last completed step's done event
  for (;;) {
    S.cv_complete.wait(lk, [&] { return !S.inflight.empty() || S.stop_complete; });
    if (S.inflight.empty()) break;
    const cudaEvent_t start = S.inflight.front().start, done = S.inflight.front().done;
    lk.unlock();
    cudaError_t e = cudaEventSynchronize(done);
    float ms = 0.f, since_prev = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, start, done);
    const float raw_ms = ms;
    // GPU time not already counted for the previous step (steps overlap by their staging)
    if (e == cudaSuccess && prev_done && cudaEventElapsedTime(&since_prev, prev_done, done) == cudaSuccess)
      ms = std::min(ms, std::max(since_prev, 0.f));
    cudaGetLastError();
    prev_done = done;
    const int status = frb::batch_device_status(S.engine);
    lk.lock();
    Step st = std::move(S.inflight.front());
    S.inflight.pop_front();
    if (e != cudaSuccess || status != FR_OK) {
      fail_all(S, e != cudaSuccess ? std::string("step failed: ") + cudaGetErrorString(e)
                                   : std::string("device-side failure in a step (status ") + std::to_string(status) + ")");
    } else {
      S.stats.steps += 1;
      S.stats.entries += st.slices.size();
      S.stats.spaces += st.spaces;
      S.stats.busy_ms += ms;
      fr_server_step_record rec{};
      rec.t_formed = st.t_formed;
      rec.t_enqueued = st.t_enqueued;
      rec.t_launched = st.t_launched;
      rec.t_retired = S.now();
      rec.gpu_ms = ms;
      rec.gpu_span_ms = raw_ms;
      rec.slices = uint32_t(st.slices.size());
      rec.spaces = st.spaces;
      std::vector<uint64_t> ids;
      for (const Slice &s : st.slices) ids.push_back(s.job);
      std::sort(ids.begin(), ids.end());
      rec.jobs = uint32_t(std::unique(ids.begin(), ids.end()) - ids.begin());
      S.step_log.push_back(rec);
      if (S.step_log.size() > kStepLog) S.step_log.pop_front();
      for (const Slice &s : st.slices) {
        auto it = S.jobs.find(s.job);
        if (it == S.jobs.end()) continue;
        Job &J = it->second;
        s.batch->inflight -= 1;
        J.spaces_done += s.take;
        while (!J.batches.empty() && J.batches.front().dispatched == J.batches.front().total
               && J.batches.front().inflight == 0) {
          J.batches.pop_front();
          J.done += 1;
        }
        finish_if_complete(S, J);
      }
      S.cv_wait.notify_all();
    }
    S.cv_dispatch.notify_all();
  }
}

int check_desc(const fr_server &S, const fr_server_job_desc *d)
{
  if (!d) return fail(FR_E_INVALID, "job description is NULL");
  if (d->fft_x < 1 || d->fft_y < 2 || d->volume_x < 3 || d->image_x < 1 || d->image_y < 1)
    return fail(FR_E_INVALID, "job sizes must be positive");
  if (d->volume_x % 2 == 0 || d->volume_y % 2 == 0 || d->volume_y != d->volume_z)
    return fail(FR_E_UNSUPPORTED, "job volume sizes must be odd with y == z");
  if (std::max(d->volume_x, d->volume_y) > S.cfg.max_volume_side)
    return fail(FR_E_UNSUPPORTED, "job volume exceeds the server's max_volume_side");
  return FR_OK;
}

}// namespace

extern "C" {

void fr_server_config_default(fr_server_config *c)
{
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  c->hbm_budget = 150ull * 1000 * 1000 * 1000;
  c->staging_bytes = 1ull << 30;
  c->max_jobs = 256;
  c->max_step_projections = 65536;
  c->max_step_entries = 256;
  c->max_volume_side = 385;
  c->table_elems = 10000;
  c->pipeline_depth = 2;
}

double fr_server_clock(const fr_server *S) { return S ? S->now() : 0.0; }

int fr_server_destroy(fr_server *S);

int fr_server_create(int device, const fr_server_config *config, const fr_settings *settings, fr_server **out)
{
  if (!out) return fail(FR_E_INVALID, "out is NULL");
  *out = nullptr;
  if (!settings) return fail(FR_E_INVALID, "settings is NULL");
  fr_server_config c;
  fr_server_config_default(&c);
  if (config) {
    c.hbm_budget = config->hbm_budget;
    if (config->staging_bytes) c.staging_bytes = config->staging_bytes;
    if (config->max_jobs) c.max_jobs = config->max_jobs;
    if (config->max_step_projections) c.max_step_projections = config->max_step_projections;
    if (config->max_step_entries) c.max_step_entries = config->max_step_entries;
    if (config->max_volume_side) c.max_volume_side = config->max_volume_side;
    if (config->table_elems) c.table_elems = config->table_elems;
    if (config->pipeline_depth) c.pipeline_depth = config->pipeline_depth;
    c.reserve_bytes = std::min(config->reserve_bytes, config->hbm_budget);
  }
  if (c.hbm_budget == 0) return fail(FR_E_INVALID, "hbm_budget must be positive");
  if (c.pipeline_depth > 2) return fail(FR_E_INVALID, "pipeline_depth must be 1 or 2");
  if (c.max_step_entries > 4096) return fail(FR_E_UNSUPPORTED, "max_step_entries above 4096");
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
    cudaGetLastError();
    return fail(FR_E_CUDA, "no such CUDA device");
  }
  DeviceGuard guard(device);
  fr_server *S = new (std::nothrow) fr_server();
  if (!S) return fail(FR_E_INVALID, "out of host memory");
  S->device = device;
  S->cfg = c;
  S->settings = *settings;
  S->t0 = Clock::now();
  S->elem = settings->storage == FR_STORAGE_FP32 ? 8 : 4;
  auto bail = [&](int code, const std::string &msg) -> int {
    const std::string m = msg;  // fr_server_destroy may overwrite the thread's message
    fr_server_destroy(S);
    return fail(code, m);
  };
  auto cu = [&](cudaError_t e, const char *what) -> int {
    if (e == cudaSuccess) return FR_OK;
    cudaGetLastError();
    return fail(FR_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  };
  int rc = cu(cudaStreamCreateWithFlags(&S->compute, cudaStreamNonBlocking), "stream");
  if (!rc) rc = cu(cudaStreamCreateWithFlags(&S->copy, cudaStreamNonBlocking), "stream");
  if (!rc) rc = cu(cudaStreamCreateWithFlags(&S->readback, cudaStreamNonBlocking), "stream");
  if (rc) return bail(rc, fr_last_error());
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.handleTypes = cudaMemHandleTypeNone;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  rc = cu(cudaMemPoolCreate(&S->pool, &props), "cudaMemPoolCreate");
  if (!rc) {
    uint64_t keep = ~0ull;
    rc = cu(cudaMemPoolSetAttribute(S->pool, cudaMemPoolAttrReleaseThreshold, &keep), "cudaMemPoolSetAttribute");
  }
  if (rc) return bail(rc, fr_last_error());
  if (c.reserve_bytes) {
    // Grow the pool by allocating the reserve in chunks that each hold the largest job, then
    // freeing them: the pool keeps the memory (release threshold above) and admissions carve
    // their volumes out of it.
    const uint64_t side = c.max_volume_side;
    const uint64_t chunk = std::max<uint64_t>(1ull << 30, align256(side * side * side * 8) + align256(side * side * side * 4));
    std::vector<void *> held;
    for (uint64_t got = 0; !rc && got < c.reserve_bytes; got += chunk) {
      void *p = nullptr;
      rc = cu(cudaMallocFromPoolAsync(&p, std::min(chunk, c.reserve_bytes - got), S->pool, S->compute),
        "reserving job memory");
      if (!rc) held.push_back(p);
    }
    for (void *p : held) cudaFreeAsync(p, S->compute);
    if (!rc) rc = cu(cudaStreamSynchronize(S->compute), "cudaStreamSynchronize");
    if (rc) return bail(rc, fr_last_error());
  }
  // the batched engine, sized for the largest step
  rc = fr_create(device, S->compute, &S->engine);
  if (rc) return bail(rc, fr_last_error());
  const uint64_t nb = (uint64_t(c.max_volume_side) + 15) / 16;
  fr_batch_limits lim{};
  lim.max_jobs = c.max_step_entries;
  lim.max_spaces = c.max_step_projections;
  lim.max_bricks = uint64_t(c.max_step_entries) * nb * nb * nb;
  lim.max_volume_side = c.max_volume_side;
  lim.table_elems = settings->interpolation == FR_INTERPOLATION_LOOKUP ? c.table_elems : 0;
  rc = fr_batch_init(S->engine, &lim, settings);
  if (rc) return bail(rc, fr_last_error());
  if (settings->interpolation == FR_INTERPOLATION_LOOKUP) {
    rc = cu(cudaMalloc(&S->table, size_t(c.table_elems) * sizeof(float)), "cudaMalloc");
    if (!rc) rc = fr_fill_blob_table(S->table, c.table_elems, settings, S->compute);
    if (rc) return bail(rc, fr_last_error());
  }
  for (auto &sl : S->slots) {
    rc = cu(cudaMalloc(reinterpret_cast<void **>(&sl.spaces), size_t(c.max_step_projections) * sizeof(fr_traverse_space)),
      "cudaMalloc");
    if (!rc) rc = cu(cudaMalloc(reinterpret_cast<void **>(&sl.stage), c.staging_bytes), "cudaMalloc");
    if (!rc) rc = cu(cudaEventCreateWithFlags(&sl.ready, cudaEventDisableTiming), "cudaEventCreate");
    if (!rc) rc = cu(cudaEventCreateWithFlags(&sl.free, cudaEventDisableTiming), "cudaEventCreate");
    if (rc) return bail(rc, fr_last_error());
  }
  for (auto &pair : S->step_events)
    for (auto &e : pair)
      if ((rc = cu(cudaEventCreateWithFlags(&e, cudaEventBlockingSync), "cudaEventCreate"))) return bail(rc, fr_last_error());
  // slots start free
  for (auto &sl : S->slots)
    if ((rc = cu(cudaEventRecord(sl.free, S->compute), "cudaEventRecord"))) return bail(rc, fr_last_error());
  if ((rc = cu(cudaStreamSynchronize(S->compute), "cudaStreamSynchronize"))) return bail(rc, fr_last_error());
  try {
    S->dispatcher = std::thread(dispatch_loop, S);
    S->completer = std::thread(complete_loop, S);
  } catch (...) {
    return bail(FR_E_INVALID, "cannot start the server threads");
  }
  *out = S;
  return FR_OK;
}

int fr_server_destroy(fr_server *S)
{
  if (!S) return FR_OK;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
    S->cv_dispatch.notify_all();
  }
  if (S->dispatcher.joinable()) S->dispatcher.join();
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop_complete = true;
    S->cv_complete.notify_all();
  }
  if (S->completer.joinable()) S->completer.join();
  DeviceGuard guard(S->device);
  if (S->compute) cudaStreamSynchronize(S->compute);
  if (S->copy) cudaStreamSynchronize(S->copy);
  for (auto &kv : S->jobs) {
    if (kv.second.volume) cudaFreeAsync(kv.second.volume, S->compute);
    if (kv.second.weight) cudaFreeAsync(kv.second.weight, S->compute);
  }
  if (S->compute) cudaStreamSynchronize(S->compute);
  if (S->engine) fr_destroy(S->engine);
  for (auto &sl : S->slots) {
    if (sl.spaces) cudaFree(sl.spaces);
    if (sl.stage) cudaFree(sl.stage);
    if (sl.ready) cudaEventDestroy(sl.ready);
    if (sl.free) cudaEventDestroy(sl.free);
  }
  for (auto &pair : S->step_events)
    for (auto &e : pair)
      if (e) cudaEventDestroy(e);
  if (S->table) cudaFree(S->table);
  if (S->pool) cudaMemPoolDestroy(S->pool);
  if (S->compute) cudaStreamDestroy(S->compute);
  if (S->copy) cudaStreamDestroy(S->copy);
  if (S->readback) cudaStreamDestroy(S->readback);
  delete S;
  return FR_OK;
}

int fr_server_open_job(fr_server *S, const fr_server_job_desc *d, uint64_t *job)
{
  if (!S || !job) return fail(FR_E_INVALID, "NULL argument");
  int rc = check_desc(*S, d);
  if (rc) return rc;
  const size_t footprint = align256(size_t(d->volume_x) * d->volume_y * d->volume_z * 8)
                           + align256(size_t(d->volume_x) * d->volume_y * d->volume_z * 4);
  std::unique_lock<std::mutex> lk(S->mu);
  if (S->failed) return fail(FR_E_CUDA, "server failed: " + S->failure);
  if (footprint > S->cfg.hbm_budget) return fail(FR_E_CAPACITY, "job volume and weights exceed the HBM budget");
  DeviceGuard guard(S->device);
  Job &J = S->jobs[S->next_id];
  J.id = S->next_id++;
  J.d = *d;
  J.footprint = footprint;
  J.t_open = S->now();
  S->queued.push_back(J.id);
  *job = J.id;
  admit(*S, lk);
  return FR_OK;
}

int fr_server_submit(fr_server *S, uint64_t job, const fr_server_batch *b)
{
  if (!S || !b) return fail(FR_E_INVALID, "NULL argument");
  if (!b->fft || b->n_projections == 0) return fail(FR_E_INVALID, "a batch needs projections");
  if (!b->rotations && (!b->spaces || b->n_spaces == 0)) return fail(FR_E_INVALID, "a batch needs rotations or spaces");
  const bool scaled = S->settings.storage != FR_STORAGE_FP32;
  if (scaled != (b->scales != nullptr)) return fail(FR_E_INVALID, "scales go with BF16/FP16 storage only");
  if (b->n_projections > (1ull << 31) || (!b->rotations && b->n_spaces > (1ull << 31)))
    return fail(FR_E_UNSUPPORTED, "batch too large");
  DeviceGuard guard(S->device);
  Batch B;
  B.b = *b;
  B.host = host_memory(b->fft);
  if (scaled && host_memory(b->scales) != B.host)
    return fail(FR_E_INVALID, "fft and scales must both be host or both be device memory");
  B.rot_host = b->rotations && host_memory(b->rotations);
  B.spaces_host = !b->rotations && host_memory(b->spaces);
  B.total = b->rotations ? b->n_projections : b->n_spaces;
  if (!b->rotations) B.b.rotations = nullptr;
  std::lock_guard<std::mutex> lk(S->mu);
  if (S->failed) return fail(FR_E_CUDA, "server failed: " + S->failure);
  auto it = S->jobs.find(job);
  if (it == S->jobs.end()) return fail(FR_E_INVALID, "no such job");
  Job &J = it->second;
  if (J.closed || (J.state != FR_JOB_QUEUED && J.state != FR_JOB_ACTIVE))
    return fail(FR_E_INVALID, "the job is closed");
  Slice probe;
  probe.b = B.b;
  probe.host = B.host;
  probe.rot_host = B.rot_host;
  probe.d = J.d;
  if (stage_bytes(*S, probe, 1) > S->cfg.staging_bytes)
    return fail(FR_E_CAPACITY, "the batch's host-resident inputs exceed the server's staging_bytes");
  J.batches.push_back(B);
  J.submitted += 1;
  S->cv_dispatch.notify_all();
  return FR_OK;
}

int fr_server_close_job(fr_server *S, uint64_t job)
{
  if (!S) return fail(FR_E_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->jobs.find(job);
  if (it == S->jobs.end()) return fail(FR_E_INVALID, "no such job");
  it->second.closed = true;
  finish_if_complete(*S, it->second);
  return FR_OK;
}

static void fill_info(const Job &J, fr_server_job_info *info)
{
  if (!info) return;
  std::memset(info, 0, sizeof(*info));
  info->state = J.state;
  info->batches_submitted = J.submitted;
  info->batches_done = J.done;
  info->spaces_done = J.spaces_done;
  info->volume = J.volume;
  info->weight = J.weight;
  info->t_open = J.t_open;
  info->t_admit = J.t_admit;
  info->t_done = J.t_done;
}

int fr_server_wait_job(fr_server *S, uint64_t job, double timeout_s, fr_server_job_info *info)
{
  if (!S) return fail(FR_E_INVALID, "NULL argument");
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->jobs.find(job);
  if (it == S->jobs.end()) return fail(FR_E_INVALID, "no such job");
  const Job &J = it->second;
  auto ready = [&] { return J.state == FR_JOB_DONE || J.state == FR_JOB_FAILED; };
  if (timeout_s < 0) {
    S->cv_wait.wait(lk, ready);
  } else if (!S->cv_wait.wait_for(lk, std::chrono::duration<double>(timeout_s), ready)) {
    fill_info(J, info);
    return fail(FR_E_CAPACITY, "timed out waiting for the job");
  }
  fill_info(J, info);
  if (J.state == FR_JOB_FAILED) return fail(FR_E_CUDA, S->failed ? "server failed: " + S->failure : "job failed");
  return FR_OK;
}

int fr_server_query_job(fr_server *S, uint64_t job, fr_server_job_info *info)
{
  if (!S || !info) return fail(FR_E_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->jobs.find(job);
  if (it == S->jobs.end()) return fail(FR_E_INVALID, "no such job");
  fill_info(it->second, info);
  return FR_OK;
}

int fr_server_read_job(fr_server *S, uint64_t job, void *volume, float *weight)
{
  if (!S) return fail(FR_E_INVALID, "NULL argument");
  void *v = nullptr;
  float *w = nullptr;
  size_t voxels = 0;
  bool empty = false;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->jobs.find(job);
    if (it == S->jobs.end()) return fail(FR_E_INVALID, "no such job");
    const Job &J = it->second;
    if (J.state != FR_JOB_DONE) return fail(FR_E_INVALID, "the job is not done");
    v = J.volume;
    w = J.weight;
    voxels = size_t(J.d.volume_x) * J.d.volume_y * J.d.volume_z;
    empty = J.spaces_done == 0;
  }
  DeviceGuard guard(S->device);
  cudaEvent_t ev = nullptr;
  if (empty) {  // nothing inserted: order the copy after the zeroing on the compute stream
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return fail(FR_E_CUDA, "cudaEventCreate failed");
    cudaEventRecord(ev, S->compute);
    cudaStreamWaitEvent(S->readback, ev, 0);
  }
  cudaError_t e = cudaSuccess;
  if (volume) e = cudaMemcpyAsync(volume, v, voxels * 8, cudaMemcpyDefault, S->readback);
  if (weight && e == cudaSuccess) e = cudaMemcpyAsync(weight, w, voxels * 4, cudaMemcpyDefault, S->readback);
  const cudaError_t es = cudaStreamSynchronize(S->readback);
  if (ev) cudaEventDestroy(ev);
  if (e != cudaSuccess || es != cudaSuccess) {
    cudaGetLastError();
    return fail(FR_E_CUDA, std::string("reading the job failed: ") + cudaGetErrorString(e != cudaSuccess ? e : es));
  }
  return FR_OK;
}

int fr_server_release_job(fr_server *S, uint64_t job)
{
  if (!S) return fail(FR_E_INVALID, "NULL argument");
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->jobs.find(job);
  // a job whose allocation is in flight is released once its admission has finished (looked
  // up again after the wait: another release of the same id may have come first)
  S->cv_wait.wait(lk, [&] {
    it = S->jobs.find(job);
    return it == S->jobs.end() || !it->second.admitting;
  });
  if (it == S->jobs.end()) return fail(FR_E_INVALID, "no such job");
  Job &J = it->second;
  if (J.state == FR_JOB_ACTIVE) return fail(FR_E_INVALID, "the job is still running");
  DeviceGuard guard(S->device);
  if (J.volume) {
    // stream-ordered: after every step that may still read or write it
    cudaFreeAsync(J.volume, S->compute);
    cudaFreeAsync(J.weight, S->compute);
    S->stats.bytes_admitted -= J.footprint;
  }
  S->queued.erase(std::remove(S->queued.begin(), S->queued.end(), job), S->queued.end());
  S->jobs.erase(it);
  admit(*S, lk);
  return FR_OK;
}

int fr_server_step_log(fr_server *S, fr_server_step_record *out, uint64_t capacity, uint64_t *count)
{
  if (!S || !count || (capacity && !out)) return fail(FR_E_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(S->mu);
  const size_t n = std::min<size_t>(capacity, S->step_log.size());
  const size_t first = S->step_log.size() - n;
  for (size_t i = 0; i < n; ++i) out[i] = S->step_log[first + i];
  *count = n;
  return FR_OK;
}

int fr_server_get_stats(fr_server *S, fr_server_stats *out)
{
  if (!S || !out) return fail(FR_E_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(S->mu);
  *out = S->stats;
  out->jobs_active = uint32_t(S->active.size());
  out->jobs_queued = uint32_t(S->queued.size());
  if (S->failed) return fail(FR_E_CUDA, "server failed: " + S->failure);
  return FR_OK;
}

}// extern "C"
