// Autotuner of the insertion launch parameters: the project's replacement for the reference's
// KTT tuning of FRCUDA.  KTT searches BLOCK_DIM / TILE / GRID_DIM_Z / SHARED_IMG on the first
// Execute of a strategy (fr_cuda.cpp:100-157, tunable_strategy.cpp:64-104) and the
// StrategyManager keeps the best configuration in one tuning file per strategy, named from the
// device and hashes of the strategy's payloads and settings (ktt_strategy_base.hpp:110-134,
// strategy_manager.cpp:14-83).  Here the search space is the engine's own launch shape --
// 256-thread groups per CTA x CTAs per SM x traverse spaces per work item -- every point that
// fits on an SM is timed with CUDA events on a sample of the caller's job, and the winner is
// written to a tuning file named by a hash of the strategy key.
#include <cuda_runtime.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <limits>
#include <sstream>
#include <string>
#include <vector>

#include "fr_device_guard.h"
#include "fr_engine.h"
#include "fr_handle.h"
#include "fr_kernels.h"
#include "umpalumpa_fr.h"

namespace {

int fail(int code, const std::string &msg) { return frb::set_last_error(code, msg.c_str()); }

// The item capacity also bounds how many contributions a brick accumulator sums in FP32 before
// the brick is added to the volume: at 20,000 the plain weights drift 4.4e-5 from FP64, so the
// search stops at 1,024 (2,048 also ran 3 % slower at box 256).
constexpr int kItemCaps[] = { 128, 256, 512, 1024 };
constexpr int kMaxCtasPerSm = 4;
constexpr uint64_t kSampleSpaces = 8192;        // single job: the first spaces of the job
constexpr uint64_t kBatchSampleSpaces = 16384;  // batch: spread over the jobs in proportion
constexpr int kRepeats = 3;                     // timed runs per candidate (the minimum counts)
constexpr double kKeepDefault = 0.98;           // a candidate must beat the default by 2%

uint64_t fnv1a(const std::string &s)
{
  uint64_t h = 1469598103934665603ull;
  for (unsigned char c : s) {
    h ^= c;
    h *= 1099511628211ull;
  }
  return h;
}

int size_class(uint64_t n)  // ceil(log2 n): jobs of one class share a tuning file
{
  int c = 0;
  while (c < 63 && (uint64_t(1) << c) < n) ++c;
  return c;
}

std::string strategy_key(const fr_handle *h)
{
  std::string dev = h->device_name;
  for (char &c : dev)
    if (c == ' ' || c == '=') c = '_';
  const fr_settings &s = h->settings;
  char buf[512];
  if (h->batch) {
    const fr_batch_limits &l = h->blim;
    std::snprintf(buf, sizeof buf,
      "fr-b200 device=%s sms=%d batch max_jobs=%llu max_spaces=%llu max_bricks=%llu max_side=%llu table=%llu",
      dev.c_str(), h->num_sms, (unsigned long long)l.max_jobs, (unsigned long long)l.max_spaces,
      (unsigned long long)l.max_bricks, (unsigned long long)l.max_volume_side, (unsigned long long)l.table_elems);
  } else {
    const fr_dims &d = h->dims;
    std::snprintf(buf, sizeof buf,
      "fr-b200 device=%s sms=%d single fft=%llux%llu volume=%llux%llux%llu table=%llu spaces_class=%d", dev.c_str(),
      h->num_sms, (unsigned long long)d.fft_x, (unsigned long long)d.fft_y, (unsigned long long)d.volume_x,
      (unsigned long long)d.volume_y, (unsigned long long)d.volume_z, (unsigned long long)d.table_elems,
      size_class(std::min<uint64_t>(d.n_spaces, 65536)));
  }
  char set[256];
  std::snprintf(set, sizeof set,
    " type=%d interpolation=%d order=%d alpha=%.9g radius=%.9g storage=%d accumulation=%d layout=%d", s.type,
    s.interpolation, s.blob_order, double(s.alpha), double(s.blob_radius), s.storage, s.accumulation, s.layout);
  return std::string(buf) + set;
}

std::string tuning_dir(const fr_handle *h)
{
  if (!h->tuning_dir.empty()) return h->tuning_dir;
  const char *e = std::getenv("UMPALUMPA_B200_TUNING_DIR");
  if (e && *e) return e;
  const char *home = std::getenv("HOME");
  return std::string(home && *home ? home : "/tmp") + "/.cache/umpalumpa_b200";
}

std::string tuning_path(const fr_handle *h, const std::string &key)
{
  char name[64];
  std::snprintf(name, sizeof name, "/fr-b200-%016llx.tune", (unsigned long long)fnv1a(key));
  return tuning_dir(h) + name;
}

bool make_dirs(const std::string &dir)
{
  for (size_t i = 1; i <= dir.size(); ++i) {
    if (i < dir.size() && dir[i] != '/') continue;
    const std::string part = dir.substr(0, i);
    if (::mkdir(part.c_str(), 0755) != 0 && errno != EEXIST) return false;
  }
  return true;
}

bool read_tuning_file(const std::string &path, const std::string &key, fr_launch_params *p)
{
  std::ifstream f(path);
  if (!f) return false;
  std::string line, k;
  int g = 0, c = 0, ic = 0;
  while (std::getline(f, line)) {
    if (line.rfind("key=", 0) == 0) k = line.substr(4);
    else if (line.rfind("groups=", 0) == 0) g = std::atoi(line.c_str() + 7);
    else if (line.rfind("ctas_per_sm=", 0) == 0) c = std::atoi(line.c_str() + 12);
    else if (line.rfind("item_capacity=", 0) == 0) ic = std::atoi(line.c_str() + 14);
  }
  if (k != key || g < 1 || c < 1 || ic < 1) return false;  // another strategy's file, or damaged
  *p = fr_launch_params{};
  p->brick = 16;
  p->groups = g;
  p->ctas_per_sm = c;
  p->item_capacity = ic;
  return true;
}

bool write_tuning_file(const std::string &path, const std::string &key, const fr_launch_params &p, double ms,
  double def_ms)
{
  const size_t slash = path.rfind('/');
  if (slash != std::string::npos && !make_dirs(path.substr(0, slash))) return false;
  const std::string tmp = path + ".tmp." + std::to_string(::getpid());
  {
    std::ofstream f(tmp);
    if (!f) return false;
    f << "key=" << key << "\n"
      << "groups=" << p.groups << "\n"
      << "ctas_per_sm=" << p.ctas_per_sm << "\n"
      << "item_capacity=" << p.item_capacity << "\n"
      << "best_ms=" << ms << "\n"
      << "default_ms=" << def_ms << "\n";
    if (!f) return false;
  }
  return std::rename(tmp.c_str(), path.c_str()) == 0;  // whole file or none
}

struct Candidate {
  int groups, ctas, item;
};

// Every launch shape of the handle's insertion kernel that fits on an SM, x the item sizes.
std::vector<Candidate> candidates(fr_handle *h, Candidate *def)
{
  std::vector<Candidate> out;
  frb::InsertConfig cfg = h->cfg;
  const int tableElems = int(h->batch ? h->blim.table_elems : h->dims.table_elems);
  const int maxg = frb::insert_max_groups(cfg);
  def->groups = maxg;
  def->ctas = 1;
  def->item = 512;
  for (int g = 1; g <= maxg; ++g) {
    cfg.groups = g;
    const size_t smem = frb::insert_smem_bytes(cfg, tableElems);
    const void *k = frb::insert_kernel_ptr(cfg);
    int occ = 0;
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess
        || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, 256 * g, smem) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    if (g == maxg) def->ctas = std::max(1, std::min(occ, kMaxCtasPerSm));
    for (int c = 1; c <= std::min(occ, kMaxCtasPerSm); ++c)
      for (int ic : kItemCaps) out.push_back({ g, c, ic });
  }
  return out;
}

bool same(const Candidate &a, const Candidate &b) { return a.groups == b.groups && a.ctas == b.ctas && a.item == b.item; }

// Times every candidate with `run` (one insertion of the sample, enqueued on the handle's
// stream) and applies the fastest.  `sync` waits for the handle and reports device errors.
template<class Run, class Sync>
int search(fr_handle *h, Run run, Sync sync, uint32_t sample, fr_tune_report *rep)
{
  Candidate def{};
  const std::vector<Candidate> cands = candidates(h, &def);
  if (cands.empty()) return fail(FR_E_UNSUPPORTED, "no launch shape of the insertion kernel fits on an SM");
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    if (e0) cudaEventDestroy(e0);
    return fail(FR_E_CUDA, "cudaEventCreate failed");
  }
  const fr_launch_params saved = h->launch;
  h->tuning_active = true;
  double best = std::numeric_limits<double>::infinity(), defMs = -1.0;
  Candidate bestC = def;
  uint32_t trials = 0;
  int rc = FR_OK;
  for (const Candidate &c : cands) {
    fr_launch_params p{};
    p.item_capacity = c.item;
    p.ctas_per_sm = c.ctas;
    p.groups = c.groups;
    if ((rc = fr_set_launch_params(h, &p)) != FR_OK) break;  // re-sizing failed: stop
    if (h->launch.ctas_per_sm != c.ctas || h->launch.groups != c.groups) continue;  // clamped: a duplicate
    if (run() != FR_OK || sync() != FR_OK) continue;  // warm-up; a failing shape is skipped
    float ms = std::numeric_limits<float>::infinity();
    bool ok = true;
    for (int r = 0; r < kRepeats && ok; ++r) {
      float t = 0.f;
      ok = cudaEventRecord(e0, h->stream) == cudaSuccess && run() == FR_OK
           && cudaEventRecord(e1, h->stream) == cudaSuccess && sync() == FR_OK
           && cudaEventElapsedTime(&t, e0, e1) == cudaSuccess;
      if (ok) ms = std::min(ms, t);
    }
    if (!ok) {
      cudaGetLastError();
      continue;
    }
    ++trials;
    if (same(c, def)) defMs = ms;
    if (ms < best) {
      best = ms;
      bestC = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc == FR_OK && trials == 0) rc = fail(FR_E_CUDA, "no launch shape ran the tuning sample");
  if (rc != FR_OK) {
    const std::string msg = fr_last_error();
    fr_set_launch_params(h, &saved);
    h->tuning_active = false;
    return fail(rc, "autotuning failed: " + msg);
  }
  if (defMs > 0 && best > kKeepDefault * defMs) {
    bestC = def;
    best = defMs;
  }
  fr_launch_params p{};
  p.item_capacity = bestC.item;
  p.ctas_per_sm = bestC.ctas;
  p.groups = bestC.groups;
  rc = fr_set_launch_params(h, &p);
  h->tuning_active = false;
  if (rc) return rc;
  h->tuned = true;
  const std::string key = strategy_key(h);
  if (h->tuning != FR_TUNING_OFF) write_tuning_file(tuning_path(h, key), key, h->launch, best, defMs);
  if (rep) {
    std::memset(rep, 0, sizeof(*rep));
    rep->best = h->launch;
    rep->best_ms = best;
    rep->default_ms = defMs;
    rep->trials = trials;
    rep->sample_spaces = sample;
    std::snprintf(rep->key, sizeof rep->key, "%s", key.c_str());
  }
  return FR_OK;
}

}// namespace

bool frb::tune_lookup(const fr_handle *h, fr_launch_params *out)
{
  const std::string key = strategy_key(h);
  return read_tuning_file(tuning_path(h, key), key, out);
}

int frb::tune_single(fr_handle *h, const void *fft, const float *scales, uint64_t nProj,
  const fr_traverse_space *spaces, uint64_t nSpaces, const float *table, fr_tune_report *rep)
{
  if (!h->initialized || h->batch) return fail(FR_E_NOT_INIT, "autotuning needs an initialised single-job handle");
  if (nSpaces == 0 || !spaces || !fft) return fail(FR_E_INVALID, "autotuning needs a job");
  const uint64_t sample = std::min<uint64_t>(nSpaces, kSampleSpaces);
  const size_t voxels = size_t(h->dims.volume_x) * h->dims.volume_y * h->dims.volume_z;
  void *vol = nullptr;
  frb::DeviceGuard guard(h->device);
  if (guard.err != cudaSuccess || cudaMalloc(&vol, voxels * 12) != cudaSuccess) {
    cudaGetLastError();
    return fail(FR_E_CUDA, "cannot allocate the tuning volume");
  }
  float *w = reinterpret_cast<float *>(static_cast<char *>(vol) + voxels * 8);
  cudaMemsetAsync(vol, 0, voxels * 12, h->stream);
  auto run = [&] { return fr_execute(h, fft, scales, nProj, vol, w, spaces, sample, table); };
  auto sync = [&] { return fr_synchronize(h); };
  const int rc = search(h, run, sync, uint32_t(sample), rep);
  cudaStreamSynchronize(h->stream);
  cudaFree(vol);
  return rc;
}

extern "C" {

int fr_set_tuning(fr_handle *h, int approach, const char *directory)
{
  if (!h) return fail(FR_E_INVALID, "handle is NULL");
  if (approach < FR_TUNING_OFF || approach > FR_TUNING_ON_EXECUTE) return fail(FR_E_INVALID, "unknown tuning approach");
  h->tuning = approach;
  h->tuning_dir = directory ? directory : "";
  h->tuned = false;
  if (h->initialized && approach != FR_TUNING_OFF) {
    fr_launch_params p{};
    if (frb::tune_lookup(h, &p)) return fr_set_launch_params(h, &p);  // re-init marks it tuned
  }
  return FR_OK;
}

int fr_autotune(fr_handle *h, const void *fft, const float *scales, uint64_t n_projections,
  const fr_traverse_space *spaces, uint64_t n_spaces, const float *table, fr_tune_report *report)
{
  if (!h) return fail(FR_E_INVALID, "handle is NULL");
  if (h->batch) return fail(FR_E_INVALID, "a batched handle is tuned with fr_batch_autotune");
  return frb::tune_single(h, fft, scales, n_projections, spaces, n_spaces, table, report);
}

int fr_batch_autotune(fr_handle *h, const fr_job *jobs, uint64_t n_jobs, const float *table, fr_tune_report *report)
{
  if (!h) return fail(FR_E_INVALID, "handle is NULL");
  if (!h->initialized || !h->batch) return fail(FR_E_NOT_INIT, "fr_batch_autotune needs a handle after fr_batch_init");
  if (!jobs || n_jobs == 0) return fail(FR_E_INVALID, "no jobs");
  if (n_jobs > h->blim.max_jobs) return fail(FR_E_MISMATCH, "more jobs than the batch limits");
  uint64_t total = 0;
  size_t bytes = 0;
  for (uint64_t j = 0; j < n_jobs; ++j) {
    total += jobs[j].n_spaces;
    const size_t v = size_t(jobs[j].volume_x) * jobs[j].volume_y * jobs[j].volume_z;
    bytes += ((v * 12) + 255) & ~size_t(255);
  }
  if (total == 0) return fail(FR_E_INVALID, "the jobs hold no traverse spaces");
  const uint64_t want = std::min<uint64_t>(total, kBatchSampleSpaces);
  void *scratch = nullptr;
  frb::DeviceGuard guard(h->device);
  if (guard.err != cudaSuccess || cudaMalloc(&scratch, bytes) != cudaSuccess) {
    cudaGetLastError();
    return fail(FR_E_CUDA, "cannot allocate the tuning volumes");
  }
  cudaMemsetAsync(scratch, 0, bytes, h->stream);
  std::vector<fr_job> sample(jobs, jobs + n_jobs);
  size_t off = 0;
  uint64_t taken = 0;
  for (fr_job &J : sample) {
    const size_t v = size_t(J.volume_x) * J.volume_y * J.volume_z;
    J.volume = static_cast<char *>(scratch) + off;
    J.weight = reinterpret_cast<float *>(static_cast<char *>(scratch) + off + v * 8);
    off += ((v * 12) + 255) & ~size_t(255);
    if (J.n_spaces) J.n_spaces = std::max<uint64_t>(1, J.n_spaces * want / total);
    taken += J.n_spaces;
  }
  auto run = [&] { return fr_batch_execute(h, sample.data(), sample.size(), table, 0); };
  auto sync = [&] { return fr_synchronize(h); };
  const int rc = search(h, run, sync, uint32_t(taken), report);
  cudaStreamSynchronize(h->stream);
  cudaFree(scratch);
  return rc;
}

int fr_tuning_key(const fr_handle *h, char *key, uint64_t key_bytes, char *path, uint64_t path_bytes)
{
  if (!h) return fail(FR_E_INVALID, "handle is NULL");
  if (!h->initialized) return fail(FR_E_NOT_INIT, "the strategy key needs an initialised handle");
  const std::string k = strategy_key(h);
  if (key && key_bytes) std::snprintf(key, size_t(key_bytes), "%s", k.c_str());
  if (path && path_bytes) std::snprintf(path, size_t(path_bytes), "%s", tuning_path(h, k).c_str());
  return FR_OK;
}

}// extern "C"
