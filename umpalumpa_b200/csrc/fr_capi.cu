// Host side of the B200 Fourier-reconstruction engine: the C-ABI declared in
// include/umpalumpa_fr.h.  Mirrors the reference operation's contract
// (libumpalumpa/operations/basic_operation.hpp:28-105, afr.hpp:35-55, fr_cuda.cpp:71-244).
#include <cuda_runtime.h>

#include "fr_device.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <array>
#include <cstring>
#include <map>
#include <new>
#include <numeric>
#include <string>
#include <vector>

#include "fr_device_guard.h"
#include "fr_engine.h"
#include "fr_handle.h"
#include "fr_kernels.h"
#include "umpalumpa_fr.h"

namespace {

thread_local std::string g_error;

int fail(int code, const std::string &msg)
{
  g_error = msg;
  return code;
}

#define FR_CUDA(call)                                                                       \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      return fail(FR_E_CUDA, std::string(#call) + " failed: " + cudaGetErrorString(e_));    \
  } while (0)

// ---- host blob math (the reference computes the constants on the host) ----------------
// Modified Bessel I0/I1 by Abramowitz & Stegun 9.8.1-9.8.4 in double, I2..I4 by upward
// recurrence (libumpalumpa/math/bessier.hpp:9-107).
double i0_host(double x)
{
  double ax = std::fabs(x);
  if (ax < 3.75) {
    double t = x / 3.75;
    t *= t;
    return 1.0
           + t * (3.5156229
                  + t * (3.0899424
                         + t * (1.2067492 + t * (0.2659732 + t * (0.360768e-1 + t * 0.45813e-2)))));
  }
  double t = 3.75 / ax;
  return (std::exp(ax) / std::sqrt(ax))
         * (0.39894228
            + t * (0.1328592e-1
                   + t * (0.225319e-2
                          + t * (-0.157565e-2
                                 + t * (0.916281e-2
                                        + t * (-0.2057706e-1
                                               + t * (0.2635537e-1
                                                      + t * (-0.1647633e-1 + t * 0.392377e-2))))))));
}

double i1_host(double x)
{
  double ax = std::fabs(x), r;
  if (ax < 3.75) {
    double t = x / 3.75;
    t *= t;
    r = ax
        * (0.5
           + t * (0.87890594
                  + t * (0.51498869
                         + t * (0.15084934 + t * (0.2658733e-1 + t * (0.301532e-2 + t * 0.32411e-3))))));
  } else {
    double t = 3.75 / ax;
    r = 0.2282967e-1 + t * (-0.2895312e-1 + t * (0.1787654e-1 - t * 0.420059e-2));
    r = 0.39894228
        + t * (-0.3988024e-1 + t * (-0.362018e-2 + t * (0.163801e-2 + t * (-0.1031555e-1 + t * r))));
    r *= std::exp(ax) / std::sqrt(ax);
  }
  return x < 0.0 ? -r : r;
}

double in_host(int order, double x)
{
  if (order == 0) return i0_host(x);
  if (order == 1) return i1_host(x);
  if (order < 0 || order > 4) return NAN;
  if (x == 0) return 0;
  double im1 = i0_host(x), i = i1_host(x);
  for (int k = 1; k < order; ++k) {
    double nx = im1 - ((2.0 * k) / x) * i;
    im1 = i;
    i = nx;
  }
  return i;
}

const float kPiF = 3.14159265358979323846f;

// Fourier transform of the blob at frequency 0, defined for order 0 only (math/kaiser.hpp:66-81).
float kaiser_fourier_value0(float radius, float alpha, int order)
{
  const float freq = 0.f;
  float sigma = std::sqrt(
    std::fabs(alpha * alpha - (2.f * kPiF * radius * freq) * (2.f * kPiF * radius * freq)));
  if (order == 0 && 2 * kPiF * radius * freq <= alpha) {
    float i15 = (sigma == 0)
                  ? 0.f
                  : std::sqrt(2.f / (kPiF * sigma)) * (std::cosh(sigma) - std::sinh(sigma) / sigma);
    return std::pow(2.f * kPiF, 1.5f) * std::pow(radius, 3.f) * i15
           / (static_cast<float>(i0_host(alpha)) * std::pow(sigma, 1.5f));
  }
  return NAN;
}

fr_constants make_constants(uint64_t vx, uint64_t vy, uint64_t tableElems, const fr_settings &s)
{
  fr_constants c;
  c.cMaxVolumeIndexX = int32_t(vx - 1);
  c.cMaxVolumeIndexYZ = int32_t(vy - 1);
  c.cBlobRadius = s.blob_radius;
  c.cOneOverBlobRadiusSqr = 1.f / (s.blob_radius * s.blob_radius);
  c.cBlobAlpha = s.alpha;
  c.cIw0 = 1.f / kaiser_fourier_value0(s.blob_radius, s.alpha, s.blob_order);
  c.cIDeltaSqrt = float(tableElems - 1) / (s.blob_radius * s.blob_radius);
  c.cOneOverBessiOrderAlpha = 1 / static_cast<float>(in_host(s.blob_order, s.alpha));
  return c;
}

// The insertion kernel's table: the caller's blob table (lookup interpolation, `lookupElems`
// entries) or the handle's Kaiser (value, slope) table (dynamic interpolation).
static void set_table(frb::InsertParams &P, const fr_handle *h, const float *table, uint64_t lookupElems)
{
  const fr_settings &s = h->settings;
  P.table = table;
  P.tableElems = 0;
  P.tableScale = 0.f;
  if (s.interpolation == FR_INTERPOLATION_LOOKUP) {
    P.tableElems = int(lookupElems);
  } else if (h->kaiser_table) {
    P.table = h->kaiser_table;
    P.tableElems = frb::kKaiserTableElems;
    P.tableScale = float(frb::kKaiserTableElems - 1) / (s.blob_radius * s.blob_radius);
  }
}

int check_settings(const fr_settings *s)
{
  if (!s) return fail(FR_E_INVALID, "settings is NULL");
  if (s->interpolation != FR_INTERPOLATION_DYNAMIC && s->interpolation != FR_INTERPOLATION_LOOKUP)
    return fail(FR_E_INVALID, "unknown interpolation");
  if (s->type != FR_TYPE_FAST && s->type != FR_TYPE_PRECISE) return fail(FR_E_INVALID, "unknown type");
  if (s->blob_order < 0 || s->blob_order > 4) return fail(FR_E_INVALID, "blob order must be 0..4");
  if (!(s->blob_radius > 0.f)) return fail(FR_E_INVALID, "blob radius must be positive");
  if (s->blob_radius >= 4.f)
    return fail(FR_E_UNSUPPORTED, "blob radius must be < 4 voxels (blob footprint of at most 8x8 pixels)");
  if (s->storage < FR_STORAGE_FP32 || s->storage > FR_STORAGE_FP16) return fail(FR_E_INVALID, "unknown storage");
  if (s->accumulation != FR_ACCUM_PLAIN && s->accumulation != FR_ACCUM_KAHAN)
    return fail(FR_E_INVALID, "unknown accumulation");
  if (s->layout < FR_LAYOUT_AUTO || s->layout > FR_LAYOUT_BANDED) return fail(FR_E_INVALID, "unknown layout");
  return FR_OK;
}

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

bool is_host_pointer(const void *p)
{
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return true;
  }
  return a.type == cudaMemoryTypeHost || a.type == cudaMemoryTypeUnregistered;
}

}// namespace

int frb::set_last_error(int code, const char *msg) { return fail(code, msg); }

// Under FR_TUNING_CACHED / ON_EXECUTE, takes the launch parameters of an equal strategy's
// tuning file (fr_init / fr_batch_init, after the dims or limits and settings are set).
static void apply_tuning_file(fr_handle *h)
{
  h->tuned = false;
  if (h->tuning == FR_TUNING_OFF || h->tuning_active) return;
  fr_launch_params p{};
  if (!frb::tune_lookup(h, &p)) return;
  h->launch.item_capacity = p.item_capacity;
  h->launch.ctas_per_sm = p.ctas_per_sm;
  h->launch.groups = p.groups;
  h->tuned = true;
}

int frb::batch_device_status(const fr_handle *h) { return h && h->host_status ? h->host_status[0] : FR_E_INVALID; }

static cudaEvent_t next_event(fr_handle *h, int &idx)
{
  if (h->ev_next == h->ev_pool.size()) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    h->ev_pool.push_back(e);
  }
  idx = int(h->ev_next++);
  return h->ev_pool[idx];
}

// Folds the recorded event pairs into h->times (call after the stream is idle).
static void collect_times(fr_handle *h)
{
  float ms = 0.f;
  for (auto &p : h->ev_bin)
    if (cudaEventElapsedTime(&ms, h->ev_pool[p.first], h->ev_pool[p.second]) == cudaSuccess) h->times.binning_ms += ms;
  for (size_t i = 0; i < h->ev_ins.size(); ++i) {
    auto &p = h->ev_ins[i];
    if (cudaEventElapsedTime(&ms, h->ev_pool[p.first], h->ev_pool[p.second]) == cudaSuccess) {
      h->times.insert_ms += ms;
      h->times.insert_launches += 1;
      h->times.insert_spaces += h->ins_spaces[i];
    }
  }
  h->ev_bin.clear();
  h->ev_ins.clear();
  h->ins_spaces.clear();
  h->ev_next = 0;
}

extern "C" {

void fr_settings_default(fr_settings *s)
{
  if (!s) return;
  s->interpolation = FR_INTERPOLATION_DYNAMIC;
  s->blob_order = 0;
  s->type = FR_TYPE_FAST;
  s->alpha = 15.f;
  s->blob_radius = 1.9f;
  s->max_resolution = 0.5f;
  s->storage = FR_STORAGE_FP32;
  s->accumulation = FR_ACCUM_PLAIN;
  s->layout = FR_LAYOUT_AUTO;
}

const char *fr_last_error(void) { return g_error.c_str(); }

int fr_create(int device, void *stream, fr_handle **out)
{
  if (!out) return fail(FR_E_INVALID, "out is NULL");
  *out = nullptr;
  int n = 0;
  FR_CUDA(cudaGetDeviceCount(&n));
  if (device < 0 || device >= n) return fail(FR_E_INVALID, "no such CUDA device");
  frb::DeviceGuard guard(device);
  FR_CUDA(guard.err);
  fr_handle *h = new (std::nothrow) fr_handle();
  if (!h) return fail(FR_E_INVALID, "out of host memory");
  h->device = device;
  h->stream = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) {
    cudaDeviceProp prop;
    e = cudaGetDeviceProperties(&prop, device);
    if (e == cudaSuccess) h->device_name = prop.name;
  }
  if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void **>(&h->host_status), 64, cudaHostAllocDefault);
  if (e == cudaSuccess)
    e = cudaHostAlloc(reinterpret_cast<void **>(&h->host_stats), 4 * sizeof(unsigned long long), cudaHostAllocDefault);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->band_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->band_fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->band_join, cudaEventDisableTiming);
  for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
    e = cudaEventCreateWithFlags(&h->slots[k].ready, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->slots[k].free, cudaEventDisableTiming);
  }
  if (e != cudaSuccess) {
    if (h->host_status) cudaFreeHost(h->host_status);
    if (h->host_stats) cudaFreeHost(h->host_stats);
    for (auto &sl : h->slots) {
      if (sl.ready) cudaEventDestroy(sl.ready);
      if (sl.free) cudaEventDestroy(sl.free);
    }
    if (h->band_fork) cudaEventDestroy(h->band_fork);
    if (h->band_join) cudaEventDestroy(h->band_join);
    if (h->band_stream) cudaStreamDestroy(h->band_stream);
    if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
    delete h;
    return fail(FR_E_CUDA, std::string("fr_create: ") + cudaGetErrorString(e));
  }
  *out = h;
  return FR_OK;
}

int fr_cleanup(fr_handle *h)
{
  if (!h) return fail(FR_E_INVALID, "handle is NULL");
  frb::DeviceGuard guard(h->device);
  if (h->scratch || h->band) {
    cudaStreamSynchronize(h->stream);
    if (h->band_stream) cudaStreamSynchronize(h->band_stream);
  }
  if (h->scratch) cudaFree(h->scratch);
  if (h->band) cudaFree(h->band);
  h->band = nullptr;
  h->band_bytes = 0;
  h->band_refused = 0;
  h->scratch = nullptr;
  h->scratch_bytes = 0;
  h->kaiser_table = nullptr;
  h->initialized = false;
  if (h->graph) cudaGraphExecDestroy(h->graph);
  h->graph = nullptr;
  h->graph_sig.clear();
  for (int k = 0; k < 2; ++k) {
    if (h->h_jobs_set[k]) cudaFreeHost(h->h_jobs_set[k]);
    if (h->h_order_set[k]) cudaFreeHost(h->h_order_set[k]);
    if (h->upload_set_done[k]) cudaEventDestroy(h->upload_set_done[k]);
    h->h_jobs_set[k] = nullptr;
    h->h_order_set[k] = nullptr;
    h->upload_set_done[k] = nullptr;
  }
  h->upload_set = 0;
  h->h_jobs = nullptr;
  h->h_order = nullptr;
  h->upload_done = nullptr;
  h->d_jobs = nullptr;
  h->batch = false;
  return FR_OK;
}

int fr_destroy(fr_handle *h)
{
  if (!h) return FR_OK;
  fr_cleanup(h);
  frb::DeviceGuard guard(h->device);
  if (h->copy_stream) cudaStreamSynchronize(h->copy_stream);
  for (auto &sl : h->slots) {
    if (sl.buf) cudaFree(sl.buf);
    if (sl.ready) cudaEventDestroy(sl.ready);
    if (sl.free) cudaEventDestroy(sl.free);
  }
  for (auto e : h->ev_pool) cudaEventDestroy(e);
  if (h->band_fork) cudaEventDestroy(h->band_fork);
  if (h->band_join) cudaEventDestroy(h->band_join);
  if (h->band_stream) cudaStreamDestroy(h->band_stream);
  if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
  if (h->host_status) cudaFreeHost(h->host_status);
  if (h->host_stats) cudaFreeHost(h->host_stats);
  delete h;
  return FR_OK;
}

int fr_make_constants(const fr_dims *d, const fr_settings *s, fr_constants *out)
{
  if (!d || !out) return fail(FR_E_INVALID, "NULL argument");
  int rc = check_settings(s);
  if (rc) return rc;
  *out = make_constants(d->volume_x, d->volume_y,
    s->interpolation == FR_INTERPOLATION_LOOKUP ? d->table_elems : 0, *s);
  return FR_OK;
}

int fr_init(fr_handle *h, const fr_dims *d, const fr_settings *s)
{
  if (!h) return fail(FR_E_INVALID, "handle is NULL");
  fr_cleanup(h);
  if (!d) return fail(FR_E_INVALID, "dims is NULL");
  int rc = check_settings(s);
  if (rc) return rc;
  // AFR::IsValid (afr.hpp:47-54) + Size validity (size.hpp:42): all payloads non-degenerate.
  if (d->fft_x < 1 || d->fft_y < 2 || d->n_projections < 1 || d->n_spaces < 1)
    return fail(FR_E_INVALID, "FFT and traverse-space payloads must be non-empty");
  if (d->volume_x < 2 || d->volume_y < 2 || d->volume_z < 2)
    return fail(FR_E_INVALID, "volume must be 3D");
  if (d->volume_x % 2 == 0)
    return fail(FR_E_UNSUPPORTED, "volume x size must be odd (fr_cuda.cpp:75)");
  if (d->volume_y != d->volume_z)
    return fail(FR_E_UNSUPPORTED, "volume y and z sizes must match (one cMaxVolumeIndexYZ)");
  // The reference centres the slab planes at maxIndex/2.f and the voxels at maxIndex/2; the
  // two agree only for odd sizes, which is what the reference's own callers produce (B+1).
  if (d->volume_y % 2 == 0)
    return fail(FR_E_UNSUPPORTED, "volume y and z sizes must be odd");
  if (d->volume_x > (1u << 14) || d->volume_y > (1u << 14) || d->fft_x > (1u << 20) || d->fft_y > (1u << 20))
    return fail(FR_E_UNSUPPORTED, "payload dimension too large");
  if (s->interpolation == FR_INTERPOLATION_LOOKUP && (d->table_elems < 2 || d->table_elems > (1u << 26)))
    return fail(FR_E_NO_TABLE, "lookup interpolation needs a blob table of at least 2 entries");

  frb::DeviceGuard guard(h->device);
  FR_CUDA(guard.err);
  h->dims = *d;
  h->settings = *s;
  h->constants = make_constants(d->volume_x, d->volume_y,
    s->interpolation == FR_INTERPOLATION_LOOKUP ? d->table_elems : 0, *s);

  frb::BinGeom &g = h->geom;
  g.vx = int(d->volume_x);
  g.vy = int(d->volume_y);
  g.vz = int(d->volume_z);
  g.nbx = (g.vx + 15) / 16;
  g.nby = (g.vy + 15) / 16;
  g.nbz = (g.vz + 15) / 16;
  g.n_bricks = g.nbx * g.nby * g.nbz;
  g.cx = h->constants.cMaxVolumeIndexX / 2;
  g.cy = h->constants.cMaxVolumeIndexYZ / 2;
  g.cz = h->constants.cMaxVolumeIndexYZ / 2;

  frb::InsertConfig &cfg = h->cfg;
  cfg.fast = s->type == FR_TYPE_FAST;
  cfg.mode = s->interpolation == FR_INTERPOLATION_LOOKUP ? 0 : (s->alpha <= 15.f ? 1 : 3);
  int taps = int(std::floor(2.f * s->blob_radius)) + 1;
  cfg.taps = taps <= 4 ? 4 : 8;  // the kernel's blob window: 4x4 for r < 2, 8x8 for r < 4
  cfg.storage = s->storage;
  cfg.kahan = s->accumulation == FR_ACCUM_KAHAN;
  cfg.jobs = false;
  cfg.banded = s->layout != FR_LAYOUT_ROWS;  // fr_execute settles it per call
  apply_tuning_file(h);
  cfg.groups = h->launch.groups;
  h->launch.groups = frb::insert_groups(cfg);

  if (h->launch.item_capacity <= 0) h->launch.item_capacity = 512;
  h->launch.brick = 16;
  size_t smem = frb::insert_smem_bytes(cfg, int(d->table_elems));
  int occ = 0;
  FR_CUDA(cudaFuncSetAttribute(frb::insert_kernel_ptr(cfg), cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  FR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, frb::insert_kernel_ptr(cfg), 256 * frb::insert_groups(cfg), smem));
  if (occ < 1) return fail(FR_E_UNSUPPORTED, "insertion kernel does not fit on an SM");
  if (h->launch.ctas_per_sm <= 0 || h->launch.ctas_per_sm > occ) h->launch.ctas_per_sm = occ;
  h->grid = h->num_sms * h->launch.ctas_per_sm;

  // Capacity of the (brick, space) list.  For a space whose normal is dominated by axis w,
  // every brick it can touch lies in one of the nb_u x nb_v brick columns along w, and
  // within one column the slab (half-width hw) spans at most
  // L = 2 (b - 1) + 2 hw sqrt(3) voxels of w, i.e. at most ceil(L / b) + 2 bricks.
  const double hw = cfg.fast ? 2.5 : double(s->blob_radius) + 1e-3;
  const int perCol = int(std::ceil((2.0 * 15.0 + 2.0 * hw * std::sqrt(3.0)) / 16.0)) + 2;
  const int64_t cols = std::max({ int64_t(g.nbx) * g.nby, int64_t(g.nbx) * g.nbz, int64_t(g.nby) * g.nbz });
  const int64_t perSpace = std::min<int64_t>(g.n_bricks, cols * perCol);
  h->chunk_cap = std::min<int64_t>(int64_t(d->n_spaces), 65536);
  while (h->chunk_cap > 1 && h->chunk_cap * perSpace > (int64_t(1) << 30)) h->chunk_cap /= 2;
  const int64_t listCap = h->chunk_cap * perSpace;
  const int64_t itemsCap = listCap / h->launch.item_capacity + g.n_bricks + 1;

  // Brick visiting order: nearest to the volume centre first (they carry the most slabs).
  std::vector<int> order(g.n_bricks);
  std::iota(order.begin(), order.end(), 0);
  std::vector<double> dist(g.n_bricks);
  for (int b = 0; b < g.n_bricks; ++b) {
    int bx = b % g.nbx, by = (b / g.nbx) % g.nby, bz = b / (g.nbx * g.nby);
    double x = bx * 16 + 7.5 - g.cx, y = by * 16 + 7.5 - g.cy, z = bz * 16 + 7.5 - g.cz;
    dist[b] = x * x + y * y + z * z;
  }
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return dist[a] < dist[b]; });

  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += align256(bytes);
    return o;
  };
  const size_t oPrep = take(size_t(h->chunk_cap) * frb::kSpacePrepBytes);
  const size_t oRec = take(size_t(h->chunk_cap) * frb::kSpaceRecBytes);
  const size_t oCounts = take(size_t(3) * g.n_bricks * sizeof(int));
  const size_t oOffsets = take((size_t(3) * g.n_bricks + 1) * sizeof(int));
  const size_t oList = take(size_t(listCap) * sizeof(int));
  const size_t oOrder = take(size_t(g.n_bricks) * sizeof(int));
  const size_t oItems = take(size_t(itemsCap) * frb::kWorkItemBytes);
  const size_t oMisc = take(64);
  const size_t oStats = take(4 * sizeof(unsigned long long));
  const size_t oKaiser = take(cfg.mode == 3 && !cfg.fast ? size_t(frb::kKaiserTableElems) * sizeof(float2) : 0);
  FR_CUDA(cudaMalloc(&h->scratch, off));
  h->scratch_bytes = off;
  char *base = static_cast<char *>(h->scratch);
  frb::BinBuffers &bb = h->bb;
  bb.prep = reinterpret_cast<frb::SpacePrep *>(base + oPrep);
  bb.rec = reinterpret_cast<frb::SpaceRec *>(base + oRec);
  bb.counts = reinterpret_cast<int *>(base + oCounts);
  bb.offsets = reinterpret_cast<int *>(base + oOffsets);
  bb.list = reinterpret_cast<int *>(base + oList);
  bb.order = reinterpret_cast<const int *>(base + oOrder);
  bb.items = reinterpret_cast<frb::WorkItem *>(base + oItems);
  int *misc = reinterpret_cast<int *>(base + oMisc);
  bb.nItems = misc;
  bb.status = misc + 1;
  h->work_counter = misc + 2;
  bb.stats = reinterpret_cast<unsigned long long *>(base + oStats);
  bb.listCap = listCap;
  bb.itemsCap = itemsCap;
  FR_CUDA(cudaMemcpyAsync(base + oOrder, order.data(), order.size() * sizeof(int), cudaMemcpyHostToDevice, h->stream));
  FR_CUDA(cudaMemsetAsync(misc, 0, 64, h->stream));
  FR_CUDA(cudaMemsetAsync(bb.stats, 0, 4 * sizeof(unsigned long long), h->stream));
  h->kaiser_table = nullptr;
  if (cfg.mode == 3 && !cfg.fast) {
    h->kaiser_table = reinterpret_cast<float *>(base + oKaiser);
    FR_CUDA(frb::launch_kaiser_table(h->kaiser_table, s->blob_order, s->alpha, s->blob_radius, h->constants.cIw0,
      h->stream));
  }
  FR_CUDA(cudaStreamSynchronize(h->stream));
  h->initialized = true;
  return FR_OK;
}

uint64_t fr_used_bytes(const fr_handle *h)
{
  return h ? uint64_t(h->scratch_bytes + h->slots[0].bytes + h->slots[1].bytes + h->band_bytes) : 0;
}

int fr_get_launch_params(const fr_handle *h, fr_launch_params *out)
{
  if (!h || !out) return fail(FR_E_INVALID, "NULL argument");
  *out = h->launch;
  return FR_OK;
}

int fr_set_launch_params(fr_handle *h, const fr_launch_params *p)
{
  if (!h || !p) return fail(FR_E_INVALID, "NULL argument");
  if (p->item_capacity < 0 || p->ctas_per_sm < 0 || p->groups < 0) return fail(FR_E_INVALID, "negative launch parameter");
  if (p->item_capacity > (1 << 20)) return fail(FR_E_UNSUPPORTED, "item_capacity above 2^20");
  if (p->item_capacity > 0) h->launch.item_capacity = p->item_capacity;
  if (p->ctas_per_sm > 0) h->launch.ctas_per_sm = p->ctas_per_sm;
  if (p->groups > 0) h->launch.groups = p->groups;
  if (h->initialized) {
    // re-size the scratch so the item buffer and grid follow the new parameters
    fr_settings s = h->settings;
    if (h->batch) {
      fr_batch_limits lim = h->blim;
      return fr_batch_init(h, &lim, &s);
    }
    fr_dims d = h->dims;
    return fr_init(h, &d, &s);
  }
  return FR_OK;
}

int fr_get_exec_stats(const fr_handle *h, fr_exec_stats *out)
{
  if (!h || !out) return fail(FR_E_INVALID, "NULL argument");
  *out = h->last;
  return FR_OK;
}

// A band buffer of at least `bytes` in h->band.  Under FR_LAYOUT_AUTO (`optional`) the copy
// is made only while it takes at most half of the device memory still free, and a size that
// could not be had is not tried again; a batch (not optional) fails without it.
static int ensure_band(fr_handle *h, size_t bytes, bool optional, bool &ok)
{
  ok = false;
  if (h->band_bytes >= bytes) {
    ok = true;
    return FR_OK;
  }
  if (optional && h->band_refused && bytes >= h->band_refused) return FR_OK;
  if (h->band) {  // the previous copy may still be read
    FR_CUDA(cudaStreamSynchronize(h->stream));
    FR_CUDA(cudaStreamSynchronize(h->band_stream));
    FR_CUDA(cudaFree(h->band));
    h->band = nullptr;
    h->band_bytes = 0;
  }
  size_t freeB = 0, totalB = 0;
  FR_CUDA(cudaMemGetInfo(&freeB, &totalB));
  if (optional && bytes > freeB / 2) {
    h->band_refused = bytes;
    return FR_OK;
  }
  if (cudaMalloc(&h->band, bytes) != cudaSuccess) {
    cudaGetLastError();
    h->band = nullptr;
    if (optional) {
      h->band_refused = bytes;
      return FR_OK;
    }
    return fail(FR_E_CUDA, "out of device memory for the banded copy of the projections");
  }
  h->band_bytes = bytes;
  ok = true;
  return FR_OK;
}

int fr_execute(fr_handle *h, const void *fft, const float *scales, uint64_t nProj, void *volume,
  float *weight, const fr_traverse_space *spaces, uint64_t nSpaces, const float *table)
{
  if (!h) return fail(FR_E_INVALID, "handle is NULL");
  if (!h->initialized || h->batch) return fail(FR_E_NOT_INIT, "Execute before a successful Init");
  // Payload::IsEquivalentTo (payload.hpp:60-63): same sizes, count <= the Init count.
  if (nProj > h->dims.n_projections || nSpaces > h->dims.n_spaces)
    return fail(FR_E_MISMATCH, "payload count exceeds the Init reference");
  // FRCUDA Strategy1::Execute (fr_cuda.cpp:165-167): FFT, volume and weight must be non-empty.
  if (!fft || !volume || !weight || nProj == 0) return fail(FR_E_INVALID, "empty payload");
  const fr_settings &s = h->settings;
  if (s.interpolation == FR_INTERPOLATION_LOOKUP && !table)
    return fail(FR_E_NO_TABLE, "lookup interpolation with an empty blob table");
  if (s.storage != FR_STORAGE_FP32 && !scales)
    return fail(FR_E_INVALID, "16-bit storage needs per-projection scales");
  if (nSpaces == 0) return FR_OK;  // nothing to insert
  if (!spaces) return fail(FR_E_INVALID, "empty traverse-space payload");
  frb::DeviceGuard guard(h->device);
  FR_CUDA(guard.err);
  if (is_host_pointer(volume) || is_host_pointer(weight))
    return fail(FR_E_INVALID, "volume and weight must be device or managed memory");
  // KTT's first-Execute tuning (tunable_strategy.cpp:64-81): search once, on these inputs
  if (h->tuning == FR_TUNING_ON_EXECUTE && !h->tuned && !h->tuning_active) {
    const int rc = frb::tune_single(h, fft, scales, nProj, spaces, nSpaces, table, nullptr);
    if (rc) return rc;
  }

  // Host-resident inputs are uploaded into a staging slot on the copy stream.
  const size_t elem = s.storage == FR_STORAGE_FP32 ? 8 : 4;
  const int fx = int(h->dims.fft_x), fy = int(h->dims.fft_y);
  const size_t bandPlaneBytes = size_t(frb::band_plane_elems(fx, fy)) * elem;
  const size_t fftBytes = size_t(nProj) * (s.layout == FR_LAYOUT_BANDED ? bandPlaneBytes : size_t(fx) * fy * elem);
  const bool hostFft = is_host_pointer(fft);
  const bool hostSp = is_host_pointer(spaces);
  const bool hostSc = s.storage != FR_STORAGE_FP32 && is_host_pointer(scales);
  const bool hostTab = s.interpolation == FR_INTERPOLATION_LOOKUP && is_host_pointer(table);
  size_t need = 0, oF = 0, oS = 0, oC = 0, oT = 0;
  if (hostFft) { oF = need; need += align256(fftBytes); }
  if (hostSp) { oS = need; need += align256(size_t(nSpaces) * sizeof(fr_traverse_space)); }
  if (hostSc) { oC = need; need += align256(size_t(nProj) * sizeof(float)); }
  if (hostTab) { oT = need; need += align256(size_t(h->dims.table_elems) * sizeof(float)); }
  StageSlot *slot = nullptr;
  if (need) {
    slot = &h->slots[h->next_slot];
    h->next_slot ^= 1;
    if (slot->bytes < need) {
      if (slot->buf) {
        FR_CUDA(cudaEventSynchronize(slot->free));
        FR_CUDA(cudaFree(slot->buf));
        slot->buf = nullptr;
        slot->bytes = 0;
      }
      FR_CUDA(cudaMalloc(&slot->buf, need));
      slot->bytes = need;
    }
    if (slot->used) FR_CUDA(cudaStreamWaitEvent(h->copy_stream, slot->free, 0));
    char *st = static_cast<char *>(slot->buf);
    auto up = [&](size_t o, const void *src, size_t bytes) {
      return cudaMemcpyAsync(st + o, src, bytes, cudaMemcpyHostToDevice, h->copy_stream);
    };
    if (hostFft) {
      FR_CUDA(up(oF, fft, fftBytes));
      fft = st + oF;
    }
    if (hostSp) {
      FR_CUDA(up(oS, spaces, size_t(nSpaces) * sizeof(fr_traverse_space)));
      spaces = reinterpret_cast<const fr_traverse_space *>(st + oS);
    }
    if (hostSc) {
      FR_CUDA(up(oC, scales, size_t(nProj) * sizeof(float)));
      scales = reinterpret_cast<const float *>(st + oC);
    }
    if (hostTab) {
      FR_CUDA(up(oT, table, size_t(h->dims.table_elems) * sizeof(float)));
      table = reinterpret_cast<const float *>(st + oT);
    }
    FR_CUDA(cudaEventRecord(slot->ready, h->copy_stream));
    FR_CUDA(cudaStreamWaitEvent(h->stream, slot->ready, 0));
  }

  // FR_LAYOUT_AUTO: the projections are copied into bands on the band stream, beside the
  // binning on the compute stream; the insertion waits for both.
  // A call that inserts few spaces of a large payload reads the rows in place: the copy (about
  // 0.1 us per box-256 projection) pays for itself from about one space per three projections.
  bool banded = s.layout == FR_LAYOUT_BANDED, bandCopy = false;
  if (s.layout == FR_LAYOUT_AUTO && nSpaces * 3 >= nProj) {
    int rc = ensure_band(h, size_t(nProj) * bandPlaneBytes, true, bandCopy);
    if (rc) return rc;
    if (bandCopy) {
      FR_CUDA(cudaEventRecord(h->band_fork, h->stream));
      FR_CUDA(cudaStreamWaitEvent(h->band_stream, h->band_fork, 0));
      FR_CUDA(frb::launch_band_projections(fft, h->band, int64_t(nProj), fx, fy, int(elem), h->band_stream));
      FR_CUDA(cudaEventRecord(h->band_join, h->band_stream));
      fft = h->band;
      banded = true;
    }
  }
  h->cfg.banded = banded;

  frb::InsertParams P{};
  P.volume = volume;
  P.weight = weight;
  P.fft = fft;
  P.scales = scales;
  P.recs = h->bb.rec;
  P.list = h->bb.list;
  P.offsets = h->bb.offsets;
  P.items = h->bb.items;
  P.nItems = h->bb.nItems;
  P.workCounter = h->work_counter;
  set_table(P, h, table, h->dims.table_elems);
  P.lutInSmem = frb::insert_lut_in_smem(h->cfg, P.tableElems);
  P.genericTaps = int(h->dims.fft_x) < h->cfg.taps || int(h->dims.fft_y) < h->cfg.taps || P.tableElems > frb::kLutSmemMax;
  P.c = h->constants;
  P.order = s.blob_order;
  P.nProj = int(nProj);
  P.fftX = int(h->dims.fft_x);
  P.fftY = int(h->dims.fft_y);
  P.bandStride = banded ? frb::band_stride(P.fftX) : 0;
  P.vx = h->geom.vx;
  P.vy = h->geom.vy;
  P.vz = h->geom.vz;
  P.nbx = h->geom.nbx;
  P.nby = h->geom.nby;
  P.nbz = h->geom.nbz;
  P.cx = h->geom.cx;
  P.cy = h->geom.cy;
  P.cz = h->geom.cz;

  uint64_t launches = 0;
  FR_CUDA(cudaMemsetAsync(h->bb.stats, 0, 4 * sizeof(unsigned long long), h->stream));
  for (uint64_t s0 = 0; s0 < nSpaces; s0 += uint64_t(h->chunk_cap)) {
    const int n = int(std::min<uint64_t>(uint64_t(h->chunk_cap), nSpaces - s0));
    int e0 = -1, e1 = -1, e2 = -1;
    if (h->profiling) FR_CUDA(cudaEventRecord(next_event(h, e0), h->stream));
    FR_CUDA(frb::launch_binning(h->geom, spaces + s0, n, int(nProj), h->cfg.fast, s.blob_radius, h->bb,
      h->launch.item_capacity, h->stream));
    FR_CUDA(cudaMemsetAsync(h->work_counter, 0, sizeof(int), h->stream));
    if (bandCopy && s0 == 0) FR_CUDA(cudaStreamWaitEvent(h->stream, h->band_join, 0));
    if (h->profiling) FR_CUDA(cudaEventRecord(next_event(h, e1), h->stream));
    FR_CUDA(frb::launch_insert(P, h->cfg, h->grid, h->stream));
    if (h->profiling) {
      FR_CUDA(cudaEventRecord(next_event(h, e2), h->stream));
      h->ev_bin.emplace_back(e0, e1);
      h->ev_ins.emplace_back(e1, e2);
      h->ins_spaces.push_back(uint64_t(n));
    }
    launches += 5;  // space prep, count, plan, fill, insert
  }
  if (slot) {
    FR_CUDA(cudaEventRecord(slot->free, h->stream));
    slot->used = true;
  }
  h->launches_pending += launches + (bandCopy ? 1 : 0);
  FR_CUDA(cudaMemcpyAsync(h->host_stats, h->bb.stats, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, h->stream));
  FR_CUDA(cudaMemcpyAsync(h->host_status, h->bb.status, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  return FR_OK;
}

// ---- batched jobs ----------------------------------------------------------------------

static void fill_config(frb::InsertConfig &cfg, const fr_settings &s)
{
  cfg.fast = s.type == FR_TYPE_FAST;
  cfg.mode = s.interpolation == FR_INTERPOLATION_LOOKUP ? 0 : (s.alpha <= 15.f ? 1 : 3);
  const int taps = int(std::floor(2.f * s.blob_radius)) + 1;
  cfg.taps = taps <= 4 ? 4 : 8;
  cfg.storage = s.storage;
  cfg.kahan = s.accumulation == FR_ACCUM_KAHAN;
}

// Worst-case bricks one space can reach in a volume of side `side` (see fr_init).
static int64_t bricks_per_space(uint64_t side, const frb::InsertConfig &cfg, float radius)
{
  const int64_t nb = int64_t((side + 15) / 16);
  const double hw = cfg.fast ? 2.5 : double(radius) + 1e-3;
  const int perCol = int(std::ceil((2.0 * 15.0 + 2.0 * hw * std::sqrt(3.0)) / 16.0)) + 2;
  return std::min<int64_t>(nb * nb * nb, nb * nb * perCol);
}

int fr_batch_init(fr_handle *h, const fr_batch_limits *lim, const fr_settings *s)
{
  if (!h) return fail(FR_E_INVALID, "handle is NULL");
  fr_cleanup(h);
  if (!lim) return fail(FR_E_INVALID, "limits is NULL");
  int rc = check_settings(s);
  if (rc) return rc;
  if (lim->max_jobs < 1 || lim->max_spaces < 1 || lim->max_bricks < 1 || lim->max_volume_side < 2)
    return fail(FR_E_INVALID, "batch limits must be positive");
  if (lim->max_jobs > (1u << 20) || lim->max_spaces > (1u << 28) || lim->max_bricks > (1u << 26)
      || lim->max_volume_side > (1u << 14))
    return fail(FR_E_UNSUPPORTED, "batch limits too large");
  if (s->interpolation == FR_INTERPOLATION_LOOKUP && (lim->table_elems < 2 || lim->table_elems > (1u << 26)))
    return fail(FR_E_NO_TABLE, "lookup interpolation needs a blob table of at least 2 entries");
  frb::DeviceGuard guard(h->device);
  FR_CUDA(guard.err);
  h->settings = *s;
  h->blim = *lim;
  h->dims = fr_dims{};
  h->dims.table_elems = lim->table_elems;
  h->constants = make_constants(3, 3, s->interpolation == FR_INTERPOLATION_LOOKUP ? lim->table_elems : 0, *s);
  frb::InsertConfig &cfg = h->cfg;
  fill_config(cfg, *s);
  cfg.jobs = true;
  cfg.banded = true;  // batches insert from banded copies
  apply_tuning_file(h);
  cfg.groups = h->launch.groups;
  h->launch.groups = frb::insert_groups(cfg);
  if (h->launch.item_capacity <= 0) h->launch.item_capacity = 512;
  h->launch.brick = 16;
  const size_t smem = frb::insert_smem_bytes(cfg, int(lim->table_elems));
  int occ = 0;
  FR_CUDA(cudaFuncSetAttribute(frb::insert_kernel_ptr(cfg), cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  FR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, frb::insert_kernel_ptr(cfg), 256 * frb::insert_groups(cfg), smem));
  if (occ < 1) return fail(FR_E_UNSUPPORTED, "insertion kernel does not fit on an SM");
  if (h->launch.ctas_per_sm <= 0 || h->launch.ctas_per_sm > occ) h->launch.ctas_per_sm = occ;
  h->grid = h->num_sms * h->launch.ctas_per_sm;

  const int64_t perSpace = bricks_per_space(lim->max_volume_side, cfg, s->blob_radius);
  const int64_t listCap = int64_t(lim->max_spaces) * perSpace;
  if (listCap > (int64_t(1) << 31) - 1) return fail(FR_E_UNSUPPORTED, "batch limits exceed the list index range");
  const int64_t nb = int64_t(lim->max_bricks);
  const int64_t itemsCap = listCap / h->launch.item_capacity + nb + 1;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += align256(bytes);
    return o;
  };
  const size_t oPrep = take(size_t(lim->max_spaces) * frb::kSpacePrepBytes);
  const size_t oRec = take(size_t(lim->max_spaces) * frb::kSpaceRecBytes);
  const size_t oCounts = take(size_t(3) * nb * sizeof(int));
  const size_t oOffsets = take((size_t(3) * nb + 1) * sizeof(int));
  const size_t oList = take(size_t(listCap) * sizeof(int));
  const size_t oOrder = take(size_t(nb) * sizeof(int));
  const size_t oItems = take(size_t(itemsCap) * frb::kWorkItemBytes);
  const size_t oJobs = take(size_t(lim->max_jobs) * sizeof(frb::JobDesc));
  const size_t oMisc = take(64);
  const size_t oStats = take(4 * sizeof(unsigned long long));
  const size_t oKaiser = take(cfg.mode == 3 && !cfg.fast ? size_t(frb::kKaiserTableElems) * sizeof(float2) : 0);
  FR_CUDA(cudaMalloc(&h->scratch, off));
  h->scratch_bytes = off;
  char *base = static_cast<char *>(h->scratch);
  frb::BinBuffers &bb = h->bb;
  bb.prep = reinterpret_cast<frb::SpacePrep *>(base + oPrep);
  bb.rec = reinterpret_cast<frb::SpaceRec *>(base + oRec);
  bb.counts = reinterpret_cast<int *>(base + oCounts);
  bb.offsets = reinterpret_cast<int *>(base + oOffsets);
  bb.list = reinterpret_cast<int *>(base + oList);
  bb.order = reinterpret_cast<const int *>(base + oOrder);
  bb.items = reinterpret_cast<frb::WorkItem *>(base + oItems);
  int *misc = reinterpret_cast<int *>(base + oMisc);
  bb.nItems = misc;
  bb.status = misc + 1;
  h->work_counter = misc + 2;
  bb.stats = reinterpret_cast<unsigned long long *>(base + oStats);
  bb.listCap = listCap;
  bb.itemsCap = itemsCap;
  h->d_jobs = reinterpret_cast<frb::JobDesc *>(base + oJobs);
  for (int k = 0; k < 2; ++k) {
    FR_CUDA(cudaHostAlloc(reinterpret_cast<void **>(&h->h_jobs_set[k]), size_t(lim->max_jobs) * sizeof(frb::JobDesc),
      cudaHostAllocDefault));
    FR_CUDA(cudaHostAlloc(reinterpret_cast<void **>(&h->h_order_set[k]), size_t(nb) * sizeof(int), cudaHostAllocDefault));
    FR_CUDA(cudaEventCreateWithFlags(&h->upload_set_done[k], cudaEventDisableTiming));
  }
  h->upload_set = 0;
  h->h_jobs = h->h_jobs_set[0];
  h->h_order = h->h_order_set[0];
  h->upload_done = h->upload_set_done[0];
  FR_CUDA(cudaMemsetAsync(misc, 0, 64, h->stream));
  FR_CUDA(cudaMemsetAsync(bb.stats, 0, 4 * sizeof(unsigned long long), h->stream));
  h->kaiser_table = nullptr;
  if (cfg.mode == 3 && !cfg.fast) {
    h->kaiser_table = reinterpret_cast<float *>(base + oKaiser);
    FR_CUDA(frb::launch_kaiser_table(h->kaiser_table, s->blob_order, s->alpha, s->blob_radius, h->constants.cIw0,
      h->stream));
  }
  FR_CUDA(cudaStreamSynchronize(h->stream));
  h->batch = true;
  h->initialized = true;
  return FR_OK;
}

// Enqueues one batch (job table and brick order already staged in pinned memory).
static int enqueue_batch(fr_handle *h, int nJobs, int totalSpaces, int totalBricks, int totalGroups,
  int64_t bandUnits, const float *table, bool capturing)
{
  const fr_settings &s = h->settings;
  FR_CUDA(cudaMemcpyAsync(h->d_jobs, h->h_jobs, size_t(nJobs) * sizeof(frb::JobDesc), cudaMemcpyHostToDevice, h->stream));
  FR_CUDA(cudaMemcpyAsync(const_cast<int *>(h->bb.order), h->h_order, size_t(totalBricks) * sizeof(int),
    cudaMemcpyHostToDevice, h->stream));
  if (!capturing) FR_CUDA(cudaEventRecord(h->upload_done, h->stream));  // graph mode records after launch
  // the jobs' projections are copied into bands on the band stream beside the binning
  FR_CUDA(cudaEventRecord(h->band_fork, h->stream));
  FR_CUDA(cudaStreamWaitEvent(h->band_stream, h->band_fork, 0));
  FR_CUDA(frb::launch_batch_band(h->d_jobs, nJobs, bandUnits, s.storage == FR_STORAGE_FP32 ? 8 : 4, h->band_stream));
  FR_CUDA(cudaEventRecord(h->band_join, h->band_stream));
  FR_CUDA(cudaMemsetAsync(h->bb.stats, 0, 4 * sizeof(unsigned long long), h->stream));
  FR_CUDA(frb::launch_batch_binning(h->d_jobs, nJobs, totalSpaces, totalBricks, totalGroups, h->cfg.fast,
    s.blob_radius, h->bb, h->launch.item_capacity, h->stream));
  FR_CUDA(cudaMemsetAsync(h->work_counter, 0, sizeof(int), h->stream));
  FR_CUDA(cudaStreamWaitEvent(h->stream, h->band_join, 0));
  frb::InsertParams P{};
  P.jobs = h->d_jobs;
  P.recs = h->bb.rec;
  P.list = h->bb.list;
  P.offsets = h->bb.offsets;
  P.items = h->bb.items;
  P.nItems = h->bb.nItems;
  P.workCounter = h->work_counter;
  set_table(P, h, table, h->blim.table_elems);
  P.lutInSmem = frb::insert_lut_in_smem(h->cfg, P.tableElems);
  P.c = h->constants;
  P.order = s.blob_order;
  FR_CUDA(frb::launch_insert(P, h->cfg, h->grid, h->stream));
  FR_CUDA(cudaMemcpyAsync(h->host_stats, h->bb.stats, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, h->stream));
  FR_CUDA(cudaMemcpyAsync(h->host_status, h->bb.status, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  return FR_OK;
}

int fr_batch_execute(fr_handle *h, const fr_job *jobs, uint64_t nJobs, const float *table, int flags)
{
  if (!h) return fail(FR_E_INVALID, "handle is NULL");
  if (!h->initialized || !h->batch) return fail(FR_E_NOT_INIT, "fr_batch_execute before a successful fr_batch_init");
  if (nJobs == 0) return FR_OK;
  if (!jobs) return fail(FR_E_INVALID, "jobs is NULL");
  if (nJobs > h->blim.max_jobs) return fail(FR_E_MISMATCH, "more jobs than the batch limits");
  const fr_settings &s = h->settings;
  if (s.interpolation == FR_INTERPOLATION_LOOKUP && !table)
    return fail(FR_E_NO_TABLE, "lookup interpolation with an empty blob table");
  if ((flags & FR_BATCH_GRAPH) && !h->stream) return fail(FR_E_INVALID, "graph capture needs a non-default stream");
  frb::DeviceGuard guard(h->device);
  FR_CUDA(guard.err);
  if (table && is_host_pointer(table)) return fail(FR_E_INVALID, "the blob table must be device memory");
  // this launch's staging set may still feed the upload of the launch before the previous one
  h->upload_set = (flags & FR_BATCH_GRAPH) ? 0 : h->upload_set ^ 1;
  h->h_jobs = h->h_jobs_set[h->upload_set];
  h->h_order = h->h_order_set[h->upload_set];
  h->upload_done = h->upload_set_done[h->upload_set];
  FR_CUDA(cudaEventSynchronize(h->upload_done));
  const bool smallTable = s.interpolation != FR_INTERPOLATION_LOOKUP || h->blim.table_elems <= frb::kLutSmemMax;
  int64_t spaceBase = 0, brickBase = 0, groupBase = 0, bandUnits = 0;
  size_t bandElems = 0;
  std::vector<size_t> bandOff(nJobs);
  for (uint64_t j = 0; j < nJobs; ++j) {
    const fr_job &J = jobs[j];
    if (!J.fft || !J.volume || !J.weight || J.n_projections == 0 || (J.n_spaces && !J.spaces))
      return fail(FR_E_INVALID, "a job has an empty payload");
    if (s.storage != FR_STORAGE_FP32 && !J.scales) return fail(FR_E_INVALID, "16-bit storage needs scales");
    if (J.volume_x < 2 || J.volume_x % 2 == 0 || J.volume_y % 2 == 0 || J.volume_y != J.volume_z || J.fft_x < 1 || J.fft_y < 2)
      return fail(FR_E_UNSUPPORTED, "job volume sizes must be odd with y == z");
    if (std::max(J.volume_x, J.volume_y) > h->blim.max_volume_side)
      return fail(FR_E_MISMATCH, "a job volume exceeds the batch limits");
    if (is_host_pointer(J.fft) || is_host_pointer(J.volume) || is_host_pointer(J.weight)
        || (J.n_spaces && is_host_pointer(J.spaces)) || (J.scales && is_host_pointer(J.scales)))
      return fail(FR_E_INVALID, "batched payloads must be device or managed memory");
    frb::JobDesc &D = h->h_jobs[j];
    std::memset(&D, 0, sizeof(D));
    D.fft = J.fft;
    D.scales = J.scales;
    D.volume = J.volume;
    D.weight = J.weight;
    D.nProj = int(J.n_projections);
    D.fftX = int(J.fft_x);
    D.fftY = int(J.fft_y);
    D.vx = int(J.volume_x);
    D.vy = int(J.volume_y);
    D.vz = int(J.volume_z);
    D.nbx = (D.vx + 15) / 16;
    D.nby = (D.vy + 15) / 16;
    D.nbz = (D.vz + 15) / 16;
    D.cx = (D.vx - 1) / 2;
    D.cy = (D.vy - 1) / 2;
    D.cz = (D.vz - 1) / 2;
    D.genericTaps = D.fftX < h->cfg.taps || D.fftY < h->cfg.taps || !smallTable;
    D.spaceBase = int(spaceBase);
    D.nSpaces = int(J.n_spaces);
    D.brickBase = int(brickBase);
    D.nBricks = D.nbx * D.nby * D.nbz;
    D.groupBase = int(groupBase);
    D.spaces = J.spaces;
    D.src = J.fft;
    D.bandStride = frb::band_stride(D.fftX);
    D.unitBase = int(bandUnits);
    bandOff[j] = bandElems;
    if (s.layout != FR_LAYOUT_BANDED) {  // banded payloads are read in place
      bandUnits += int64_t(D.nProj) * ((D.fftY + 3) / 4);
      bandElems += size_t(D.nProj) * size_t(frb::band_plane_elems(D.fftX, D.fftY));
    }
    spaceBase += int64_t(J.n_spaces);
    brickBase += D.nBricks;
    groupBase += (D.nBricks + 7) / 8;
    if (bandUnits > int64_t(INT32_MAX)) return fail(FR_E_UNSUPPORTED, "too many projection rows in one batch");
  }
  if (spaceBase > int64_t(h->blim.max_spaces) || brickBase > int64_t(h->blim.max_bricks))
    return fail(FR_E_MISMATCH, "batch exceeds the spaces or bricks of the batch limits");
  if (spaceBase == 0) return FR_OK;
  if (s.layout != FR_LAYOUT_BANDED) {  // the batch inserts from a banded copy of every job's projections
    bool ok = false;
    const size_t elem = s.storage == FR_STORAGE_FP32 ? 8 : 4;
    const int rc = ensure_band(h, bandElems * elem, false, ok);
    if (rc) return rc;
    for (uint64_t j = 0; j < nJobs; ++j) h->h_jobs[j].fft = static_cast<char *>(h->band) + bandOff[j] * elem;
  }
  // brick order: heavier jobs first (spaces x voxels), each job's bricks nearest its centre first
  std::vector<int> jo(nJobs);
  std::iota(jo.begin(), jo.end(), 0);
  std::stable_sort(jo.begin(), jo.end(), [&](int a, int b) {
    const double wa = double(h->h_jobs[a].nSpaces) * h->h_jobs[a].vx * h->h_jobs[a].vx;
    const double wb = double(h->h_jobs[b].nSpaces) * h->h_jobs[b].vx * h->h_jobs[b].vx;
    return wa > wb;
  });
  int64_t k = 0;
  for (int j : jo) {
    const frb::JobDesc &D = h->h_jobs[j];
    std::vector<int> &ord = h->brick_order[{ D.vx, D.vy, D.vz }];
    if (ord.empty()) {
      std::vector<std::pair<double, int>> bd(size_t(D.nBricks));
      for (int b = 0; b < D.nBricks; ++b) {
        const int bx = b % D.nbx, by = (b / D.nbx) % D.nby, bz = b / (D.nbx * D.nby);
        const double x = bx * 16 + 7.5 - D.cx, y = by * 16 + 7.5 - D.cy, z = bz * 16 + 7.5 - D.cz;
        bd[size_t(b)] = { x * x + y * y + z * z, b };
      }
      std::stable_sort(bd.begin(), bd.end());
      ord.reserve(bd.size());
      for (const auto &e : bd) ord.push_back(e.second);
    }
    for (int b : ord) h->h_order[k++] = D.brickBase + b;
  }
  const int nj = int(nJobs), ts = int(spaceBase), tb = int(brickBase), tg = int(groupBase);
  h->launches_pending += 6;
  if (!(flags & FR_BATCH_GRAPH)) return enqueue_batch(h, nj, ts, tb, tg, bandUnits, table, false);
  // graph mode: replay while the job table (and table pointer) repeats
  std::vector<unsigned char> sig(size_t(nJobs) * sizeof(frb::JobDesc) + sizeof(table));
  std::memcpy(sig.data(), h->h_jobs, size_t(nJobs) * sizeof(frb::JobDesc));
  std::memcpy(sig.data() + size_t(nJobs) * sizeof(frb::JobDesc), &table, sizeof(table));
  if (!h->graph || sig != h->graph_sig) {
    if (h->graph) cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
    cudaGraph_t g = nullptr;
    FR_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = enqueue_batch(h, nj, ts, tb, tg, bandUnits, table, true);
    const cudaError_t ec = cudaStreamEndCapture(h->stream, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    FR_CUDA(ec);
    const cudaError_t ei = cudaGraphInstantiate(&h->graph, g, 0);
    cudaGraphDestroy(g);
    FR_CUDA(ei);
    h->graph_sig.swap(sig);
  }
  FR_CUDA(cudaGraphLaunch(h->graph, h->stream));
  FR_CUDA(cudaEventRecord(h->upload_done, h->stream));  // the graph reads the staging buffers
  return FR_OK;
}

int fr_set_profiling(fr_handle *h, int enable)
{
  if (!h) return fail(FR_E_INVALID, "handle is NULL");
  h->profiling = enable != 0;
  return FR_OK;
}

int fr_get_phase_times(fr_handle *h, fr_phase_times *out, int reset)
{
  if (!h || !out) return fail(FR_E_INVALID, "NULL argument");
  frb::DeviceGuard guard(h->device);
  FR_CUDA(guard.err);
  FR_CUDA(cudaStreamSynchronize(h->stream));
  collect_times(h);
  *out = h->times;
  if (reset) h->times = fr_phase_times{};
  return FR_OK;
}

int fr_synchronize(fr_handle *h)
{
  if (!h) return fail(FR_E_INVALID, "handle is NULL");
  frb::DeviceGuard guard(h->device);
  FR_CUDA(guard.err);
  FR_CUDA(cudaStreamSynchronize(h->stream));
  FR_CUDA(cudaGetLastError());
  h->last.pairs = h->host_stats[0];
  h->last.items = h->host_stats[1];
  h->last.chunks = h->host_stats[2];
  h->last.launches = h->launches_pending;
  h->launches_pending = 0;
  int st = h->host_status[0];
  if (st != 0) {
    h->host_status[0] = 0;
    if (h->initialized) {
      FR_CUDA(cudaMemsetAsync(h->bb.status, 0, sizeof(int), h->stream));
      FR_CUDA(cudaStreamSynchronize(h->stream));
    }
    return fail(st, st == FR_E_CAPACITY ? "device-side failure: binned work exceeded the engine's list capacity"
                                        : "a traverse space addresses a projection outside the FFT payload");
  }
  return FR_OK;
}

int fr_fill_blob_table(float *table, uint64_t n, const fr_settings *s, void *stream)
{
  int rc = check_settings(s);
  if (rc) return rc;
  if (!table || n < 2) return fail(FR_E_INVALID, "blob table needs at least 2 entries");
  const float iw0 = 1.f / kaiser_fourier_value0(s->blob_radius, s->alpha, s->blob_order);
  FR_CUDA(frb::launch_blob_table(table, int64_t(n), s->blob_order, s->alpha, s->blob_radius, iw0,
    static_cast<cudaStream_t>(stream)));
  return FR_OK;
}

int fr_quantize_projections(const void *fft, uint64_t n, uint64_t fftX, uint64_t fftY, int storage,
  void *out, float *scales, void *stream)
{
  if (storage != FR_STORAGE_BF16 && storage != FR_STORAGE_FP16)
    return fail(FR_E_INVALID, "storage must be FR_STORAGE_BF16 or FR_STORAGE_FP16");
  if (n == 0) return FR_OK;
  if (!fft || !out || !scales || fftX == 0 || fftY == 0) return fail(FR_E_INVALID, "NULL or empty argument");
  if (n > (1u << 31)) return fail(FR_E_UNSUPPORTED, "too many projections for one call");
  FR_CUDA(frb::launch_quantize(fft, int64_t(n), int64_t(fftX * fftY), storage, out, scales,
    static_cast<cudaStream_t>(stream)));
  return FR_OK;
}

uint64_t fr_band_plane_elems(uint64_t fftX, uint64_t fftY)
{
  if (fftX == 0 || fftY == 0 || fftX > (1u << 20) || fftY > (1u << 20)) return 0;
  return uint64_t(frb::band_plane_elems(int(fftX), int(fftY)));
}

int fr_band_projections(const void *fft, uint64_t n, uint64_t fftX, uint64_t fftY, int storage, void *out,
  void *stream)
{
  if (storage < FR_STORAGE_FP32 || storage > FR_STORAGE_FP16) return fail(FR_E_INVALID, "unknown storage");
  if (n == 0) return FR_OK;
  if (!fft || !out || fftX == 0 || fftY == 0) return fail(FR_E_INVALID, "NULL or empty argument");
  if (fftX > (1u << 20) || fftY > (1u << 20)) return fail(FR_E_UNSUPPORTED, "payload dimension too large");
  if (is_host_pointer(fft) || is_host_pointer(out)) return fail(FR_E_INVALID, "fft and out must be device memory");
  FR_CUDA(frb::launch_band_projections(fft, out, int64_t(n), int(fftX), int(fftY), storage == FR_STORAGE_FP32 ? 8 : 4,
    static_cast<cudaStream_t>(stream)));
  return FR_OK;
}

int fr_compute_traverse_spaces(const float *rotations, uint64_t n, uint32_t imgX, uint32_t imgY,
  uint32_t maxVX, uint32_t maxVYZ, int useFast, float radius, float weight, int32_t first,
  fr_traverse_space *out, void *stream)
{
  if (n == 0) return FR_OK;
  if (!rotations || !out) return fail(FR_E_INVALID, "NULL argument");
  FR_CUDA(frb::launch_traverse_spaces(rotations, int64_t(n), imgX, imgY, maxVX, maxVYZ, useFast,
    radius, weight, first, out, static_cast<cudaStream_t>(stream)));
  return FR_OK;
}

int fr_compute_traverse_spaces_sym(const float *rotations, uint64_t n, const float *symmetries, uint32_t nSym,
  uint32_t imgX, uint32_t imgY, uint32_t maxVX, uint32_t maxVYZ, int useFast, float radius, float weight,
  int32_t first, fr_traverse_space *out, void *stream)
{
  if (n == 0 || nSym == 0) return FR_OK;
  if (!rotations || !symmetries || !out) return fail(FR_E_INVALID, "NULL argument");
  if (n * uint64_t(nSym) > (uint64_t(1) << 31)) return fail(FR_E_UNSUPPORTED, "too many spaces");
  if (is_host_pointer(rotations) || is_host_pointer(symmetries) || is_host_pointer(out))
    return fail(FR_E_INVALID, "rotations, symmetries and spaces must be device memory");
  FR_CUDA(frb::launch_traverse_spaces_sym(rotations, int64_t(n), symmetries, int(nSym), imgX, imgY, maxVX, maxVYZ,
    useFast, radius, weight, first, out, static_cast<cudaStream_t>(stream)));
  return FR_OK;
}

}// extern "C"
