// fr_insert_noalloc: a Fourier-reconstruction insertion that allocates no memory.
//
// Some hosts cannot let a plugin call cudaMalloc: an application that owns its GPU memory
// through its own pool or budget, a real-time or audio-style thread where an allocation may
// block on the driver, or a framework that must not see device memory appear outside its
// allocator.  fr_init sizes and allocates the engine's scratch (binning lists, work items);
// this entry point instead takes its scratch from one fixed array compiled into the library,
// so the caller only provides the inputs and outputs.
//
// The array below is part of the library image: every GPU on which the library is loaded
// holds its kScratchBytes until the process exits.  All calls on a device share it and it
// keeps whatever the previous call left there, so the parts that must start at zero (status,
// counters) are cleared at the start of every call, and two calls whose work overlaps on the
// GPU (for example on two streams) would race on it -- run them one after the other.
//
// Every call looks the array's device address up again (cudaGetSymbolAddress, with the
// call's device current), so a device reset or a reloaded module never leaves a stale
// address behind.  The first call on a device loads the library's kernels there: make it
// before any stream capture.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>

#include "fr_device.cuh"
#include "fr_device_guard.h"
#include "fr_kernels.h"
#include "umpalumpa_fr.h"

namespace {

constexpr size_t kScratchBytes = size_t(32) << 20;  // 32 MiB per device
constexpr int kMaxDevices = 64;
constexpr int kItemCapacity = 512;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// In host code the name g_noalloc_scratch is only a host-side stand-in for the array, never
// a device address: kernels get the address cudaGetSymbolAddress returns.

int fail(int code, const char *msg) { return frb::set_last_error(code, msg); }

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

bool is_device_accessible(const void *p)
{
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Bricks nearest the volume centre first (they carry the most slabs), by a counting sort on
// the squared distance: one CTA, 1024 distance buckets.
__global__ void __launch_bounds__(1024) noalloc_order_kernel(frb::BinGeom g, int *__restrict__ order)
{
  __shared__ int hist[1024];
  const int tid = threadIdx.x;
  hist[tid] = 0;
  __syncthreads();
  const float maxD2 = 3.f * 0.25f * float(max(g.vx, max(g.vy, g.vz))) * float(max(g.vx, max(g.vy, g.vz))) + 1.f;
  auto bucket = [&](int b) {
    const int bx = b % g.nbx, by = (b / g.nbx) % g.nby, bz = b / (g.nbx * g.nby);
    const float x = bx * 16 + 7.5f - g.cx, y = by * 16 + 7.5f - g.cy, z = bz * 16 + 7.5f - g.cz;
    return min(1023, int((x * x + y * y + z * z) / maxD2 * 1024.f));
  };
  for (int b = tid; b < g.n_bricks; b += 1024) atomicAdd(&hist[bucket(b)], 1);
  __syncthreads();
  if (tid == 0) {
    int run = 0;
    for (int k = 0; k < 1024; ++k) {
      const int c = hist[k];
      hist[k] = run;
      run += c;
    }
  }
  __syncthreads();
  for (int b = tid; b < g.n_bricks; b += 1024) order[atomicAdd(&hist[bucket(b)], 1)] = b;
}

}// namespace

extern "C" int fr_insert_noalloc(int device, void *stream, const fr_dims *d, const fr_settings *s,
  const void *fft, const float *scales, uint64_t nProj, void *volume, float *weight,
  const fr_traverse_space *spaces, uint64_t nSpaces, const float *table)
{
  if (!d || !s) return fail(FR_E_INVALID, "dims and settings are required");
  fr_constants c;
  int rc = fr_make_constants(d, s, &c);  // validates the settings
  if (rc) return rc;
  if (d->volume_x < 2 || d->volume_y < 2 || d->volume_z < 2 || d->fft_x < 1 || d->fft_y < 2)
    return fail(FR_E_INVALID, "malformed payload sizes");
  if (d->volume_x % 2 == 0 || d->volume_y % 2 == 0 || d->volume_y != d->volume_z)
    return fail(FR_E_UNSUPPORTED, "volume sizes must be odd with y == z");
  if (nProj == 0 || !fft || !volume || !weight) return fail(FR_E_INVALID, "empty payload");
  // Payload::IsEquivalentTo (payload.hpp:60-63): counts within the sizes described by `d`
  if (nProj > d->n_projections || nSpaces > d->n_spaces)
    return fail(FR_E_MISMATCH, "payload count exceeds the sizes in dims");
  if (nProj > uint64_t(INT32_MAX) || nSpaces > uint64_t(INT32_MAX))
    return fail(FR_E_UNSUPPORTED, "more than 2^31 - 1 projections or traverse spaces");
  if (s->interpolation == FR_INTERPOLATION_LOOKUP && (!table || d->table_elems < 2))
    return fail(FR_E_NO_TABLE, "lookup interpolation with an empty blob table");
  if (s->storage != FR_STORAGE_FP32 && !scales) return fail(FR_E_INVALID, "16-bit storage needs scales");
  if (nSpaces == 0) return FR_OK;
  if (!spaces) return fail(FR_E_INVALID, "empty traverse-space payload");
  if (device < 0 || device >= kMaxDevices) return fail(FR_E_INVALID, "device index out of range");
  frb::DeviceGuard guard(device);
  if (guard.err != cudaSuccess) {
    cudaGetLastError();
    return fail(FR_E_CUDA, "cudaSetDevice failed");
  }
  if (!is_device_accessible(fft) || !is_device_accessible(volume) || !is_device_accessible(weight)
      || !is_device_accessible(spaces) || (table && !is_device_accessible(table))
      || (scales && !is_device_accessible(scales)))
    return fail(FR_E_INVALID, "every payload must be device or managed memory");

  // The array's device address on this device (the call's device is current).
  void *base = nullptr;
  {
    const cudaError_t e = cudaGetSymbolAddress(&base, g_noalloc_scratch);
    if (e != cudaSuccess || !base) {
      cudaGetLastError();
      return fail(FR_E_CUDA, "cudaGetSymbolAddress of the scratch array failed");
    }
  }
  const cudaStream_t st = static_cast<cudaStream_t>(stream);

  frb::BinGeom g;
  g.vx = int(d->volume_x);
  g.vy = int(d->volume_y);
  g.vz = int(d->volume_z);
  g.nbx = (g.vx + 15) / 16;
  g.nby = (g.vy + 15) / 16;
  g.nbz = (g.vz + 15) / 16;
  g.n_bricks = g.nbx * g.nby * g.nbz;
  g.cx = c.cMaxVolumeIndexX / 2;
  g.cy = c.cMaxVolumeIndexYZ / 2;
  g.cz = c.cMaxVolumeIndexYZ / 2;

  frb::InsertConfig cfg{};
  cfg.fast = s->type == FR_TYPE_FAST;
  // the kernel modes of fr_execute: above alpha 15 the interpolated Kaiser table, built in
  // the scratch array by every call
  cfg.mode = s->interpolation == FR_INTERPOLATION_LOOKUP ? 0 : (s->alpha <= 15.f ? 1 : 3);
  const bool kaiserTable = cfg.mode == 3 && !cfg.fast;
  cfg.taps = int(std::floor(2.f * s->blob_radius)) + 1 <= 4 ? 4 : 8;
  cfg.storage = s->storage;
  cfg.kahan = s->accumulation == FR_ACCUM_KAHAN;
  cfg.banded = s->layout == FR_LAYOUT_BANDED;  // no room for a banded copy: rows unless given bands

  // Carve the array: per-brick arrays first, then as many traverse spaces per chunk as fit
  // (same list-capacity bound as fr_init: ceil(L / 16) + 2 bricks per brick column).
  const double hw = cfg.fast ? 2.5 : double(s->blob_radius) + 1e-3;
  const int perCol = int(std::ceil((2.0 * 15.0 + 2.0 * hw * std::sqrt(3.0)) / 16.0)) + 2;
  const int64_t cols = std::max({ int64_t(g.nbx) * g.nby, int64_t(g.nbx) * g.nbz, int64_t(g.nby) * g.nbz });
  const int64_t perSpace = std::min<int64_t>(g.n_bricks, cols * perCol);
  size_t off = 0;
  const size_t oMisc = off;
  off += 256;
  const size_t oStats = off;
  off += 256;
  const size_t oCounts = off;
  off += align256(size_t(3) * g.n_bricks * sizeof(int));
  const size_t oOffsets = off;
  off += align256((size_t(3) * g.n_bricks + 1) * sizeof(int));
  const size_t oOrder = off;
  off += align256(size_t(g.n_bricks) * sizeof(int));
  const size_t oKaiser = off;
  off += kaiserTable ? align256(size_t(frb::kKaiserTableElems) * sizeof(float2)) : 0;
  if (off >= kScratchBytes) return fail(FR_E_UNSUPPORTED, "volume too large for the 32 MiB scratch");
  const double perSpaceBytes = double(frb::kSpacePrepBytes + frb::kSpaceRecBytes) + double(perSpace) * 4.0
                               + double(perSpace) / kItemCapacity * frb::kWorkItemBytes;
  const double room = double(kScratchBytes - off) - double(g.n_bricks + 1) * frb::kWorkItemBytes - 4 * 256.0;
  int64_t chunk = room > 0 ? int64_t(room / perSpaceBytes) : 0;
  chunk = std::min<int64_t>(chunk, int64_t(nSpaces));
  if (chunk < 1) return fail(FR_E_UNSUPPORTED, "volume too large for the 32 MiB scratch");
  const int64_t listCap = chunk * perSpace;
  const int64_t itemsCap = listCap / kItemCapacity + g.n_bricks + 1;
  const size_t oPrep = off;
  off += align256(size_t(chunk) * frb::kSpacePrepBytes);
  const size_t oRec = off;
  off += align256(size_t(chunk) * frb::kSpaceRecBytes);
  const size_t oList = off;
  off += align256(size_t(listCap) * sizeof(int));
  const size_t oItems = off;
  off += align256(size_t(itemsCap) * frb::kWorkItemBytes);
  if (off > kScratchBytes) return fail(FR_E_UNSUPPORTED, "volume too large for the 32 MiB scratch");

  char *sb = static_cast<char *>(base);
  int *misc = reinterpret_cast<int *>(sb + oMisc);
  frb::BinBuffers bb;
  bb.prep = reinterpret_cast<frb::SpacePrep *>(sb + oPrep);
  bb.rec = reinterpret_cast<frb::SpaceRec *>(sb + oRec);
  bb.counts = reinterpret_cast<int *>(sb + oCounts);
  bb.offsets = reinterpret_cast<int *>(sb + oOffsets);
  bb.list = reinterpret_cast<int *>(sb + oList);
  bb.order = reinterpret_cast<const int *>(sb + oOrder);
  bb.items = reinterpret_cast<frb::WorkItem *>(sb + oItems);
  bb.nItems = misc;
  bb.status = misc + 1;
  int *workCounter = misc + 2;
  bb.stats = reinterpret_cast<unsigned long long *>(sb + oStats);
  bb.listCap = listCap;
  bb.itemsCap = itemsCap;

  // the array keeps the previous call's contents: clear what must start at zero
  cudaError_t e = cudaMemsetAsync(misc, 0, 256, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(bb.stats, 0, 256, st);
  if (e == cudaSuccess) {
    noalloc_order_kernel<<<1, 1024, 0, st>>>(g, reinterpret_cast<int *>(sb + oOrder));
    e = cudaGetLastError();
  }
  float *kaiser = kaiserTable ? reinterpret_cast<float *>(sb + oKaiser) : nullptr;
  if (e == cudaSuccess && kaiserTable)
    e = frb::launch_kaiser_table(kaiser, s->blob_order, s->alpha, s->blob_radius, c.cIw0, st);

  const size_t smem = frb::insert_smem_bytes(cfg, int(d->table_elems));
  int occ = 0, sms = 0;
  if (e == cudaSuccess) e = cudaFuncSetAttribute(frb::insert_kernel_ptr(cfg), cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, frb::insert_kernel_ptr(cfg), 256 * frb::insert_groups(cfg), smem);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(FR_E_CUDA, cudaGetErrorString(e));
  }
  if (occ < 1) return fail(FR_E_UNSUPPORTED, "insertion kernel does not fit on an SM");

  frb::InsertParams P{};
  P.volume = volume;
  P.weight = weight;
  P.fft = fft;
  P.scales = scales;
  P.recs = bb.rec;
  P.list = bb.list;
  P.offsets = bb.offsets;
  P.items = bb.items;
  P.nItems = bb.nItems;
  P.workCounter = workCounter;
  P.table = kaiserTable ? kaiser : table;
  P.tableElems = kaiserTable ? frb::kKaiserTableElems
                             : int(s->interpolation == FR_INTERPOLATION_LOOKUP ? d->table_elems : 0);
  P.tableScale = kaiserTable ? float(frb::kKaiserTableElems - 1) / (s->blob_radius * s->blob_radius) : 0.f;
  P.lutInSmem = frb::insert_lut_in_smem(cfg, P.tableElems);
  P.genericTaps = int(d->fft_x) < cfg.taps || int(d->fft_y) < cfg.taps || P.tableElems > frb::kLutSmemMax;
  P.c = c;
  P.order = s->blob_order;
  P.nProj = int(nProj);
  P.fftX = int(d->fft_x);
  P.fftY = int(d->fft_y);
  P.bandStride = cfg.banded ? frb::band_stride(P.fftX) : 0;
  P.vx = g.vx;
  P.vy = g.vy;
  P.vz = g.vz;
  P.nbx = g.nbx;
  P.nby = g.nby;
  P.nbz = g.nbz;
  P.cx = g.cx;
  P.cy = g.cy;
  P.cz = g.cz;
  for (uint64_t s0 = 0; s0 < nSpaces && e == cudaSuccess; s0 += uint64_t(chunk)) {
    const int n = int(std::min<uint64_t>(uint64_t(chunk), nSpaces - s0));
    e = frb::launch_binning(g, spaces + s0, n, int(nProj), cfg.fast, s->blob_radius, bb, kItemCapacity, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(workCounter, 0, sizeof(int), st);
    if (e == cudaSuccess) e = frb::launch_insert(P, cfg, sms * occ, st);
  }
  int status = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&status, bb.status, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(FR_E_CUDA, cudaGetErrorString(e));
  }
  if (status == FR_E_CAPACITY) return fail(FR_E_CAPACITY, "binned work exceeded the scratch list capacity");
  if (status != 0) return fail(status, "a traverse space addresses a projection outside the FFT payload");
  return FR_OK;
}
