// Internal interface between the host engine (fr_capi.cu) and the kernels (fr_kernels.cu).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "umpalumpa_fr.h"

namespace frb {

struct SpacePrep;
struct SpaceRec;
struct WorkItem;
struct JobDesc;

// Brick grid over the volume and the reference's integer volume centre
// (cMaxVolumeIndex / 2, fr_cpu_kernels.hpp:34-36).
struct BinGeom {
  int vx, vy, vz;
  int nbx, nby, nbz, n_bricks;
  int cx, cy, cz;
};

// Scratch of one binning + insertion chunk.
struct BinBuffers {
  SpacePrep *prep;        // [chunk capacity]
  SpaceRec *rec;          // [chunk capacity]
  int *counts;            // [3 * n_bricks]
  int *offsets;           // [3 * n_bricks + 1]
  int *list;              // [listCap] space indices, grouped by (brick, direction)
  const int *order;       // [n_bricks] brick visiting order (heaviest expected first)
  WorkItem *items;        // [itemsCap]
  int *nItems;            // [1]
  int *status;            // [1] sticky FR_E_* of device-side failures
  unsigned long long *stats;  // [4] pairs, items, chunks
  int64_t listCap;
  int64_t itemsCap;
};

struct InsertParams {
  const JobDesc *jobs;  // batched launches: the job table (the per-job fields below unused)
  void *volume;
  float *weight;
  const void *fft;
  const float *scales;
  const SpaceRec *recs;
  const int *list;
  const int *offsets;
  const WorkItem *items;
  const int *nItems;
  int *workCounter;
  const float *table;  // lookup: the blob table; dynamic: the Kaiser (value, slope) table
  int tableElems;      // entries (float2 entries for the Kaiser table)
  float tableScale;    // Kaiser table: nodes per unit of d^2, (N - 1) / r^2
  int lutInSmem;
  int genericTaps;  // bounds-checked taps with a clamped table index: half-plane narrower or
                    // shorter than the blob window, or a blob table above kLutSmemMax entries
  fr_constants c;
  int order;
  int nProj;
  int fftX, fftY;
  int vx, vy, vz;
  int nbx, nby, nbz;
  int cx, cy, cz;
  int bandStride;  // banded half-planes: elements per 4-row band (band_stride); row-major: 0
};

// Which insertion kernel variant runs.
struct InsertConfig {
  int mode;     // 0 lookup table, 1 fast Kaiser (alpha <= 15), 2 Kaiser of any order per tap,
                // 3 Kaiser of any order from the interpolated (value, slope) table (alpha > 15)
  int taps;     // blob footprint per axis: floor(2 r) + 1
  bool fast;    // nearest-pixel insertion (Settings::Type::kFast)
  int storage;  // FR_STORAGE_*
  bool kahan;   // Kahan-compensated brick accumulators
  bool jobs;    // batched launch over a job table
  int groups;   // 256-thread groups per CTA (launch shape); 0 = the most that fit
  bool banded;  // half-planes in 4-row bands (always for a batch); else row-major
};

using InsertFn = void (*)(InsertParams);
// One insertion-kernel variant per storage type and layout, each in its own translation unit.
InsertFn pick_insert_fp32(const InsertConfig &cfg);
InsertFn pick_insert_bf16(const InsertConfig &cfg);
InsertFn pick_insert_fp16(const InsertConfig &cfg);
InsertFn pick_insert_band_fp32(const InsertConfig &cfg);
InsertFn pick_insert_band_bf16(const InsertConfig &cfg);
InsertFn pick_insert_band_fp16(const InsertConfig &cfg);
InsertFn pick_insert_batch_fp32(const InsertConfig &cfg);
InsertFn pick_insert_batch_bf16(const InsertConfig &cfg);
InsertFn pick_insert_batch_fp16(const InsertConfig &cfg);

// Dynamic interpolation's Kaiser (value, slope) table: kKaiserTableElems float2 entries.
cudaError_t launch_kaiser_table(float *table, int order, float alpha, float radius, float iw0, cudaStream_t st);
cudaError_t launch_blob_table(float *table, int64_t n, int order, float alpha, float radius,
  float iw0, cudaStream_t st);
cudaError_t launch_traverse_spaces(const float *rot, int64_t n, uint32_t imgX, uint32_t imgY,
  uint32_t maxVX, uint32_t maxVYZ, int useFast, float radius, float weight, int32_t first,
  fr_traverse_space *out, cudaStream_t st);
cudaError_t launch_traverse_spaces_sym(const float *rot, int64_t n, const float *sym, int nSym, uint32_t imgX,
  uint32_t imgY, uint32_t maxVX, uint32_t maxVYZ, int useFast, float radius, float weight, int32_t first,
  fr_traverse_space *out, cudaStream_t st);
cudaError_t launch_quantize(const void *in, int64_t n, int64_t elems, int storage, void *out, float *scales,
  cudaStream_t st);

// Banded half-planes: rows grouped in bands of four, each band stored column by column, the
// band pitch rounded up to 8 columns (whole 128-byte lines for 8- and 4-byte pixels).
__host__ __device__ inline int band_pitch(int fftX) { return (fftX + 7) & ~7; }
__host__ __device__ inline int band_stride(int fftX) { return 4 * band_pitch(fftX); }
__host__ __device__ inline int64_t band_plane_elems(int fftX, int fftY)
{
  return int64_t((fftY + 3) / 4) * band_stride(fftX);
}
// Copies n row-major half-planes [n][fftY][fftX] of elemBytes-byte pixels (8: complex64, 4: a
// 16-bit pair) into bands; padding columns and rows are written as zeros.
cudaError_t launch_band_projections(const void *src, void *dst, int64_t n, int fftX, int fftY, int elemBytes,
  cudaStream_t st);
// The same for every job of a batch: job j's projections go from its `src` to its `fft`, its
// bands numbered from its `unitBase` (totalUnits bands in all).
cudaError_t launch_batch_band(const JobDesc *jobs, int nJobs, int64_t totalUnits, int elemBytes, cudaStream_t st);
cudaError_t launch_binning(const BinGeom &g, const fr_traverse_space *spaces, int n, int nProj,
  bool fast, float radius, const BinBuffers &b, int itemCap, cudaStream_t st);
// Binning of a batch: jobs (device job table, nJobs entries) with totalSpaces spaces,
// totalBricks bricks and totalGroups 8-brick binning groups in all.
cudaError_t launch_batch_binning(const JobDesc *jobs, int nJobs, int totalSpaces, int totalBricks,
  int totalGroups, bool fast, float radius, const BinBuffers &b, int itemCap, cudaStream_t st);
cudaError_t launch_insert(const InsertParams &P, const InsertConfig &cfg, int grid, cudaStream_t st);
size_t insert_smem_bytes(const InsertConfig &cfg, int tableElems);
int insert_groups(const InsertConfig &cfg);      // 256-thread groups per insertion CTA
int insert_max_groups(const InsertConfig &cfg);  // the most groups a CTA of this variant holds
// Whether the kernel's table goes to shared memory beside the launch's brick accumulators (a
// lookup table of at most kLutSmemMax entries, or the Kaiser table, with room left); else it
// is read from global memory.
bool insert_lut_in_smem(const InsertConfig &cfg, int tableElems);
const void *insert_kernel_ptr(const InsertConfig &cfg);

// Records `msg` as the calling thread's fr_last_error() and returns `code`.
int set_last_error(int code, const char *msg);

constexpr size_t kSpacePrepBytes = 64;
constexpr size_t kSpaceRecBytes = 128;
constexpr size_t kWorkItemBytes = 16;

}// namespace frb
