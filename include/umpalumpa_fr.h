/*
 * umpalumpa_fr.h -- C-ABI of the B200 (sm_100a) Fourier-reconstruction insertion engine.
 *
 * This is the drop-in boundary for Umpalumpa's AFR operation
 * (libumpalumpa/operations/fourier_reconstruction/afr.hpp:35-55).  The engine inserts
 * centred half-plane FFTs of 2D projections into a complex64 Fourier volume and a float
 * weight volume with a Kaiser-Bessel blob (or nearest-pixel) gather, exactly as the
 * reference's FRCPU/FRCUDA do, and replaces the KTT-tuned FRCUDA strategy
 * (fr_cuda.cpp:71-236, fr_cuda_kernels.cu:468-523).  Paths are relative to the reference
 * project root.
 *
 * Conventions
 *  - Every function returns FR_OK (0) or a negative FR_E* status; fr_last_error() returns
 *    the calling thread's last message.  A C++ wrapper maps these onto the reference's
 *    bool/exception conventions (include/umpalumpa_fr_afr.hpp).
 *  - All payload pointers passed to fr_execute are device pointers (cudaMalloc or
 *    cudaMallocManaged).  The projection FFTs may also be host memory (pinned or pageable);
 *    they are then staged to the device inside the call, as FRCUDA's argument upload does.
 *  - fr_execute is asynchronous on the handle's stream (FRCUDA: RunKernelAsync,
 *    fr_cuda.cpp:227-229); call fr_synchronize before reading results.
 *  - Execute ACCUMULATES into volume and weight and never zeroes them
 *    (fr_cpu_kernels.hpp:149-151); zeroing is the caller's job.
 *  - One handle per stream/thread; a handle is not re-entrant (same as one reference
 *    operation instance per worker, fr_starpu.cpp:91-120).
 */
#ifndef UMPALUMPA_FR_H
#define UMPALUMPA_FR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FR_ABI_VERSION 1

/* ---- status codes ------------------------------------------------------------------- */
enum {
  FR_OK = 0,
  FR_E_INVALID = -1,    /* malformed argument or payload (reference: Init/Execute -> false) */
  FR_E_NOT_INIT = -2,   /* Execute before a successful Init (basic_operation.hpp:60-66)     */
  FR_E_MISMATCH = -3,   /* payload not equivalent to the Init reference (size.hpp:77-80)    */
  FR_E_NO_TABLE = -4,   /* lookup interpolation with an empty blob table (fr_cpu.cpp:27-29) */
  FR_E_CUDA = -5,       /* CUDA runtime failure (reference: CudaErrchk throws, cuda.cpp:7-14)*/
  FR_E_CAPACITY = -6,   /* internal work list overflow (reported at fr_synchronize)         */
  FR_E_UNSUPPORTED = -7 /* e.g. even-sized volume (fr_cuda.cpp:75), blob order without a
                           Fourier value (kaiser.hpp:74-80)                                 */
};

/* ---- settings: libumpalumpa/operations/fourier_reconstruction/settings.hpp:8-67 ------- */
enum { FR_INTERPOLATION_DYNAMIC = 0, FR_INTERPOLATION_LOOKUP = 1 };  /* settings.hpp:12 */
enum { FR_TYPE_FAST = 0, FR_TYPE_PRECISE = 1 };                     /* settings.hpp:14 */
enum { FR_DIR_XY = 0, FR_DIR_XZ = 1, FR_DIR_YZ = 2 };               /* traverse_space.hpp:24-28 */
/* Storage of the projection FFTs handed to fr_execute.  FP32 = interleaved complex64 (the
 * reference's only format).  BF16/FP16 = interleaved 2x16-bit complex with one float scale
 * per projection (value = stored * scale); accumulation stays FP32. */
enum { FR_STORAGE_FP32 = 0, FR_STORAGE_BF16 = 1, FR_STORAGE_FP16 = 2 };
/* Voxel accumulation: plain FP32 adds (reference behaviour) or FP32 with Kahan compensation
 * inside each on-chip brick accumulator (the compensation terms held in BF16). */
enum { FR_ACCUM_PLAIN = 0, FR_ACCUM_KAHAN = 1 };
/* Layout of the half-planes the insertion kernel reads (no reference counterpart).  The
 * payload handed to fr_execute is row-major [n][fft_y][fft_x] (the reference's layout) unless
 * the layout is FR_LAYOUT_BANDED.
 *   FR_LAYOUT_AUTO:   fr_execute copies the projections into bands (fr_band_projections) in
 *                     device memory of its own and inserts from the copy (at box 256 the
 *                     insertion is 12 % faster, the whole call 7 %), or reads the rows in
 *                     place where that memory cannot be had or the call inserts fewer spaces
 *                     than a third of the payload's projections;
 *   FR_LAYOUT_ROWS:   reads the caller's rows in place (no copy, no extra memory);
 *   FR_LAYOUT_BANDED: the payload is already banded (fr_band_projections, or fr_prep with
 *                     out_layout FR_LAYOUT_BANDED); fr_execute reads it in place.
 * Banded: the rows of each half-plane are grouped in bands of four, and each band is stored
 * column by column: pixel (y, x) of projection p at element
 * p * fr_band_plane_elems(fft_x, fft_y) + (y / 4) * 4 * P + 4 * x + y % 4, with the band pitch
 * P = fft_x rounded up to a multiple of 8; padding pixels are never read (fr_band_projections
 * writes zeros there, fr_prep leaves them as they were).  A warp's blob taps then touch
 * fewer cache lines.  Batched launches (fr_batch_execute) always insert from bands: they copy
 * row-major payloads (FR_LAYOUT_AUTO or _ROWS) and read FR_LAYOUT_BANDED payloads in place. */
enum { FR_LAYOUT_AUTO = 0, FR_LAYOUT_ROWS = 1, FR_LAYOUT_BANDED = 2 };

typedef struct fr_settings {
  int32_t interpolation;  /* FR_INTERPOLATION_*; reference default kDynamic (settings.hpp:62) */
  int32_t blob_order;     /* 0..4 (blob_order.hpp:5); only 0 has a Fourier value             */
  int32_t type;           /* FR_TYPE_*; reference default kFast (settings.hpp:64)            */
  float alpha;            /* Kaiser-Bessel alpha, default 15                                  */
  float blob_radius;      /* default 1.9                                                      */
  float max_resolution;   /* fraction of the box inserted; the traverse-space image size is
                             max_resolution * box.  0.5 reproduces the reference (which has no
                             such field and uses imgSizeX = Y/2, afr_common.hpp:50-68)        */
  int32_t storage;        /* FR_STORAGE_*                                                     */
  int32_t accumulation;   /* FR_ACCUM_*                                                       */
  int32_t layout;         /* FR_LAYOUT_*                                                      */
} fr_settings;

/* Fills the reference defaults (interpolation dynamic, order 0, type fast, alpha 15,
 * radius 1.9) plus max_resolution 0.5, FP32 storage, plain accumulation, layout auto. */
void fr_settings_default(fr_settings *s);

/* ---- POD types, byte-compatible with the reference ---------------------------------- */
/* traverse_space.hpp:14-48, 112 bytes */
typedef struct fr_traverse_space {
  int32_t minY, minX, minZ;
  int32_t maxY, maxX, maxZ;
  float maxDistanceSqr;
  int32_t dir;                 /* FR_DIR_* */
  float unitNormal[3];
  float topOrigin[3];
  float bottomOrigin[3];
  int32_t projectionIndex;
  float transformInv[3][3];
  float weight;
} fr_traverse_space;

/* constants.hpp:6-16, 32 bytes */
typedef struct fr_constants {
  int32_t cMaxVolumeIndexX;
  int32_t cMaxVolumeIndexYZ;
  float cBlobRadius;
  float cOneOverBlobRadiusSqr;
  float cBlobAlpha;
  float cIw0;
  float cIDeltaSqrt;
  float cOneOverBessiOrderAlpha;
} fr_constants;

/* Sizes of the AFR payloads (afr.hpp:13-33).  An Execute payload is equivalent to the Init
 * one when all sizes match and its count is <= the Init count (payload.hpp:60-63). */
typedef struct fr_dims {
  uint64_t fft_x;          /* half-plane columns X (B/2+1 for a B x B projection)      */
  uint64_t fft_y;          /* half-plane rows Y (B)                                    */
  uint64_t n_projections;  /* FFT payload count N                                      */
  uint64_t volume_x;       /* volume sizes (B+1); volume_x must be odd (fr_cuda.cpp:75) */
  uint64_t volume_y;
  uint64_t volume_z;
  uint64_t n_spaces;       /* traverse-space payload count                             */
  uint64_t table_elems;    /* blob table entries (10,000 in the reference) or 0        */
} fr_dims;

typedef struct fr_handle fr_handle;

/* ---- operation lifecycle: basic_operation.hpp:28-105 ---------------------------------- */

/* FRCUDA(workerId, streams) (fr_cuda.hpp:8-20, ktt_base.hpp:19-34).  `stream` is a
 * cudaStream_t (NULL = the legacy default stream) on CUDA device `device`. */
int fr_create(int device, void *stream, fr_handle **out);
int fr_destroy(fr_handle *h);

/* AFR::Init (basic_operation.hpp:28-48 + afr.hpp:47-54 + fr_cuda.cpp:71-159): validates the
 * payload sizes and settings, sizes the engine's scratch and picks launch parameters (from
 * the tuning cache when one is loaded). */
int fr_init(fr_handle *h, const fr_dims *dims, const fr_settings *settings);

/* AFR::Execute (basic_operation.hpp:60-66 + fr_cuda.cpp:163-236).  Inserts `n_spaces`
 * traverse spaces; each addresses projection `projectionIndex` of `fft`, which holds
 * `n_projections` half-planes [n][fft_y][fft_x].  `scales` (one float per projection) is
 * required for BF16/FP16 storage and ignored for FP32.  `table` (device, table_elems floats)
 * is required for lookup interpolation.  Asynchronous. */
int fr_execute(fr_handle *h, const void *fft, const float *scales, uint64_t n_projections,
  void *volume, float *weight, const fr_traverse_space *spaces, uint64_t n_spaces,
  const float *table);

/* AFR::Synchronize (fr_cuda.cpp:241-244): waits for the handle's work and reports any
 * deferred device-side error (e.g. FR_E_CAPACITY). */
int fr_synchronize(fr_handle *h);

/* BasicOperation::Cleanup (basic_operation.hpp:72-80): drops Init state and scratch. */
int fr_cleanup(fr_handle *h);

/* BasicOperation::GetUsedBytes (basic_operation.hpp:100): device bytes held as scratch
 * (binning buffers, staging of host inputs, the banded copy of the projections). */
uint64_t fr_used_bytes(const fr_handle *h);

/* The calling thread's last error message ("" when none). */
const char *fr_last_error(void);

/* ---- static helpers of AFR ----------------------------------------------------------- */

/* AFR::CreateConstants (afr.cpp:6-19).  Host computation. */
int fr_make_constants(const fr_dims *dims, const fr_settings *settings, fr_constants *out);

/* AFR::FillBlobTable (afr.cpp:22-34) as a GPU kernel with FP64 Bessel functions.  `table`
 * is a device (or managed) pointer of `table_elems` floats; asynchronous on `stream`. */
int fr_fill_blob_table(float *table, uint64_t table_elems, const fr_settings *settings,
  void *stream);

/* ComputeTraverseSpace (traverse_space_generator.hpp:94-145) as a GPU kernel with FP64
 * setup, one space per 3x3 row-major rotation.  `rotations` (9*n floats) and `out` are
 * device pointers.  Space i gets projectionIndex = first_projection_index + i.  The image
 * size used for the cuboid is (img_size_x, img_size_y); the reference passes Y/2 for x
 * (afr_common.hpp:60-63), which fr_settings.max_resolution * box reproduces. */
int fr_compute_traverse_spaces(const float *rotations, uint64_t n, uint32_t img_size_x,
  uint32_t img_size_y, uint32_t max_volume_index_x, uint32_t max_volume_index_yz,
  int use_fast, float blob_radius, float weight, int32_t first_projection_index,
  fr_traverse_space *out, void *stream);
/* Symmetry expansion (examples/fourier_reconstruction/fr.cpp:293-309): n projections under
 * n_symmetries row-major 3x3 operations S_k give n * n_symmetries spaces, image-major: space
 * i * n_symmetries + k uses the transform R_i * S_k (single-precision product in the
 * reference's order, fr.hpp:123-130) and projectionIndex first_projection_index + i.  All
 * pointers are device memory. */
int fr_compute_traverse_spaces_sym(const float *rotations, uint64_t n, const float *symmetries,
  uint32_t n_symmetries, uint32_t img_size_x, uint32_t img_size_y, uint32_t max_volume_index_x,
  uint32_t max_volume_index_yz, int use_fast, float blob_radius, float weight,
  int32_t first_projection_index, fr_traverse_space *out, void *stream);

/* ---- input preparation: FFT + Fourier processing straight into the insertion layout ------
 * Replaces the two reference operations the example driver runs before insertion: AFFT, a
 * batched real-to-complex cuFFT (fft_cuda.cpp:92-95), then AFP, which crops, shifts, centres
 * and normalises the spectra into a new buffer (scaleFFT2DKernel, fp_cuda_kernels.cu:9-61;
 * ScaleFFT2DCPU, fp_cpu_kernels.hpp:8-41; settings as in examples/fourier_reconstruction/
 * fr.cpp:166-204).  Here the images are transformed in large chunks and one kernel per chunk
 * reads each spectrum once and writes the processed half-planes straight into the layout
 * fr_execute reads -- optionally quantised to BF16/FP16 with a per-projection scale exactly as
 * fr_quantize_projections does -- instead of separate processing and quantisation passes. */
typedef struct fr_prep_settings {
  uint32_t size_x, size_y;  /* spatial image size (the FFT size), both even                   */
  uint32_t out_x, out_y;    /* output half-plane, out_x <= size_x/2+1, out_y <= size_y, out_y
                               even (0: the full size_x/2+1 x size_y)                          */
  int32_t normalize;        /* x 1/(size_x size_y)       (AFP Settings::SetNormalize)          */
  int32_t center;           /* x (1 - 2((x + y) & 1))    (SetCenter)                           */
  int32_t shift;            /* output row (y + out_y/2) mod out_y  (SetShift)                  */
  int32_t crop_freq;        /* zero coefficients whose squared digital frequency exceeds
                               max_freq (SetMaxFreq; FPCPU compares |f|^2 with the value
                               itself, fp_cpu.cpp:43)                                          */
  float max_freq;
  int32_t storage;          /* FR_STORAGE_FP32 (complex64) or _BF16 / _FP16 with scales        */
  uint32_t chunk;           /* images per FFT chunk of the cuFFT route (0: about 1 GiB of
                               spectra)                                                       */
  uint32_t fft;             /* FR_PREP_FFT_*: the route of the FFT                             */
  uint32_t out_layout;      /* FR_LAYOUT_BANDED: half-planes written in bands (fr_execute with
                               layout FR_LAYOUT_BANDED reads them in place); else row-major     */
} fr_prep_settings;

/* FR_PREP_FFT_FUSED: square images of side 64, 128 or 256 go through the engine's own FFT fused
 * with the processing (each image read once, each half-plane written once, the row spectra kept
 * in an L2-resident scratch); other sizes take the cuFFT route.  FR_PREP_FFT_CUFFT: cuFFT R2C
 * into a chunk of spectra, then one processing pass.  FR_PREP_FFT_AUTO (0, the default): the
 * fused route for FP32 output, the cuFFT route for 16-bit output. */
enum { FR_PREP_FFT_AUTO = 0, FR_PREP_FFT_CUFFT = 1, FR_PREP_FFT_FUSED = 2 };

typedef struct fr_prep fr_prep;
/* Plans the FFT and allocates the chunk workspace on `device` / `stream` (a cudaStream_t). */
int fr_prep_create(int device, void *stream, const fr_prep_settings *settings, fr_prep **out);
int fr_prep_destroy(fr_prep *p);
/* images: device float [n][size_y][size_x]; out: device [n][out_y][out_x] complex in the
 * storage type, or n banded planes of fr_band_plane_elems(out_x, out_y) with out_layout
 * FR_LAYOUT_BANDED; scales: device float [n] (16-bit storage, else NULL).  Asynchronous on the
 * handle's stream. */
int fr_prep_execute(fr_prep *p, const float *images, uint64_t n, void *out, float *scales);

/* Input preparation for 16-bit storage (no reference counterpart): converts `n` complex64
 * half-planes of fft_x * fft_y (device memory) to 2 x bf16 / 2 x fp16 complex in `out` with
 * one float scale per projection in `scales` (value = stored * scale; the largest component
 * of each projection is stored as 2^14).  Asynchronous on `stream`. */
int fr_quantize_projections(const void *fft, uint64_t n, uint64_t fft_x, uint64_t fft_y, int storage,
  void *out, float *scales, void *stream);

/* Elements (pixels) of one banded half-plane of fft_x * fft_y (see FR_LAYOUT_BANDED). */
uint64_t fr_band_plane_elems(uint64_t fft_x, uint64_t fft_y);
/* Copies `n` row-major half-planes of fft_x * fft_y pixels of `storage` (device memory) into
 * the banded layout at `out` (n * fr_band_plane_elems pixels, device memory).  Asynchronous
 * on `stream`. */
int fr_band_projections(const void *fft, uint64_t n, uint64_t fft_x, uint64_t fft_y, int storage, void *out,
  void *stream);

/* ---- engine introspection (no reference counterpart; used by the tuner and tests) ----- */

/* Launch parameters of the insertion kernel, picked at fr_init / fr_batch_init (or by the
 * autotuner): brick edge (voxels), traverse spaces per work item, CTAs per SM, and 256-thread
 * groups per CTA (the thread-block shape; each group accumulates one brick in shared memory,
 * the groups of a CTA share one copy of the blob table).  These are what the reference's KTT
 * search varies for FRCUDA (BLOCK_DIM, TILE, GRID_DIM_Z, fr_cuda.cpp:100-157). */
typedef struct fr_launch_params {
  int32_t brick;
  int32_t item_capacity;
  int32_t ctas_per_sm;
  int32_t groups;
} fr_launch_params;

int fr_get_launch_params(const fr_handle *h, fr_launch_params *out);
/* Overrides the launch parameters (0 keeps a field) and re-sizes the handle's scratch;
 * takes effect at the next fr_execute / fr_batch_execute. */
int fr_set_launch_params(fr_handle *h, const fr_launch_params *p);

/* Per-call statistics of the last fr_execute, read after fr_synchronize: number of
 * (brick, projection) pairs and work items the binning produced. */
typedef struct fr_exec_stats {
  uint64_t pairs;     /* (brick, space) pairs binned */
  uint64_t items;     /* work items executed */
  uint64_t chunks;    /* internal chunks (binning + insertion rounds) */
  uint64_t launches;  /* engine kernels launched by the call */
} fr_exec_stats;

int fr_get_exec_stats(const fr_handle *h, fr_exec_stats *out);

/* Per-phase device time, measured with CUDA events on the handle's stream around every
 * binning round and every insertion launch while profiling is on (off by default).
 * Accumulates over fr_execute calls until reset. */
typedef struct fr_phase_times {
  double binning_ms;
  double insert_ms;
  uint64_t insert_launches;
  uint64_t insert_spaces;   /* traverse spaces covered by the timed insertion launches */
} fr_phase_times;

int fr_set_profiling(fr_handle *h, int enable);
int fr_get_phase_times(fr_handle *h, fr_phase_times *out, int reset);

/* ---- batched jobs -----------------------------------------------------------------------
 * No counterpart in the reference (which runs one operation per job).  Several independent
 * reconstructions -- each with its own projections, traverse spaces, volume and weights, of
 * any box size -- are binned together and inserted by one persistent kernel launch, so small
 * and uneven jobs share the GPU instead of queueing behind each other.  All jobs share the
 * handle's settings and blob table. */
typedef struct fr_job {
  const void *fft;                 /* device: n_projections half-planes [n][fft_y][fft_x]  */
  const float *scales;             /* device: per-projection scales (16-bit storage only)  */
  uint64_t n_projections;
  void *volume;                    /* device: complex64 [volume_z][volume_y][volume_x]     */
  float *weight;                   /* device: float [volume_z][volume_y][volume_x]         */
  const fr_traverse_space *spaces; /* device: n_spaces traverse spaces                     */
  uint64_t n_spaces;
  uint64_t fft_x, fft_y;
  uint64_t volume_x, volume_y, volume_z;
} fr_job;

typedef struct fr_batch_limits {
  uint64_t max_jobs;         /* jobs per fr_batch_execute                                   */
  uint64_t max_spaces;       /* traverse spaces per fr_batch_execute, all jobs together      */
  uint64_t max_bricks;       /* 16^3-voxel bricks per call, all jobs: sum of ceil(v/16)^3    */
  uint64_t max_volume_side;  /* largest volume side of any job                               */
  uint64_t table_elems;      /* blob table entries (lookup interpolation) or 0               */
} fr_batch_limits;

enum { FR_BATCH_GRAPH = 1 }; /* capture the call in a CUDA graph; replay it while the job
                                table stays the same (needs a non-default stream)            */

/* Sizes the batch scratch (allocates); the handle then serves fr_batch_execute. */
int fr_batch_init(fr_handle *h, const fr_batch_limits *limits, const fr_settings *settings);
/* Inserts every job's spaces into its volume and weights.  Asynchronous; fr_synchronize waits
 * and reports deferred device errors.  `table` (device) for lookup interpolation. */
int fr_batch_execute(fr_handle *h, const fr_job *jobs, uint64_t n_jobs, const float *table, int flags);

/* ---- autotuning -------------------------------------------------------------------------
 * Replaces the reference's KTT tuning of FRCUDA: KTT searches the kernel's launch space on the
 * first Execute of a strategy, blocking (fr_cuda.cpp:100-157, tunable_strategy.cpp:64-104), and
 * the StrategyManager keeps the best configuration in one tuning file per strategy, reused by
 * every equal strategy (strategy_manager.cpp:14-83, ktt_strategy_base.hpp:110-134).  Here the
 * search is over fr_launch_params -- groups per CTA x CTAs per SM x traverse spaces per work
 * item, every combination that fits on an SM -- each timed with CUDA events on the handle's
 * stream, and the best is stored in a tuning file named by the strategy key: device name and SM
 * count, payload sizes (for a batch: its limits), settings, and the size class of the job. */
enum {
  FR_TUNING_OFF = 0,        /* defaults, no tuning files (the default)                        */
  FR_TUNING_CACHED = 1,     /* fr_init / fr_batch_init use the tuning file of an equal strategy */
  FR_TUNING_ON_EXECUTE = 2  /* as CACHED; without a file, the first fr_execute tunes on its own
                               inputs first (blocking, into scratch volumes) and writes one   */
};

typedef struct fr_tune_report {
  fr_launch_params best;    /* the parameters applied                                         */
  double best_ms;           /* sample insertion time with them                                */
  double default_ms;        /* sample insertion time with the defaults                        */
  uint32_t trials;          /* configurations timed (0: taken from a tuning file)             */
  uint32_t sample_spaces;   /* traverse spaces in the timed sample                            */
  char key[256];            /* strategy key of the tuning file                                */
} fr_tune_report;

/* Sets the handle's tuning approach (FR_TUNING_*) and tuning-file directory (NULL: the
 * environment variable UMPALUMPA_B200_TUNING_DIR, else $HOME/.cache/umpalumpa_b200).  Takes
 * effect at the next fr_init / fr_batch_init / fr_execute. */
int fr_set_tuning(fr_handle *h, int approach, const char *directory);
/* Tunes an initialised single-job handle now on a sample of the given job (the arguments of
 * fr_execute without volume and weight: the trials insert into scratch volumes), applies the
 * best parameters and writes the tuning file (unless the approach is FR_TUNING_OFF). */
int fr_autotune(fr_handle *h, const void *fft, const float *scales, uint64_t n_projections,
                const fr_traverse_space *spaces, uint64_t n_spaces, const float *table, fr_tune_report *report);
/* The same for a batched handle on a job table (each job's traverse spaces are sampled in
 * proportion; the jobs' volume and weight are not touched). */
int fr_batch_autotune(fr_handle *h, const fr_job *jobs, uint64_t n_jobs, const float *table,
                      fr_tune_report *report);
/* The strategy key and tuning-file path the handle's current Init maps to. */
int fr_tuning_key(const fr_handle *h, char *key, uint64_t key_bytes, char *path, uint64_t path_bytes);

/* ---- insertion without any memory allocation ------------------------------------------
 * No counterpart in the reference.  For callers that are not allowed to allocate device
 * memory -- a host application that owns the GPU through its own pool or memory budget, a
 * latency-critical thread where cudaMalloc may block on the driver, a framework whose
 * allocator must account for every byte -- this one call inserts `n_spaces` traverse spaces
 * like fr_create + fr_init + fr_execute + fr_synchronize, but allocates nothing: its
 * working memory is a fixed 32 MiB array inside the library (present on every GPU that
 * loads the library, until the process exits).  All payloads must be device or managed
 * memory; the call returns when the insertion has finished on `stream` (a cudaStream_t).
 *  - Every call looks up the array's device address with `device` current (so a reset
 *    device or a reloaded library never leaves a stale address); the first call on a device
 *    also loads the library's kernels there, so make it before any stream capture.
 *  - The caller's current device is restored before the call returns.
 *  - n_projections and n_spaces may not exceed dims->n_projections / dims->n_spaces
 *    (FR_E_MISMATCH), nor 2^31 - 1 (FR_E_UNSUPPORTED).
 *  - The kernel modes are fr_execute's, including the interpolated Kaiser table of dynamic
 *    interpolation above alpha 15 (built in the array by every such call).  There is no room
 *    for a banded copy: the half-planes are read as given, row-major unless settings->layout
 *    is FR_LAYOUT_BANDED.
 *  - Jobs larger than the array are processed in several internal rounds; volumes whose
 *    per-brick tables alone do not fit (beyond about 1000^3 voxels) return FR_E_UNSUPPORTED.
 *  - All calls on a device share the array: calls whose GPU work overlaps (e.g. issued from
 *    two threads or on two streams at once) race and must be serialised by the caller.
 * Accumulates into volume and weight like fr_execute; errors are reported as FR_E_* and
 * fr_last_error(). */
int fr_insert_noalloc(int device, void *stream, const fr_dims *dims, const fr_settings *settings,
  const void *fft, const float *scales, uint64_t n_projections, void *volume, float *weight,
  const fr_traverse_space *spaces, uint64_t n_spaces, const float *table);

#ifdef __cplusplus
}
#endif
#endif /* UMPALUMPA_FR_H */
