/*
 * TEST INFRASTRUCTURE ONLY -- the oracle.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load it, and only as the checker.  The product never
 * links or calls it.
 *
 * A plain-C restatement of the reference's CPU Fourier-reconstruction path (FRCPU), in the
 * reference's own single-precision operation order, plus an FP64 variant of the same
 * algorithm.  Each function cites the reference file:line it restates (paths relative to the
 * reference project root).  The structs are byte-compatible with the reference's
 * TraverseSpace (112 B) and Constants (32 B).
 */
#ifndef FR_ORACLE_H
#define FR_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* libumpalumpa/operations/fourier_reconstruction/traverse_space.hpp:14-48 */
typedef struct or_traverse_space {
  int32_t minY, minX, minZ;
  int32_t maxY, maxX, maxZ;
  float maxDistanceSqr;
  int32_t dir; /* 0 = XY, 1 = XZ, 2 = YZ */
  float unitNormal[3];
  float topOrigin[3];
  float bottomOrigin[3];
  int32_t projectionIndex;
  float transformInv[3][3];
  float weight;
} or_traverse_space;

/* libumpalumpa/operations/fourier_reconstruction/constants.hpp:6-16 */
typedef struct or_constants {
  int32_t cMaxVolumeIndexX;
  int32_t cMaxVolumeIndexYZ;
  float cBlobRadius;
  float cOneOverBlobRadiusSqr;
  float cBlobAlpha;
  float cIw0;
  float cIDeltaSqrt;
  float cOneOverBessiOrderAlpha;
} or_constants;

/* interpolation: 0 = dynamic, 1 = lookup; type: 0 = fast (nearest), 1 = precise (blob) */
void or_make_constants(size_t vx, size_t vy, size_t tableElems, int order, float alpha,
  float radius, or_constants *out);
void or_fill_blob_table(float *table, size_t tableElems, int order, float alpha, float radius);
void or_compute_traverse_space(uint32_t imgSizeX, uint32_t imgSizeY, const float *transform9,
  uint32_t maxVolumeIndexX, uint32_t maxVolumeIndexYZ, int useFast, float blobRadius,
  float weight, or_traverse_space *out);

/* Single-precision restatement of FRCPU::Execute.  volume is interleaved complex64
 * [vz][vy][vx], weight is float [vz][vy][vx], fft is interleaved complex64 [n][fftY][fftX].
 * Accumulates (never zeroes).  Returns 0, or 1 when lookup is requested without a table. */
int or_fr_execute(float *volume, float *weight, size_t vx, size_t vy, size_t vz,
  const float *fft, size_t fftX, size_t fftY, const or_traverse_space *spaces, size_t nSpaces,
  const float *table, size_t tableElems, int interpolation, int order, int type, float alpha,
  float radius);

/* The same algorithm in FP64: float inputs are promoted, the blob table is rebuilt in double
 * with the same index rule, and volume/weight accumulate in double.  `threads` host threads
 * insert contiguous space ranges into private partials, added in thread order.  Accumulates
 * into volume/weight; returns 0, 1 (no table), 2 (out of memory) or 3 (thread start). */
int or_fr_execute_f64(double *volume, double *weight, size_t vx, size_t vy, size_t vz,
  const float *fft, size_t fftX, size_t fftY, const or_traverse_space *spaces, size_t nSpaces,
  size_t tableElems, int interpolation, int order, int type, float alpha, float radius, int threads);

/* The reference's float decisions with FP64 arithmetic after them: the voxel rotation and
 * rejection tests, the blob box, d^2, the table index (int)(d^2 cIDeltaSqrt + 0.5f) and the
 * blob weight (table entry, or the float Kaiser evaluation) are computed exactly as FRCPU
 * computes them in single precision (fr_cpu_kernels.hpp:70-152); every product with the
 * space weight and the pixel, and every sum, is taken in double.  It isolates accumulation
 * error from table-index choices.  Threads as in or_fr_execute_f64. */
int or_fr_execute_fd64(double *volume, double *weight, size_t vx, size_t vy, size_t vz,
  const float *fft, size_t fftX, size_t fftY, const or_traverse_space *spaces, size_t nSpaces,
  const float *table, size_t tableElems, int interpolation, int order, int type, float alpha,
  float radius, int threads);

/* Number of voxels that receive a contribution from each space (precise and fast). */
void or_count_slab_voxels(size_t vx, size_t vy, size_t vz, size_t fftX, size_t fftY,
  const or_traverse_space *spaces, size_t nSpaces, int type, float radius, int64_t *counts);

#ifdef __cplusplus
}
#endif
#endif
