// TEST INFRASTRUCTURE ONLY -- a launcher for the reference's own GPU insertion kernel.
//
// The reference's FRCUDA strategy compiles ProcessKernel (fr_cuda_kernels.cu:468-523) at run
// time through KTT with the tuning parameters of its default configuration
// (fr_cuda.cpp:32-39: BLOCK_DIM 16, SHARED_IMG 0, TILE 2, GRID_DIM_Z 1; the parameters the
// default leaves open take the first value of their lists, fr_cuda.cpp:100-111:
// SHARED_BLOB_TABLE 0, PRECOMPUTE_BLOB_VAL = lookup interpolation, BLOB_TABLE_SIZE_SQRT = the
// table size) and launches it with a grid of the volume face rounded up to the block
// (fr_cuda.cpp:211-224).  KTT is not available here, so oracle/Makefile compiles that same
// kernel source in place from the reference tree with nvcc for sm_100a, with those values as
// macros, into oracle/_ref/libfrcuda_ref.so, and this file launches it the way the launcher
// does.  It is timed beside the engine as the reference's GPU baseline; nothing in the
// product links it.
#ifndef BLOCK_DIM
#define BLOCK_DIM 16
#endif
#define TILE 2
#define SHARED_IMG 0
#define GRID_DIM_Z 1
#define SHARED_BLOB_TABLE 0
#define PRECOMPUTE_BLOB_VAL 1
#define BLOB_TABLE_SIZE_SQRT 10000
#include <libumpalumpa/operations/fourier_reconstruction/fr_cuda_kernels.cu>

#include <cuda_runtime.h>

// Inserts n_spaces traverse spaces (device, 112-byte TraverseSpace each) of `fft` (device,
// complex64 [n_proj][fft_y][fft_x]) into volume / weight (device, [vz][vy][vx]) with the
// reference's kernel on `stream`: kPrecise blob gather from the lookup table (device,
// table_elems == 10,000 floats).  `constants` is the reference's 32-byte Constants
// (AFR::CreateConstants).  Returns a cudaError_t value.
extern "C" int frcuda_ref_execute(void *volume, float *weight, unsigned long long vx, unsigned long long vy,
  const void *fft, unsigned long long fft_x, unsigned long long fft_y, unsigned long long n_proj,
  const void *spaces, int n_spaces, const float *table, unsigned long long table_elems,
  const void *constants, void *stream)
{
  if (table_elems != BLOB_TABLE_SIZE_SQRT) return int(cudaErrorInvalidValue);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemcpyToSymbolAsync(::constants, constants, sizeof(Constants), 0, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return int(e);
  const umpalumpa::data::Size size(fft_x, fft_y, 1, n_proj);
  const dim3 block(BLOCK_DIM, BLOCK_DIM);
  const dim3 grid(unsigned((vx + BLOCK_DIM - 1) / BLOCK_DIM), unsigned((vy + BLOCK_DIM - 1) / BLOCK_DIM), GRID_DIM_Z);
  ProcessKernel<0, false, true><<<grid, block, 0, st>>>(static_cast<float2 *>(volume), weight, size, n_spaces,
    static_cast<const TraverseSpace *>(spaces), static_cast<const float2 *>(fft), table, 0);
  return int(cudaGetLastError());
}
