// Input preparation for insertion: real-to-complex FFT of the projection images and the
// reference's Fourier processing -- crop, row shift, centring, normalisation, optional
// frequency crop -- writing the half-planes in the layout fr_execute reads, optionally quantised
// to 16 bits with a per-projection scale.  Square images of side 64, 128 or 256 go through the
// engine's own FFT fused with the processing (fr_prep_fft.cuh); other sizes, or
// FR_PREP_FFT_CUFFT, through cuFFT and one processing pass (below).  The C-ABI is declared in
// include/umpalumpa_fr.h.
//
// The reference runs this as two operations with a full buffer between them: AFFT's batched
// cuFFT (libumpalumpa/operations/fourier_transformation/fft_cuda.cpp:92-95) writes every
// spectrum and AFP's scaleFFT2DKernel (fourier_processing/fp_cuda_kernels.cu:9-61) makes a
// second buffer from it, which a 16-bit store would quantise in a third pass.  Here the images
// go through the FFT in chunks of about 1 GiB of spectra (large batches keep cuFFT at full rate;
// chunks sized to stay in L2 measured 25 % slower), and one kernel per chunk reads each
// spectrum once and writes the finished half-planes, quantised if asked.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <new>
#include <string>

#include "fr_device_guard.h"
#include "fr_kernels.h"
#include "fr_prep_fft.cuh"
#include "umpalumpa_fr.h"

#include <cmath>
#include <vector>

namespace {

int fail(int code, const std::string &msg) { return frb::set_last_error(code, msg.c_str()); }

constexpr size_t kChunkBytes = size_t(1) << 30;  // spectra bytes per FFT chunk
constexpr int kThreads = 512;

// Idx2Freq (fourier_processing/fp_common_kernels.hpp:13-20): digital frequency of index idx.
__device__ __forceinline__ float idx2freq(int idx, int size)
{
  if (size <= 1) return 0.f;
  const float t = idx <= size / 2 ? float(idx) : __fsub_rn(float(idx), float(size));
  return __fdiv_rn(t, float(size));
}

struct PrepArgs {
  const float2 *spectra;  // chunk of [inY][inX] spectra
  int inX, inY;           // spectrum size: size_x/2+1 x size_y
  int spX, spY;           // spatial size
  int outX, outY;
  int normalize, center, shift, crop;
  float maxFreq, norm;
  void *out;              // [n][outY][outX] complex in the storage type, or n banded planes
  float *scales;
  int64_t first;          // index of the chunk's first image in `out`
  int bandStride;         // banded output: elements per 4-row band (frb::band_stride); rows: 0
  int64_t outPlane;       // elements per output plane
};

// Output coefficient (y, x) (y before the row shift) of one spectrum, as ScaleFFT2DCPU computes
// it (fp_cpu_kernels.hpp:24-36): source row, frequency crop, then normalisation and centring,
// each product rounded separately.
__device__ __forceinline__ float2 processed_yx(const PrepArgs &a, const float2 *S, int y, int x)
{
  const int origY = y <= a.outY / 2 ? y : a.inY - (a.outY - y);
  float2 v = S[size_t(origY) * a.inX + x];
  if (a.crop) {
    const float fx = idx2freq(x, a.spX), fy = idx2freq(origY, a.spY);
    if (__fadd_rn(__fmul_rn(fx, fx), __fmul_rn(fy, fy)) > a.maxFreq) v = make_float2(0.f, 0.f);
  }
  if (a.normalize) v = make_float2(__fmul_rn(v.x, a.norm), __fmul_rn(v.y, a.norm));
  if (a.center) {
    const float c = float(1 - 2 * ((x + y) & 1));
    v = make_float2(__fmul_rn(v.x, c), __fmul_rn(v.y, c));
  }
  return v;
}

// Output coefficient e of one image in the order it is stored: row-major over the shifted
// rows, or banded (band, column, row within the band; padding positions return false).
__device__ __forceinline__ bool processed(const PrepArgs &a, const float2 *S, int e, float2 &v)
{
  int row, x;
  if (a.bandStride) {
    const int b = e / a.bandStride, r = e - b * a.bandStride;
    x = r >> 2;
    row = 4 * b + (r & 3);
    if (x >= a.outX || row >= a.outY) return false;
  } else {
    row = e / a.outX;
    x = e - row * a.outX;
  }
  const int h = a.outY / 2;  // the shift moves row y to (y + h) mod outY (outY even)
  const int y = a.shift ? (row >= h ? row - h : row + h) : row;
  v = processed_yx(a, S, y, x);
  return true;
}

// One CTA per image of the chunk.  16-bit storage: a first pass finds the largest |re|, |im|
// of the processed coefficients and the scale max / 2^14 (1 for a zero image), exactly as
// fr_quantize_projections does; the second pass stores value / scale rounded to nearest.
template<int STORAGE>
__global__ void __launch_bounds__(kThreads) prep_kernel(PrepArgs a)
{
  const int img = blockIdx.x;
  const float2 *S = a.spectra + size_t(img) * a.inX * a.inY;
  const int elems = int(a.outPlane);
  const int64_t o = a.first + img;
  if (STORAGE == FR_STORAGE_FP32) {
    float2 *O = static_cast<float2 *>(a.out) + o * a.outPlane;
    for (int e = threadIdx.x; e < elems; e += kThreads) {
      float2 v;
      if (processed(a, S, e, v)) O[e] = v;
    }
    return;
  }
  float m = 0.f;
  for (int e = threadIdx.x; e < elems; e += kThreads) {
    float2 v;
    if (processed(a, S, e, v)) m = fmaxf(m, fmaxf(fabsf(v.x), fabsf(v.y)));
  }
  for (int s = 16; s > 0; s >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, s));
  __shared__ float wm[kThreads / 32];
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < kThreads / 32 ? wm[threadIdx.x] : 0.f;
    for (int s = 8; s > 0; s >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, s));
    if (threadIdx.x == 0) wm[0] = m;
  }
  __syncthreads();
  const float scale = wm[0] > 0.f ? wm[0] / 16384.f : 1.f;
  const float inv = 1.f / scale;
  if (threadIdx.x == 0) a.scales[o] = scale;
  for (int e = threadIdx.x; e < elems; e += kThreads) {
    float2 v;
    if (!processed(a, S, e, v)) continue;
    const size_t d = size_t(o) * a.outPlane + e;
    if (STORAGE == FR_STORAGE_BF16)
      static_cast<__nv_bfloat162 *>(a.out)[d] = __floats2bfloat162_rn(v.x * inv, v.y * inv);
    else
      static_cast<__half2 *>(a.out)[d] = __floats2half2_rn(v.x * inv, v.y * inv);
  }
}

bool host_memory(const void *p)
{
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return true;
  }
  return at.type == cudaMemoryTypeHost || at.type == cudaMemoryTypeUnregistered;
}

}// namespace

struct fr_prep {
  int device = 0;
  cudaStream_t stream = nullptr;
  fr_prep_settings s{};
  int chunk = 0;
  cufftHandle plan = 0, tail = 0;
  int tail_batch = 0;
  float2 *spectra = nullptr;
  // fused route: side N, one scratch of (N/2 + 1) x N per persistent CTA, the twiddle table
  int fused = 0;
  int ctas = 0;
  float2 *scratch = nullptr;
  float2 *twiddles = nullptr;
};

namespace {

// Side of the fused route for these settings (0: cuFFT route).  FR_PREP_FFT_AUTO takes the
// fused route for FP32 output only: with 16-bit output its extra transpose pass through the
// scratch made it slower than the cuFFT route (1.96 M against 2.49 M box-256 images/s on a
// B200, FP32 2.95 M against 2.92 M).
int fused_side(const fr_prep_settings &s)
{
  if (s.fft == FR_PREP_FFT_CUFFT || s.size_x != s.size_y) return 0;
  if (s.fft == FR_PREP_FFT_AUTO && s.storage != FR_STORAGE_FP32) return 0;
  return (s.size_x == 64 || s.size_x == 128 || s.size_x == 256) ? int(s.size_x) : 0;
}

template<int N> cudaError_t launch_fused(fr_prep *p, const frb::prepfft::Args &a)
{
  const size_t smem = frb::prepfft::smem_bytes<N>();
  const int grid = std::min(a.n, p->ctas);
  cudaError_t e;
  switch (p->s.storage) {
  case FR_STORAGE_BF16:
    e = cudaFuncSetAttribute(frb::prepfft::prep_fft_kernel<N, FR_STORAGE_BF16>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e == cudaSuccess)
      frb::prepfft::prep_fft_kernel<N, FR_STORAGE_BF16><<<grid, frb::prepfft::kThreads, smem, p->stream>>>(a);
    break;
  case FR_STORAGE_FP16:
    e = cudaFuncSetAttribute(frb::prepfft::prep_fft_kernel<N, FR_STORAGE_FP16>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e == cudaSuccess)
      frb::prepfft::prep_fft_kernel<N, FR_STORAGE_FP16><<<grid, frb::prepfft::kThreads, smem, p->stream>>>(a);
    break;
  default:
    e = cudaFuncSetAttribute(frb::prepfft::prep_fft_kernel<N, FR_STORAGE_FP32>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e == cudaSuccess)
      frb::prepfft::prep_fft_kernel<N, FR_STORAGE_FP32><<<grid, frb::prepfft::kThreads, smem, p->stream>>>(a);
    break;
  }
  return e == cudaSuccess ? cudaGetLastError() : e;
}

}// namespace

static int plan_for(fr_prep *p, int batch, cufftHandle *h)
{
  int dims[2] = { int(p->s.size_y), int(p->s.size_x) };
  cufftResult r = cufftPlanMany(h, 2, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_R2C, batch);
  if (r == CUFFT_SUCCESS) r = cufftSetStream(*h, p->stream);
  if (r != CUFFT_SUCCESS) {
    if (*h) cufftDestroy(*h);
    *h = 0;
    return fail(FR_E_CUDA, "cuFFT plan failed (cufftResult " + std::to_string(int(r)) + ")");
  }
  return FR_OK;
}

extern "C" {

int fr_prep_destroy(fr_prep *p)
{
  if (!p) return FR_OK;
  frb::DeviceGuard guard(p->device);
  if (p->stream) cudaStreamSynchronize(p->stream);
  if (p->plan) cufftDestroy(p->plan);
  if (p->tail) cufftDestroy(p->tail);
  if (p->spectra) cudaFree(p->spectra);
  if (p->scratch) cudaFree(p->scratch);
  if (p->twiddles) cudaFree(p->twiddles);
  delete p;
  return FR_OK;
}

int fr_prep_create(int device, void *stream, const fr_prep_settings *s, fr_prep **out)
{
  if (!out || !s) return fail(FR_E_INVALID, "NULL argument");
  *out = nullptr;
  if (s->size_x < 2 || s->size_y < 2 || s->size_x % 2 || s->size_y % 2)
    return fail(FR_E_UNSUPPORTED, "image sizes must be even and at least 2 (the centring assumes even sizes)");
  if (s->size_x > 16384 || s->size_y > 16384) return fail(FR_E_UNSUPPORTED, "image too large");
  const uint32_t fullX = s->size_x / 2 + 1;
  const uint32_t outX = s->out_x ? s->out_x : fullX, outY = s->out_y ? s->out_y : s->size_y;
  if (outX > fullX || outY > s->size_y || outY % 2 || outY < 2)
    return fail(FR_E_UNSUPPORTED, "output half-plane must fit the spectrum and have an even row count");
  if (s->storage < FR_STORAGE_FP32 || s->storage > FR_STORAGE_FP16) return fail(FR_E_INVALID, "unknown storage");
  if (s->fft != FR_PREP_FFT_AUTO && s->fft != FR_PREP_FFT_FUSED && s->fft != FR_PREP_FFT_CUFFT)
    return fail(FR_E_INVALID, "unknown FFT route");
  if (s->out_layout > FR_LAYOUT_BANDED) return fail(FR_E_INVALID, "unknown output layout");
  frb::DeviceGuard guard(device);
  if (guard.err != cudaSuccess) {
    cudaGetLastError();
    return fail(FR_E_CUDA, "no such CUDA device");
  }
  fr_prep *p = new (std::nothrow) fr_prep();
  if (!p) return fail(FR_E_INVALID, "out of host memory");
  p->device = device;
  p->stream = static_cast<cudaStream_t>(stream);
  p->s = *s;
  p->s.out_x = outX;
  p->s.out_y = outY;

  int rc = FR_OK;
  p->fused = fused_side(*s);
  if (p->fused) {
    // persistent CTAs (kCtasPerSm per SM), each with its own column-major scratch of the row spectra
    const int N = p->fused;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) sms = 1;
    p->ctas = std::max(1, sms) * frb::prepfft::kCtasPerSm;
    std::vector<float2> tw(N);
    for (int t = 0; t < N; ++t) {
      const double a = -2.0 * 3.14159265358979323846 * double(t) / double(N);
      tw[t] = make_float2(float(std::cos(a)), float(std::sin(a)));
    }
    const size_t scratchBytes = size_t(p->ctas) * size_t(N / 2 + 1) * N * sizeof(float2);
    if (cudaMalloc(reinterpret_cast<void **>(&p->scratch), scratchBytes) != cudaSuccess
        || cudaMalloc(reinterpret_cast<void **>(&p->twiddles), N * sizeof(float2)) != cudaSuccess
        || cudaMemcpy(p->twiddles, tw.data(), N * sizeof(float2), cudaMemcpyHostToDevice) != cudaSuccess) {
      cudaGetLastError();
      rc = fail(FR_E_CUDA, "cannot allocate the FFT workspace");
    }
  } else {
    const size_t specBytes = size_t(fullX) * s->size_y * sizeof(float2);
    p->chunk = s->chunk ? int(std::min<uint32_t>(s->chunk, 1u << 16))
                        : int(std::max<size_t>(1, std::min<size_t>(16384, kChunkBytes / specBytes)));
    rc = plan_for(p, p->chunk, &p->plan);
    if (!rc && cudaMalloc(reinterpret_cast<void **>(&p->spectra), specBytes * p->chunk) != cudaSuccess) {
      cudaGetLastError();
      rc = fail(FR_E_CUDA, "cannot allocate the spectrum workspace");
    }
  }
  if (rc) {
    const std::string m = fr_last_error();
    fr_prep_destroy(p);
    return fail(rc, m);
  }
  *out = p;
  return FR_OK;
}

int fr_prep_execute(fr_prep *p, const float *images, uint64_t n, void *out, float *scales)
{
  if (!p) return fail(FR_E_INVALID, "handle is NULL");
  if (n == 0) return FR_OK;
  if (!images || !out) return fail(FR_E_INVALID, "NULL argument");
  frb::DeviceGuard guard(p->device);
  if (guard.err != cudaSuccess) return fail(FR_E_CUDA, "cudaSetDevice failed");
  const bool scaled = p->s.storage != FR_STORAGE_FP32;
  if (scaled != (scales != nullptr)) return fail(FR_E_INVALID, "scales go with BF16/FP16 storage only");
  if (host_memory(images) || host_memory(out) || (scales && host_memory(scales)))
    return fail(FR_E_INVALID, "images, output and scales must be device memory");
  const bool banded = p->s.out_layout == FR_LAYOUT_BANDED;
  if (p->fused) {
    if (n > uint64_t(INT32_MAX)) return fail(FR_E_UNSUPPORTED, "more than 2^31 - 1 images in one call");
    frb::prepfft::Args f{};
    f.images = images;
    f.n = int(n);
    f.scratch = p->scratch;
    f.tw = p->twiddles;
    f.outX = int(p->s.out_x);
    f.outY = int(p->s.out_y);
    f.normalize = p->s.normalize != 0;
    f.center = p->s.center != 0;
    f.shift = p->s.shift != 0;
    f.crop = p->s.crop_freq != 0;
    f.maxFreq = p->s.max_freq;
    f.norm = 1.f / float(uint64_t(p->s.size_x) * p->s.size_y);  // as FPCPU: 1 / padded spatial size
    f.out = out;
    f.scales = scales;
    f.bandStride = banded ? frb::band_stride(f.outX) : 0;
    f.outPlane = banded ? frb::band_plane_elems(f.outX, f.outY) : int64_t(f.outX) * f.outY;
    cudaError_t e = p->fused == 256 ? launch_fused<256>(p, f)
                    : p->fused == 128 ? launch_fused<128>(p, f)
                                      : launch_fused<64>(p, f);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(FR_E_CUDA, std::string("fused prep launch failed: ") + cudaGetErrorString(e));
    }
    return FR_OK;
  }
  PrepArgs a{};
  a.spectra = p->spectra;
  a.inX = int(p->s.size_x / 2 + 1);
  a.inY = int(p->s.size_y);
  a.spX = int(p->s.size_x);
  a.spY = int(p->s.size_y);
  a.outX = int(p->s.out_x);
  a.outY = int(p->s.out_y);
  a.normalize = p->s.normalize != 0;
  a.center = p->s.center != 0;
  a.shift = p->s.shift != 0;
  a.crop = p->s.crop_freq != 0;
  a.maxFreq = p->s.max_freq;
  a.norm = 1.f / float(uint64_t(p->s.size_x) * p->s.size_y);  // as FPCPU: 1 / padded spatial size
  a.out = out;
  a.scales = scales;
  a.bandStride = banded ? frb::band_stride(a.outX) : 0;
  a.outPlane = banded ? frb::band_plane_elems(a.outX, a.outY) : int64_t(a.outX) * a.outY;
  const size_t imgElems = size_t(p->s.size_x) * p->s.size_y;
  for (uint64_t b = 0; b < n; b += uint64_t(p->chunk)) {
    const int batch = int(std::min<uint64_t>(uint64_t(p->chunk), n - b));
    cufftHandle h = p->plan;
    if (batch != p->chunk) {
      if (p->tail_batch != batch) {
        if (p->tail) cufftDestroy(p->tail);
        p->tail = 0;
        p->tail_batch = 0;
        const int rc = plan_for(p, batch, &p->tail);
        if (rc) return rc;
        p->tail_batch = batch;
      }
      h = p->tail;
    }
    const cufftResult r = cufftExecR2C(h, const_cast<cufftReal *>(images + b * imgElems),
      reinterpret_cast<cufftComplex *>(p->spectra));
    if (r != CUFFT_SUCCESS) return fail(FR_E_CUDA, "cufftExecR2C failed (cufftResult " + std::to_string(int(r)) + ")");
    a.first = int64_t(b);
    switch (p->s.storage) {
    case FR_STORAGE_BF16: prep_kernel<FR_STORAGE_BF16><<<batch, kThreads, 0, p->stream>>>(a); break;
    case FR_STORAGE_FP16: prep_kernel<FR_STORAGE_FP16><<<batch, kThreads, 0, p->stream>>>(a); break;
    default: prep_kernel<FR_STORAGE_FP32><<<batch, kThreads, 0, p->stream>>>(a); break;
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(FR_E_CUDA, std::string("prep kernel launch failed: ") + cudaGetErrorString(e));
  }
  return FR_OK;
}

}// extern "C"
