// Fused input preparation for square power-of-two images (N = 64, 128, 256): the real-to-complex
// 2D FFT and the reference's Fourier processing in one kernel that reads each image once and
// writes its finished half-plane once.
//
// The reference runs AFFT (batched cuFFT R2C, fourier_transformation/fft_cuda.cpp:92-95), whose
// spectra go to a buffer, and AFP (scaleFFT2DKernel, fourier_processing/fp_cuda_kernels.cu:9-61),
// which reads that buffer and writes a second one.  Here persistent CTAs (two per SM) take images
// in turn:
//   1. row pass: two image rows form one complex sequence z = a + ib; its N-point DFT Z gives
//      both rows' half spectra, A[k] = (Z[k] + conj Z[N-k]) / 2 and B[k] = (Z[k] - conj Z[N-k]) / 2i,
//      k = 0..N/2, staged in shared memory and written column-major to the CTA's own scratch
//      (N/2+1 columns of N values, 264 KB at N = 256: two per SM stay in L2);
//   2. column pass: every needed column x < out_x goes through an N-point DFT; its values are
//      processed exactly like ScaleFFT2DCPU (fp_cpu_kernels.hpp:24-36, crop / normalise /
//      centre / row shift, each product rounded separately) and written to the output rows
//      through a shared-memory transpose -- FP32 directly; for 16-bit storage written back to the
//      column's scratch slot while the largest |re|, |im| is reduced, then quantised exactly like
//      fr_quantize_projections in a tiled transpose pass from the scratch.
// An N-point DFT is done by a team of N/16 threads holding 16 points each: a 16-point DFT per
// thread (radix 4 x 4), twiddles e^{-2 pi i j k1 / N} from a table built in double precision on the host, a
// transpose through the team's shared buffer, and N/16-point DFTs over the other index
// (Cooley-Tukey with n = j + (N/16) m, k = k1 + 16 k2).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "umpalumpa_fr.h"

namespace frb {
namespace prepfft {

constexpr int kThreads = 256;
constexpr int kCtasPerSm = 2;

// cos and sin of 2 pi t / 16, t = 0..7
__device__ __constant__ float kCos16[8] = { 1.0f, 0.92387953251128674f, 0.70710678118654752f, 0.38268343236508977f,
  0.0f, -0.38268343236508977f, -0.70710678118654752f, -0.92387953251128674f };
__device__ __constant__ float kSin16[8] = { 0.0f, 0.38268343236508977f, 0.70710678118654752f, 0.92387953251128674f,
  1.0f, 0.92387953251128674f, 0.70710678118654752f, 0.38268343236508977f };

// Bit-reversed index of i among S = 4, 8 or 16 points.
template<int S, int I> struct BitRev {
  static constexpr int value = S == 4 ? ((I & 1) << 1 | (I >> 1 & 1))
                               : S == 8 ? ((I & 1) << 2 | (I & 2) | (I >> 2 & 1))
                                        : ((I & 1) << 3 | (I & 2) << 1 | (I >> 1 & 2) | (I >> 3 & 1));
};

template<int S, int I = 0> __device__ __forceinline__ void bitrev_permute(float2 (&v)[S])
{
  if constexpr (I < S) {
    constexpr int J = BitRev<S, I>::value;
    if constexpr (J > I) {
      const float2 t = v[I];
      v[I] = v[J];
      v[J] = t;
    }
    bitrev_permute<S, I + 1>(v);
  }
}

// Forward DFT (e^{-2 pi i n k / S}) of S = 4, 8 or 16 points in registers, natural order in and
// out: radix-2 decimation in time after a bit-reversed permutation.
// One radix-2 stage of butterflies of span LEN (all indices compile-time).
template<int S, int LEN> __device__ __forceinline__ void dft_stage(float2 (&v)[S])
{
#pragma unroll
  for (int i = 0; i < S; i += LEN) {
#pragma unroll
    for (int k = 0; k < LEN / 2; ++k) {
      const int t = k * (16 / LEN);  // e^{-2 pi i k / LEN} = e^{-2 pi i t / 16}
      const float c = t == 0 ? 1.f : kCos16[t], s = t == 0 ? 0.f : kSin16[t];
      const float2 a = v[i + k], b = v[i + k + LEN / 2];
      const float2 tb = make_float2(fmaf(b.x, c, b.y * s), fmaf(b.y, c, -b.x * s));
      v[i + k] = make_float2(a.x + tb.x, a.y + tb.y);
      v[i + k + LEN / 2] = make_float2(a.x - tb.x, a.y - tb.y);
    }
  }
  if constexpr (LEN < S) dft_stage<S, 2 * LEN>(v);
}

// 4-point forward DFT of v[o], v[o + s], v[o + 2s], v[o + 3s] in place.
template<int O, int ST, int S> __device__ __forceinline__ void dft4(float2 (&v)[S])
{
  const float2 x0 = v[O], x1 = v[O + ST], x2 = v[O + 2 * ST], x3 = v[O + 3 * ST];
  const float2 a0 = make_float2(x0.x + x2.x, x0.y + x2.y), a1 = make_float2(x0.x - x2.x, x0.y - x2.y);
  const float2 b0 = make_float2(x1.x + x3.x, x1.y + x3.y), b1 = make_float2(x1.x - x3.x, x1.y - x3.y);
  v[O] = make_float2(a0.x + b0.x, a0.y + b0.y);
  v[O + 2 * ST] = make_float2(a0.x - b0.x, a0.y - b0.y);
  v[O + ST] = make_float2(a1.x + b1.y, a1.y - b1.x);       // a1 - i b1
  v[O + 3 * ST] = make_float2(a1.x - b1.y, a1.y + b1.x);   // a1 + i b1
}

// e^{-2 pi i e / 16} for a compile-time exponent e
template<int E> __device__ __forceinline__ float2 w16()
{
  constexpr int e = E & 15;
  if constexpr (e == 0) return make_float2(1.f, 0.f);
  else if constexpr (e == 4) return make_float2(0.f, -1.f);
  else if constexpr (e == 8) return make_float2(-1.f, 0.f);
  else if constexpr (e == 12) return make_float2(0.f, 1.f);
  else if constexpr (e < 8) return make_float2(kCos16[e], -kSin16[e]);
  else return make_float2(-kCos16[e - 8], kSin16[e - 8]);
}

template<int N2, int K1> __device__ __forceinline__ void twiddle16(float2 (&v)[16])
{
  if constexpr (N2 * K1 != 0) {
    const float2 w = w16<N2 * K1>();
    const float2 a = v[4 * K1 + N2];
    v[4 * K1 + N2] = make_float2(fmaf(a.x, w.x, -a.y * w.y), fmaf(a.x, w.y, a.y * w.x));
  }
}

// Forward DFT (e^{-2 pi i n k / S}) of S = 4, 8 or 16 points in registers, natural order in and
// out.  16 points: radix 4 x 4 (n = 4 n1 + n2, k = k1 + 4 k2); 8: radix 2 after a bit-reversed
// permutation; 4: one radix-4 butterfly.
template<int S> __device__ __forceinline__ void dft(float2 (&v)[S])
{
  static_assert(S == 4 || S == 8 || S == 16, "4, 8 or 16 points");
  if constexpr (S == 4) {
    dft4<0, 1>(v);
  } else if constexpr (S == 8) {
    bitrev_permute<S>(v);
    dft_stage<S, 2>(v);
  } else {
    // 4-point DFTs over n1 for each n2: x[4 n1 + n2] -> Y[n2][k1] held at v[4 k1 + n2]
    dft4<0, 4>(v);
    dft4<1, 4>(v);
    dft4<2, 4>(v);
    dft4<3, 4>(v);
    // twiddles e^{-2 pi i n2 k1 / 16}
    twiddle16<1, 1>(v); twiddle16<1, 2>(v); twiddle16<1, 3>(v);
    twiddle16<2, 1>(v); twiddle16<2, 2>(v); twiddle16<2, 3>(v);
    twiddle16<3, 1>(v); twiddle16<3, 2>(v); twiddle16<3, 3>(v);
    // 4-point DFTs over n2 for each k1: v[4 k1 + n2] -> X[k1 + 4 k2] at v[4 k1 + k2]
    dft4<0, 1>(v);
    dft4<4, 1>(v);
    dft4<8, 1>(v);
    dft4<12, 1>(v);
    // transpose the 4 x 4 index: X[k1 + 4 k2] sits at v[4 k1 + k2]
    float2 t[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) t[i] = v[i];
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1)
#pragma unroll
      for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = t[4 * k1 + k2];
  }
}

// N-point forward DFT by a team of TT = N / 16 lanes (lane j of the team holds x[j + TT m] in
// v[m]); leaves Z[k] in natural order in buf[0..N) (the team's shared buffer of 16 x (TT + 1)
// float2).  tw[t] = e^{-2 pi i t / N}.  Every lane of the warp calls it (teams tile the warp).
template<int N> __device__ __forceinline__ void team_dft(float2 (&v)[16], int j, float2 *buf, const float2 *tw)
{
  constexpr int TT = N / 16, P = TT + 1;
  dft<16>(v);
#pragma unroll
  for (int k1 = 1; k1 < 16; ++k1) {
    const float2 w = tw[j * k1];  // j k1 < TT * 16 = N
    const float2 a = v[k1];
    v[k1] = make_float2(fmaf(a.x, w.x, -a.y * w.y), fmaf(a.x, w.y, a.y * w.x));
  }
#pragma unroll
  for (int k1 = 0; k1 < 16; ++k1) buf[k1 * P + j] = v[k1];
  __syncwarp();
  constexpr int Q = 16 / TT;  // k1 values per lane: k1 = j + TT q
  float2 o[Q][TT];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
#pragma unroll
    for (int jj = 0; jj < TT; ++jj) o[q][jj] = buf[(j + TT * q) * P + jj];
    dft<TT>(o[q]);
  }
  __syncwarp();
#pragma unroll
  for (int q = 0; q < Q; ++q)
#pragma unroll
    for (int k2 = 0; k2 < TT; ++k2) buf[(j + TT * q) + 16 * k2] = o[q][k2];
  __syncwarp();
}

struct Args {
  const float *images;   // [n][N][N]
  int n;
  float2 *scratch;       // per CTA: [N/2 + 1][N]
  const float2 *tw;      // [N]
  int outX, outY;
  int normalize, center, shift, crop;
  float maxFreq, norm;
  void *out;             // [n][outY][outX] in the storage type, or n banded planes
  float *scales;
  int bandStride;        // banded output: elements per 4-row band (frb::band_stride); rows: 0
  int64_t outPlane;      // elements per output plane
};

// Idx2Freq (fourier_processing/fp_common_kernels.hpp:13-20)
__device__ __forceinline__ float idx2freq_(int idx, int size)
{
  if (size <= 1) return 0.f;
  const float t = idx <= size / 2 ? float(idx) : __fsub_rn(float(idx), float(size));
  return __fdiv_rn(t, float(size));
}

template<int N> __host__ __device__ constexpr size_t smem_bytes()
{
  // twiddles + team buffers + the staging area (row pass [rows][N/2+1], column pass [N][teams],
  // 16-bit transpose tiles)
  constexpr int TT = N / 16, TEAMS = kThreads / TT;
  constexpr int rows = 2 * TEAMS < N ? 2 * TEAMS : N;
  constexpr size_t rowStage = size_t(rows) * (N / 2 + 1);
  constexpr size_t colStage = size_t(N) * TEAMS;
  constexpr size_t stage = rowStage > colStage ? rowStage : colStage;
  return (size_t(N) + size_t(TEAMS) * 16 * (TT + 1) + (stage > 32 * 33 ? stage : 32 * 33)) * sizeof(float2) + 64;
}

template<int N, int STORAGE> __global__ void __launch_bounds__(kThreads, kCtasPerSm) prep_fft_kernel(Args a)
{
  constexpr int TT = N / 16, P = TT + 1, TEAMS = kThreads / TT, H = N / 2 + 1;
  constexpr int ROWS = 2 * TEAMS < N ? 2 * TEAMS : N;  // image rows per row pass
  extern __shared__ float2 sm[];
  float2 *tw = sm;
  float2 *teamBuf = tw + N;
  float2 *stage = teamBuf + TEAMS * 16 * P;
  __shared__ float red[kThreads / 32];
  const int tid = threadIdx.x, team = tid / TT, j = tid % TT;
  float2 *buf = teamBuf + team * 16 * P;
  for (int i = tid; i < N; i += kThreads) tw[i] = a.tw[i];
  float2 *S = a.scratch + size_t(blockIdx.x) * H * N;  // [H][N], column-major
  __syncthreads();

  for (int img = blockIdx.x; img < a.n; img += gridDim.x) {
    const float *I = a.images + size_t(img) * N * N;
    // ---- 1. row pass: pairs of rows -> half spectra, staged, then written column-major
    for (int y0 = 0; y0 < N; y0 += ROWS) {
      const int r0 = min(2 * team, ROWS - 2);  // teams beyond the pass compute a row pair again
      const float *ra = I + size_t(y0 + r0) * N, *rb = ra + N;
      float2 v[16];
#pragma unroll
      for (int m = 0; m < 16; ++m) v[m] = make_float2(__ldg(ra + j + TT * m), __ldg(rb + j + TT * m));
      team_dft<N>(v, j, buf, tw);
      if (2 * team < ROWS) {
        for (int k = j; k < H; k += TT) {
          const float2 z = buf[k], zr = buf[(N - k) & (N - 1)];
          stage[(2 * team) * H + k] = make_float2(0.5f * (z.x + zr.x), 0.5f * (z.y - zr.y));
          stage[(2 * team + 1) * H + k] = make_float2(0.5f * (z.y + zr.y), -0.5f * (z.x - zr.x));
        }
      }
      __syncthreads();
      for (int i = tid; i < ROWS * H; i += kThreads) {
        const int k = i / ROWS, r = i - k * ROWS;
        S[size_t(k) * N + y0 + r] = stage[r * H + k];
      }
      __syncthreads();
    }
    // ---- 2. column pass
    float amax = 0.f;
    for (int x0 = 0; x0 < a.outX; x0 += TEAMS) {
      const int x = min(x0 + team, a.outX - 1);  // teams beyond the last column repeat it
      const bool live = x0 + team < a.outX;
      float2 v[16];
#pragma unroll
      for (int m = 0; m < 16; ++m) v[m] = S[size_t(x) * N + j + TT * m];
      team_dft<N>(v, j, buf, tw);
      // ScaleFFT2DCPU on column x (fp_cpu_kernels.hpp:24-36)
      for (int y = j; y < a.outY; y += TT) {
        const int origY = y <= a.outY / 2 ? y : N - (a.outY - y);
        float2 w = buf[origY];
        if (a.crop) {
          const float fx = idx2freq_(x, N), fy = idx2freq_(origY, N);
          if (__fadd_rn(__fmul_rn(fx, fx), __fmul_rn(fy, fy)) > a.maxFreq) w = make_float2(0.f, 0.f);
        }
        if (a.normalize) w = make_float2(__fmul_rn(w.x, a.norm), __fmul_rn(w.y, a.norm));
        if (a.center) {
          const float c = float(1 - 2 * ((x + y) & 1));
          w = make_float2(__fmul_rn(w.x, c), __fmul_rn(w.y, c));
        }
        const int t = y + a.outY / 2;
        const int row = a.shift ? (t >= a.outY ? t - a.outY : t) : y;
        if (STORAGE == FR_STORAGE_FP32) {
          stage[row * TEAMS + team] = w;
        } else if (live) {
          amax = fmaxf(amax, fmaxf(fabsf(w.x), fabsf(w.y)));
          S[size_t(x) * N + row] = w;  // the column was read whole above (v, then buf)
        }
      }
      if (STORAGE == FR_STORAGE_FP32) {
        __syncthreads();
        const int cols = min(TEAMS, a.outX - x0);
        float2 *O = static_cast<float2 *>(a.out) + size_t(img) * a.outPlane;
        if (a.bandStride) {  // (band, column, row within the band): contiguous runs of 4 cols
          for (int i = tid; i < (a.outY + 3) / 4 * 4 * cols; i += kThreads) {
            const int b = i / (4 * cols), r = i - b * 4 * cols, c = r >> 2, row = 4 * b + (r & 3);
            if (row < a.outY) O[size_t(b) * a.bandStride + 4 * (x0 + c) + (row & 3)] = stage[row * TEAMS + c];
          }
        } else {
          for (int i = tid; i < a.outY * cols; i += kThreads) {
            const int row = i / cols, c = i - row * cols;
            O[size_t(row) * a.outX + x0 + c] = stage[row * TEAMS + c];
          }
        }
      }
      __syncthreads();
    }
    if (STORAGE != FR_STORAGE_FP32) {
      // the image's largest |re|, |im|, then the quantised rows from the scratch by 32 x 32 tiles
      for (int s = 16; s > 0; s >>= 1) amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, s));
      if ((tid & 31) == 0) red[tid >> 5] = amax;
      __syncthreads();
      if (tid < 32) {
        float m = tid < kThreads / 32 ? red[tid] : 0.f;
        for (int s = 16; s > 0; s >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, s));
        if (tid == 0) red[0] = m;
      }
      __syncthreads();
      const float scale = red[0] > 0.f ? red[0] / 16384.f : 1.f;
      const float inv = 1.f / scale;
      if (tid == 0) a.scales[img] = scale;
      float2 *tile = stage;  // [32][33]
      for (int xb = 0; xb < a.outX; xb += 32)
        for (int yb = 0; yb < a.outY; yb += 32) {
          __syncthreads();
          for (int i = tid; i < 32 * 32; i += kThreads) {
            const int c = i / 32, r = i - c * 32;  // read down columns (contiguous rows)
            if (xb + c < a.outX && yb + r < a.outY) tile[c * 33 + r] = S[size_t(xb + c) * N + yb + r];
          }
          __syncthreads();
          for (int i = tid; i < 32 * 32; i += kThreads) {
            // write along rows, or banded: (band, column, row within the band)
            const int r = a.bandStride ? 4 * (i >> 7) + (i & 3) : i / 32;
            const int c = a.bandStride ? (i >> 2) & 31 : i - r * 32;
            if (xb + c < a.outX && yb + r < a.outY) {
              const float2 w = tile[c * 33 + r];
              const int y = yb + r, x = xb + c;
              const size_t d = size_t(img) * a.outPlane
                               + (a.bandStride ? size_t(y >> 2) * a.bandStride + 4 * x + (y & 3) : size_t(y) * a.outX + x);
              if (STORAGE == FR_STORAGE_BF16)
                static_cast<__nv_bfloat162 *>(a.out)[d] = __floats2bfloat162_rn(w.x * inv, w.y * inv);
              else
                static_cast<__half2 *>(a.out)[d] = __floats2half2_rn(w.x * inv, w.y * inv);
            }
          }
        }
      __syncthreads();
    }
  }
}

}// namespace prepfft
}// namespace frb
