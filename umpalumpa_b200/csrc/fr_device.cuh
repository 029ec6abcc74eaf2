// Device-side building blocks of the B200 Fourier-reconstruction engine: layouts shared by
// the kernels, the Kaiser-Bessel blob math and the slab geometry.  Reference citations are
// path:line relative to the Umpalumpa project root.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include "umpalumpa_fr.h"

namespace frb {

static_assert(sizeof(fr_traverse_space) == 112, "TraverseSpace must stay 112 bytes");
static_assert(sizeof(fr_constants) == 32, "Constants must stay 32 bytes");

constexpr int kThreads = 256;     // insertion CTA: 16 x 16 columns of one brick face
constexpr int kBrick = 16;        // brick edge in voxels (16^3 voxels = 48 KB of accumulators)
constexpr int kBrickVox = kBrick * kBrick * kBrick;
constexpr int kLutSmemMax = 16384;// blob tables up to 64 KB live in shared memory
// Dynamic interpolation's Kaiser table for alpha > 15: (value, slope) at nodes equally spaced
// in d^2 over [0, r^2], interpolated linearly (32 KB; at r 1.9 its error is 5.4e-7 of the
// peak weight at alpha 18, 1.1e-6 at alpha 25, 2.8e-6 at alpha 40).
constexpr int kKaiserTableElems = 4096;

// Compact per-space record used by the binning passes (64 bytes).  t0/t2 are rows 0 and 2
// of transformInv: t0.p is the image x of voxel offset p, t2.p its distance from the
// projection plane.  lo/hi are the traversal-AABB limits on the two axes the reference's
// traversal constrains for this direction (fr_cpu_kernels.hpp:166-238); the third axis is
// left open.  All thresholds carry a small outward margin so the test is conservative.
struct SpacePrep {
  float t0[3];
  float maxDist2;
  float t2[3];
  float halfWidth;
  int lo[3];
  int dir;
  int hi[3];
  float xMin;
};
static_assert(sizeof(SpacePrep) == 64, "SpacePrep is 64 bytes");

// Per-space record read by the insertion kernel (128 bytes = eight 16-byte loads), built
// once per space by the binning prep pass.  The axes U, V are the traversal plane of the
// space's direction and W its column axis (XY: x, y | z;  XZ: x, z | y;  YZ: y, z | x).
//  - T, maxDist2, weight, proj: as in the TraverseSpace.
//  - lo0/hi0/lo1/hi1: the traversal AABB on U and V (fr_cpu_kernels.hpp:166-238).
//  - w0, wu, wv, hw (blob mode): the slab |t2.(q - c)| <= r crosses column (U, V) at
//    W = w0 + wu U + wv V with half-width hw along W (plus a margin).  A voxel contributes
//    only if its float |t2.(q - c)| <= r, and the reference's column range
//    [floor(min(z1,z2)), ceil(max(z1,z2))] always contains every such voxel, so visiting
//    [ceil(wc - hw), floor(wc + hw)] instead yields the same contributing voxels.
//  - nu, nv, nw, bu, bv, bw (nearest mode): the plane normal and bottom origin on U, V, W,
//    for the reference's exact rounded plane hit.
//  - xu, xv, xw, xwInv: row 0 of transformInv on U, V, W; a voxel contributes only if its
//    image x' = t0.(q - c) >= -r (>= 0 in nearest mode), which bounds each column on one side.
struct SpaceRec {
  float T[9];
  float maxDist2;
  float weight;
  int proj;
  int lo0, hi0, lo1, hi1;
  float w0, wu, wv, hw;
  float nu, nv, nw, bu, bv, bw;
  float xu, xv;         // half-space x' >= -r per column: row 0 of transformInv on U, V,
  float xwInv, xw;      // 1/t0_W (0 when |t0_W| <= 1e-3) and t0_W
  int dir;
  int pad;
};
static_assert(sizeof(SpaceRec) == 128, "SpaceRec is 128 bytes");

// One unit of insertion work: a brick and a range [begin, end) of its binned list; in a
// batched launch also the job the brick belongs to.
struct WorkItem {
  int brick;
  int begin;
  int end;
  int job;
};

// One job of a batched launch (128 bytes): its payloads, sizes, brick grid and the offsets
// of its traverse spaces and bricks in the batch-wide arrays.
struct JobDesc {
  const void *fft;
  const float *scales;
  void *volume;
  float *weight;
  int nProj, fftX, fftY, vx;
  int vy, vz, nbx, nby;
  int nbz, cx, cy, cz;
  int genericTaps, spaceBase, nSpaces, brickBase;
  int nBricks, groupBase;              // bricks; first 8-brick binning group of the job
  const fr_traverse_space *spaces;     // the job's traverse spaces (device memory)
  const void *src;                     // the caller's row-major half-planes (fft: their bands)
  int bandStride;                      // elements per 4-row band of fft
  int unitBase;                        // the job's first band in the batch's band copy
};
static_assert(sizeof(JobDesc) == 128, "JobDesc is 128 bytes");

// ------------------------------------------------------------------------------------
// Exact-rounding helpers.  The reference's geometry is evaluated without fused
// multiply-adds (its ISO-mode host build); the helpers keep nvcc from contracting them so
// slab bounds and blob boxes round the same way.
// ------------------------------------------------------------------------------------
__device__ __forceinline__ float mul_(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add_(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub_(float a, float b) { return __fsub_rn(a, b); }

// Plane intersection along one axis: from n.(q - p0) = 0 solve for the free coordinate
// (libumpalumpa/math/geometry.hpp:11-33).  (u, v) are the two fixed coordinates, nu/nv
// their normal components, nw the normal component of the solved axis.
__device__ __forceinline__ float plane_hit(float u, float v, float nu, float nv, float nw,
  float pu, float pv, float pw)
{
  float a = mul_(-nu, sub_(u, pu));
  float b = mul_(nv, sub_(v, pv));
  return add_(__fdiv_rn(sub_(a, b), nw), pw);
}

__device__ __forceinline__ float clampf_(float v, float lo, float hi)
{
  float r = (v > hi) ? hi : v;
  return (r < lo) ? lo : r;
}

// ------------------------------------------------------------------------------------
// Bessel functions.  I0/I1 by the polynomial approximations of Abramowitz & Stegun
// 9.8.1-9.8.4 and I2..I4 by upward recurrence -- the reference's choice
// (libumpalumpa/math/bessier.hpp:9-63 in double; fr_common_kernels.hpp:55-127 in float).
// The double forms use explicit round-to-nearest operations in the reference's
// evaluation order so the blob table matches the reference's host table.
// ------------------------------------------------------------------------------------
__device__ __forceinline__ double dm(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double da(double a, double b) { return __dadd_rn(a, b); }

__device__ inline double bessel_i0_d(double x)
{
  double ax = fabs(x);
  if (ax < 3.75) {
    double t = x / 3.75;
    t = dm(t, t);
    double p = 0.45813e-2;
    p = da(0.360768e-1, dm(t, p));
    p = da(0.2659732, dm(t, p));
    p = da(1.2067492, dm(t, p));
    p = da(3.0899424, dm(t, p));
    p = da(3.5156229, dm(t, p));
    return da(1.0, dm(t, p));
  }
  double t = 3.75 / ax;
  double p = 0.392377e-2;
  p = da(-0.1647633e-1, dm(t, p));
  p = da(0.2635537e-1, dm(t, p));
  p = da(-0.2057706e-1, dm(t, p));
  p = da(0.916281e-2, dm(t, p));
  p = da(-0.157565e-2, dm(t, p));
  p = da(0.225319e-2, dm(t, p));
  p = da(0.1328592e-1, dm(t, p));
  p = da(0.39894228, dm(t, p));
  return dm(exp(ax) / sqrt(ax), p);
}

__device__ inline double bessel_i1_d(double x)
{
  double ax = fabs(x), r;
  if (ax < 3.75) {
    double t = x / 3.75;
    t = dm(t, t);
    double p = 0.32411e-3;
    p = da(0.301532e-2, dm(t, p));
    p = da(0.2658733e-1, dm(t, p));
    p = da(0.15084934, dm(t, p));
    p = da(0.51498869, dm(t, p));
    p = da(0.87890594, dm(t, p));
    p = da(0.5, dm(t, p));
    r = dm(ax, p);
  } else {
    double t = 3.75 / ax;
    double q = __dsub_rn(0.1787654e-1, dm(t, 0.420059e-2));
    q = da(-0.2895312e-1, dm(t, q));
    q = da(0.2282967e-1, dm(t, q));
    double p = da(-0.1031555e-1, dm(t, q));
    p = da(0.163801e-2, dm(t, p));
    p = da(-0.362018e-2, dm(t, p));
    p = da(-0.3988024e-1, dm(t, p));
    p = da(0.39894228, dm(t, p));
    r = dm(p, exp(ax) / sqrt(ax));
  }
  return x < 0.0 ? -r : r;
}

__device__ inline double bessel_in_d(int order, double x)
{
  if (order == 0) return bessel_i0_d(x);
  if (order == 1) return bessel_i1_d(x);
  if (x == 0) return 0;
  double im1 = bessel_i0_d(x), i = bessel_i1_d(x);
  for (int k = 1; k < order; ++k) {
    double nx = __dsub_rn(im1, dm((2.0 * k) / x, i));
    im1 = i;
    i = nx;
  }
  return i;
}

__device__ inline float bessel_i0_f(float x)
{
  float ax = fabsf(x), t;
  if (ax < 3.75f) {
    t = x / 3.75f;
    t *= t;
    return 1.f
           + t * (3.5156229f
                  + t * (3.0899424f
                         + t * (1.2067492f + t * (0.2659732f + t * (0.360768e-1f + t * 0.45813e-2f)))));
  }
  t = 3.75f / ax;
  return (expf(ax) * (1 / sqrtf(ax)))
         * (0.39894228f
            + t * (0.1328592e-1f
                   + t * (0.225319e-2f
                          + t * (-0.157565e-2f
                                 + t * (0.916281e-2f
                                        + t * (-0.2057706e-1f
                                               + t * (0.2635537e-1f
                                                      + t * (-0.1647633e-1f + t * 0.392377e-2f))))))));
}

__device__ inline float bessel_i1_f(float x)
{
  float ax = fabsf(x), r, t;
  if (ax < 3.75f) {
    t = x / 3.75f;
    t *= t;
    r = ax
        * (0.5f
           + t * (0.87890594f
                  + t * (0.51498869f
                         + t * (0.15084934f + t * (0.2658733e-1f + t * (0.301532e-2f + t * 0.32411e-3f))))));
  } else {
    t = 3.75f / ax;
    r = 0.2282967e-1f + t * (-0.2895312e-1f + t * (0.1787654e-1f - t * 0.420059e-2f));
    r = 0.39894228f
        + t * (-0.3988024e-1f + t * (-0.362018e-2f + t * (0.163801e-2f + t * (-0.1031555e-1f + t * r))));
    r *= (expf(ax) * (1 / sqrtf(ax)));
  }
  return x < 0.f ? -r : r;
}

__device__ inline float bessel_in_f(int order, float x)
{
  if (order == 0) return bessel_i0_f(x);
  if (order == 1) return bessel_i1_f(x);
  if (x == 0) return 0;
  float im1 = bessel_i0_f(x), i = bessel_i1_f(x);
  for (int k = 1; k < order; ++k) {
    float nx = im1 - ((2 * k) / x) * i;
    im1 = i;
    i = nx;
  }
  return i;
}

// The fast dynamic blob (fr_common_kernels.hpp:163-170: bessi0Fast(alpha sqrt(1 - d2/r^2))
// / I0(alpha) * cIw0) for two taps at once, for the insertion's tap pairs.  I0 is the rational
// minimax approximation of Blair & Edwards (AECL-4928, 1974, table 5; valid for x <= 15, the
// reference's bessi0Fast, fr_common_kernels.hpp:30-53): P(x^2) / (x^2 + q0) with P of degree
// 11, coefficients below from the highest power down.  The quotient is a function of x^2
// only, so x^2 is taken as alpha^2 (1 - d2/r^2)
// instead of squaring alpha sqrt(1 - d2/r^2) (no square root), both numerators and
// denominators run in packed FP32x2, and the quotient is a fast divide.  The weights differ
// from the reference's scalar form by a few ulps (relative 1e-6 at most), far inside the
// insertion's 1e-5 bar.  1 - d2/r^2 is formed unfused and clamped at 0, so a tap on the blob
// boundary cannot turn negative (the reference's fused GPU form can, giving NaN).
// ks = cOneOverBessiOrderAlpha * cIw0; d2 beyond r^2 gives x^2 = 0.
__device__ __forceinline__ float2 kaiser_value_fast2(float2 d2, float alpha2, float oneOverR2, float ks)
{
  const float2 u = make_float2(fmaxf(0.f, __fsub_rn(1.f, __fmul_rn(d2.x, oneOverR2))),
                               fmaxf(0.f, __fsub_rn(1.f, __fmul_rn(d2.y, oneOverR2))));
  const float2 x2 = __fmul2_rn(u, make_float2(alpha2, alpha2));
  constexpr float kNum[12] = { -0.8436825781374849e-19f, -0.93466495199548700e-17f, -0.15716375332511895e-13f,
    -0.42520971595532318e-11f, -0.13704363824102120e-8f, -0.28508770483148419e-6f, -0.44322160233346062e-4f,
    -0.46703811755736946e-2f, -0.31112484643702141e-0f, -0.11512633616429962e+2f, -0.18720283332732112e+3f,
    -0.75281108169006924e+3f };
  float2 num = make_float2(kNum[0], kNum[0]);
#pragma unroll
  for (int k = 1; k < 12; ++k) num = __ffma2_rn(num, x2, make_float2(kNum[k], kNum[k]));
  const float2 den = __fadd2_rn(x2, make_float2(-0.75281109410939403e+3f, -0.75281109410939403e+3f));
  return make_float2(__fdividef(num.x, den.x) * ks, __fdividef(num.y, den.y) * ks);
}

// Blob value at distance r for a blob of radius a, in the device form of the reference
// (fr_common_kernels.hpp:129-161): the Bessel ratio is scaled by 1/I_order(alpha).
__device__ inline float kaiser_value_f(float r, float a, float alpha, float oneOverBessi, int order)
{
  float rda = r / a;
  if (!(rda <= 1.f)) return 0.f;
  float rdas = rda * rda;
  float arg = alpha * sqrtf(1.f - rdas);
  if (order == 0) return bessel_i0_f(arg) * oneOverBessi;
  float w = sqrtf(1.f - rdas);
  if (order == 2) w = w * w;
  if (order == 3) w = w * w * w;
  if (order == 4) w = w * w * w * w;
  return w * (bessel_in_f(order, arg) * oneOverBessi);
}

// ------------------------------------------------------------------------------------
// Projection storage: complex64, or 2 x 16-bit complex with a per-projection scale.
// ------------------------------------------------------------------------------------
template<int STORAGE> struct Pixel;

template<> struct Pixel<FR_STORAGE_FP32> {
  using T = float2;
  static constexpr int kBytes = 8;
  __device__ __forceinline__ static float2 load(const T *p) { return __ldg(p); }
};

template<> struct Pixel<FR_STORAGE_BF16> {
  using T = __nv_bfloat162;
  static constexpr int kBytes = 4;
  // A BF16 value is the upper half of the FP32 one: the pair's low half (re) shifted up, the
  // high half (im) masked -- two integer operations (2.3 % faster insertion than the library
  // conversion at box 256).
  __device__ __forceinline__ static float2 load(const T *p)
  {
    const unsigned u = __ldg(reinterpret_cast<const unsigned *>(p));
    return make_float2(__uint_as_float(u << 16), __uint_as_float(u & 0xffff0000u));
  }
};

template<> struct Pixel<FR_STORAGE_FP16> {
  using T = __half2;
  static constexpr int kBytes = 4;
  __device__ __forceinline__ static float2 load(const T *p) { return __half22float2(__ldg(p)); }
};

}// namespace frb
