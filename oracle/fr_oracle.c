/*
 * TEST INFRASTRUCTURE ONLY -- the oracle (see fr_oracle.h).  Plain C restatement of the
 * reference's CPU Fourier-reconstruction path in its single-precision operation order,
 * plus an FP64 variant of the same algorithm.  Compiled with -ffp-contract=off so that no
 * a*b+c is fused, as in the reference's own ISO-mode build.  References are
 * path:line relative to the reference project root.
 */
#include "fr_oracle.h"

#include <float.h>
#include <pthread.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

static const float kPiF = 3.14159265358979323846f;
static const double kPiD = 3.14159265358979323846;

/* ---------------------------------------------------------------------------------------
 * Modified Bessel functions I0, I1 by the polynomial approximations of Abramowitz & Stegun
 * 9.8.1-9.8.4, and I2..I4 by the upward recurrence I(n+1) = I(n-1) - (2n/x) I(n).
 * Double precision: libumpalumpa/math/bessier.hpp:9-63.  Single precision (device form):
 * libumpalumpa/operations/fourier_reconstruction/fr_common_kernels.hpp:55-127.
 * ------------------------------------------------------------------------------------- */
static double as_i0(double x)
{
  double ax = fabs(x);
  if (ax < 3.75) {
    double t = x / 3.75;
    t *= t;
    return 1.0
           + t * (3.5156229
                  + t * (3.0899424
                         + t * (1.2067492 + t * (0.2659732 + t * (0.360768e-1 + t * 0.45813e-2)))));
  }
  double t = 3.75 / ax;
  return (exp(ax) / sqrt(ax))
         * (0.39894228
            + t * (0.1328592e-1
                   + t * (0.225319e-2
                          + t * (-0.157565e-2
                                 + t * (0.916281e-2
                                        + t * (-0.2057706e-1
                                               + t * (0.2635537e-1
                                                      + t * (-0.1647633e-1 + t * 0.392377e-2))))))));
}

static double as_i1(double x)
{
  double ax = fabs(x), r;
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
    r *= exp(ax) / sqrt(ax);
  }
  return x < 0.0 ? -r : r;
}

static double as_i2(double x) { return x == 0 ? 0 : as_i0(x) - (2.0 / x) * as_i1(x); }
static double as_i3(double x) { return x == 0 ? 0 : as_i1(x) - (4.0 / x) * as_i2(x); }
static double as_i4(double x) { return x == 0 ? 0 : as_i2(x) - (6.0 / x) * as_i3(x); }

static double as_in(int order, double x)
{
  switch (order) {
  case 0: return as_i0(x);
  case 1: return as_i1(x);
  case 2: return as_i2(x);
  case 3: return as_i3(x);
  case 4: return as_i4(x);
  default: return NAN;
  }
}

static float as_i0f(float x)
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

static float as_i1f(float x)
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

static float as_i2f(float x) { return (x == 0) ? 0 : as_i0f(x) - ((2 * 1) / x) * as_i1f(x); }
static float as_i3f(float x) { return (x == 0) ? 0 : as_i1f(x) - ((2 * 2) / x) * as_i2f(x); }
static float as_i4f(float x) { return (x == 0) ? 0 : as_i2f(x) - ((2 * 3) / x) * as_i3f(x); }

/* I0 by the rational minimax approximation of Blair & Edwards (1974, table 5), valid for
 * x <= 15, evaluated with explicit fused multiply-adds in the given precision.
 * fr_common_kernels.hpp:30-53 */
static const double kBE_P[12] = { -0.8436825781374849e-19, -0.93466495199548700e-17,
  -0.15716375332511895e-13, -0.42520971595532318e-11, -0.13704363824102120e-8,
  -0.28508770483148419e-6, -0.44322160233346062e-4, -0.46703811755736946e-2,
  -0.31112484643702141e-0, -0.11512633616429962e+2, -0.18720283332732112e+3,
  -0.75281108169006924e+3 };
static const double kBE_Q0 = -0.75281109410939403e+3;

static float be_i0f(float x)
{
  float x2 = x * x;
  float num = (float)kBE_P[0];
  for (int k = 1; k < 12; ++k) num = fmaf(num, x2, (float)kBE_P[k]);
  float den = fmaf(1.f, x2, (float)kBE_Q0);
  return num / den;
}

static double be_i0(double x)
{
  double x2 = x * x;
  double num = kBE_P[0];
  for (int k = 1; k < 12; ++k) num = fma(num, x2, kBE_P[k]);
  return num / (x2 + kBE_Q0);
}

/* ---------------------------------------------------------------------------------------
 * Kaiser-Bessel blob value and its Fourier value.
 * libumpalumpa/math/kaiser.hpp:19-81 (host; float args with double Bessel functions)
 * ------------------------------------------------------------------------------------- */
static float kaiser_value_host(float freq, float radius, float alpha, int order)
{
  float w = 0;
  float rda = freq / radius;
  if (rda <= 1.f) {
    float rdas = rda * rda;
    float arg = alpha * sqrtf(1 - rdas);
    switch (order) {
    case 0: w = (float)(as_i0(arg) / as_i0(alpha)); break;
    case 1:
      w = sqrtf(1 - rdas);
      if (alpha != 0) w *= (float)(as_i1(arg) / as_i1(alpha));
      break;
    case 2:
      w = sqrtf(1 - rdas);
      w = w * w;
      if (alpha != 0) w *= (float)(as_i2(arg) / as_i2(alpha));
      break;
    case 3:
      w = sqrtf(1 - rdas);
      w = w * w * w;
      if (alpha != 0) w *= (float)(as_i3(arg) / as_i3(alpha));
      break;
    case 4:
      w = sqrtf(1 - rdas);
      w = w * w * w * w;
      if (alpha != 0) w *= (float)(as_i4(arg) / as_i4(alpha));
      break;
    default: break;
    }
  }
  return w;
}

static double kaiser_value_d(double freq, double radius, double alpha, int order)
{
  double w = 0;
  double rda = freq / radius;
  if (rda <= 1.0) {
    double rdas = rda * rda;
    double arg = alpha * sqrt(1 - rdas);
    double s = sqrt(1 - rdas);
    switch (order) {
    case 0: w = as_i0(arg) / as_i0(alpha); break;
    case 1: w = s * (alpha != 0 ? as_i1(arg) / as_i1(alpha) : 1.0); break;
    case 2: w = s * s * (alpha != 0 ? as_i2(arg) / as_i2(alpha) : 1.0); break;
    case 3: w = s * s * s * (alpha != 0 ? as_i3(arg) / as_i3(alpha) : 1.0); break;
    case 4: w = s * s * s * s * (alpha != 0 ? as_i4(arg) / as_i4(alpha) : 1.0); break;
    default: break;
    }
  }
  return w;
}

/* Modified spherical Bessel function of order 3/2, bessier.hpp:65-70 */
static float i1_5f(float x)
{
  return (x == 0) ? 0 : sqrtf(2.f / (kPiF * x)) * (coshf(x) - sinhf(x) / x);
}
static double i1_5d(double x)
{
  return (x == 0) ? 0 : sqrt(2.0 / (kPiD * x)) * (cosh(x) - sinh(x) / x);
}

/* kaiser.hpp:66-81; defined only for blob order 0, NaN otherwise. */
static float kaiser_fourier_value_host(float freq, float radius, float alpha, int order)
{
  float sigma = sqrtf(
    fabsf(alpha * alpha - (2.f * kPiF * radius * freq) * (2.f * kPiF * radius * freq)));
  if (order == 0 && 2 * kPiF * radius * freq <= alpha) {
    return powf(2.f * kPiF, 1.5f) * powf(radius, 3.f) * i1_5f(sigma)
           / ((float)as_i0(alpha) * powf(sigma, 1.5f));
  }
  return NAN;
}

static double kaiser_fourier_value_d(double freq, double radius, double alpha, int order)
{
  double sigma =
    sqrt(fabs(alpha * alpha - (2.0 * kPiD * radius * freq) * (2.0 * kPiD * radius * freq)));
  if (order == 0 && 2 * kPiD * radius * freq <= alpha) {
    return pow(2.0 * kPiD, 1.5) * pow(radius, 3.0) * i1_5d(sigma)
           / (as_i0(alpha) * pow(sigma, 1.5));
  }
  return NAN;
}

/* AFR::CreateConstants, afr.cpp:6-19 */
void or_make_constants(size_t vx, size_t vy, size_t tableElems, int order, float alpha,
  float radius, or_constants *c)
{
  memset(c, 0, sizeof(*c));
  c->cMaxVolumeIndexX = (int32_t)(vx - 1);
  c->cMaxVolumeIndexYZ = (int32_t)(vy - 1);
  c->cBlobRadius = radius;
  c->cOneOverBlobRadiusSqr = 1.f / (radius * radius);
  c->cBlobAlpha = alpha;
  c->cIw0 = 1.f / kaiser_fourier_value_host(0.f, radius, alpha, order);
  c->cIDeltaSqrt = (float)(tableElems - 1) / (radius * radius);
  c->cOneOverBessiOrderAlpha = 1 / (float)as_in(order, alpha);
}

/* AFR::FillBlobTable, afr.cpp:22-34: entry i holds the blob at distance r*sqrt(i/(N-1)),
 * i.e. the table is indexed by squared distance. */
void or_fill_blob_table(float *table, size_t n, int order, float alpha, float radius)
{
  or_constants c;
  or_make_constants(3, 3, n, order, alpha, radius, &c);
  float freq = radius * sqrtf(1.f / (float)(n - 1));
  for (size_t i = 0; i < n; ++i) {
    table[i] = kaiser_value_host(freq * (float)sqrt((double)i), radius, alpha, order) * c.cIw0;
  }
}

/* ---------------------------------------------------------------------------------------
 * Traverse space: traverse_space_generator.hpp:30-145
 * ------------------------------------------------------------------------------------- */
static void mul3f(const float t[3][3], float v[3])
{
  float a = t[0][0] * v[0] + t[0][1] * v[1] + t[0][2] * v[2];
  float b = t[1][0] * v[0] + t[1][1] * v[1] + t[1][2] * v[2];
  float c = t[2][0] * v[0] + t[2][1] * v[1] + t[2][2] * v[2];
  v[0] = a;
  v[1] = b;
  v[2] = c;
}

void or_compute_traverse_space(uint32_t imgSizeX, uint32_t imgSizeY, const float *transform9,
  uint32_t maxVolumeIndexX, uint32_t maxVolumeIndexYZ, int useFast, float blobRadius,
  float weight, or_traverse_space *s)
{
  float t[3][3];
  for (int i = 0; i < 9; ++i) t[i / 3][i % 3] = transform9[i];
  memset(s, 0, sizeof(*s));

  /* The projection plane padded by the blob radius, as a cuboid with corners 0..7:
   * x in {-b, X+b}, y in {-(Y/2+b), Y/2+b}, z in {+b, -b}.  (:30-40) */
  float b = useFast ? 0.f : blobRadius;
  float sizeX = (float)imgSizeX, sizeY = (float)imgSizeY;
  float halfY = sizeY / 2.0f;
  float cub[8][3];
  const int xHi[8] = { 1, 1, 0, 0, 1, 1, 0, 0 };
  const int yHi[8] = { 0, 1, 1, 0, 0, 1, 1, 0 };
  const int zHi[8] = { 1, 1, 1, 1, 0, 0, 0, 0 };
  for (int i = 0; i < 8; ++i) {
    cub[i][0] = xHi[i] ? sizeX + b : 0.f - b;
    cub[i][1] = yHi[i] ? halfY + b : -(halfY + b);
    cub[i][2] = zHi[i] ? 0.f + b : 0.f - b;
  }
  float origin[3] = { maxVolumeIndexX / 2.f, maxVolumeIndexYZ / 2.f, maxVolumeIndexYZ / 2.f };
  for (int i = 0; i < 8; ++i) {
    mul3f(t, cub[i]);
    for (int k = 0; k < 3; ++k) cub[i][k] += origin[k];
  }
  /* AABB; note the reference starts the maxima at FLT_MIN (the smallest positive float). */
  float lo[3] = { FLT_MAX, FLT_MAX, FLT_MAX }, hi[3] = { FLT_MIN, FLT_MIN, FLT_MIN };
  for (int i = 0; i < 8; ++i)
    for (int k = 0; k < 3; ++k) {
      if (lo[k] > cub[i][k]) lo[k] = cub[i][k];
      if (hi[k] < cub[i][k]) hi[k] = cub[i][k];
    }
  float lim[3] = { (float)maxVolumeIndexX, (float)maxVolumeIndexYZ, (float)maxVolumeIndexYZ };
  for (int k = 0; k < 3; ++k) {
    if (lo[k] < 0.f) lo[k] = 0.f;
    if (hi[k] > lim[k]) hi[k] = lim[k];
  }
  s->minZ = (int32_t)floorf(lo[2]);
  s->minY = (int32_t)floorf(lo[1]);
  s->minX = (int32_t)floorf(lo[0]);
  s->maxZ = (int32_t)ceilf(hi[2]);
  s->maxY = (int32_t)ceilf(hi[1]);
  s->maxX = (int32_t)ceilf(hi[0]);
  memcpy(s->topOrigin, cub[4], sizeof(s->topOrigin));
  memcpy(s->bottomOrigin, cub[0], sizeof(s->bottomOrigin));
  float rr = (float)imgSizeX + b;
  s->maxDistanceSqr = rr * rr;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) s->transformInv[i][j] = t[j][i];
  float n[3] = { 0.f, 0.f, 1.f };
  mul3f(t, n);
  memcpy(s->unitNormal, n, sizeof(n));
  float nX = fabsf(n[0]), nY = fabsf(n[1]), nZ = fabsf(n[2]);
  /* dominant normal component picks the traversal plane; tie order YZ, XZ, XY (:136-142) */
  if (nX >= nY && nX >= nZ)
    s->dir = 2;
  else if (nY >= nX && nY >= nZ)
    s->dir = 1;
  else if (nZ >= nX && nZ >= nY)
    s->dir = 0;
  s->weight = weight;
}

/* ---------------------------------------------------------------------------------------
 * Insertion: fr_cpu_kernels.hpp:18-277, single precision.
 * ------------------------------------------------------------------------------------- */
typedef struct {
  float *volume, *weight;
  double *volume64, *weight64;
  int64_t *count;
  size_t vx, vy, vz;
  int xSize, ySize;
  const float *fft; /* interleaved complex, already offset to the projection */
  const float *table;
  const double *table64;
  or_constants c;
  double cIDeltaSqrt64, cIw0_64, cOneOverBessi64;
  int interpolation, order, fastKaiser;
  int mode; /* 0 = float accumulate, 1 = double accumulate, 2 = count,
              3 = float decisions (the reference's own), double products and sums */
} ctx_t;

static inline int clampi(int v, int lo, int hi) { return v > hi ? hi : (v < lo ? lo : v); }
static inline float clampf(float v, float lo, float hi)
{
  float r = (v > hi) ? hi : v;
  return (r < lo) ? lo : r;
}

static int in_volume(const ctx_t *x, int X, int Y, int Z)
{
  return X >= 0 && Y >= 0 && Z >= 0 && (size_t)X < x->vx && (size_t)Y < x->vy
         && (size_t)Z < x->vz;
}

/* kaiserValue<order> and kaiserValueFast, fr_common_kernels.hpp:129-170 */
static float kaiser_value_dev(float r, float a, const or_constants *c, int order)
{
  float w;
  float rda = r / a;
  if (rda <= 1.f) {
    float rdas = rda * rda;
    float arg = c->cBlobAlpha * sqrtf(1.f - rdas);
    if (order == 0) {
      w = as_i0f(arg) * c->cOneOverBessiOrderAlpha;
    } else {
      w = sqrtf(1.f - rdas);
      if (order == 2) w = w * w;
      if (order == 3) w = w * w * w;
      if (order == 4) w = w * w * w * w;
      float bi = order == 1 ? as_i1f(arg) : order == 2 ? as_i2f(arg) : order == 3 ? as_i3f(arg) : as_i4f(arg);
      w *= bi * c->cOneOverBessiOrderAlpha;
    }
  } else
    w = 0.f;
  return w;
}

static float kaiser_value_fast_dev(float distSqr, const or_constants *c)
{
  float arg = c->cBlobAlpha * sqrtf(1.f - (distSqr * c->cOneOverBlobRadiusSqr));
  return be_i0f(arg) * c->cOneOverBessiOrderAlpha * c->cIw0;
}

/* FR<>::ProcessVoxelBlob, fr_cpu_kernels.hpp:70-152 */
static void voxel_blob_f(ctx_t *x, const or_traverse_space *s, int X, int Y, int Z)
{
  const or_constants *c = &x->c;
  float p[3] = { (float)(X - c->cMaxVolumeIndexX / 2), (float)(Y - c->cMaxVolumeIndexYZ / 2),
    (float)(Z - c->cMaxVolumeIndexYZ / 2) };
  if ((p[0] * p[0] + p[1] * p[1] + p[2] * p[2]) > s->maxDistanceSqr) return;
  mul3f(s->transformInv, p);
  if (p[0] < -c->cBlobRadius) return;
  p[1] += (float)(c->cMaxVolumeIndexYZ / 2);
  float radiusSqr = c->cBlobRadius * c->cBlobRadius;
  float zSqr = p[2] * p[2];
  if (zSqr > radiusSqr) return;
  int minX = (int)ceilf(p[0] - c->cBlobRadius);
  int maxX = (int)floorf(p[0] + c->cBlobRadius);
  int minY = (int)ceilf(p[1] - c->cBlobRadius);
  int maxY = (int)floorf(p[1] + c->cBlobRadius);
  if (minX < 0) minX = 0;
  if (minY < 0) minY = 0;
  if (maxX > x->xSize - 1) maxX = x->xSize - 1;
  if (maxY > x->ySize - 1) maxY = x->ySize - 1;
  if (!in_volume(x, X, Y, Z)) return;
  size_t idx3 = ((size_t)Z * x->vy + (size_t)Y) * x->vx + (size_t)X;
  float w = 0.f, re = 0.f, im = 0.f;
  double w64 = 0.0, re64 = 0.0, im64 = 0.0; /* mode 3 */
  float dataWeight = s->weight;
  int64_t taps = 0;
  for (int i = minY; i <= maxY; i++) {
    float ySqr = (p[1] - (float)i) * (p[1] - (float)i);
    float yzSqr = ySqr + zSqr;
    if (yzSqr > radiusSqr) continue;
    for (int j = minX; j <= maxX; j++) {
      float xD = p[0] - (float)j;
      float d2 = xD * xD + yzSqr;
      if (d2 > radiusSqr) continue;
      ++taps;
      if (x->mode == 2) continue;
      float wBlob;
      if (x->interpolation == 1) {
        int aux = (int)(d2 * c->cIDeltaSqrt + 0.5f);
        wBlob = x->table[aux];
      } else if (x->fastKaiser) {
        wBlob = kaiser_value_fast_dev(d2, c);
      } else {
        wBlob = kaiser_value_dev(sqrtf(d2), c->cBlobRadius, c, x->order) * c->cIw0;
      }
      const float *px = x->fft + 2 * ((size_t)i * (size_t)x->xSize + (size_t)j);
      if (x->mode == 3) {
        double weight64 = (double)wBlob * (double)dataWeight;
        w64 += weight64;
        re64 += (double)px[0] * weight64;
        im64 += (double)px[1] * weight64;
        continue;
      }
      float weight = wBlob * dataWeight;
      w += weight;
      re += px[0] * weight;
      im += px[1] * weight;
    }
  }
  if (x->mode == 2) {
    if (taps) x->count[0]++;
    return;
  }
  if (x->mode == 3) {
    x->volume64[2 * idx3 + 0] += re64;
    x->volume64[2 * idx3 + 1] += im64;
    x->weight64[idx3] += w64;
    return;
  }
  x->volume[2 * idx3 + 0] += re;
  x->volume[2 * idx3 + 1] += im;
  x->weight[idx3] += w;
}

/* FR<>::ProcessVoxel (nearest pixel), fr_cpu_kernels.hpp:18-68 */
static void voxel_nearest_f(ctx_t *x, const or_traverse_space *s, int X, int Y, int Z)
{
  const or_constants *c = &x->c;
  float p[3] = { (float)(X - c->cMaxVolumeIndexX / 2), (float)(Y - c->cMaxVolumeIndexYZ / 2),
    (float)(Z - c->cMaxVolumeIndexYZ / 2) };
  if (p[0] * p[0] + p[1] * p[1] + p[2] * p[2] > s->maxDistanceSqr) return;
  mul3f(s->transformInv, p);
  if (p[0] < 0.f) return;
  int imgX = clampi((int)(p[0] + 0.5f), 0, x->xSize - 1);
  int imgY = clampi((int)(p[1] + 0.5f + (float)(c->cMaxVolumeIndexYZ / 2)), 0, x->ySize - 1);
  if (!in_volume(x, X, Y, Z)) return;
  if (x->mode == 2) {
    x->count[0]++;
    return;
  }
  size_t idx3 = ((size_t)Z * x->vy + (size_t)Y) * x->vx + (size_t)X;
  const float *px = x->fft + 2 * ((size_t)imgY * (size_t)x->xSize + (size_t)imgX);
  if (x->mode == 3) {
    double w64 = (double)s->weight;
    x->volume64[2 * idx3 + 0] += (double)px[0] * w64;
    x->volume64[2 * idx3 + 1] += (double)px[1] * w64;
    x->weight64[idx3] += w64;
    return;
  }
  float w = 1.f * s->weight;
  x->volume[2 * idx3 + 0] += px[0] * w;
  x->volume[2 * idx3 + 1] += px[1] * w;
  x->weight[idx3] += w;
}

/* The same voxel update in FP64 (blob gather or nearest pixel). */
static void voxel_d(ctx_t *x, const or_traverse_space *s, int X, int Y, int Z, int fast)
{
  const or_constants *c = &x->c;
  double p0 = X - c->cMaxVolumeIndexX / 2, p1 = Y - c->cMaxVolumeIndexYZ / 2,
         p2 = Z - c->cMaxVolumeIndexYZ / 2;
  if (p0 * p0 + p1 * p1 + p2 * p2 > (double)s->maxDistanceSqr) return;
  const float(*T)[3] = s->transformInv;
  double q0 = (double)T[0][0] * p0 + (double)T[0][1] * p1 + (double)T[0][2] * p2;
  double q1 = (double)T[1][0] * p0 + (double)T[1][1] * p1 + (double)T[1][2] * p2;
  double q2 = (double)T[2][0] * p0 + (double)T[2][1] * p1 + (double)T[2][2] * p2;
  if (!in_volume(x, X, Y, Z)) return;
  size_t idx3 = ((size_t)Z * x->vy + (size_t)Y) * x->vx + (size_t)X;
  double dataWeight = s->weight;
  double r = c->cBlobRadius;
  if (fast) {
    if (q0 < 0.0) return;
    int imgX = clampi((int)(q0 + 0.5), 0, x->xSize - 1);
    int imgY = clampi((int)(q1 + 0.5 + (double)(c->cMaxVolumeIndexYZ / 2)), 0, x->ySize - 1);
    const float *px = x->fft + 2 * ((size_t)imgY * (size_t)x->xSize + (size_t)imgX);
    x->volume64[2 * idx3 + 0] += px[0] * dataWeight;
    x->volume64[2 * idx3 + 1] += px[1] * dataWeight;
    x->weight64[idx3] += dataWeight;
    return;
  }
  if (q0 < -r) return;
  q1 += (double)(c->cMaxVolumeIndexYZ / 2);
  double rSq = r * r, zSq = q2 * q2;
  if (zSq > rSq) return;
  int minX = (int)ceil(q0 - r), maxX = (int)floor(q0 + r);
  int minY = (int)ceil(q1 - r), maxY = (int)floor(q1 + r);
  if (minX < 0) minX = 0;
  if (minY < 0) minY = 0;
  if (maxX > x->xSize - 1) maxX = x->xSize - 1;
  if (maxY > x->ySize - 1) maxY = x->ySize - 1;
  double w = 0, re = 0, im = 0;
  for (int i = minY; i <= maxY; i++) {
    double yzSq = (q1 - i) * (q1 - i) + zSq;
    if (yzSq > rSq) continue;
    for (int j = minX; j <= maxX; j++) {
      double d2 = (q0 - j) * (q0 - j) + yzSq;
      if (d2 > rSq) continue;
      double wb;
      if (x->interpolation == 1) {
        wb = x->table64[(int)(d2 * x->cIDeltaSqrt64 + 0.5)];
      } else if (x->fastKaiser) {
        double arg = (double)c->cBlobAlpha * sqrt(1.0 - d2 / rSq);
        wb = be_i0(arg) * x->cOneOverBessi64 * x->cIw0_64;
      } else {
        wb = kaiser_value_d(sqrt(d2), r, c->cBlobAlpha, x->order) * x->cIw0_64;
      }
      double wt = wb * dataWeight;
      const float *px = x->fft + 2 * ((size_t)i * (size_t)x->xSize + (size_t)j);
      w += wt;
      re += px[0] * wt;
      im += px[1] * wt;
    }
  }
  x->volume64[2 * idx3 + 0] += re;
  x->volume64[2 * idx3 + 1] += im;
  x->weight64[idx3] += w;
}

static void visit(ctx_t *x, const or_traverse_space *s, int X, int Y, int Z, int fast)
{
  if (x->mode == 1)
    voxel_d(x, s, X, Y, Z, fast);
  else if (fast)
    voxel_nearest_f(x, s, X, Y, Z);
  else
    voxel_blob_f(x, s, X, Y, Z);
}

/* Plane intersections, libumpalumpa/math/geometry.hpp:11-33 */
static inline float plane_z(float x, float y, const float *n, const float *p0)
{
  return (-n[0] * (x - p0[0]) - n[1] * (y - p0[1])) / n[2] + p0[2];
}
static inline float plane_y(float x, float z, const float *n, const float *p0)
{
  return (-n[0] * (x - p0[0]) - n[2] * (z - p0[2])) / n[1] + p0[1];
}
static inline float plane_x(float y, float z, const float *n, const float *p0)
{
  return (-n[1] * (y - p0[1]) - n[2] * (z - p0[2])) / n[0] + p0[0];
}

/* FR<>::Execute<order>: walk the traverse space's AABB along its dominant plane and the
 * blob slab between the two padded planes (fr_cpu_kernels.hpp:154-240). */
static void traverse(ctx_t *x, const or_traverse_space *s, int fast)
{
  const or_constants *c = &x->c;
  const float *n = s->unitNormal;
  if (s->dir == 0) { /* XY */
    for (int b = s->minY; b <= s->maxY; b++)
      for (int a = s->minX; a <= s->maxX; a++) {
        if (fast) {
          visit(x, s, a, b, (int)(plane_z((float)a, (float)b, n, s->bottomOrigin) + 0.5f), 1);
          continue;
        }
        float z1 = clampf(plane_z((float)a, (float)b, n, s->bottomOrigin), 0.f, (float)c->cMaxVolumeIndexYZ);
        float z2 = clampf(plane_z((float)a, (float)b, n, s->topOrigin), 0.f, (float)c->cMaxVolumeIndexYZ);
        int lo = (int)floorf(fminf(z1, z2)), hi = (int)ceilf(fmaxf(z1, z2));
        for (int z = lo; z <= hi; z++) visit(x, s, a, b, z, 0);
      }
  } else if (s->dir == 1) { /* XZ */
    for (int b = s->minZ; b <= s->maxZ; b++)
      for (int a = s->minX; a <= s->maxX; a++) {
        if (fast) {
          visit(x, s, a, (int)(plane_y((float)a, (float)b, n, s->bottomOrigin) + 0.5f), b, 1);
          continue;
        }
        float y1 = clampf(plane_y((float)a, (float)b, n, s->bottomOrigin), 0.f, (float)c->cMaxVolumeIndexYZ);
        float y2 = clampf(plane_y((float)a, (float)b, n, s->topOrigin), 0.f, (float)c->cMaxVolumeIndexYZ);
        int lo = (int)floorf(fminf(y1, y2)), hi = (int)ceilf(fmaxf(y1, y2));
        for (int y = lo; y <= hi; y++) visit(x, s, a, y, b, 0);
      }
  } else { /* YZ */
    for (int b = s->minZ; b <= s->maxZ; b++)
      for (int a = s->minY; a <= s->maxY; a++) {
        if (fast) {
          visit(x, s, (int)(plane_x((float)a, (float)b, n, s->bottomOrigin) + 0.5f), a, b, 1);
          continue;
        }
        float x1 = clampf(plane_x((float)a, (float)b, n, s->bottomOrigin), 0.f, (float)c->cMaxVolumeIndexX);
        float x2 = clampf(plane_x((float)a, (float)b, n, s->topOrigin), 0.f, (float)c->cMaxVolumeIndexX);
        int lo = (int)floorf(fminf(x1, x2)), hi = (int)ceilf(fmaxf(x1, x2));
        for (int xx = lo; xx <= hi; xx++) visit(x, s, xx, a, b, 0);
      }
  }
}

static void run_all(ctx_t *x, const float *fft, const or_traverse_space *spaces, size_t n, int fast)
{
  size_t plane = (size_t)x->xSize * (size_t)x->ySize;
  for (size_t i = 0; i < n; ++i) {
    x->fft = fft ? fft + 2 * plane * (size_t)spaces[i].projectionIndex : NULL;
    traverse(x, &spaces[i], fast);
  }
}

/* Double-precision runs (modes 1 and 3) over `threads` host threads: thread t inserts the
 * contiguous space range [t n / T, (t + 1) n / T) into private zeroed volume and weights, and
 * the partials are added into the caller's arrays in thread order (a fixed summation order
 * for a given T; the reference's Execute is serial over spaces, fr_cpu_kernels.hpp:254). */
typedef struct {
  ctx_t x;
  const float *fft;
  const or_traverse_space *spaces;
  size_t n;
  int fast;
} job_t;

static void *run_job(void *arg)
{
  job_t *j = (job_t *)arg;
  run_all(&j->x, j->fft, j->spaces, j->n, j->fast);
  return NULL;
}

static int run_all_double(ctx_t *x, const float *fft, const or_traverse_space *spaces, size_t n, int fast,
  int threads)
{
  const size_t vox = x->vx * x->vy * x->vz;
  if (threads < 1) threads = 1;
  if ((size_t)threads > n) threads = n > 0 ? (int)n : 1;
  if (threads == 1) {
    run_all(x, fft, spaces, n, fast);
    return 0;
  }
  job_t *jobs = (job_t *)calloc((size_t)threads, sizeof(job_t));
  pthread_t *tids = (pthread_t *)calloc((size_t)threads, sizeof(pthread_t));
  if (!jobs || !tids) {
    free(jobs);
    free(tids);
    return 2;
  }
  int rc = 0, started = 0;
  for (int t = 0; t < threads; ++t) {
    job_t *j = &jobs[t];
    j->x = *x;
    j->x.volume64 = (double *)calloc(2 * vox, sizeof(double));
    j->x.weight64 = (double *)calloc(vox, sizeof(double));
    if (!j->x.volume64 || !j->x.weight64) {
      rc = 2;
      break;
    }
    const size_t b = n * (size_t)t / (size_t)threads, e = n * (size_t)(t + 1) / (size_t)threads;
    j->fft = fft;
    j->spaces = spaces + b;
    j->n = e - b;
    j->fast = fast;
  }
  if (rc == 0) {
    for (; started < threads; ++started)
      if (pthread_create(&tids[started], NULL, run_job, &jobs[started]) != 0) {
        rc = 3;
        break;
      }
    for (int t = 0; t < started; ++t) pthread_join(tids[t], NULL);
  }
  if (rc == 0)
    for (int t = 0; t < threads; ++t) {
      for (size_t i = 0; i < 2 * vox; ++i) x->volume64[i] += jobs[t].x.volume64[i];
      for (size_t i = 0; i < vox; ++i) x->weight64[i] += jobs[t].x.weight64[i];
    }
  for (int t = 0; t < threads; ++t) {
    free(jobs[t].x.volume64);
    free(jobs[t].x.weight64);
  }
  free(jobs);
  free(tids);
  return rc;
}

int or_fr_execute(float *volume, float *weight, size_t vx, size_t vy, size_t vz,
  const float *fft, size_t fftX, size_t fftY, const or_traverse_space *spaces, size_t nSpaces,
  const float *table, size_t tableElems, int interpolation, int order, int type, float alpha,
  float radius)
{
  if (interpolation == 1 && (table == NULL || tableElems == 0)) return 1; /* fr_cpu.cpp:27-29 */
  ctx_t x;
  memset(&x, 0, sizeof(x));
  x.volume = volume;
  x.weight = weight;
  x.vx = vx;
  x.vy = vy;
  x.vz = vz;
  x.xSize = (int)fftX;
  x.ySize = (int)fftY;
  x.table = table;
  x.interpolation = interpolation;
  x.order = order;
  x.fastKaiser = alpha <= 15.f; /* fr_cpu.cpp:31 */
  x.mode = 0;
  or_make_constants(vx, vy, interpolation == 1 ? tableElems : 0, order, alpha, radius, &x.c);
  run_all(&x, fft, spaces, nSpaces, type == 0);
  return 0;
}

int or_fr_execute_f64(double *volume, double *weight, size_t vx, size_t vy, size_t vz,
  const float *fft, size_t fftX, size_t fftY, const or_traverse_space *spaces, size_t nSpaces,
  size_t tableElems, int interpolation, int order, int type, float alpha, float radius, int threads)
{
  if (interpolation == 1 && tableElems < 2) return 1;
  ctx_t x;
  memset(&x, 0, sizeof(x));
  x.volume64 = volume;
  x.weight64 = weight;
  x.vx = vx;
  x.vy = vy;
  x.vz = vz;
  x.xSize = (int)fftX;
  x.ySize = (int)fftY;
  x.interpolation = interpolation;
  x.order = order;
  x.fastKaiser = alpha <= 15.f;
  x.mode = 1;
  or_make_constants(vx, vy, interpolation == 1 ? tableElems : 0, order, alpha, radius, &x.c);
  double r = radius;
  x.cIw0_64 = 1.0 / kaiser_fourier_value_d(0.0, r, alpha, order);
  x.cOneOverBessi64 = 1.0 / as_in(order, alpha);
  double *t64 = NULL;
  if (interpolation == 1) {
    t64 = (double *)malloc(tableElems * sizeof(double));
    if (!t64) return 2;
    double freq = r * sqrt(1.0 / (double)(tableElems - 1));
    for (size_t i = 0; i < tableElems; ++i)
      t64[i] = kaiser_value_d(freq * sqrt((double)i), r, alpha, order) * x.cIw0_64;
    x.cIDeltaSqrt64 = (double)(tableElems - 1) / (r * r);
  }
  x.table64 = t64;
  int rc = run_all_double(&x, fft, spaces, nSpaces, type == 0, threads);
  free(t64);
  return rc;
}

int or_fr_execute_fd64(double *volume, double *weight, size_t vx, size_t vy, size_t vz,
  const float *fft, size_t fftX, size_t fftY, const or_traverse_space *spaces, size_t nSpaces,
  const float *table, size_t tableElems, int interpolation, int order, int type, float alpha,
  float radius, int threads)
{
  if (interpolation == 1 && (table == NULL || tableElems == 0)) return 1; /* fr_cpu.cpp:27-29 */
  ctx_t x;
  memset(&x, 0, sizeof(x));
  x.volume64 = volume;
  x.weight64 = weight;
  x.vx = vx;
  x.vy = vy;
  x.vz = vz;
  x.xSize = (int)fftX;
  x.ySize = (int)fftY;
  x.table = table;
  x.interpolation = interpolation;
  x.order = order;
  x.fastKaiser = alpha <= 15.f; /* fr_cpu.cpp:31 */
  x.mode = 3;
  or_make_constants(vx, vy, interpolation == 1 ? tableElems : 0, order, alpha, radius, &x.c);
  return run_all_double(&x, fft, spaces, nSpaces, type == 0, threads);
}

void or_count_slab_voxels(size_t vx, size_t vy, size_t vz, size_t fftX, size_t fftY,
  const or_traverse_space *spaces, size_t nSpaces, int type, float radius, int64_t *counts)
{
  ctx_t x;
  memset(&x, 0, sizeof(x));
  x.vx = vx;
  x.vy = vy;
  x.vz = vz;
  x.xSize = (int)fftX;
  x.ySize = (int)fftY;
  x.mode = 2;
  or_make_constants(vx, vy, 0, 0, 15.f, radius, &x.c);
  for (size_t i = 0; i < nSpaces; ++i) {
    counts[i] = 0;
    x.count = &counts[i];
    traverse(&x, &spaces[i], type == 0);
  }
}
