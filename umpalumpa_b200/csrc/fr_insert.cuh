// The insertion kernel of the B200 Fourier-reconstruction engine.
//
// Why it is not the reference's ProcessKernel: the reference launches a 2D grid over the
// volume face and lets every CTA walk every traverse space, doing three global float
// atomics per voxel per projection (fr_cuda_kernels.cu:362-365,468-523).  Here the volume is
// cut into 16^3-voxel bricks.  The binning passes (fr_kernels.cu) list, per brick, the
// traverse spaces whose blob slab can touch it, grouped by traversal direction; this
// persistent kernel takes (brick, list range) work items, accumulates all their
// projections into shared-memory accumulators and adds the brick into the caller's volume
// once per item.
//
// The per-voxel arithmetic is the reference's ProcessVoxelBlob / ProcessVoxel
// (fr_cpu_kernels.hpp:18-152); the voxels visited are the reference's traversal
// (fr_cpu_kernels.hpp:154-240): for a space of direction XY the column (x, y) of the
// traversal AABB is walked along z across the blob slab, for XZ along y, for YZ along x.
//
// Work split: a CTA runs several independent 256-thread groups, each working on its own
// brick (Groups below); a batched launch (JOBS) takes the items of several jobs, each item
// naming its job in the job table.  Warp w of a group owns the 32 brick columns (U, V) = (tx, w + 8 ty),
// tx < 16, ty < 2, of the current direction.  Per projection each lane finds its column's voxel range;
// the warp then deals the warp's voxels out to its lanes 32 at a time (prefix sum + binary
// search over shuffles), so lanes stay busy whatever the column lengths.  Within one
// direction a warp touches only its own columns, so projections need no synchronisation
// beyond __syncwarp; a group synchronises (named barrier) only when the direction changes.
//
// Half-plane layouts (BANDED): the caller's row-major half-planes, or the same pixels in bands
// of four rows stored column by column (pixel (y, x) at (y / 4) * bandStride + 4 x + y % 4,
// band_projections in fr_kernels.cu).  A warp's 32 voxels map to a compact patch of the image;
// in bands a blob tap of the patch touches about 3 cache lines where rows take about 5, which
// cuts the L1 wavefronts of the pixel gathers by about a quarter.
#pragma once

#include "fr_device.cuh"
#include "fr_kernels.h"

namespace frb {

enum { kModeLut = 0, kModeFastKaiser = 1, kModeKaiser = 2, kModeKaiserTable = 3 };

// Traversal plane axes (U, V) and column axis W per direction (traverse_space.hpp:24-28).
template<int DIR> struct Axes;
template<> struct Axes<FR_DIR_XY> { static constexpr int U = 0, V = 1, W = 2; };
template<> struct Axes<FR_DIR_XZ> { static constexpr int U = 0, V = 2, W = 1; };
template<> struct Axes<FR_DIR_YZ> { static constexpr int U = 1, V = 2, W = 0; };

template<int K, typename T> __device__ __forceinline__ T pick3(T a, T b, T c)
{
  return K == 0 ? a : (K == 1 ? b : c);
}

// Brick accumulators are [z][y][x] with x swizzled by (z + y/2) mod 16, so that the voxels
// of any x-, y- or z-column fall into distinct shared-memory banks.
__device__ __forceinline__ int acc_index(int x, int y, int z)
{
  return (z * kBrick + y) * kBrick + (x ^ ((z + (y >> 1)) & (kBrick - 1)));
}

// Sizes and payloads of the job a work item belongs to.  A single-job launch builds it from
// the launch parameters (so the compiler reads them as constant operands); a batched launch
// loads it from the job table for every work item.
struct JobGeom {
  const void *fft;
  const float *scales;
  void *volume;
  float *weight;
  int fftX, fftY, vx, vy, vz, nbx, nby, cx, cy, cz;
  int genericTaps;
  int bandStride;  // banded half-planes: elements per 4-row band
};

__device__ __forceinline__ JobGeom geom_of(const InsertParams &P)
{
  JobGeom g;
  g.fft = P.fft;
  g.scales = P.scales;
  g.volume = P.volume;
  g.weight = P.weight;
  g.fftX = P.fftX;
  g.fftY = P.fftY;
  g.vx = P.vx;
  g.vy = P.vy;
  g.vz = P.vz;
  g.nbx = P.nbx;
  g.nby = P.nby;
  g.cx = P.cx;
  g.cy = P.cy;
  g.cz = P.cz;
  g.genericTaps = P.genericTaps;
  g.bandStride = P.bandStride;
  return g;
}

__device__ __forceinline__ JobGeom geom_of(const JobDesc &J)
{
  JobGeom g;
  g.fft = J.fft;
  g.scales = J.scales;
  g.volume = J.volume;
  g.weight = J.weight;
  g.fftX = J.fftX;
  g.fftY = J.fftY;
  g.vx = J.vx;
  g.vy = J.vy;
  g.vz = J.vz;
  g.nbx = J.nbx;
  g.nby = J.nby;
  g.cx = J.cx;
  g.cy = J.cy;
  g.cz = J.cz;
  g.genericTaps = J.genericTaps;
  g.bandStride = J.bandStride;
  return g;
}

struct Accum {
  float *re, *im, *w;              // brick accumulators
  __nv_bfloat16 *cre, *cim, *cw;   // Kahan compensations (KAHAN only)
};

// Kahan-compensated add.  The compensation -- the rounding error of the previous add, at most
// half an ulp of the sum -- is kept in BF16: its 8 significant bits leave each add at most
// 1/256 of plain FP32's rounding residual, and 18 instead of 24 bytes per voxel let the blob
// table stay in shared memory beside two brick groups.
template<bool KAHAN>
__device__ __forceinline__ void acc_add(float *sum, __nv_bfloat16 *comp, int i, float v)
{
  if (KAHAN) {
    const float y = __fsub_rn(v, __bfloat162float(comp[i]));
    const float t = __fadd_rn(sum[i], y);
    comp[i] = __float2bfloat16_rn(__fsub_rn(__fsub_rn(t, sum[i]), y));
    sum[i] = t;
  } else {
    sum[i] += v;
  }
}

// The fields of a SpaceRec the kernel reads, loaded with 16-byte broadcast loads: load_rec
// reads what the column phase needs, run_direction the voxel fields after it (the rotation, in
// banded kernels, for every voxel: load_rotation).
struct RecView {
  float T[9];
  float maxDist2, weight;
  int proj;
  int lo0, hi0, lo1, hi1;
  float w0, wu, wv, hw;
  float nu, nv, nw, bu, bv, bw;
  float xu, xv, xw, xwInv;
};

template<bool FAST>
__device__ __forceinline__ void load_rec(const SpaceRec *r, RecView &v)
{
  const float4 *q = reinterpret_cast<const float4 *>(r);
  const float4 f2 = __ldg(q + 2), f3 = __ldg(q + 3);
  const float4 f4 = __ldg(q + 4);
  v.maxDist2 = f2.y;
  v.lo0 = __float_as_int(f3.x);
  v.hi0 = __float_as_int(f3.y);
  v.lo1 = __float_as_int(f3.z);
  v.hi1 = __float_as_int(f3.w);
  v.w0 = f4.x; v.wu = f4.y; v.wv = f4.z; v.hw = f4.w;
  if (FAST) {
    const float4 f5 = __ldg(q + 5), f6 = __ldg(q + 6);
    v.nu = f5.x; v.nv = f5.y; v.nw = f5.z; v.bu = f5.w; v.bv = f6.x; v.bw = f6.y;
  } else {
    const float4 f6 = __ldg(q + 6), f7 = __ldg(q + 7);
    v.xu = f6.z; v.xv = f6.w; v.xwInv = f7.x; v.xw = f7.y;
  }
}

// The nine entries of transformInv (the record's first 36 bytes).  Volatile, so that the
// compiler re-reads them where they are used instead of keeping them live in registers.
__device__ __forceinline__ void load_rotation(const float4 *rec, float *T)
{
  asm volatile("ld.global.nc.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(T[0]), "=f"(T[1]), "=f"(T[2]), "=f"(T[3]) : "l"(rec));
  asm volatile("ld.global.nc.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(T[4]), "=f"(T[5]), "=f"(T[6]), "=f"(T[7]) : "l"(rec + 1));
  asm volatile("ld.global.nc.f32 %0, [%1];" : "=f"(T[8]) : "l"(rec + 2));
}

// FR<>::ProcessVoxelBlob (fr_cpu_kernels.hpp:70-152) for voxel (X, Y, Z): Kaiser-Bessel
// gather of the projection pixels within the blob radius.  The blob weights are summed raw
// and scaled by the space weight (and the storage scale) once at the end.  Returns false if
// the voxel is rejected.
template<int MODE, int TAPS, int STORAGE, bool GENERIC, bool BANDED>
__device__ __forceinline__ bool voxel_blob(const InsertParams &P, const JobGeom &G, const RecView &s,
  const typename Pixel<STORAGE>::T *__restrict__ img, int bandStride, float scale, const float *lut, int X,
  int Y, int Z, float &ore, float &oim, float &ow)
{
  const fr_constants &c = P.c;
  const float px = float(X - G.cx), py = float(Y - G.cy), pz = float(Z - G.cz);
  if (px * px + py * py + pz * pz > s.maxDist2) return false;  // integer-valued: exact
  const float qx = add_(add_(mul_(s.T[0], px), mul_(s.T[1], py)), mul_(s.T[2], pz));
  const float qy0 = add_(add_(mul_(s.T[3], px), mul_(s.T[4], py)), mul_(s.T[5], pz));
  const float qz = add_(add_(mul_(s.T[6], px), mul_(s.T[7], py)), mul_(s.T[8], pz));
  const float r = c.cBlobRadius;
  if (qx < -r) return false;
  const float qy = add_(qy0, float(G.cy));
  const float rSq = mul_(r, r);
  const float zSq = mul_(qz, qz);
  if (zSq > rSq) return false;
  // no pixel lies within the blob radius (also rejects non-finite coordinates)
  if (!(qx <= float(G.fftX) + r && qy >= -r && qy <= float(G.fftY) + r)) return false;
  // The TAPS x TAPS window starts at (ceil(qx - r), ceil(qy - r)) shifted into the image, so
  // it covers the reference's clamped blob box [max(ceil(q - r), 0), min(floor(q + r), X-1)]
  // and lies inside the image; candidates outside the blob box have d2 > r^2, so d2 <= r^2
  // is the only per-tap test (FR::ProcessVoxelBlob's radius test, fr_cpu_kernels.hpp:128-134).
  // GENERIC (a half-plane narrower or shorter than the window) tests the blob box explicitly.
  int minX = max(int(ceilf(sub_(qx, r))), 0);
  int minY = max(int(ceilf(sub_(qy, r))), 0);
  const int maxX = min(int(floorf(add_(qx, r))), G.fftX - 1);
  const int maxY = min(int(floorf(add_(qy, r))), G.fftY - 1);
  if (!GENERIC) {
    minX = min(minX, G.fftX - TAPS);
    minY = min(minY, G.fftY - TAPS);
  }
  const float dx0 = sub_(qx, float(minX));
  // Taps are evaluated in pairs with packed FP32x2 arithmetic: per pair one fused d2 and one
  // fused table position, per tap one fused complex accumulation.  Each lane rounds exactly
  // like the scalar fmaf it replaces.
  float2 dxp[TAPS / 2];
#pragma unroll
  for (int k = 0; k < TAPS / 2; ++k) dxp[k] = make_float2(dx0 - float(2 * k), dx0 - float(2 * k + 1));
  const float2 cI2 = make_float2(c.cIDeltaSqrt, c.cIDeltaSqrt);
  const float2 kt2 = make_float2(P.tableScale, P.tableScale);
  const float alpha2 = c.cBlobAlpha * c.cBlobAlpha, ks = c.cOneOverBessiOrderAlpha * c.cIw0;
  const float2 half2 = make_float2(0.5f, 0.5f);
  float2 acc = make_float2(0.f, 0.f);
  float w = 0.f;
  auto tap = [&](const typename Pixel<STORAGE>::T *row, int ii, int jj, float d2, float pos) {
    const bool inBox = !GENERIC || (minY + ii <= maxY && minX + jj <= maxX);
    if (inBox && d2 <= rSq) {
      float wb;
      if (MODE == kModeLut) {
        // With at most 16,384 table entries (cIDeltaSqrt = (N-1)/r^2; the table in shared or,
        // beside Kahan accumulators, global memory), d2 <= r^2 bounds the position by
        // N - 1 + 0.5 + N * 2^-23 < N: no clamp needed.
        const int li = int(pos);
        wb = lut[GENERIC ? min(li, P.tableElems - 1) : li];
      } else if (MODE == kModeKaiserTable) {
        // pos = d2 (N-1) / r^2 in [0, N-1] (d2 <= r^2, rounding keeps it below N): node and
        // fraction, then value + slope * fraction
        const int li = GENERIC ? min(int(pos), P.tableElems - 1) : int(pos);
        const float2 e = reinterpret_cast<const float2 *>(lut)[li];
        wb = fmaf(e.y, pos - float(li), e.x);
      } else if (MODE == kModeFastKaiser) {
        wb = pos;  // the pair's weights, computed below with kaiser_value_fast2
      } else {
        wb = kaiser_value_f(sqrtf(d2), r, c.cBlobAlpha, c.cOneOverBessiOrderAlpha, P.order) * c.cIw0;
      }
      const float2 v = Pixel<STORAGE>::load(row + (BANDED ? 4 * jj : jj));
      w += wb;
      acc = __ffma2_rn(v, make_float2(wb, wb), acc);
    }
  };
#pragma unroll
  for (int ii = 0; ii < TAPS; ++ii) {
    const float dy = sub_(qy, float(minY + ii));
    const float yz = add_(mul_(dy, dy), zSq);
    const float2 yz2 = make_float2(yz, yz);
    const int ry = minY + ii;
    const typename Pixel<STORAGE>::T *row =
      BANDED ? img + size_t(ry / 4) * size_t(bandStride) + (ry % 4) + 4 * minX : img + size_t(ry) * G.fftX + minX;
#pragma unroll
    for (int k = 0; k < TAPS / 2; ++k) {
      const float2 d2 = __ffma2_rn(dxp[k], dxp[k], yz2);
      // per tap: the table position (lookup), the blob weight (fast Kaiser) or d2
      const float2 pos = MODE == kModeLut            ? __ffma2_rn(d2, cI2, half2)
                         : MODE == kModeKaiserTable ? __fmul2_rn(d2, kt2)
                         : MODE == kModeFastKaiser  ? kaiser_value_fast2(d2, alpha2, c.cOneOverBlobRadiusSqr, ks)
                                                    : d2;
      tap(row, ii, 2 * k, d2.x, pos.x);
      tap(row, ii, 2 * k + 1, d2.y, pos.y);
    }
  }
  const float dw = mul_(s.weight, scale);
  const float2 o = __fmul2_rn(acc, make_float2(dw, dw));
  ore = o.x;
  oim = o.y;
  ow = mul_(w, s.weight);
  return true;
}

// FR<>::ProcessVoxel (fr_cpu_kernels.hpp:18-68): nearest pixel.
template<int STORAGE, bool BANDED>
__device__ __forceinline__ bool voxel_nearest(const JobGeom &G, const RecView &s,
  const typename Pixel<STORAGE>::T *__restrict__ img, int bandStride, float scale, int X, int Y, int Z,
  float &ore, float &oim, float &ow)
{
  const float px = float(X - G.cx), py = float(Y - G.cy), pz = float(Z - G.cz);
  if (px * px + py * py + pz * pz > s.maxDist2) return false;
  const float qx = add_(add_(mul_(s.T[0], px), mul_(s.T[1], py)), mul_(s.T[2], pz));
  const float qy = add_(add_(mul_(s.T[3], px), mul_(s.T[4], py)), mul_(s.T[5], pz));
  if (qx < 0.f) return false;
  const int imgX = min(max(int(add_(qx, 0.5f)), 0), G.fftX - 1);
  const int imgY = min(max(int(add_(add_(qy, 0.5f), float(G.cy))), 0), G.fftY - 1);
  const float2 v = Pixel<STORAGE>::load(BANDED ? img + size_t(imgY / 4) * size_t(bandStride) + 4 * imgX + imgY % 4
                                               : img + size_t(imgY) * G.fftX + imgX);
  const float w = s.weight;
  const float wt = mul_(w, scale);
  ore = mul_(v.x, wt);
  oim = mul_(v.y, wt);
  ow = w;
  return true;
}

// All list entries [e0, e1) of one direction for the brick at (ox, oy, oz).
template<int DIR, int MODE, int TAPS, bool FAST, int STORAGE, bool KAHAN, bool JOBS, bool BANDED>
__device__ __forceinline__ void run_direction(const InsertParams &P, const JobGeom &G, const Accum &A,
  const float *lut, int ox, int oy, int oz, int warp, int lane, int e0, int e1)
{
  using AX = Axes<DIR>;
  using PT = typename Pixel<STORAGE>::T;
  const PT *fft = reinterpret_cast<const PT *>(G.fft);
  // a single-job launch reads the band stride as a constant operand of the launch parameters
  const int bandStride = JOBS ? G.bandStride : P.bandStride;
  const size_t plane = BANDED ? size_t((G.fftY + 3) / 4) * size_t(bandStride) : size_t(G.fftX) * size_t(G.fftY);
  const int oU = pick3<AX::U>(ox, oy, oz), oV = pick3<AX::V>(ox, oy, oz), oW = pick3<AX::W>(ox, oy, oz);
  const int nU = pick3<AX::U>(G.vx, G.vy, G.vz), nV = pick3<AX::V>(G.vx, G.vy, G.vz);
  const int nW = pick3<AX::W>(G.vx, G.vy, G.vz);
  // warp w owns column rows w and w + 8: a slab that crosses part of the brick face spreads
  // over the warps instead of piling onto a few (2 % faster than adjacent rows)
  const int tu = lane & (kBrick - 1), tv = warp + 8 * (lane >> 4);
  const int U = oU + tu, V = oV + tv;
  const bool colIn = U < nU && V < nV;
  const int wLo = oW, wHi = min(oW + kBrick, nW) - 1;
  const float uf = float(U), vf = float(V);
  const float du = float(U - pick3<AX::U>(G.cx, G.cy, G.cz)), dv = float(V - pick3<AX::V>(G.cx, G.cy, G.cz));
  const float cw = float(pick3<AX::W>(G.cx, G.cy, G.cz));
  const float r = P.c.cBlobRadius;
  for (int e = e0; e < e1; ++e) {
    const int si = __ldg(P.list + e);
    RecView s;
    load_rec<FAST>(P.recs + si, s);
    // this lane's column range
    int lo = 1, hi = 0;
    if (colIn && U >= s.lo0 && U <= s.hi0 && V >= s.lo1 && V <= s.hi1) {
      if (FAST) {
        lo = hi = int(add_(plane_hit(uf, vf, s.nu, s.nv, s.nw, s.bu, s.bv, s.bw), 0.5f));
      } else {
        // slab |t2.p| <= r, frequency sphere |p|^2 <= maxDist2 and image half-space
        // t0.p >= -r, each widened by a margin; the voxel checks decide exactly
        const float wc = fmaf(s.wu, uf, fmaf(s.wv, vf, s.w0));
        float flo = wc - s.hw, fhi = wc + s.hw;
        const float rem = s.maxDist2 - du * du - dv * dv;
        const float sq = sqrtf(fmaxf(rem, 0.f)) + 1e-3f;
        flo = fmaxf(flo, cw - sq);
        fhi = fminf(fhi, cw + sq);
        if (s.xwInv != 0.f) {
          const float b = cw + (-r - 0.01f - s.xu * du - s.xv * dv) * s.xwInv;
          if (s.xw > 0.f) flo = fmaxf(flo, b);
          else fhi = fminf(fhi, b);
        }
        lo = rem >= 0.f ? int(ceilf(flo)) : 1;
        hi = rem >= 0.f ? int(floorf(fhi)) : 0;
      }
      lo = max(lo, wLo);
      hi = min(hi, wHi);
    }
    const int cnt = max(hi - lo + 1, 0);
    // warp prefix sum of the column lengths
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    if (total == 0) continue;  // warp-uniform
    const int excl = incl - cnt;
    // Banded kernels read the rotation rows again (L1 hits) for every voxel instead of holding
    // them in registers through the voxel loop: they run at their register cap, and the nine
    // registers let the tap loads of a voxel stay in flight together (6 % faster).  The
    // row-major kernels keep them (re-reading costs them 3 %).
    const float4 *rec4 = reinterpret_cast<const float4 *>(P.recs + si);
    {
      const float4 f2 = __ldg(rec4 + 2);
      s.weight = f2.z;
      s.proj = __float_as_int(f2.w);
      if (!BANDED) {
        const float4 f0 = __ldg(rec4), f1 = __ldg(rec4 + 1);
        s.T[0] = f0.x; s.T[1] = f0.y; s.T[2] = f0.z; s.T[3] = f0.w;
        s.T[4] = f1.x; s.T[5] = f1.y; s.T[6] = f1.z; s.T[7] = f1.w;
        s.T[8] = f2.x;
      }
    }
    const float scale = STORAGE == FR_STORAGE_FP32 ? 1.f : __ldg(G.scales + s.proj);
    const PT *img = fft + size_t(s.proj) * plane;
    for (int base = 0; base < total; base += 32) {
      const int k = base + lane;
      // source lane: the largest s with excl_s <= k
      int src = 0;
#pragma unroll
      for (int step = 16; step >= 1; step >>= 1) {
        const int ex = __shfl_sync(0xffffffffu, excl, src + step);
        if (ex <= k) src += step;
      }
      const int wv = __shfl_sync(0xffffffffu, lo, src) + (k - __shfl_sync(0xffffffffu, excl, src));
      if (k < total) {
        if (BANDED) load_rotation(rec4, s.T);
        const int Uv = oU + (src & (kBrick - 1)), Vv = oV + warp + 8 * (src >> 4);
        const int X = AX::W == 0 ? wv : (AX::U == 0 ? Uv : Vv);
        const int Y = AX::W == 1 ? wv : (AX::U == 1 ? Uv : Vv);
        const int Z = AX::W == 2 ? wv : Vv;
        float re, im, w;
        bool ok;
        if (FAST)
          ok = voxel_nearest<STORAGE, BANDED>(G, s, img, bandStride, scale, X, Y, Z, re, im, w);
        else if (G.genericTaps)
          ok = voxel_blob<MODE, TAPS, STORAGE, true, BANDED>(P, G, s, img, bandStride, scale, lut, X, Y, Z, re, im, w);
        else
          ok = voxel_blob<MODE, TAPS, STORAGE, false, BANDED>(P, G, s, img, bandStride, scale, lut, X, Y, Z, re, im, w);
        if (ok) {
          const int li = acc_index(X - ox, Y - oy, Z - oz);
          acc_add<KAHAN>(A.re, A.cre, li, re);
          acc_add<KAHAN>(A.im, A.cim, li, im);
          acc_add<KAHAN>(A.w, A.cw, li, w);
        }
      }
    }
    __syncwarp();  // the next projection may revisit these voxels from other lanes
  }
}

// Shared-memory groups per CTA: one 256-thread group per brick in flight.  The groups of a CTA
// share one copy of the blob table, so three plain-accumulator groups (3 x 48 KB + 40 KB)
// fit on an SM where three separate CTAs would not.  Kahan accumulators (72 KB: FP32 sums and
// BF16 compensations) allow two groups beside the table.
// This is the most a CTA may hold; the launch picks 1..value groups (blockDim.x / 256).
template<bool KAHAN> struct Groups { static constexpr int value = KAHAN ? 2 : 3; };

__device__ __forceinline__ void group_sync(int group)
{
  asm volatile("bar.sync %0, %1;" ::"r"(group + 1), "r"(kThreads) : "memory");
}

template<int MODE, int TAPS, bool FAST, int STORAGE, bool KAHAN, bool JOBS, bool BANDED>
__global__ void __launch_bounds__(kThreads *Groups<KAHAN>::value, 1) insert_kernel(InsertParams P)
{
  constexpr int kMaxGroups = Groups<KAHAN>::value;
  constexpr int kAccFloats = (KAHAN ? 9 * kBrickVox / 2 : 3 * kBrickVox);  // 32-bit words
  const int nGroups = int(blockDim.x) / kThreads;  // launch shape: 1..kMaxGroups
  extern __shared__ float4 smem4[];
  float *smem = reinterpret_cast<float *>(smem4);
  __shared__ int sItem[kMaxGroups];
  // Batched launches: the current job's geometry, one copy per group in shared memory.  Held
  // in registers (as the single-job kernel may, where the values are constant operands of the
  // launch parameters) its 20 words spilled 80 bytes at the register cap.
  __shared__ JobGeom sGeom[kMaxGroups];
  const int group = threadIdx.x / kThreads;
  const int tid = threadIdx.x % kThreads;
  const int warp = tid >> 5, lane = tid & 31;
  float *acc = smem + group * kAccFloats;
  Accum A;
  A.re = acc;
  A.im = acc + kBrickVox;
  A.w = acc + 2 * kBrickVox;
  A.cre = reinterpret_cast<__nv_bfloat16 *>(acc + 3 * kBrickVox);
  A.cim = A.cre + kBrickVox;
  A.cw = A.cim + kBrickVox;
  float *lutS = smem + nGroups * kAccFloats;

  const float *lut = P.table;
  if ((MODE == kModeLut || MODE == kModeKaiserTable) && !FAST && P.lutInSmem) {
    const int nf = MODE == kModeKaiserTable ? 2 * P.tableElems : P.tableElems;  // float2 entries
    for (int i = threadIdx.x; i < nf; i += int(blockDim.x)) lutS[i] = __ldg(P.table + i);
    lut = lutS;
  }
  __syncthreads();
  const int nItems = *P.nItems;

  for (;;) {
    group_sync(group);
    if (tid == 0) sItem[group] = atomicAdd(P.workCounter, 1);
    group_sync(group);
    const int itIdx = sItem[group];
    if (itIdx >= nItems) break;
    const WorkItem it = P.items[itIdx];
    // (the group finished its previous item, flush included, before the barrier above)
    if (JOBS && tid == 0) sGeom[group] = geom_of(P.jobs[it.job]);
    for (int i = tid; i < kAccFloats; i += kThreads) acc[i] = 0.f;
    group_sync(group);
    JobGeom Gl;
    if (!JOBS) Gl = geom_of(P);
    const JobGeom &G = JOBS ? sGeom[group] : Gl;
    // batch-wide brick index; offsets and lists are batch-wide
    const int brick = it.brick - (JOBS ? P.jobs[it.job].brickBase : 0);
    const int bx = brick % G.nbx, by = (brick / G.nbx) % G.nby, bz = brick / (G.nbx * G.nby);
    const int ox = bx * kBrick, oy = by * kBrick, oz = bz * kBrick;
    const int base = 3 * it.brick;
    for (int dir = 0; dir < 3; ++dir) {
      const int e0 = max(it.begin, P.offsets[base + dir]);
      const int e1 = min(it.end, P.offsets[base + dir + 1]);
      if (e0 >= e1) continue;  // uniform across the group
      if (dir == FR_DIR_XY)
        run_direction<FR_DIR_XY, MODE, TAPS, FAST, STORAGE, KAHAN, JOBS, BANDED>(P, G, A, lut, ox, oy, oz, warp, lane,
          e0, e1);
      else if (dir == FR_DIR_XZ)
        run_direction<FR_DIR_XZ, MODE, TAPS, FAST, STORAGE, KAHAN, JOBS, BANDED>(P, G, A, lut, ox, oy, oz, warp, lane,
          e0, e1);
      else
        run_direction<FR_DIR_YZ, MODE, TAPS, FAST, STORAGE, KAHAN, JOBS, BANDED>(P, G, A, lut, ox, oy, oz, warp, lane,
          e0, e1);
      group_sync(group);  // the next direction maps warps to other voxels
    }
    // add the brick into the caller's volume
    for (int li = tid; li < kBrickVox; li += kThreads) {
      const int lz = li / (kBrick * kBrick), ly = (li / kBrick) & (kBrick - 1);
      const int lx = (li & (kBrick - 1)) ^ ((lz + (ly >> 1)) & (kBrick - 1));
      const int X = ox + lx, Y = oy + ly, Z = oz + lz;
      if (X >= G.vx || Y >= G.vy || Z >= G.vz) continue;
      float re = A.re[li], im = A.im[li], w = A.w[li];
      if (KAHAN) {
        re = __fsub_rn(re, __bfloat162float(A.cre[li]));
        im = __fsub_rn(im, __bfloat162float(A.cim[li]));
        w = __fsub_rn(w, __bfloat162float(A.cw[li]));
      }
      if (__float_as_uint(re) == 0u && __float_as_uint(im) == 0u && __float_as_uint(w) == 0u) continue;
      const size_t g = (size_t(Z) * G.vy + Y) * G.vx + X;
      atomicAdd(reinterpret_cast<float2 *>(G.volume) + g, make_float2(re, im));
      atomicAdd(G.weight + g, w);
    }
  }
}

template<int MODE, bool FAST, int STORAGE, bool KAHAN, bool JOBS, bool BANDED>
static InsertFn pick_taps(int taps)
{
  if (taps <= 4) return insert_kernel<MODE, 4, FAST, STORAGE, KAHAN, JOBS, BANDED>;
  return insert_kernel<MODE, 8, FAST, STORAGE, KAHAN, JOBS, BANDED>;
}

template<int STORAGE, bool KAHAN, bool JOBS, bool BANDED>
static InsertFn pick_mode(const InsertConfig &cfg)
{
  if (cfg.fast) return insert_kernel<kModeLut, 4, true, STORAGE, KAHAN, JOBS, BANDED>;
  switch (cfg.mode) {
  case kModeLut: return pick_taps<kModeLut, false, STORAGE, KAHAN, JOBS, BANDED>(cfg.taps);
  case kModeFastKaiser: return pick_taps<kModeFastKaiser, false, STORAGE, KAHAN, JOBS, BANDED>(cfg.taps);
  case kModeKaiserTable: return pick_taps<kModeKaiserTable, false, STORAGE, KAHAN, JOBS, BANDED>(cfg.taps);
  default: return pick_taps<kModeKaiser, false, STORAGE, KAHAN, JOBS, BANDED>(cfg.taps);
  }
}

// Single-job kernels (accumulation plain or Kahan) over row-major or banded half-planes.
template<int STORAGE, bool BANDED>
static InsertFn pick_storage(const InsertConfig &cfg)
{
  return cfg.kahan ? pick_mode<STORAGE, true, false, BANDED>(cfg) : pick_mode<STORAGE, false, false, BANDED>(cfg);
}

// Batched kernels (work items of several jobs in one launch); a batch always reads banded
// half-planes (fr_batch_execute copies every job's projections into bands).
template<int STORAGE>
static InsertFn pick_storage_jobs(const InsertConfig &cfg)
{
  return cfg.kahan ? pick_mode<STORAGE, true, true, true>(cfg) : pick_mode<STORAGE, false, true, true>(cfg);
}

}// namespace frb
