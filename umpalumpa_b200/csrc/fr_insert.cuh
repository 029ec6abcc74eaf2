// The insertion kernel of the B200 Fourier-reconstruction engine.
//
// Why it is not the reference's ProcessKernel: the reference launches a 2D grid over the
// volume face and lets every CTA walk every traverse space, doing three global float
// atomics per voxel per projection (fr_cuda_kernels.cu:362-365,468-523).  Here the volume is
// cut into 16^3-voxel bricks.  The binning passes (fr_kernels.cu) list, per brick, the
// traverse spaces whose blob slab can touch it, grouped by traversal direction; this
// persistent kernel takes (brick, list range) work items, accumulates all their
// projections into shared-memory accumulators and adds the brick into the caller's volume
// once per item.  The per-voxel arithmetic is the reference's ProcessVoxelBlob /
// ProcessVoxel (fr_cpu_kernels.hpp:18-152) and the voxel set of each projection is the
// reference's traversal (fr_cpu_kernels.hpp:154-240): for a space of direction XY the
// thread owning column (x, y) of the brick visits z in [floor(min(z1,z2)), ceil(max(z1,z2))]
// between the two padded planes, and likewise for XZ (column along y) and YZ (along x).
// Within one direction every thread owns its column, so consecutive projections need no
// synchronisation; the CTA synchronises only when the direction changes.
#pragma once

#include "fr_device.cuh"
#include "fr_kernels.h"

namespace frb {

enum { kModeLut = 0, kModeFastKaiser = 1, kModeKaiser = 2 };

// Traversal plane axes (U, V) and column axis W per direction (traverse_space.hpp:24-28).
template<int DIR> struct Axes;
template<> struct Axes<FR_DIR_XY> { static constexpr int U = 0, V = 1, W = 2; };
template<> struct Axes<FR_DIR_XZ> { static constexpr int U = 0, V = 2, W = 1; };
template<> struct Axes<FR_DIR_YZ> { static constexpr int U = 1, V = 2, W = 0; };

template<int K, typename T> __device__ __forceinline__ T pick3(T a, T b, T c)
{
  return K == 0 ? a : (K == 1 ? b : c);
}

struct SpaceView {
  int lo0, hi0, lo1, hi1;  // traversal AABB on the plane axes U, V
  float nu, nv, nw;        // plane normal on U, V, W
  float bu, bv, bw;        // bottom-plane origin
  float tu, tv, tw;        // top-plane origin
  float maxDist2;
  float T[9];              // transformInv, row-major
  float weight;
  int proj;
};

// One 112-byte TraverseSpace as seven 16-byte loads; every thread of the CTA reads the
// same record, so these are broadcasts served from L1.
template<int DIR>
__device__ __forceinline__ void load_space(const fr_traverse_space *sp, SpaceView &v)
{
  const float4 *q = reinterpret_cast<const float4 *>(sp);
  const float4 f0 = __ldg(q + 0), f1 = __ldg(q + 1), f2 = __ldg(q + 2), f3 = __ldg(q + 3);
  const float4 f4 = __ldg(q + 4), f5 = __ldg(q + 5), f6 = __ldg(q + 6);
  // f0 = minY minX minZ maxY | f1 = maxX maxZ maxDist dir | f2 = n0 n1 n2 top0
  // f3 = top1 top2 bot0 bot1 | f4 = bot2 proj T00 T01    | f5 = T02 T10 T11 T12
  // f6 = T20 T21 T22 weight
  const int mn[3] = { __float_as_int(f0.y), __float_as_int(f0.x), __float_as_int(f0.z) };
  const int mx[3] = { __float_as_int(f1.x), __float_as_int(f0.w), __float_as_int(f1.y) };
  using AX = Axes<DIR>;
  v.lo0 = mn[AX::U];
  v.hi0 = mx[AX::U];
  v.lo1 = mn[AX::V];
  v.hi1 = mx[AX::V];
  v.maxDist2 = f1.z;
  v.nu = pick3<AX::U>(f2.x, f2.y, f2.z);
  v.nv = pick3<AX::V>(f2.x, f2.y, f2.z);
  v.nw = pick3<AX::W>(f2.x, f2.y, f2.z);
  v.tu = pick3<AX::U>(f2.w, f3.x, f3.y);
  v.tv = pick3<AX::V>(f2.w, f3.x, f3.y);
  v.tw = pick3<AX::W>(f2.w, f3.x, f3.y);
  v.bu = pick3<AX::U>(f3.z, f3.w, f4.x);
  v.bv = pick3<AX::V>(f3.z, f3.w, f4.x);
  v.bw = pick3<AX::W>(f3.z, f3.w, f4.x);
  v.proj = __float_as_int(f4.y);
  v.T[0] = f4.z; v.T[1] = f4.w; v.T[2] = f5.x;
  v.T[3] = f5.y; v.T[4] = f5.z; v.T[5] = f5.w;
  v.T[6] = f6.x; v.T[7] = f6.y; v.T[8] = f6.z;
  v.weight = f6.w;
}

struct Accum {
  float *re, *im, *w;     // brick accumulators [z][y][x]
  float *cre, *cim, *cw;  // Kahan compensations (KAHAN only)
};

template<bool KAHAN>
__device__ __forceinline__ void acc_add(float *sum, float *comp, int i, float v)
{
  if (KAHAN) {
    const float y = __fsub_rn(v, comp[i]);
    const float t = __fadd_rn(sum[i], y);
    comp[i] = __fsub_rn(__fsub_rn(t, sum[i]), y);
    sum[i] = t;
  } else {
    sum[i] += v;
  }
}

// FR<>::ProcessVoxelBlob (fr_cpu_kernels.hpp:70-152) for voxel (X, Y, Z): Kaiser-Bessel
// gather of the projection pixels within the blob radius.  False if the voxel is rejected.
template<int MODE, int TAPS, int STORAGE>
__device__ __forceinline__ bool voxel_blob(const InsertParams &P, const SpaceView &s,
  const typename Pixel<STORAGE>::T *__restrict__ img, float scale, const float *lut, int X, int Y,
  int Z, float &ore, float &oim, float &ow)
{
  const fr_constants &c = P.c;
  const float px = float(X - P.cx), py = float(Y - P.cy), pz = float(Z - P.cz);
  if (px * px + py * py + pz * pz > s.maxDist2) return false;  // integer-valued: exact
  const float qx = add_(add_(mul_(s.T[0], px), mul_(s.T[1], py)), mul_(s.T[2], pz));
  const float qy0 = add_(add_(mul_(s.T[3], px), mul_(s.T[4], py)), mul_(s.T[5], pz));
  const float qz = add_(add_(mul_(s.T[6], px), mul_(s.T[7], py)), mul_(s.T[8], pz));
  const float r = c.cBlobRadius;
  if (qx < -r) return false;
  const float qy = add_(qy0, float(P.cy));
  // no pixel lies within the blob radius (also rejects non-finite coordinates)
  if (!(qx <= float(P.fftX) + r && qy >= -r && qy <= float(P.fftY) + r)) return false;
  const float rSq = mul_(r, r);
  const float zSq = mul_(qz, qz);
  if (zSq > rSq) return false;
  const int minX = max(int(ceilf(sub_(qx, r))), 0);
  const int maxX = min(int(floorf(add_(qx, r))), P.fftX - 1);
  const int minY = max(int(ceilf(sub_(qy, r))), 0);
  const int maxY = min(int(floorf(add_(qy, r))), P.fftY - 1);
  float re = 0.f, im = 0.f, w = 0.f;
  const float dataWeight = mul_(s.weight, scale);
  const float wOnly = s.weight;
#pragma unroll
  for (int ii = 0; ii < TAPS; ++ii) {
    const int i = minY + ii;
    const float dy = sub_(qy, float(i));
    const float yz = add_(mul_(dy, dy), zSq);
    const bool rowOk = i <= maxY && yz <= rSq;
    const typename Pixel<STORAGE>::T *row = img + size_t(i) * P.fftX;
#pragma unroll
    for (int jj = 0; jj < TAPS; ++jj) {
      const int j = minX + jj;
      const float dx = qx - float(j);
      const float d2 = fmaf(dx, dx, yz);
      if (rowOk && j <= maxX && d2 <= rSq) {
        float wb;
        if (MODE == kModeLut) {
          wb = lut[min(int(fmaf(d2, c.cIDeltaSqrt, 0.5f)), P.tableElems - 1)];
        } else if (MODE == kModeFastKaiser) {
          wb = kaiser_value_fast(d2, c);
        } else {
          wb = kaiser_value_f(sqrtf(d2), r, c.cBlobAlpha, c.cOneOverBessiOrderAlpha, P.order) * c.cIw0;
        }
        const float2 v = Pixel<STORAGE>::load(row + j);
        w = fmaf(wb, wOnly, w);
        const float wt = wb * dataWeight;
        re = fmaf(v.x, wt, re);
        im = fmaf(v.y, wt, im);
      }
    }
  }
  ore = re;
  oim = im;
  ow = w;
  return true;
}

// FR<>::ProcessVoxel (fr_cpu_kernels.hpp:18-68): nearest pixel.
template<int STORAGE>
__device__ __forceinline__ bool voxel_nearest(const InsertParams &P, const SpaceView &s,
  const typename Pixel<STORAGE>::T *__restrict__ img, float scale, int X, int Y, int Z,
  float &ore, float &oim, float &ow)
{
  const float px = float(X - P.cx), py = float(Y - P.cy), pz = float(Z - P.cz);
  if (px * px + py * py + pz * pz > s.maxDist2) return false;
  const float qx = add_(add_(mul_(s.T[0], px), mul_(s.T[1], py)), mul_(s.T[2], pz));
  const float qy = add_(add_(mul_(s.T[3], px), mul_(s.T[4], py)), mul_(s.T[5], pz));
  if (qx < 0.f) return false;
  const int imgX = min(max(int(add_(qx, 0.5f)), 0), P.fftX - 1);
  const int imgY = min(max(int(add_(add_(qy, 0.5f), float(P.cy))), 0), P.fftY - 1);
  const float2 v = Pixel<STORAGE>::load(img + size_t(imgY) * P.fftX + imgX);
  const float w = s.weight;
  const float wt = mul_(w, scale);
  ore = mul_(v.x, wt);
  oim = mul_(v.y, wt);
  ow = w;
  return true;
}

// All list entries [e0, e1) of one direction for the brick at (ox, oy, oz).
template<int DIR, int MODE, int TAPS, bool FAST, int STORAGE, bool KAHAN>
__device__ __forceinline__ void run_direction(const InsertParams &P, const Accum &A,
  const float *lut, int ox, int oy, int oz, int tx, int ty, int e0, int e1)
{
  using AX = Axes<DIR>;
  using PT = typename Pixel<STORAGE>::T;
  const PT *fft = reinterpret_cast<const PT *>(P.fft);
  const size_t plane = size_t(P.fftX) * size_t(P.fftY);
  const int oU = pick3<AX::U>(ox, oy, oz), oV = pick3<AX::V>(ox, oy, oz), oW = pick3<AX::W>(ox, oy, oz);
  const int nU = pick3<AX::U>(P.vx, P.vy, P.vz), nV = pick3<AX::V>(P.vx, P.vy, P.vz);
  const int nW = pick3<AX::W>(P.vx, P.vy, P.vz);
  const int U = oU + tx, V = oV + ty;
  const bool colIn = U < nU && V < nV;
  const int wLo = oW, wHi = min(oW + kBrick, nW) - 1;
  const float wMax = float(AX::W == 0 ? P.c.cMaxVolumeIndexX : P.c.cMaxVolumeIndexYZ);
  const float uf = float(U), vf = float(V);
  for (int e = e0; e < e1; ++e) {
    const int si = __ldg(P.list + e);
    SpaceView s;
    load_space<DIR>(P.spaces + si, s);
    if (!colIn || U < s.lo0 || U > s.hi0 || V < s.lo1 || V > s.hi1) continue;
    if (unsigned(s.proj) >= unsigned(P.nProj)) continue;  // never binned; kept as a guard
    int lo, hi;
    if (FAST) {
      lo = hi = int(add_(plane_hit(uf, vf, s.nu, s.nv, s.nw, s.bu, s.bv, s.bw), 0.5f));
    } else {
      const float h1 = clampf_(plane_hit(uf, vf, s.nu, s.nv, s.nw, s.bu, s.bv, s.bw), 0.f, wMax);
      const float h2 = clampf_(plane_hit(uf, vf, s.nu, s.nv, s.nw, s.tu, s.tv, s.tw), 0.f, wMax);
      lo = int(floorf(fminf(h1, h2)));
      hi = int(ceilf(fmaxf(h1, h2)));
    }
    lo = max(lo, wLo);
    hi = min(hi, wHi);
    if (lo > hi) continue;
    const float scale = STORAGE == FR_STORAGE_FP32 ? 1.f : __ldg(P.scales + s.proj);
    const PT *img = fft + size_t(s.proj) * plane;
    for (int wv = lo; wv <= hi; ++wv) {
      const int X = AX::W == 0 ? wv : (AX::U == 0 ? U : V);
      const int Y = AX::W == 1 ? wv : (AX::U == 1 ? U : V);
      const int Z = AX::W == 2 ? wv : V;
      float re, im, w;
      bool ok;
      if (FAST)
        ok = voxel_nearest<STORAGE>(P, s, img, scale, X, Y, Z, re, im, w);
      else
        ok = voxel_blob<MODE, TAPS, STORAGE>(P, s, img, scale, lut, X, Y, Z, re, im, w);
      if (ok) {
        const int li = ((Z - oz) * kBrick + (Y - oy)) * kBrick + (X - ox);
        acc_add<KAHAN>(A.re, A.cre, li, re);
        acc_add<KAHAN>(A.im, A.cim, li, im);
        acc_add<KAHAN>(A.w, A.cw, li, w);
      }
    }
  }
}

template<int MODE, int TAPS, bool FAST, int STORAGE, bool KAHAN>
__global__ void __launch_bounds__(kThreads, 2) insert_kernel(InsertParams P)
{
  extern __shared__ float4 smem4[];
  float *smem = reinterpret_cast<float *>(smem4);
  Accum A;
  A.re = smem;
  A.im = smem + kBrickVox;
  A.w = smem + 2 * kBrickVox;
  A.cre = smem + 3 * kBrickVox;
  A.cim = smem + 4 * kBrickVox;
  A.cw = smem + 5 * kBrickVox;
  constexpr int kAccFloats = (KAHAN ? 6 : 3) * kBrickVox;
  float *lutS = smem + kAccFloats;
  __shared__ int sItem;

  const int tid = threadIdx.x;
  const float *lut = P.table;
  if (MODE == kModeLut && !FAST && P.lutInSmem) {
    for (int i = tid; i < P.tableElems; i += kThreads) lutS[i] = __ldg(P.table + i);
    lut = lutS;
  }
  const int nItems = *P.nItems;
  const int tx = tid & (kBrick - 1), ty = tid / kBrick;

  for (;;) {
    __syncthreads();
    if (tid == 0) sItem = atomicAdd(P.workCounter, 1);
    __syncthreads();
    const int itIdx = sItem;
    if (itIdx >= nItems) break;
    const WorkItem it = P.items[itIdx];
    for (int i = tid; i < kAccFloats; i += kThreads) smem[i] = 0.f;
    __syncthreads();
    const int bx = it.brick % P.nbx, by = (it.brick / P.nbx) % P.nby, bz = it.brick / (P.nbx * P.nby);
    const int ox = bx * kBrick, oy = by * kBrick, oz = bz * kBrick;
    const int base = 3 * it.brick;
    for (int dir = 0; dir < 3; ++dir) {
      const int e0 = max(it.begin, P.offsets[base + dir]);
      const int e1 = min(it.end, P.offsets[base + dir + 1]);
      if (e0 >= e1) continue;  // uniform across the CTA
      if (dir == FR_DIR_XY)
        run_direction<FR_DIR_XY, MODE, TAPS, FAST, STORAGE, KAHAN>(P, A, lut, ox, oy, oz, tx, ty, e0, e1);
      else if (dir == FR_DIR_XZ)
        run_direction<FR_DIR_XZ, MODE, TAPS, FAST, STORAGE, KAHAN>(P, A, lut, ox, oy, oz, tx, ty, e0, e1);
      else
        run_direction<FR_DIR_YZ, MODE, TAPS, FAST, STORAGE, KAHAN>(P, A, lut, ox, oy, oz, tx, ty, e0, e1);
      __syncthreads();  // the next direction maps threads to other voxels
    }
    // add the brick into the caller's volume
    for (int li = tid; li < kBrickVox; li += kThreads) {
      const int X = ox + (li & (kBrick - 1)), Y = oy + ((li / kBrick) & (kBrick - 1)),
                Z = oz + li / (kBrick * kBrick);
      if (X >= P.vx || Y >= P.vy || Z >= P.vz) continue;
      float re = A.re[li], im = A.im[li], w = A.w[li];
      if (KAHAN) {
        re = __fsub_rn(re, A.cre[li]);
        im = __fsub_rn(im, A.cim[li]);
        w = __fsub_rn(w, A.cw[li]);
      }
      if (__float_as_uint(re) == 0u && __float_as_uint(im) == 0u && __float_as_uint(w) == 0u) continue;
      const size_t g = (size_t(Z) * P.vy + Y) * P.vx + X;
      atomicAdd(reinterpret_cast<float2 *>(P.volume) + g, make_float2(re, im));
      atomicAdd(P.weight + g, w);
    }
  }
}

template<int MODE, bool FAST, int STORAGE, bool KAHAN>
static InsertFn pick_taps(int taps)
{
  if (taps <= 4) return insert_kernel<MODE, 4, FAST, STORAGE, KAHAN>;
  return insert_kernel<MODE, 8, FAST, STORAGE, KAHAN>;
}

template<int STORAGE, bool KAHAN>
static InsertFn pick_mode(const InsertConfig &cfg)
{
  if (cfg.fast) return insert_kernel<kModeLut, 4, true, STORAGE, KAHAN>;
  switch (cfg.mode) {
  case kModeLut: return pick_taps<kModeLut, false, STORAGE, KAHAN>(cfg.taps);
  case kModeFastKaiser: return pick_taps<kModeFastKaiser, false, STORAGE, KAHAN>(cfg.taps);
  default: return pick_taps<kModeKaiser, false, STORAGE, KAHAN>(cfg.taps);
  }
}

template<int STORAGE>
static InsertFn pick_storage(const InsertConfig &cfg)
{
  return cfg.kahan ? pick_mode<STORAGE, true>(cfg) : pick_mode<STORAGE, false>(cfg);
}

}// namespace frb
