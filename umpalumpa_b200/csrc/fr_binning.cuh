// Binning building blocks shared by the single-job and the batched passes.
#pragma once

#include "fr_device.cuh"
#include "fr_kernels.h"

namespace frb {

// Builds, for one space, the binning record (SpacePrep) and the insertion record (SpaceRec)
// relative to the volume centre (cx, cy, cz).  A space whose projectionIndex is outside the
// FFT payload is given direction -1, so it is never binned (never read); returns false then.
__device__ __forceinline__ bool prep_space(const fr_traverse_space &s, float halfWidth, float xMin,
  float radius, int cx, int cy, int cz, int nProj, SpacePrep &p, SpaceRec &r)
{
  for (int k = 0; k < 3; ++k) {
    p.t0[k] = s.transformInv[0][k];
    p.t2[k] = s.transformInv[2][k];
  }
  p.maxDist2 = s.maxDistanceSqr * 1.00001f + 1e-2f;
  p.halfWidth = halfWidth;
  p.xMin = xMin;
  const int open = 1 << 30;
  int lo[3] = { s.minX, s.minY, s.minZ }, hi[3] = { s.maxX, s.maxY, s.maxZ };
  const int dir = s.dir;
  const int ua = dir == FR_DIR_YZ ? 1 : 0;
  const int va = dir == FR_DIR_XY ? 1 : 2;
  const int wa = dir == FR_DIR_XY ? 2 : (dir == FR_DIR_XZ ? 1 : 0);
  r.lo0 = lo[ua];
  r.hi0 = hi[ua];
  r.lo1 = lo[va];
  r.hi1 = hi[va];
  lo[wa] = -open;
  hi[wa] = open;
  for (int k = 0; k < 3; ++k) {
    p.lo[k] = lo[k];
    p.hi[k] = hi[k];
  }
  p.dir = dir;
  const bool bad = s.projectionIndex < 0 || s.projectionIndex >= nProj;
  if (bad) p.dir = -1;  // matches no direction segment

  for (int k = 0; k < 9; ++k) r.T[k] = s.transformInv[k / 3][k % 3];
  r.maxDist2 = s.maxDistanceSqr;
  r.weight = s.weight;
  r.proj = s.projectionIndex;
  const double c[3] = { double(cx), double(cy), double(cz) };
  const double nrm[3] = { s.transformInv[2][0], s.transformInv[2][1], s.transformInv[2][2] };
  const double nw = nrm[wa];
  if (fabs(nw) > 1e-6) {
    r.w0 = float(c[wa] + (nrm[ua] * c[ua] + nrm[va] * c[va]) / nw);
    r.wu = float(-nrm[ua] / nw);
    r.wv = float(-nrm[va] / nw);
    r.hw = float(double(radius) / fabs(nw) + 2e-3);
  } else {  // degenerate normal: visit the whole column, the voxel checks decide
    r.w0 = 0.f;
    r.wu = 0.f;
    r.wv = 0.f;
    r.hw = 1e9f;
  }
  const double t0[3] = { s.transformInv[0][0], s.transformInv[0][1], s.transformInv[0][2] };
  r.xu = float(t0[ua]);
  r.xv = float(t0[va]);
  r.xw = float(t0[wa]);
  r.xwInv = fabs(t0[wa]) > 1e-3 ? float(1.0 / t0[wa]) : 0.f;
  const float *un = s.unitNormal, *bo = s.bottomOrigin;
  r.nu = un[ua];
  r.nv = un[va];
  r.nw = un[wa];
  r.bu = bo[ua];
  r.bv = bo[va];
  r.bw = bo[wa];
  r.dir = bad ? -1 : dir;
  r.pad = 0;
  return !bad;
}

// Conservative test: can any voxel of the brick [b0, b1] (inclusive voxel coordinates)
// receive a contribution from this space?  Centre (cx, cy, cz) is the reference's integer
// volume centre.
__device__ __forceinline__ bool brick_hit(const SpacePrep &p, const int b0[3], const int b1[3],
  const float a[3], const float e[3])
{
  for (int k = 0; k < 3; ++k)
    if (b1[k] < p.lo[k] || b0[k] > p.hi[k]) return false;
  float zlo = 0.f, zhi = 0.f, xhi = 0.f, d2 = 0.f;
  for (int k = 0; k < 3; ++k) {
    float u = p.t2[k] * a[k], v = p.t2[k] * e[k];
    zlo += fminf(u, v);
    zhi += fmaxf(u, v);
    xhi += fmaxf(p.t0[k] * a[k], p.t0[k] * e[k]);
    float c = fminf(fmaxf(0.f, a[k]), e[k]);
    d2 += c * c;
  }
  return zlo <= p.halfWidth && zhi >= -p.halfWidth && xhi >= p.xMin && d2 <= p.maxDist2;
}

__device__ __forceinline__ void brick_box(const BinGeom &g, int b, int b0[3], int b1[3], float a[3],
  float e[3])
{
  int bx = b % g.nbx, by = (b / g.nbx) % g.nby, bz = b / (g.nbx * g.nby);
  int v[3] = { g.vx, g.vy, g.vz };
  int c[3] = { g.cx, g.cy, g.cz };
  int o[3] = { bx * kBrick, by * kBrick, bz * kBrick };
  for (int k = 0; k < 3; ++k) {
    b0[k] = o[k];
    b1[k] = min(o[k] + kBrick, v[k]) - 1;
    a[k] = float(b0[k] - c[k]);
    e[k] = float(b1[k] - c[k]);
  }
}

// Union box of the bricks a binning CTA owns (bricks first .. first + count - 1): every space
// that can touch one of them touches the union, so brick_hit on the union is a conservative
// pre-test (the AABB overlap, the slab range, the half-space maximum and the distance of the
// nearest point all widen with the box).
__device__ __forceinline__ void union_box(const BinGeom &g, int first, int count, int u0[3], int u1[3], float ua[3],
  float ue[3])
{
  for (int k = 0; k < 3; ++k) {
    u0[k] = 1 << 30;
    u1[k] = -(1 << 30);
  }
  for (int w = 0; w < count; ++w) {
    int b0[3], b1[3];
    float a[3], e[3];
    brick_box(g, first + w, b0, b1, a, e);
    for (int k = 0; k < 3; ++k) {
      u0[k] = min(u0[k], b0[k]);
      u1[k] = max(u1[k], b1[k]);
    }
  }
  const int c[3] = { g.cx, g.cy, g.cz };
  for (int k = 0; k < 3; ++k) {
    ua[k] = float(u0[k] - c[k]);
    ue[k] = float(u1[k] - c[k]);
  }
}

// Compacts, in ascending order, the tile entries [0, m) that hit the union box into idx[0, *n)
// (every thread of the 256-thread CTA calls it; ends with a barrier).
__device__ __forceinline__ void compact_tile_hits(const SpacePrep *tile, int m, const int u0[3], const int u1[3],
  const float ua[3], const float ue[3], int *idx, int *n, int *warpBase)
{
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const bool h = t < m && brick_hit(tile[t], u0, u1, ua, ue);
  const unsigned mask = __ballot_sync(0xffffffffu, h);
  if (lane == 0) warpBase[warp] = __popc(mask);
  __syncthreads();
  if (t == 0) {
    int run = 0;
    for (int w = 0; w < 8; ++w) {
      const int c = warpBase[w];
      warpBase[w] = run;
      run += c;
    }
    *n = run;
  }
  __syncthreads();
  if (h) idx[warpBase[warp] + __popc(mask & ((1u << lane) - 1u))] = t;
  __syncthreads();
}

}// namespace frb
