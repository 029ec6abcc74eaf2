// Kernels of the B200 Fourier-reconstruction engine.
//
// Design (why it is not the reference's ProcessKernel): the reference launches a 2D grid over
// the volume face and lets every CTA walk every traverse space, doing three global float
// atomics per voxel per projection (fr_cuda_kernels.cu:362-365,468-523).  Here the volume is
// cut into 16^3-voxel bricks.  A binning pass lists, per brick, the traverse spaces whose
// blob slab can touch it; a persistent kernel then takes (brick, list range) work items,
// accumulates all their projections into shared-memory accumulators, and adds each brick
// into the caller's volume once per item.  The per-voxel arithmetic is the reference's
// ProcessVoxelBlob / ProcessVoxel (fr_cpu_kernels.hpp:18-152), and the voxel set of every
// projection is the reference's traversal (fr_cpu_kernels.hpp:154-240).
#include "fr_binning.cuh"
#include "fr_device.cuh"
#include "fr_kernels.h"

#include <float.h>

#include <algorithm>

#include <type_traits>

namespace frb {

// =====================================================================================
// Setup kernels (FP64)
// =====================================================================================

// AFR::FillBlobTable (afr.cpp:22-34) with KaiserValue (math/kaiser.hpp:19-56): entry i is
// the blob at distance r*sqrt(i/(N-1)), evaluated with the reference's float arguments and
// double-precision Bessel ratio, scaled by cIw0.
__global__ void blob_table_kernel(float *table, int64_t n, int order, float alpha, float radius,
  float iw0)
{
  int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float freq = __fmul_rn(radius, __fsqrt_rn(__fdiv_rn(1.f, float(n - 1))));
  float f = __fmul_rn(freq, float(sqrt(double(i))));
  float w = 0.f;
  float rda = __fdiv_rn(f, radius);
  if (rda <= 1.f) {
    float rdas = __fmul_rn(rda, rda);
    float s = __fsqrt_rn(__fsub_rn(1.f, rdas));
    float arg = __fmul_rn(alpha, s);
    if (order == 0) {
      w = float(bessel_i0_d(arg) / bessel_i0_d(alpha));
    } else {
      w = s;
      if (order == 2) w = __fmul_rn(w, w);
      if (order == 3) w = __fmul_rn(__fmul_rn(w, w), w);
      if (order == 4) w = __fmul_rn(__fmul_rn(__fmul_rn(w, w), w), w);
      if (alpha != 0.f) w = __fmul_rn(w, float(bessel_in_d(order, arg) / bessel_in_d(order, alpha)));
    }
  }
  table[i] = __fmul_rn(w, iw0);
}

// Dynamic interpolation's Kaiser weight (KaiserValue, math/kaiser.hpp:19-56, times cIw0 as
// FR<>::ProcessVoxelBlob applies it, fr_cpu_kernels.hpp:137-141) as a function of the squared
// distance: entry i holds the value at d2_i = i r^2 / (N-1) and the step to the next node,
// both evaluated in FP64 and rounded once.  The weight is analytic in d2 for every order
// (s^m I_m(alpha s) is a power series in s^2 = 1 - d2/r^2), so linear interpolation in d2
// converges quadratically; the last node (d2 = r^2) has slope 0.
__device__ double kaiser_of_d2(double d2, double r2, int order, double alpha, double iw0)
{
  const double u = fmax(0.0, 1.0 - d2 / r2);
  const double s = sqrt(u);
  double w;
  if (order == 0) {
    w = bessel_i0_d(alpha * s) / bessel_i0_d(alpha);
  } else {
    w = s;
    for (int k = 1; k < order; ++k) w *= s;
    if (alpha != 0.0) w *= bessel_in_d(order, alpha * s) / bessel_in_d(order, alpha);
  }
  return w * iw0;
}

__global__ void kaiser_table_kernel(float2 *table, int n, int order, float alpha, float radius, float iw0)
{
  const int i = int(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double r2 = double(radius) * double(radius);
  const double h = r2 / double(n - 1);
  const double v = kaiser_of_d2(double(i) * h, r2, order, double(alpha), double(iw0));
  const double next = i + 1 < n ? kaiser_of_d2(double(i + 1) * h, r2, order, double(alpha), double(iw0)) : v;
  table[i] = make_float2(float(v), float(next - v));
}

// ComputeTraverseSpace (traverse_space_generator.hpp:94-145) in the reference's own single-
// precision evaluation, operation by operation (products and sums rounded separately, no
// fused multiply-add -- the reference's ISO-mode host build), so that every field a caller or
// the insertion reads comes out bit for bit as the reference's host code makes it: the
// cuboid [-b, X+b] x [-(Y/2+b), Y/2+b] x [+b, -b] (corner order of :30-40) is rotated
// (multiply, :10-17: ((t0 x + t1 y) + t2 z) per row), moved to the volume centre and bounded
// by an AABB clamped to the volume (the maxima start at FLT_MIN, :66); corner 4 is the "top"
// and corner 0 the "bottom" origin; the normal is the transform applied to z, and its dominant
// component picks the traversal plane, ties YZ > XZ > XY.  The nearest-pixel insertion rounds
// its plane hit from bottomOrigin, so those bits decide which voxel a pixel lands in.
__device__ __forceinline__ void rotate_ref(const float t[3][3], float v[3])
{
  float o[3];
  for (int r = 0; r < 3; ++r)
    o[r] = __fadd_rn(__fadd_rn(__fmul_rn(t[r][0], v[0]), __fmul_rn(t[r][1], v[1])), __fmul_rn(t[r][2], v[2]));
  for (int r = 0; r < 3; ++r) v[r] = o[r];
}

__device__ void traverse_space_of(const float *rot, uint32_t imgX, uint32_t imgY, uint32_t maxVX,
  uint32_t maxVYZ, int useFast, float blobRadius, float weight, int32_t projectionIndex,
  fr_traverse_space *__restrict__ dst)
{
  float t[3][3];
  for (int k = 0; k < 9; ++k) t[k / 3][k % 3] = rot[k];
  const float b = useFast ? 0.f : blobRadius;
  const float sizeX = float(imgX), halfY = __fdiv_rn(float(imgY), 2.0f);
  const float origin[3] = { __fdiv_rn(float(maxVX), 2.f), __fdiv_rn(float(maxVYZ), 2.f), __fdiv_rn(float(maxVYZ), 2.f) };
  const int xHi[8] = { 1, 1, 0, 0, 1, 1, 0, 0 };
  const int yHi[8] = { 0, 1, 1, 0, 0, 1, 1, 0 };
  const int zHi[8] = { 1, 1, 1, 1, 0, 0, 0, 0 };
  float lo[3] = { FLT_MAX, FLT_MAX, FLT_MAX };
  float hi[3] = { FLT_MIN, FLT_MIN, FLT_MIN };
  float c0[3] = {}, c4[3] = {};
  for (int i = 0; i < 8; ++i) {
    float v[3] = { xHi[i] ? __fadd_rn(sizeX, b) : __fsub_rn(0.f, b),
                   yHi[i] ? __fadd_rn(halfY, b) : -__fadd_rn(halfY, b), zHi[i] ? __fadd_rn(0.f, b) : __fsub_rn(0.f, b) };
    rotate_ref(t, v);
    for (int r = 0; r < 3; ++r) {
      v[r] = __fadd_rn(v[r], origin[r]);
      if (lo[r] > v[r]) lo[r] = v[r];
      if (hi[r] < v[r]) hi[r] = v[r];
    }
    if (i == 0)
      for (int r = 0; r < 3; ++r) c0[r] = v[r];
    if (i == 4)
      for (int r = 0; r < 3; ++r) c4[r] = v[r];
  }
  const float lim[3] = { float(maxVX), float(maxVYZ), float(maxVYZ) };
  for (int r = 0; r < 3; ++r) {
    if (lo[r] < 0.f) lo[r] = 0.f;
    if (hi[r] > lim[r]) hi[r] = lim[r];
  }
  fr_traverse_space s;
  s.minX = int32_t(floorf(lo[0]));
  s.minY = int32_t(floorf(lo[1]));
  s.minZ = int32_t(floorf(lo[2]));
  s.maxX = int32_t(ceilf(hi[0]));
  s.maxY = int32_t(ceilf(hi[1]));
  s.maxZ = int32_t(ceilf(hi[2]));
  const float rr = __fadd_rn(sizeX, b);
  s.maxDistanceSqr = __fmul_rn(rr, rr);
  float n[3] = { 0.f, 0.f, 1.f };
  rotate_ref(t, n);
  for (int r = 0; r < 3; ++r) {
    s.topOrigin[r] = c4[r];
    s.bottomOrigin[r] = c0[r];
    s.unitNormal[r] = n[r];
    for (int c = 0; c < 3; ++c) s.transformInv[r][c] = t[c][r];
  }
  const float nX = fabsf(n[0]), nY = fabsf(n[1]), nZ = fabsf(n[2]);
  s.dir = (nX >= nY && nX >= nZ) ? FR_DIR_YZ : (nY >= nX && nY >= nZ) ? FR_DIR_XZ : FR_DIR_XY;
  s.projectionIndex = projectionIndex;
  s.weight = weight;
  *dst = s;
}

__global__ void traverse_space_kernel(const float *__restrict__ rot, int64_t n, uint32_t imgX,
  uint32_t imgY, uint32_t maxVX, uint32_t maxVYZ, int useFast, float blobRadius, float weight,
  int32_t firstIndex, fr_traverse_space *__restrict__ out)
{
  const int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p >= n) return;
  traverse_space_of(rot + p * 9, imgX, imgY, maxVX, maxVYZ, useFast, blobRadius, weight,
    firstIndex + int32_t(p), out + p);
}

// Symmetry expansion (examples/fourier_reconstruction/fr.cpp:293-309): space i * nSym + k
// inserts projection firstIndex + i under the transform R_i * S_k, the product formed in
// single precision in the reference's order (Multiply, fr.hpp:123-130: each entry summed
// over k from 0, products and sums rounded separately).
__global__ void traverse_space_sym_kernel(const float *__restrict__ rot, int64_t n,
  const float *__restrict__ sym, int nSym, uint32_t imgX, uint32_t imgY, uint32_t maxVX, uint32_t maxVYZ,
  int useFast, float blobRadius, float weight, int32_t firstIndex, fr_traverse_space *__restrict__ out)
{
  const int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (q >= n * nSym) return;
  const int64_t p = q / nSym;
  const int k = int(q - p * nSym);
  const float *l = rot + p * 9, *r = sym + int64_t(k) * 9;
  float t[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      float acc = 0.f;
      for (int m = 0; m < 3; ++m) acc = __fadd_rn(acc, __fmul_rn(l[i * 3 + m], r[m * 3 + j]));
      t[i * 3 + j] = acc;
    }
  traverse_space_of(t, imgX, imgY, maxVX, maxVYZ, useFast, blobRadius, weight, firstIndex + int32_t(p), out + q);
}

// Projection storage in 16 bits: one CTA per projection finds the largest |re|, |im| and
// stores value / scale with scale = max / 2^14 (round to nearest), so the largest component
// sits at 2^14 -- inside FP16's range with headroom, and irrelevant to BF16's range.  A zero
// projection gets scale 1.
template<typename T>
__global__ void __launch_bounds__(256) quantize_kernel(const float2 *__restrict__ in, int64_t elems,
  T *__restrict__ out, float *__restrict__ scales)
{
  const int64_t p = blockIdx.x;
  const float2 *src = in + p * elems;
  float m = 0.f;
  for (int64_t i = threadIdx.x; i < elems; i += blockDim.x) {
    const float2 v = src[i];
    m = fmaxf(m, fmaxf(fabsf(v.x), fabsf(v.y)));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ float wm[8];
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < 8 ? wm[threadIdx.x] : 0.f;
    for (int o = 4; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) wm[0] = m;
  }
  __syncthreads();
  const float scale = wm[0] > 0.f ? wm[0] / 16384.f : 1.f;
  const float inv = 1.f / scale;
  if (threadIdx.x == 0) scales[p] = scale;
  T *dst = out + p * elems;
  for (int64_t i = threadIdx.x; i < elems; i += blockDim.x) {
    const float2 v = src[i];
    if constexpr (sizeof(T) == 4 && std::is_same<T, __nv_bfloat162>::value)
      dst[i] = __floats2bfloat162_rn(v.x * inv, v.y * inv);
    else
      dst[i] = __floats2half2_rn(v.x * inv, v.y * inv);
  }
}

// =====================================================================================
// Binning
// =====================================================================================

// Per-space record for the brick tests (see SpacePrep).
// Per space of a single-job chunk: the binning and insertion records (prep_space); a space
// whose projectionIndex is outside the FFT payload is not binned and flags FR_E_INVALID for
// fr_synchronize.
__global__ void space_prep_kernel(const fr_traverse_space *__restrict__ spaces, int n,
  float halfWidth, float xMin, float radius, int cx, int cy, int cz, int nProj,
  SpacePrep *__restrict__ out, SpaceRec *__restrict__ rec, int *__restrict__ status)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  SpacePrep p;
  SpaceRec r;
  if (!prep_space(spaces[i], halfWidth, xMin, radius, cx, cy, cz, nProj, p, r)) atomicCAS(status, 0, FR_E_INVALID);
  out[i] = p;
  rec[i] = r;
}

// One warp per brick, 8 bricks per CTA; the CTA stages 256 space records at a time in
// shared memory, keeps those that hit the union box of its bricks (in ascending order) and
// only those are tested per brick.  FILL = false counts hits per (brick, direction); FILL =
// true writes the hit space indices in ascending order into the brick's three direction
// segments.
// The band copy, the binning and the insertion all ask for the largest shared-memory carve-out,
// so that an SM running copy CTAs (which need no shared memory) can take binning CTAs beside
// them instead of waiting for the copy to end.
template<typename K> static void prefer_max_shared(K *kernel)
{
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared)
      != cudaSuccess)
    cudaGetLastError();  // a hint only
}

// One binning record through four 16-byte read-only loads.  The binning kernels fetch the next
// 256 records into registers while they test the staged ones, so the load latency hides behind
// the tests (without it the stages waited on their loads, and a copy kernel running beside the
// binning, as the band copy does, doubled the binning time).
__device__ __forceinline__ SpacePrep load_prep(const SpacePrep *p)
{
  const float4 *q = reinterpret_cast<const float4 *>(p);
  SpacePrep r;
  float4 *d = reinterpret_cast<float4 *>(&r);
  d[0] = __ldg(q);
  d[1] = __ldg(q + 1);
  d[2] = __ldg(q + 2);
  d[3] = __ldg(q + 3);
  return r;
}

template<bool FILL>
__global__ void __launch_bounds__(256) bin_kernel(BinGeom g, const SpacePrep *__restrict__ prep,
  int n, int *__restrict__ counts, const int *__restrict__ offsets, int *__restrict__ list,
  const int *__restrict__ status)
{
  __shared__ SpacePrep tile[256];
  __shared__ int hitIdx[256];
  __shared__ int hitN, warpBase[8];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int b = blockIdx.x * 8 + warp;
  const bool active = b < g.n_bricks;
  if (FILL && *status != 0) return;
  int b0[3] = {}, b1[3] = {};
  float a[3] = {}, e[3] = {};
  if (active) brick_box(g, b, b0, b1, a, e);
  int u0[3], u1[3];
  float ua[3], ue[3];
  union_box(g, blockIdx.x * 8, min(8, g.n_bricks - int(blockIdx.x) * 8), u0, u1, ua, ue);
  int cnt[3] = { 0, 0, 0 };
  if (FILL && active)
    for (int d = 0; d < 3; ++d) cnt[d] = offsets[3 * b + d];
  SpacePrep next;
  if (int(threadIdx.x) < n) next = load_prep(prep + threadIdx.x);
  for (int base = 0; base < n; base += 256) {
    __syncthreads();
    if (base + int(threadIdx.x) < n) tile[threadIdx.x] = next;
    __syncthreads();
    if (base + 256 + int(threadIdx.x) < n) next = load_prep(prep + base + 256 + threadIdx.x);
    const int m = min(256, n - base);
    compact_tile_hits(tile, m, u0, u1, ua, ue, hitIdx, &hitN, warpBase);
    if (!active) continue;
    const int hn = hitN;
    for (int r = 0; r < hn; r += 32) {
      const int jj = r + lane;
      bool hit = false;
      int dir = 0, j = 0;
      if (jj < hn) {
        j = hitIdx[jj];
        hit = brick_hit(tile[j], b0, b1, a, e);
        dir = tile[j].dir;
      }
      for (int d = 0; d < 3; ++d) {
        unsigned mask = __ballot_sync(0xffffffffu, hit && dir == d);
        if (FILL && hit && dir == d) list[cnt[d] + __popc(mask & ((1u << lane) - 1u))] = base + j;
        cnt[d] += __popc(mask);
      }
    }
  }
  if (!FILL && active && lane == 0)
    for (int d = 0; d < 3; ++d) counts[3 * b + d] = cnt[d];
}

// ---- batched binning: the spaces and bricks of several jobs, indexed batch-wide ----------

// The job whose range [base(j), base(j+1)) holds the batch-wide index i (uniform lookups).
template<typename F>
__device__ __forceinline__ int job_of(const JobDesc *jobs, int nJobs, int i, F base)
{
  int lo = 0, hi = nJobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (base(jobs[mid]) <= i) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__global__ void batch_prep_kernel(const JobDesc *__restrict__ jobs, int nJobs, int total, float halfWidth,
  float xMin, float radius, SpacePrep *__restrict__ out, SpaceRec *__restrict__ rec, int *__restrict__ status)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int j = job_of(jobs, nJobs, i, [](const JobDesc &J) { return J.spaceBase; });
  const JobDesc &J = jobs[j];
  SpacePrep p;
  SpaceRec r;
  if (!prep_space(J.spaces[i - J.spaceBase], halfWidth, xMin, radius, J.cx, J.cy, J.cz, J.nProj, p, r))
    atomicCAS(status, 0, FR_E_INVALID);
  out[i] = p;
  rec[i] = r;
}

// As bin_kernel, for a batch: CTA c bins 8 bricks of the job whose binning groups hold c,
// against that job's spaces only; counts, offsets and list entries are batch-wide.
template<bool FILL>
__global__ void __launch_bounds__(256) batch_bin_kernel(const JobDesc *__restrict__ jobs, int nJobs,
  const SpacePrep *__restrict__ prep, int *__restrict__ counts, const int *__restrict__ offsets,
  int *__restrict__ list, const int *__restrict__ status)
{
  __shared__ SpacePrep tile[256];
  __shared__ int hitIdx[256];
  __shared__ int hitN, warpBase[8];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int j = job_of(jobs, nJobs, int(blockIdx.x), [](const JobDesc &J) { return J.groupBase; });
  const JobDesc &J = jobs[j];
  const int local = (int(blockIdx.x) - J.groupBase) * 8 + warp;
  const bool active = local < J.nBricks;
  const int b = J.brickBase + local;
  if (FILL && *status != 0) return;
  BinGeom g;
  g.vx = J.vx;
  g.vy = J.vy;
  g.vz = J.vz;
  g.nbx = J.nbx;
  g.nby = J.nby;
  g.nbz = J.nbz;
  g.n_bricks = J.nBricks;
  g.cx = J.cx;
  g.cy = J.cy;
  g.cz = J.cz;
  int b0[3] = {}, b1[3] = {};
  float a[3] = {}, e[3] = {};
  if (active) brick_box(g, local, b0, b1, a, e);
  int u0[3], u1[3];
  float ua[3], ue[3];
  const int first = (int(blockIdx.x) - J.groupBase) * 8;
  union_box(g, first, min(8, J.nBricks - first), u0, u1, ua, ue);
  int cnt[3] = { 0, 0, 0 };
  if (FILL && active)
    for (int d = 0; d < 3; ++d) cnt[d] = offsets[3 * b + d];
  const int n = J.nSpaces;
  SpacePrep next;
  if (int(threadIdx.x) < n) next = load_prep(prep + J.spaceBase + threadIdx.x);
  for (int base = 0; base < n; base += 256) {
    __syncthreads();
    if (base + int(threadIdx.x) < n) tile[threadIdx.x] = next;
    __syncthreads();
    if (base + 256 + int(threadIdx.x) < n) next = load_prep(prep + J.spaceBase + base + 256 + threadIdx.x);
    const int m = min(256, n - base);
    compact_tile_hits(tile, m, u0, u1, ua, ue, hitIdx, &hitN, warpBase);
    if (!active) continue;
    const int hn = hitN;
    for (int r = 0; r < hn; r += 32) {
      const int qq = r + lane;
      bool hit = false;
      int dir = 0, q = 0;
      if (qq < hn) {
        q = hitIdx[qq];
        hit = brick_hit(tile[q], b0, b1, a, e);
        dir = tile[q].dir;
      }
      for (int d = 0; d < 3; ++d) {
        unsigned mask = __ballot_sync(0xffffffffu, hit && dir == d);
        if (FILL && hit && dir == d) list[cnt[d] + __popc(mask & ((1u << lane) - 1u))] = J.spaceBase + base + q;
        cnt[d] += __popc(mask);
      }
    }
  }
  if (!FILL && active && lane == 0)
    for (int d = 0; d < 3; ++d) counts[3 * b + d] = cnt[d];
}

// Single-CTA planner: exclusive scan of the (brick, direction) counts into list offsets,
// then cuts every brick's list into work items of at most `itemCap` entries, bricks taken
// in `order` (heaviest expected first).  Sets status = FR_E_CAPACITY instead of
// overflowing the list or item buffers.  When the status is already set (a space with a
// projection outside the FFT payload, or an earlier failure), the fill pass writes no lists,
// so no work items are published either: the insertion then reads no list entry.
__global__ void __launch_bounds__(1024) plan_kernel(BinGeom g, const int *__restrict__ counts,
  int *__restrict__ offsets, const int *__restrict__ order, int itemCap, int64_t listCap,
  int64_t itemsCap, WorkItem *__restrict__ items, int *__restrict__ nItems, int *__restrict__ status,
  unsigned long long *__restrict__ stats, const JobDesc *__restrict__ jobs, int nJobs)
{
  __shared__ long long part[1024];
  const int tid = threadIdx.x, T = blockDim.x;
  const int prior = *status;  // read before this kernel writes it
  // pass 1: offsets over 3*n_bricks counts
  const int M = 3 * g.n_bricks;
  const int per = (M + T - 1) / T;
  long long s = 0;
  for (int k = tid * per; k < min(M, (tid + 1) * per); ++k) s += counts[k];
  part[tid] = s;
  __syncthreads();
  for (int off = 1; off < T; off <<= 1) {
    long long v = tid >= off ? part[tid - off] : 0;
    __syncthreads();
    part[tid] += v;
    __syncthreads();
  }
  long long run = part[tid] - s;
  const long long total = part[T - 1];
  for (int k = tid * per; k < min(M, (tid + 1) * per); ++k) {
    offsets[k] = int(min(run, (long long)listCap));
    run += counts[k];
  }
  if (tid == 0) offsets[M] = int(min(total, (long long)listCap));
  __syncthreads();
  // pass 2: items per brick in `order`
  const int NB = g.n_bricks;
  const int perb = (NB + T - 1) / T;
  s = 0;
  for (int k = tid * perb; k < min(NB, (tid + 1) * perb); ++k) {
    int bb = order[k];
    long long len = (long long)offsets[3 * bb + 3] - offsets[3 * bb];
    s += (len + itemCap - 1) / itemCap;
  }
  __syncthreads();
  part[tid] = s;
  __syncthreads();
  for (int off = 1; off < T; off <<= 1) {
    long long v = tid >= off ? part[tid - off] : 0;
    __syncthreads();
    part[tid] += v;
    __syncthreads();
  }
  run = part[tid] - s;
  const long long totalItems = part[T - 1];
  const bool fits = total <= listCap && totalItems <= itemsCap;
  const bool ok = fits && prior == 0;
  if (ok) {
    for (int k = tid * perb; k < min(NB, (tid + 1) * perb); ++k) {
      int bb = order[k];
      int beg = offsets[3 * bb], end = offsets[3 * bb + 3];
      int job = 0;  // batched plans: the job whose brick range holds bb
      if (jobs) {
        int lo = 0, hi = nJobs - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (jobs[mid].brickBase <= bb) lo = mid;
          else hi = mid - 1;
        }
        job = lo;
      }
      for (int q = beg; q < end; q += itemCap) {
        WorkItem it;
        it.brick = bb;
        it.begin = q;
        it.end = min(end, q + itemCap);
        it.job = job;
        items[run++] = it;
      }
    }
  }
  if (tid == 0) {
    *nItems = ok ? int(totalItems) : 0;
    if (!fits && prior == 0) *status = FR_E_CAPACITY;
    stats[0] += (unsigned long long)total;
    stats[1] += ok ? (unsigned long long)totalItems : 0ull;
    stats[2] += 1ull;
  }
}

// =====================================================================================
// Host-side launchers
// =====================================================================================

cudaError_t launch_blob_table(float *table, int64_t n, int order, float alpha, float radius,
  float iw0, cudaStream_t st)
{
  if (n <= 0) return cudaSuccess;
  int blocks = int((n + 255) / 256);
  blob_table_kernel<<<blocks, 256, 0, st>>>(table, n, order, alpha, radius, iw0);
  return cudaGetLastError();
}

cudaError_t launch_kaiser_table(float *table, int order, float alpha, float radius, float iw0, cudaStream_t st)
{
  kaiser_table_kernel<<<(kKaiserTableElems + 255) / 256, 256, 0, st>>>(reinterpret_cast<float2 *>(table),
    kKaiserTableElems, order, alpha, radius, iw0);
  return cudaGetLastError();
}

cudaError_t launch_traverse_spaces_sym(const float *rot, int64_t n, const float *sym, int nSym, uint32_t imgX,
  uint32_t imgY, uint32_t maxVX, uint32_t maxVYZ, int useFast, float radius, float weight, int32_t first,
  fr_traverse_space *out, cudaStream_t st)
{
  const int64_t total = n * nSym;
  if (total <= 0) return cudaSuccess;
  traverse_space_sym_kernel<<<unsigned((total + 127) / 128), 128, 0, st>>>(rot, n, sym, nSym, imgX, imgY, maxVX,
    maxVYZ, useFast, radius, weight, first, out);
  return cudaGetLastError();
}

cudaError_t launch_traverse_spaces(const float *rot, int64_t n, uint32_t imgX, uint32_t imgY,
  uint32_t maxVX, uint32_t maxVYZ, int useFast, float radius, float weight, int32_t first,
  fr_traverse_space *out, cudaStream_t st)
{
  if (n <= 0) return cudaSuccess;
  int blocks = int((n + 127) / 128);
  traverse_space_kernel<<<blocks, 128, 0, st>>>(rot, n, imgX, imgY, maxVX, maxVYZ, useFast, radius,
    weight, first, out);
  return cudaGetLastError();
}

cudaError_t launch_batch_binning(const JobDesc *jobs, int nJobs, int totalSpaces, int totalBricks,
  int totalGroups, bool fast, float radius, const BinBuffers &b, int itemCap, cudaStream_t st)
{
  const float hw = fast ? 2.5f : radius + 1e-3f;
  const float xmin = fast ? -1e-3f : -radius - 1e-3f;
  if (totalSpaces > 0)
    batch_prep_kernel<<<(totalSpaces + 255) / 256, 256, 0, st>>>(jobs, nJobs, totalSpaces, hw, xmin, radius,
      b.prep, b.rec, b.status);
  prefer_max_shared(batch_bin_kernel<false>);
  prefer_max_shared(batch_bin_kernel<true>);
  batch_bin_kernel<false><<<totalGroups, 256, 0, st>>>(jobs, nJobs, b.prep, b.counts, nullptr, nullptr, b.status);
  BinGeom g{};
  g.n_bricks = totalBricks;
  plan_kernel<<<1, 1024, 0, st>>>(g, b.counts, b.offsets, b.order, itemCap, b.listCap, b.itemsCap, b.items,
    b.nItems, b.status, b.stats, jobs, nJobs);
  batch_bin_kernel<true><<<totalGroups, 256, 0, st>>>(jobs, nJobs, b.prep, nullptr, b.offsets, b.list, b.status);
  return cudaGetLastError();
}

cudaError_t launch_quantize(const void *in, int64_t n, int64_t elems, int storage, void *out, float *scales,
  cudaStream_t st)
{
  if (n <= 0) return cudaSuccess;
  if (storage == FR_STORAGE_BF16)
    quantize_kernel<__nv_bfloat162><<<unsigned(n), 256, 0, st>>>(static_cast<const float2 *>(in), elems,
      static_cast<__nv_bfloat162 *>(out), scales);
  else
    quantize_kernel<__half2><<<unsigned(n), 256, 0, st>>>(static_cast<const float2 *>(in), elems,
      static_cast<__half2 *>(out), scales);
  return cudaGetLastError();
}

// ---- banded half-planes -------------------------------------------------------------------

// One band (4 rows of one projection) per warp: lane x reads the band's four rows at column x
// (runs of 32 consecutive columns per row) and writes them as one 4-pixel group, so the warp's
// stores form one contiguous run.  Columns beyond fftX and rows beyond fftY are zeros.
__device__ __forceinline__ void store4(float2 *d, const float2 (&v)[4])
{
  reinterpret_cast<float4 *>(d)[0] = make_float4(v[0].x, v[0].y, v[1].x, v[1].y);
  reinterpret_cast<float4 *>(d)[1] = make_float4(v[2].x, v[2].y, v[3].x, v[3].y);
}

__device__ __forceinline__ void store4(uint32_t *d, const uint32_t (&v)[4])
{
  *reinterpret_cast<uint4 *>(d) = make_uint4(v[0], v[1], v[2], v[3]);
}

template<typename E>
__device__ __forceinline__ void band_unit(const E *__restrict__ src, E *__restrict__ dst, int fftX, int fftY,
  int band, int lane)
{
  const int pitch = band_pitch(fftX);
  // two 32-column runs per round: eight loads of a lane in flight before its stores
  for (int x0 = lane; x0 < pitch; x0 += 64) {
    E v[2][4];
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int x = x0 + 32 * h, y = 4 * band + r;
        v[h][r] = x < fftX && y < fftY ? __ldg(src + size_t(y) * fftX + x) : E{};
      }
#pragma unroll
    for (int h = 0; h < 2; ++h)
      if (x0 + 32 * h < pitch) store4(dst + 4 * (x0 + 32 * h), v[h]);
  }
}

template<typename E>
__global__ void band_kernel(const E *__restrict__ src, E *__restrict__ dst, int64_t n, int fftX, int fftY)
{
  const int bands = (fftY + 3) / 4;
  const int64_t plane = int64_t(fftY) * fftX, bplane = band_plane_elems(fftX, fftY);
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t u = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; u < n * bands; u += warps) {
    const int64_t p = u / bands;
    const int b = int(u - p * bands);
    band_unit(src + p * plane, dst + p * bplane + int64_t(b) * band_stride(fftX), fftX, fftY, b, lane);
  }
}

template<typename E>
__global__ void batch_band_kernel(const JobDesc *__restrict__ jobs, int nJobs, int64_t total)
{
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t u = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; u < total; u += warps) {
    const int j = job_of(jobs, nJobs, int(u), [](const JobDesc &J) { return J.unitBase; });
    const JobDesc &J = jobs[j];
    const int bands = (J.fftY + 3) / 4;
    const int local = int(u) - J.unitBase;
    const int p = local / bands, b = local - p * bands;
    band_unit(static_cast<const E *>(J.src) + int64_t(p) * J.fftY * J.fftX,
      static_cast<E *>(const_cast<void *>(J.fft)) + int64_t(p) * band_plane_elems(J.fftX, J.fftY)
        + int64_t(b) * J.bandStride,
      J.fftX, J.fftY, b, lane);
  }
}

// Two 256-thread CTAs per SM: enough loads in flight to run near the copy bandwidth, and room
// left on every SM for the binning kernels that run beside the copy on the other stream
// (prefer_max_shared).
static int band_blocks(int64_t units)
{
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return int(std::max<int64_t>(1, std::min<int64_t>((units + 7) / 8, int64_t(sms) * 2)));
}

cudaError_t launch_band_projections(const void *src, void *dst, int64_t n, int fftX, int fftY, int elemBytes,
  cudaStream_t st)
{
  if (n <= 0) return cudaSuccess;
  const int blocks = band_blocks(n * ((fftY + 3) / 4));
  prefer_max_shared(band_kernel<float2>);
  prefer_max_shared(band_kernel<uint32_t>);
  if (elemBytes == 8)
    band_kernel<float2><<<blocks, 256, 0, st>>>(static_cast<const float2 *>(src), static_cast<float2 *>(dst), n, fftX,
      fftY);
  else
    band_kernel<uint32_t><<<blocks, 256, 0, st>>>(static_cast<const uint32_t *>(src), static_cast<uint32_t *>(dst), n,
      fftX, fftY);
  return cudaGetLastError();
}

cudaError_t launch_batch_band(const JobDesc *jobs, int nJobs, int64_t totalUnits, int elemBytes, cudaStream_t st)
{
  if (totalUnits <= 0) return cudaSuccess;
  const int blocks = band_blocks(totalUnits);
  prefer_max_shared(batch_band_kernel<float2>);
  prefer_max_shared(batch_band_kernel<uint32_t>);
  if (elemBytes == 8) batch_band_kernel<float2><<<blocks, 256, 0, st>>>(jobs, nJobs, totalUnits);
  else batch_band_kernel<uint32_t><<<blocks, 256, 0, st>>>(jobs, nJobs, totalUnits);
  return cudaGetLastError();
}

cudaError_t launch_binning(const BinGeom &g, const fr_traverse_space *spaces, int n, int nProj,
  bool fast, float radius, const BinBuffers &b, int itemCap, cudaStream_t st)
{
  const float hw = fast ? 2.5f : radius + 1e-3f;
  const float xmin = fast ? -1e-3f : -radius - 1e-3f;
  prefer_max_shared(space_prep_kernel);
  prefer_max_shared(bin_kernel<false>);
  prefer_max_shared(bin_kernel<true>);
  space_prep_kernel<<<(n + 255) / 256, 256, 0, st>>>(spaces, n, hw, xmin, radius, g.cx, g.cy, g.cz, nProj,
    b.prep, b.rec, b.status);
  const int blocks = (g.n_bricks + 7) / 8;
  bin_kernel<false><<<blocks, 256, 0, st>>>(g, b.prep, n, b.counts, nullptr, nullptr, b.status);
  plan_kernel<<<1, 1024, 0, st>>>(g, b.counts, b.offsets, b.order, itemCap, b.listCap, b.itemsCap,
    b.items, b.nItems, b.status, b.stats, nullptr, 0);
  bin_kernel<true><<<blocks, 256, 0, st>>>(g, b.prep, n, nullptr, b.offsets, b.list, b.status);
  return cudaGetLastError();
}

int insert_max_groups(const InsertConfig &cfg) { return cfg.kahan ? 2 : 3; }

int insert_groups(const InsertConfig &cfg)
{
  const int mx = insert_max_groups(cfg);
  return cfg.groups > 0 && cfg.groups < mx ? cfg.groups : mx;
}

// Bytes of the kernel's table (the lookup table's entries, or the fixed Kaiser table of
// dynamic interpolation); 0 when the mode reads none.
static size_t table_bytes(const InsertConfig &cfg, int tableElems)
{
  if (cfg.fast) return 0;
  if (cfg.mode == 0) return tableElems <= kLutSmemMax ? size_t(tableElems) * sizeof(float) : 0;
  if (cfg.mode == 3) return size_t(kKaiserTableElems) * sizeof(float2);
  return 0;
}

bool insert_lut_in_smem(const InsertConfig &cfg, int tableElems)
{
  const size_t acc = size_t(insert_groups(cfg)) * size_t(cfg.kahan ? 18 : 12) * kBrickVox;
  const size_t t = table_bytes(cfg, tableElems);
  return t > 0 && acc + t <= (227u << 10);
}

size_t insert_smem_bytes(const InsertConfig &cfg, int tableElems)
{
  size_t acc = size_t(insert_groups(cfg)) * size_t(cfg.kahan ? 18 : 12) * kBrickVox;
  return acc + (insert_lut_in_smem(cfg, tableElems) ? table_bytes(cfg, tableElems) : 0);
}

static InsertFn pick_kernel(const InsertConfig &cfg)
{
  if (cfg.jobs) {
    switch (cfg.storage) {
    case FR_STORAGE_BF16: return pick_insert_batch_bf16(cfg);
    case FR_STORAGE_FP16: return pick_insert_batch_fp16(cfg);
    default: return pick_insert_batch_fp32(cfg);
    }
  }
  if (cfg.banded) {
    switch (cfg.storage) {
    case FR_STORAGE_BF16: return pick_insert_band_bf16(cfg);
    case FR_STORAGE_FP16: return pick_insert_band_fp16(cfg);
    default: return pick_insert_band_fp32(cfg);
    }
  }
  switch (cfg.storage) {
  case FR_STORAGE_BF16: return pick_insert_bf16(cfg);
  case FR_STORAGE_FP16: return pick_insert_fp16(cfg);
  default: return pick_insert_fp32(cfg);
  }
}

const void *insert_kernel_ptr(const InsertConfig &cfg)
{
  return reinterpret_cast<const void *>(pick_kernel(cfg));
}

cudaError_t launch_insert(const InsertParams &P, const InsertConfig &cfg, int grid, cudaStream_t st)
{
  const size_t smem = insert_smem_bytes(cfg, P.tableElems);
  InsertFn k = pick_kernel(cfg);
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  k<<<grid, kThreads * insert_groups(cfg), smem, st>>>(P);
  return cudaGetLastError();
}

}// namespace frb
