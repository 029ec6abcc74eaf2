// The reference's twelve AFR unit cases, run through the reference's own operation API and
// payload types with the B200 engine as the strategy (include/umpalumpa_fr_afr.hpp).
//
// Cases as in tests/operations/fourier_reconstruction/fr_tests.hpp:7-101: a 5x6 projection
// (a 3x6 half-plane) into a 7^3 volume, one axis-permutation rotation per plane (XY, YZ, XZ),
// kFast/kPrecise x kDynamic/kLookup; payloads in CUDA managed memory as the reference's CUDA
// tests allocate them (tests/operations/fourier_reconstruction/fr_cuda.cpp:11-27).  Each case
// checks the traverse space the reference generator produced, then the structure of the
// inserted volume (afr_common.hpp:256-314): zero outside the frequency sphere, behind the
// image or off the slab; non-zero real, imaginary and weight elsewhere.
// Exit status 0 when every case passes.
#include <cuda_runtime.h>

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <numeric>

#include <libumpalumpa/operations/fourier_reconstruction/afr.hpp>
#include <libumpalumpa/operations/fourier_reconstruction/traverse_space_generator.hpp>

#include "umpalumpa_fr_afr.hpp"

using namespace umpalumpa::fourier_reconstruction;
using namespace umpalumpa::data;

namespace {

void *Managed(size_t bytes)
{
  void *p = nullptr;
  if (cudaMallocManaged(&p, bytes) != cudaSuccess) throw std::runtime_error("cudaMallocManaged");
  std::memset(p, 0, bytes);
  return p;
}

PhysicalDescriptor PD(void *p, size_t bytes, DataType t)
{
  return PhysicalDescriptor(p, bytes, t, ManagedBy::CUDA, nullptr);
}

int Check(const float2 *vol, const float *w, const TraverseSpace &s, float maxDistance)
{
  int bad = 0;
  const int n = 7, c = 3;
  for (int z = 0; z < n; ++z)
    for (int y = 0; y < n; ++y)
      for (int x = 0; x < n; ++x) {
        const float p[3] = { float(x - c), float(y - c), float(z - c) };
        const size_t i = (size_t(z) * n + y) * n + x;
        const bool zero = vol[i].x == 0.f && vol[i].y == 0.f && w[i] == 0.f;
        const bool nonzero = vol[i].x != 0.f && vol[i].y != 0.f && w[i] != 0.f;
        bool expectZero;
        if (p[0] * p[0] + p[1] * p[1] + p[2] * p[2] > s.maxDistanceSqr) {
          expectZero = true;
        } else {
          const float ix = s.transformInv[0][0] * p[0] + s.transformInv[0][1] * p[1] + s.transformInv[0][2] * p[2];
          const float d = std::fabs(s.unitNormal.x * p[0] + s.unitNormal.y * p[1] + s.unitNormal.z * p[2]);
          expectZero = ix < -maxDistance || d > maxDistance;
        }
        if (expectZero ? !zero : !nonzero) ++bad;
      }
  return bad;
}

int RunCase(const char *plane, Settings::Type type, Settings::Interpolation interp)
{
  Settings s;
  s.SetType(type);
  s.SetInterpolation(interp);
  const auto c2 = DataType::Get<std::complex<float>>();
  const auto f1 = DataType::Get<float>();
  auto fsd = FourierDescriptor::FourierSpaceDescriptor{};
  auto fftLd = FourierDescriptor(Size(5, 6, 1, 1), PaddingDescriptor(), fsd);
  auto vfsd = fsd;
  vfsd.hasSymetry = true;
  auto volLd = FourierDescriptor(Size(7, 7, 7, 1), PaddingDescriptor(), vfsd);
  auto wLd = LogicalDescriptor(Size(7, 7, 7, 1));
  auto spLd = LogicalDescriptor(Size(1, 1, 1, 1));
  const size_t tableN = interp == Settings::Interpolation::kLookup ? 10000 : 0;
  auto tabLd = LogicalDescriptor(Size(tableN, 1, 1, 1));

  Payload<FourierDescriptor> fft(fftLd, PD(Managed(fftLd.Elems() * 8), fftLd.Elems() * 8, c2));
  Payload<FourierDescriptor> vol(volLd, PD(Managed(volLd.Elems() * 8), volLd.Elems() * 8, c2));
  Payload<LogicalDescriptor> wgt(wLd, PD(Managed(wLd.Elems() * 4), wLd.Elems() * 4, f1));
  Payload<LogicalDescriptor> sp(spLd, PD(Managed(sizeof(TraverseSpace)), sizeof(TraverseSpace), DataType::Get<TraverseSpace>()));
  Payload<LogicalDescriptor> tab(tabLd, tableN ? PD(Managed(tableN * 4), tableN * 4, f1) : PD(nullptr, 0, f1));

  float t[3][3] = {};
  if (plane[0] == 'x' && plane[1] == 'y') {
    t[0][0] = t[1][1] = t[2][2] = 1.f;
  } else if (plane[0] == 'y') {
    t[0][2] = t[1][1] = 1.f;
    t[2][0] = -1.f;
  } else {
    t[0][1] = t[2][0] = -1.f;
    t[1][2] = 1.f;
  }
  auto &space = *static_cast<TraverseSpace *>(sp.GetPtr());
  ComputeTraverseSpace(6 / 2, 6, t, space, 7 - 1, 7 - 1, type == Settings::Type::kFast, s.GetBlobRadius(), 1.f);

  auto out = AFR::OutputData(vol, wgt);
  auto in = AFR::InputData(fft, vol, wgt, sp, tab);
  if (tableN) AFR::FillBlobTable(in, s);
  float *f = static_cast<float *>(fft.GetPtr());
  const size_t nf = fftLd.Elems() * 2;
  if (plane[0] == 'x' && plane[1] == 'y')
    std::fill(f, f + nf, 1.f);
  else
    std::iota(f, f + nf, 1.f);

  FRB200 op(0, nullptr);
  int bad = 0;
  if (!op.Init(out, in, s)) {
    std::printf("FAIL %s: Init returned false: %s\n", plane, fr_last_error());
    return 1;
  }
  if (!op.Execute(out, in)) {
    std::printf("FAIL %s: Execute returned false: %s\n", plane, fr_last_error());
    return 1;
  }
  op.Synchronize();
  bad = Check(static_cast<const float2 *>(vol.GetPtr()), static_cast<const float *>(wgt.GetPtr()), space,
    type == Settings::Type::kFast ? 0.f : s.GetBlobRadius());
  std::printf("%s %s %s %s (%d mismatching voxels)\n", bad ? "FAIL" : "PASS", plane,
    type == Settings::Type::kFast ? "fast" : "precise",
    interp == Settings::Interpolation::kLookup ? "lookup" : "dynamic", bad);
  for (void *p : { fft.GetPtr(), vol.GetPtr(), wgt.GetPtr(), sp.GetPtr(), tab.GetPtr() })
    if (p) cudaFree(p);
  return bad ? 1 : 0;
}

}// namespace

int main()
{
  int failures = 0;
  for (const char *plane : { "xy", "yz", "xz" })
    for (auto type : { Settings::Type::kPrecise, Settings::Type::kFast })
      for (auto interp : { Settings::Interpolation::kDynamic, Settings::Interpolation::kLookup })
        failures += RunCase(plane, type, interp);
  std::printf("%d of 12 cases failed\n", failures);
  return failures ? 1 : 0;
}
