// TEST INFRASTRUCTURE ONLY. Never linked into the product.
//
// A thin extern "C" harness around the reference's own CPU implementation (FRCPU) of the
// Fourier-reconstruction insertion, so that the Python tests and the CPU baseline can drive
// the unmodified reference code.  The reference sources are compiled in place from the
// read-only reference tree by oracle/Makefile; nothing from them is copied here.
//
// Reference entry points driven here (paths relative to the reference project root):
//   AFR::CreateConstants / AFR::FillBlobTable   libumpalumpa/operations/fourier_reconstruction/afr.cpp:6-34
//   ComputeTraverseSpace                          libumpalumpa/operations/fourier_reconstruction/traverse_space_generator.hpp:94-145
//   FRCPU Init / Execute                          libumpalumpa/operations/fourier_reconstruction/fr_cpu.cpp:9-45
//                                                 libumpalumpa/operations/basic_operation.hpp:28-66
#include <cstdint>
#include <cstring>
#include <complex>
#include <thread>
#include <vector>
#include <libumpalumpa/operations/fourier_reconstruction/fr_cpu.hpp>
#include <libumpalumpa/operations/fourier_reconstruction/traverse_space_generator.hpp>

using namespace umpalumpa::fourier_reconstruction;
using namespace umpalumpa::data;

static_assert(sizeof(TraverseSpace) == 112, "reference TraverseSpace layout changed");
static_assert(sizeof(Constants) == 32, "reference Constants layout changed");

namespace {

Settings MakeSettings(int interpolation, int order, int type, float alpha, float radius)
{
  Settings s;
  s.SetInterpolation(interpolation == 1 ? Settings::Interpolation::kLookup
                                        : Settings::Interpolation::kDynamic);
  s.SetBlobOrder(static_cast<BlobOrder>(order));
  s.SetType(type == 1 ? Settings::Type::kPrecise : Settings::Type::kFast);
  s.SetAlpha(alpha);
  s.SetBlobRadius(radius);
  return s;
}

PhysicalDescriptor Phys(void *p, size_t bytes, DataType t)
{
  return PhysicalDescriptor(p, bytes, t, ManagedBy::Manually, nullptr);
}

// The five reference payloads for one call.  The FFT payload is described in the spatial
// domain with width 2*(fftX-1), so that its frequency-domain size is exactly fftX x fftY.
struct Payloads
{
  Payload<FourierDescriptor> fft, volume;
  Payload<LogicalDescriptor> weight, spaces, table;

  Payloads(void *fftPtr, size_t fftX, size_t fftY, size_t nProj, void *vol, void *wgt,
    size_t vx, size_t vy, size_t vz, void *sp, size_t nSpaces, void *tab, size_t tabElems)
    : fft(FourierDescriptor(Size(2 * (fftX - 1), fftY, 1, nProj), PaddingDescriptor(),
            FourierDescriptor::FourierSpaceDescriptor{}),
        Phys(fftPtr, fftX * fftY * nProj * sizeof(std::complex<float>),
          DataType::Get<std::complex<float>>())),
      volume(FourierDescriptor(Size(vx, vy, vz, 1), PaddingDescriptor(), VolumeFsd()),
        Phys(vol, vx * vy * vz * sizeof(std::complex<float>), DataType::Get<std::complex<float>>())),
      weight(LogicalDescriptor(Size(vx, vy, vz, 1)),
        Phys(wgt, vx * vy * vz * sizeof(float), DataType::Get<float>())),
      spaces(LogicalDescriptor(Size(1, 1, 1, nSpaces)),
        Phys(sp, nSpaces * sizeof(TraverseSpace), DataType::Get<TraverseSpace>())),
      table(LogicalDescriptor(Size(tabElems, 1, 1, 1)),
        Phys(tabElems ? tab : nullptr, tabElems * sizeof(float), DataType::Get<float>()))
  {}

  static FourierDescriptor::FourierSpaceDescriptor VolumeFsd()
  {
    auto f = FourierDescriptor::FourierSpaceDescriptor{};
    f.hasSymetry = true;
    return f;
  }
};

// One FRCPU Init+Execute over `nSpaces` traverse spaces.  Returns 0 on success.
int RunOnce(const Settings &s, void *fft, size_t fftX, size_t fftY, size_t nProj, void *vol,
  void *wgt, size_t vx, size_t vy, size_t vz, TraverseSpace *sp, size_t nSpaces, float *tab,
  size_t tabElems)
{
  if (nSpaces == 0) return 0;
  Payloads p(fft, fftX, fftY, nProj, vol, wgt, vx, vy, vz, sp, nSpaces, tab, tabElems);
  auto in = AFR::InputData(p.fft, p.volume, p.weight, p.spaces, p.table);
  auto out = AFR::OutputData(p.volume, p.weight);
  FRCPU op;
  if (!op.Init(out, in, s)) return 1;
  if (!op.Execute(out, in)) return 2;
  op.Synchronize();
  return 0;
}

// FRCPU forms the projection offset as int(xSize*ySize*projectionIndex)
// (fr_cpu_kernels.hpp:256), which overflows once that product passes 2^31.  Split the
// spaces into runs whose projection indices fit, rebase the FFT pointer and indices.
int RunChunked(const Settings &s, std::complex<float> *fft, size_t fftX, size_t fftY,
  size_t nProj, void *vol, void *wgt, size_t vx, size_t vy, size_t vz, const TraverseSpace *sp,
  size_t nSpaces, float *tab, size_t tabElems)
{
  const size_t plane = fftX * fftY;
  const size_t maxIdx = (size_t(1) << 31) / plane - 1;// largest safe projection index per run
  size_t i = 0;
  std::vector<TraverseSpace> run;
  while (i < nSpaces) {
    size_t base = size_t(sp[i].projectionIndex);
    run.clear();
    size_t lo = base, hi = base;
    while (i < nSpaces) {
      size_t pi = size_t(sp[i].projectionIndex);
      size_t nlo = std::min(lo, pi), nhi = std::max(hi, pi);
      if (nhi - nlo > maxIdx) break;
      lo = nlo;
      hi = nhi;
      run.push_back(sp[i]);
      ++i;
    }
    for (auto &t : run) t.projectionIndex = int(size_t(t.projectionIndex) - lo);
    int rc = RunOnce(s, fft + lo * plane, fftX, fftY, hi - lo + 1, vol, wgt, vx, vy, vz,
      run.data(), run.size(), tab, tabElems);
    if (rc) return rc;
  }
  return 0;
}

}// namespace

extern "C" {

int ref_sizeof_traverse_space() { return int(sizeof(TraverseSpace)); }

void ref_compute_traverse_space(uint32_t imgSizeX, uint32_t imgSizeY, const float *transform9,
  void *spaceOut, uint32_t maxVolumeIndexX, uint32_t maxVolumeIndexYZ, int useFast,
  float blobRadius, float weight, int projectionIndex)
{
  float t[3][3];
  for (int i = 0; i < 9; ++i) t[i / 3][i % 3] = transform9[i];
  TraverseSpace ts{};
  ComputeTraverseSpace(
    imgSizeX, imgSizeY, t, ts, maxVolumeIndexX, maxVolumeIndexYZ, useFast != 0, blobRadius, weight);
  ts.projectionIndex = projectionIndex;
  std::memcpy(spaceOut, &ts, sizeof(ts));
}

void ref_make_constants(size_t vx, size_t vy, size_t vz, size_t tableElems, int interpolation,
  int order, int type, float alpha, float radius, void *constantsOut)
{
  auto s = MakeSettings(interpolation, order, type, alpha, radius);
  std::vector<float> dummyTable(tableElems ? tableElems : 1);
  Payloads p(nullptr, 2, 2, 1, nullptr, nullptr, vx, vy, vz, nullptr, 1, dummyTable.data(),
    tableElems);
  auto in = AFR::InputData(p.fft, p.volume, p.weight, p.spaces, p.table);
  Constants c = AFR::CreateConstants(in, s);
  std::memcpy(constantsOut, &c, sizeof(c));
}

void ref_fill_blob_table(float *table, size_t tableElems, int order, float alpha, float radius)
{
  auto s = MakeSettings(1, order, 1, alpha, radius);
  Payloads p(nullptr, 2, 2, 1, nullptr, nullptr, 3, 3, 3, nullptr, 1, table, tableElems);
  auto in = AFR::InputData(p.fft, p.volume, p.weight, p.spaces, p.table);
  AFR::FillBlobTable(in, s);
}

// Reference FRCPU over all spaces, split across `threads` host threads (each with its own
// FRCPU instance over a contiguous range of spaces; the reference's CAS float atomics make
// the shared accumulation race-free).  threads <= 1 runs the reference serially.
int ref_fr_execute(void *fft, size_t fftX, size_t fftY, size_t nProj, void *volume, void *weight,
  size_t vx, size_t vy, size_t vz, const void *spaces, size_t nSpaces, float *table,
  size_t tableElems, int interpolation, int order, int type, float alpha, float radius,
  int threads)
{
  auto s = MakeSettings(interpolation, order, type, alpha, radius);
  auto *f = reinterpret_cast<std::complex<float> *>(fft);
  auto *sp = reinterpret_cast<const TraverseSpace *>(spaces);
  if (threads <= 1 || nSpaces < 2) {
    return RunChunked(
      s, f, fftX, fftY, nProj, volume, weight, vx, vy, vz, sp, nSpaces, table, tableElems);
  }
  size_t T = std::min<size_t>(size_t(threads), nSpaces);
  std::vector<int> rcs(T, 0);
  std::vector<std::thread> pool;
  for (size_t t = 0; t < T; ++t) {
    size_t b = nSpaces * t / T, e = nSpaces * (t + 1) / T;
    pool.emplace_back([&, t, b, e]() {
      rcs[t] = RunChunked(
        s, f, fftX, fftY, nProj, volume, weight, vx, vy, vz, sp + b, e - b, table, tableElems);
    });
  }
  for (auto &th : pool) th.join();
  for (int rc : rcs)
    if (rc) return rc;
  return 0;
}

}// extern "C"
