// TEST INFRASTRUCTURE ONLY. Never linked into the product.
//
// An extern "C" harness around the reference's own CPU Fourier-processing kernel, so that the
// Python tests can check the restatement in oracle/__init__.py against the unmodified
// reference code.  The reference header is compiled in place from the read-only reference
// tree by oracle/Makefile; nothing from it is copied here.
//
// Reference entry points driven here (paths relative to the reference project root):
//   ScaleFFT2DCPU<applyFilter, normalize, center, cropFreq, shift>::Execute
//       libumpalumpa/operations/fourier_processing/fp_cpu_kernels.hpp:8-41
//   its arguments as FPCPU's Strategy1 passes them (normFactor = 1/padded spatial size, the
//   max frequency unsquared as maxFreqSquare)
//       libumpalumpa/operations/fourier_processing/fp_cpu.cpp:25-46
#include <complex>
#include <cstdint>
#include <libumpalumpa/operations/fourier_processing/fp_cpu_kernels.hpp>

using umpalumpa::data::Size;
using umpalumpa::fourier_processing::ScaleFFT2DCPU;

namespace {

template<bool N, bool C, bool F, bool S>
void run(const std::complex<float> *in, std::complex<float> *out, const Size &inSize, const Size &spatial,
  const Size &outSize, float norm, float maxFreq)
{
  ScaleFFT2DCPU<false, N, C, F, S>::template Execute<float, std::complex<float>>(
    in, out, inSize, spatial, outSize, nullptr, norm, maxFreq);
}

}// namespace

extern "C" int fpref_scale_fft2d(const float *in, float *out, uint64_t inX, uint64_t inY, uint64_t n,
  uint64_t spatialX, uint64_t spatialY, uint64_t outX, uint64_t outY, int normalize, int center, int cropFreq,
  int shift, float maxFreq)
{
  const Size inSize(inX, inY, 1, n), spatial(spatialX, spatialY, 1, n), outSize(outX, outY, 1, n);
  const float norm = 1.f / static_cast<float>(spatial.single);
  auto *i = reinterpret_cast<const std::complex<float> *>(in);
  auto *o = reinterpret_cast<std::complex<float> *>(out);
  const int key = (normalize ? 8 : 0) | (center ? 4 : 0) | (cropFreq ? 2 : 0) | (shift ? 1 : 0);
  switch (key) {
  case 0: run<false, false, false, false>(i, o, inSize, spatial, outSize, norm, maxFreq); break;
  case 1: run<false, false, false, true>(i, o, inSize, spatial, outSize, norm, maxFreq); break;
  case 2: run<false, false, true, false>(i, o, inSize, spatial, outSize, norm, maxFreq); break;
  case 3: run<false, false, true, true>(i, o, inSize, spatial, outSize, norm, maxFreq); break;
  case 4: run<false, true, false, false>(i, o, inSize, spatial, outSize, norm, maxFreq); break;
  case 5: run<false, true, false, true>(i, o, inSize, spatial, outSize, norm, maxFreq); break;
  case 6: run<false, true, true, false>(i, o, inSize, spatial, outSize, norm, maxFreq); break;
  case 7: run<false, true, true, true>(i, o, inSize, spatial, outSize, norm, maxFreq); break;
  case 8: run<true, false, false, false>(i, o, inSize, spatial, outSize, norm, maxFreq); break;
  case 9: run<true, false, false, true>(i, o, inSize, spatial, outSize, norm, maxFreq); break;
  case 10: run<true, false, true, false>(i, o, inSize, spatial, outSize, norm, maxFreq); break;
  case 11: run<true, false, true, true>(i, o, inSize, spatial, outSize, norm, maxFreq); break;
  case 12: run<true, true, false, false>(i, o, inSize, spatial, outSize, norm, maxFreq); break;
  case 13: run<true, true, false, true>(i, o, inSize, spatial, outSize, norm, maxFreq); break;
  case 14: run<true, true, true, false>(i, o, inSize, spatial, outSize, norm, maxFreq); break;
  default: run<true, true, true, true>(i, o, inSize, spatial, outSize, norm, maxFreq); break;
  }
  return 0;
}
