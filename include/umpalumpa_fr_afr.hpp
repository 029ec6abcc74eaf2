// umpalumpa_fr_afr.hpp -- the B200 engine as an AFR strategy of the Umpalumpa reference.
//
// Header-only shim for a maintainer of the reference tree: include it after the reference's
// afr.hpp (libumpalumpa/operations/fourier_reconstruction/afr.hpp:35-55) and construct an
// FRB200 where an FRCUDA (fr_cuda.hpp:8-20) was constructed.  It keeps the reference's
// operation contract (basic_operation.hpp:28-105): Init and Execute return false for invalid
// or non-equivalent payloads, Execute is asynchronous, Synchronize waits; CUDA failures throw
// std::runtime_error as the reference's CudaErrchk does (utils/cuda.cpp:7-14).  Link with
// libfr_b200.so.
#pragma once

#include <cstring>
#include <stdexcept>
#include <string>

#include <libumpalumpa/operations/fourier_reconstruction/afr.hpp>
#include <libumpalumpa/operations/fourier_reconstruction/traverse_space.hpp>

#include "umpalumpa_fr.h"

namespace umpalumpa::fourier_reconstruction {

static_assert(sizeof(TraverseSpace) == sizeof(fr_traverse_space), "TraverseSpace layout");
static_assert(sizeof(Constants) == sizeof(fr_constants), "Constants layout");

class FRB200 : public AFR
{
public:
  // device: CUDA device ordinal; stream: a cudaStream_t (nullptr = the default stream).
  explicit FRB200(int device = 0, void *stream = nullptr)
  {
    if (fr_create(device, stream, &handle) != FR_OK) throw std::runtime_error(fr_last_error());
  }
  ~FRB200() override
  {
    if (handle) fr_destroy(handle);
    handle = nullptr;
  }
  FRB200(const FRB200 &) = delete;
  FRB200 &operator=(const FRB200 &) = delete;

  void Synchronize() override
  {
    const int rc = fr_synchronize(handle);
    if (rc != FR_OK) throw std::runtime_error(fr_last_error());
  }

  void Cleanup() override
  {
    if (handle) fr_cleanup(handle);
    AFR::Cleanup();
  }

  size_t GetUsedBytes() const override { return size_t(fr_used_bytes(handle)); }

  // Settings of the engine beyond the reference's (settings.hpp:8-67).
  void SetMaxResolution(float m) { maxResolution = m; }
  void SetStorage(int s) { storage = s; }
  void SetAccumulation(int a) { accumulation = a; }
  void SetLayout(int l) { layout = l; }  // FR_LAYOUT_*; the reference's callers pass row-major FFTs

protected:
  bool InitImpl() override
  {
    const fr_dims d = Dims(GetInputRef());
    const fr_settings s = ToC(GetSettings());
    const int rc = fr_init(handle, &d, &s);
    if (rc == FR_E_CUDA) throw std::runtime_error(fr_last_error());
    return rc == FR_OK;
  }

  bool ExecuteImpl(const OutputData &, const InputData &in) override
  {
    const fr_dims d = Dims(in);
    const int rc = fr_execute(handle, in.GetFFT().GetPtr(), nullptr, d.n_projections,
      in.GetVolume().GetPtr(), static_cast<float *>(in.GetWeight().GetPtr()),
      static_cast<const fr_traverse_space *>(in.GetTraverseSpace().GetPtr()), d.n_spaces,
      static_cast<const float *>(in.GetBlobTable().GetPtr()));
    if (rc == FR_E_CUDA) throw std::runtime_error(fr_last_error());
    return rc == FR_OK;
  }

private:
  fr_handle *handle = nullptr;
  float maxResolution = 0.5f;
  int storage = FR_STORAGE_FP32;
  int accumulation = FR_ACCUM_PLAIN;
  int layout = FR_LAYOUT_AUTO;

  static fr_dims Dims(const InputData &in)
  {
    fr_dims d;
    const auto &f = in.GetFFT().info.GetSize();  // frequency-domain size X x Y x 1 x N
    const auto &v = in.GetVolume().info.GetSize();
    d.fft_x = f.x;
    d.fft_y = f.y;
    d.n_projections = f.n;
    d.volume_x = v.x;
    d.volume_y = v.y;
    d.volume_z = v.z;
    d.n_spaces = in.GetTraverseSpace().info.GetSize().total;  // as FRCPU counts (fr_cpu.cpp:40)
    d.table_elems = in.GetBlobTable().info.Elems();
    return d;
  }

  fr_settings ToC(const Settings &s) const
  {
    fr_settings c;
    fr_settings_default(&c);
    c.interpolation = s.GetInterpolation() == Settings::Interpolation::kLookup ? FR_INTERPOLATION_LOOKUP
                                                                               : FR_INTERPOLATION_DYNAMIC;
    c.blob_order = ToInt(s.GetBlobOrder());
    c.type = s.GetType() == Settings::Type::kPrecise ? FR_TYPE_PRECISE : FR_TYPE_FAST;
    c.alpha = s.GetAlpha();
    c.blob_radius = s.GetBlobRadius();
    c.max_resolution = maxResolution;
    c.storage = storage;
    c.accumulation = accumulation;
    c.layout = layout;
    return c;
  }
};

}// namespace umpalumpa::fourier_reconstruction
