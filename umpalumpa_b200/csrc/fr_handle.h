// Internal: the engine handle behind the C-ABI's opaque fr_handle, shared by the host engine
// (fr_capi.cu) and the autotuner (fr_tune.cu).
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "fr_device.cuh"
#include "fr_kernels.h"
#include "umpalumpa_fr.h"

// Device staging of host-resident inputs: two slots used alternately, each filled on the
// copy stream once the insertion work that last read it has finished, so the upload of one
// Execute batch overlaps the insertion of the previous one.
struct StageSlot {
  void *buf = nullptr;
  size_t bytes = 0;
  cudaEvent_t ready = nullptr;  // upload finished (copy stream)
  cudaEvent_t free = nullptr;   // last reader finished (compute stream)
  bool used = false;
};

struct fr_handle {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_stream = nullptr;
  int num_sms = 0;
  bool initialized = false;
  fr_dims dims{};
  fr_settings settings{};
  fr_constants constants{};
  frb::BinGeom geom{};
  frb::InsertConfig cfg{};
  fr_launch_params launch{};
  int64_t chunk_cap = 0;
  int grid = 0;
  void *scratch = nullptr;
  size_t scratch_bytes = 0;
  frb::BinBuffers bb{};
  int *work_counter = nullptr;
  int *host_status = nullptr;                 // pinned: status + padding
  unsigned long long *host_stats = nullptr;   // pinned: 4 counters
  StageSlot slots[2];
  int next_slot = 0;
  // Banded copy of the projections (FR_LAYOUT_AUTO and batches): written on band_stream while
  // the binning runs on `stream`, between the events band_fork and band_join.
  void *band = nullptr;
  size_t band_bytes = 0;
  size_t band_refused = 0;  // smallest size that could not be had (AUTO reads rows above it)
  cudaStream_t band_stream = nullptr;
  cudaEvent_t band_fork = nullptr, band_join = nullptr;
  fr_exec_stats last{};
  uint64_t launches_pending = 0;
  // profiling: event pairs recorded around binning rounds and insertion launches
  bool profiling = false;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<int, int>> ev_bin, ev_ins;  // indices into ev_pool
  std::vector<uint64_t> ins_spaces;
  size_t ev_next = 0;
  fr_phase_times times{};
  // batched mode (fr_batch_init / fr_batch_execute)
  bool batch = false;
  fr_batch_limits blim{};
  frb::JobDesc *d_jobs = nullptr;     // in scratch
  float *kaiser_table = nullptr;      // dynamic interpolation: Kaiser (value, slope) table in scratch
  frb::JobDesc *h_jobs = nullptr;     // pinned staging of the job table (the set in use)
  int *h_order = nullptr;             // pinned staging of the brick order (the set in use)
  cudaEvent_t upload_done = nullptr;  // the set may be rewritten once its last upload finished
  // Two staging sets, used in turn by eager launches: a launch fills one set while the other's
  // upload still waits in the stream behind the previous launch's kernels (graph mode keeps
  // set 0, which its captured copies read).
  frb::JobDesc *h_jobs_set[2] = {};
  int *h_order_set[2] = {};
  cudaEvent_t upload_set_done[2] = {};
  int upload_set = 0;
  cudaGraphExec_t graph = nullptr;    // captured batch, replayed while the job table repeats
  std::vector<unsigned char> graph_sig;
  // brick visiting order of each volume shape: bricks nearest the volume centre first
  std::map<std::array<int, 3>, std::vector<int>> brick_order;
  // autotuning (fr_tune.cu)
  std::string device_name;
  int tuning = FR_TUNING_OFF;
  std::string tuning_dir;      // empty: the default directory
  bool tuned = false;          // this Init's parameters came from a tuning file or a search
  bool tuning_active = false;  // a search is running: no tuning-file lookups, no nested search
};
