// Internal hooks between the host engine (fr_capi.cu), the serving layer (fr_server.cu) and
// the autotuner (fr_tune.cu).
#pragma once

#include "umpalumpa_fr.h"

namespace frb {

// Sticky device-side status (FR_OK or an FR_E_* code) as copied back by the handle's last
// finished batched launch; valid once that launch's work has completed on the stream.
int batch_device_status(const fr_handle *h);

// Autotuner hooks (fr_tune.cu).  tune_lookup: the launch parameters of the tuning file of the
// handle's current strategy (dims/limits and settings set), if the file exists.  tune_single:
// the search of fr_autotune, run by fr_execute under FR_TUNING_ON_EXECUTE.
bool tune_lookup(const fr_handle *h, fr_launch_params *out);
int tune_single(fr_handle *h, const void *fft, const float *scales, uint64_t nProj,
  const fr_traverse_space *spaces, uint64_t nSpaces, const float *table, fr_tune_report *report);

}// namespace frb
