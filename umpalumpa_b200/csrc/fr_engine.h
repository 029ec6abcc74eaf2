// Internal hooks of the host engine (fr_capi.cu) for the serving layer (fr_server.cu).
#pragma once

#include "umpalumpa_fr.h"

namespace frb {

// Sticky device-side status (FR_OK or an FR_E_* code) as copied back by the handle's last
// finished batched launch; valid once that launch's work has completed on the stream.
int batch_device_status(const fr_handle *h);

}// namespace frb
