// Insertion-kernel variants for FP16 projection storage, banded half-planes (see fr_insert.cuh).
#include "fr_insert.cuh"

namespace frb {
InsertFn pick_insert_band_fp16(const InsertConfig &cfg) { return pick_storage<FR_STORAGE_FP16, true>(cfg); }
}// namespace frb
