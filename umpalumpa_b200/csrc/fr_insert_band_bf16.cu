// Insertion-kernel variants for BF16 projection storage, banded half-planes (see fr_insert.cuh).
#include "fr_insert.cuh"

namespace frb {
InsertFn pick_insert_band_bf16(const InsertConfig &cfg) { return pick_storage<FR_STORAGE_BF16, true>(cfg); }
}// namespace frb
