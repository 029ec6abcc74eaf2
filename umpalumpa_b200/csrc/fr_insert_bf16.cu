// Insertion-kernel variants for BF16 projection storage, row-major half-planes (see fr_insert.cuh).
#include "fr_insert.cuh"

namespace frb {
InsertFn pick_insert_bf16(const InsertConfig &cfg) { return pick_storage<FR_STORAGE_BF16, false>(cfg); }
}// namespace frb
