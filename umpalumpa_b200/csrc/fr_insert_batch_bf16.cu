// Batched insertion-kernel variants for BF16 projection storage (see fr_insert.cuh).
#include "fr_insert.cuh"

namespace frb {
InsertFn pick_insert_batch_bf16(const InsertConfig &cfg) { return pick_storage_jobs<FR_STORAGE_BF16>(cfg); }
}// namespace frb
