// Batched insertion-kernel variants for FP32 projection storage (see fr_insert.cuh).
#include "fr_insert.cuh"

namespace frb {
InsertFn pick_insert_batch_fp32(const InsertConfig &cfg) { return pick_storage_jobs<FR_STORAGE_FP32>(cfg); }
}// namespace frb
