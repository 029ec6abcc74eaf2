// Batched insertion-kernel variants for FP16 projection storage (see fr_insert.cuh).
#include "fr_insert.cuh"

namespace frb {
InsertFn pick_insert_batch_fp16(const InsertConfig &cfg) { return pick_storage_jobs<FR_STORAGE_FP16>(cfg); }
}// namespace frb
