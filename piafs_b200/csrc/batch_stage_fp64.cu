// Stage kernels of the batched engine for FP64 members (batch_tile.cuh).
#include <algorithm>
#define PIAFS_BATCH_STAGE_IMPL
#include "batch_tile.cuh"

namespace piafs {
namespace batch {
template struct StageTable<false>;
}  // namespace batch
}  // namespace piafs
