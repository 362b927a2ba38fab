// Stage kernels of the batched engine for mixed-precision members
// (batch_tile.cuh, MX = true).
#include <algorithm>
#define PIAFS_BATCH_STAGE_IMPL
#include "batch_tile.cuh"

namespace piafs {
namespace batch {
template struct StageTable<true>;
}  // namespace batch
}  // namespace piafs
