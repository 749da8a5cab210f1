// Internal interface of the grouped (batched) launch shared by the batch
// plans and the serving engine. Not part of the public ABI.
#pragma once

#include <vector>

#include "skg_fp64_types.h"
#include "skg_runtime.h"

namespace skg {

struct GroupTables {
  std::vector<Fp64Params> params;
  std::vector<CUtensorMap> maps;
  std::vector<int64_t> iter_begin;
  double useful = 0.0, issued = 0.0;  // MACs
};

// Problems with work in `order` (1 as given, 2 most work first), their TMA
// descriptors for `tile` x `tile` output tiles and the iteration prefix.
int build_group_tables(const std::vector<Fp64Problem>& probs, int tile, int order,
                       GroupTables* T);
// Cost-model tile shape (128 or 64) for a set of problems.
int model_tile(const std::vector<Fp64Problem>& probs);
// Cost-model device time (s) of `p` on the FP64 Stream-K kernels (issued
// MACs at the sustained DMMA rate); compared with ozaki_time_estimate to
// resolve SKGEMM_PREC_AUTO.
double batch_native_estimate(const Fp64Problem& p);

// A ring of `depth` grouped-launch workspaces for a stream of batches.
struct GroupRing;
GroupRing* group_ring_create(DeviceState* dev, int depth);
void group_ring_destroy(GroupRing* R);
// Grows every slot for up to `max_problems` problems and the largest grid.
int group_ring_reserve(GroupRing* R, int max_problems);
// Enqueues one grouped launch of `probs` (K == 0 problems included) on `s`.
int group_ring_submit(GroupRing* R, const std::vector<Fp64Problem>& probs, cudaStream_t s,
                      int* tile_out);
// Reads and clears the slots' error words (call after synchronising).
int group_ring_error(GroupRing* R);

}  // namespace skg
