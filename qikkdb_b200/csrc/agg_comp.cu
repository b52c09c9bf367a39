// Aggregation pass instantiations for composite (int32, int32) keys.
#include "groupby_agg.cuh"

namespace qdb {
int32_t launch_agg_comp(const AggArgs& a, ValKind vk, int32_t ptype, bool nulls, size_t smem, cudaStream_t st) {
    return launch_agg_k<int32_t, true>(a, vk, ptype, nulls, smem, st);
}
}  // namespace qdb
