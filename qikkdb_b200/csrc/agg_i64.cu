// Aggregation pass instantiations for int64_t keys.
#include "groupby_agg.cuh"

namespace qdb {
int32_t launch_agg_i64(const AggArgs& a, ValKind vk, int32_t ptype, bool nulls, size_t smem, cudaStream_t st) {
    return launch_agg_k<int64_t, false>(a, vk, ptype, nulls, smem, st);
}
}  // namespace qdb
