// Aggregation pass instantiations for double keys.
#include "groupby_agg.cuh"

namespace qdb {
int32_t launch_agg_f64(const AggArgs& a, ValKind vk, int32_t ptype, bool nulls, size_t smem, cudaStream_t st) {
    return launch_agg_k<double, false>(a, vk, ptype, nulls, smem, st);
}
}  // namespace qdb
