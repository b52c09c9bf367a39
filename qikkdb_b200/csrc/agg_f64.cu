// Aggregation pass instantiations for double keys.
#include "groupby_agg.cuh"

namespace qdb {
int32_t launch_agg_f64(const AggArgs& a, ValKind vk, int32_t ptype, size_t smem, cudaStream_t st) {
    return launch_agg_k<double, false>(a, vk, ptype, smem, st);
}
}  // namespace qdb
