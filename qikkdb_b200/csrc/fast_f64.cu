// Fast aggregation pass instantiations for double keys.
#include "groupby_fast.cuh"

namespace qdb {
int32_t launch_fast_f64(const AggArgs& a, ValKind vk, int32_t ptype, size_t smem, cudaStream_t st) {
    return launch_fast_k<double, false>(a, vk, ptype, smem, st);
}
}  // namespace qdb
