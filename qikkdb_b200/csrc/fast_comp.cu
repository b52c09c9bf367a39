// Fast aggregation pass instantiations for composite (int32, int32) keys.
#include "groupby_fast.cuh"

namespace qdb {
int32_t launch_fast_comp(const AggArgs& a, ValKind vk, int32_t ptype, size_t smem, cudaStream_t st) {
    return launch_fast_k<int32_t, true>(a, vk, ptype, smem, st);
}
}  // namespace qdb
