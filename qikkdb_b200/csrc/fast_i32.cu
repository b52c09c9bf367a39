// Fast aggregation pass instantiations for int32_t keys.
#include "groupby_fast.cuh"

namespace qdb {
int32_t launch_fast_i32(const AggArgs& a, ValKind vk, int32_t ptype, size_t smem, cudaStream_t st) {
    return launch_fast_k<int32_t, false>(a, vk, ptype, smem, st);
}
}  // namespace qdb
