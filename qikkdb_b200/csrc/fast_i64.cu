// Fast aggregation pass instantiations for int64_t keys.
#include "groupby_fast.cuh"

namespace qdb {
int32_t launch_fast_i64(const AggArgs& a, ValKind vk, int32_t ptype, size_t smem, cudaStream_t st) {
    return launch_fast_k<int64_t, false>(a, vk, ptype, smem, st);
}
}  // namespace qdb
