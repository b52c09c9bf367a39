// Fast aggregation pass instantiations for int64_t keys grouped by key % m (the remainder taken as the keys are read).
#include "groupby_fast.cuh"

namespace qdb {
int32_t launch_fast_i64_mod(const AggArgs& a, ValKind vk, int32_t ptype, size_t smem, cudaStream_t st) {
    return launch_fast_k<int64_t, false, true>(a, vk, ptype, smem, st);
}
}  // namespace qdb
