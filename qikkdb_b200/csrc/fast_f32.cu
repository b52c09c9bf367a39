// Fast aggregation pass instantiations for float keys.
#include "groupby_fast.cuh"

namespace qdb {
int32_t launch_fast_f32(const AggArgs& a, ValKind vk, int32_t ptype, size_t smem, cudaStream_t st) {
    return launch_fast_k<float, false>(a, vk, ptype, smem, st);
}
}  // namespace qdb
