// Partial-state export and merge: the building blocks of merging GROUP BY tables held on several GPUs.
// The reference merges per-GPU tables by copying every table to host vectors (ReconstructRawNumbers,
// qikkDB/QueryEngine/GPUCore/GPUGroupBy.cuh:433-471) and re-grouping the concatenation on device 0
// (GPUGroupBy.cuh:594-790).  Here each table exports its occupied slots bucketed by the rank that owns
// the key (owner = hash(key) mod ranks), the buckets travel rank to rank (an NCCL all-to-all driven by
// the host), and each owner merges what it receives straight into its own table, so no data passes
// through host memory and no rank holds the whole key set.
#include <vector>

#include "groupby_agg.cuh"

namespace qdb {

constexpr int kExThreads = 256;

enum ExportFlag : uint8_t { EX_NULL_KEY = 1, EX_ESCAPE_KEY = 2, EX_AUX_KEY = 4 };

__device__ __forceinline__ int owner_of(const SlotSpace& sp, uint64_t v, uint64_t kw, int n_parts) {
    const uint64_t per = sp.cap + 2;
    if (v == per - 2 || v == per - 1) return 0;  // special slots live on rank 0
    return static_cast<int>(static_cast<uint32_t>(mix64(kw) >> 32) % static_cast<uint32_t>(n_parts));
}

__global__ void ex_hist_kernel(SlotSpace sp, int n_parts, unsigned long long* part_counts) {
    extern __shared__ unsigned int hist[];
    for (int i = threadIdx.x; i < n_parts; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    for (uint64_t v = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; v < sp.total;
         v += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t kw = slot_at(sp, v)[0];
        if (kw != kEmpty) atomicAdd(&hist[owner_of(sp, v, kw, n_parts)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n_parts; i += blockDim.x)
        if (hist[i]) atomicAdd(&part_counts[i], static_cast<unsigned long long>(hist[i]));
}

__global__ void ex_scatter_kernel(SlotSpace sp, int n_parts, unsigned long long* cursors, uint64_t* keys,
                                  uint64_t* state, uint8_t* flags) {
    const uint64_t per = sp.cap + 2;
    const int sw = sp.W - 1;
    for (uint64_t v = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; v < sp.total;
         v += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t* slot = slot_at(sp, v);
        const uint64_t kw = slot[0];
        if (kw == kEmpty) continue;
        const unsigned long long pos = atomicAdd(&cursors[owner_of(sp, v, kw, n_parts)], 1ull);
        uint8_t f = 0;
        if (v == per - 2) f = EX_NULL_KEY;
        else if (v == per - 1) f = EX_ESCAPE_KEY;
        else if (v >= per) f = EX_AUX_KEY;
        keys[pos] = kw;
        flags[pos] = f;
        for (int w = 0; w < sw; ++w) state[pos * sw + w] = slot[1 + w];
    }
}

__global__ void merge_partial_kernel(Region main, Region aux, Layout L, int32_t has_sum, int32_t has_min,
                                     int32_t has_max, int32_t v32, int32_t vfloat, const uint64_t* keys,
                                     const uint64_t* state, const uint8_t* flags, int64_t n,
                                     unsigned long long* counters, unsigned long long capacity) {
    const int sw = L.W - 1;
    __shared__ unsigned long long s_claims;
    if (threadIdx.x == 0) s_claims = 0;
    __syncthreads();
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const uint8_t f = flags[i];
        const uint64_t kw = keys[i];
        uint64_t* slot;
        if (f & EX_NULL_KEY) slot = g_special(main, L.W, 0, &s_claims);
        else if (f & EX_ESCAPE_KEY) slot = g_special(main, L.W, 1, &s_claims);
        else if (f & EX_AUX_KEY) slot = aux.slots ? g_find(aux, L.W, kw, mix64(kw), counters, &s_claims) : nullptr;
        else slot = g_find(main, L.W, kw, mix64(kw), counters, &s_claims);
        if (!slot || sw == 0) continue;
        const uint64_t* st = state + i * sw;
        const unsigned long long c = (L.cnt >= 0) ? st[L.cnt - 1] : 0ull;
        const uint64_t sumbits = (L.sum >= 0) ? st[L.sum - 1] : 0ull;
        long long mn = 0, mx = 0;
        if (L.packed) {
            const uint64_t w = st[L.mn - 1];
            mn = static_cast<int32_t>(w & 0xffffffffull);
            mx = static_cast<int32_t>(w >> 32);
        } else {
            if (L.mn >= 0) mn = static_cast<long long>(st[L.mn - 1]);
            if (L.mx >= 0) mx = static_cast<long long>(st[L.mx - 1]);
        }
        if (L.cnt >= 0 && !has_sum && !has_min && !has_max) {
            if (c) atomicAdd(reinterpret_cast<unsigned long long*>(slot + L.cnt), c);
        } else {
            g_merge(slot, L, has_sum, has_min, has_max, v32, vfloat, c, sumbits, mn, mx);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) publish_claims(counters, capacity, s_claims);
}

}  // namespace qdb

using namespace qdb;

extern "C" {

int32_t qdb_gb_state_words(qdb_gb* gb, int32_t* out_words) {
    if (!gb || !out_words) return fail(QDB_ERR_INVALID, "qdb_gb_state_words: null argument");
    *out_words = gb->L.W - 1;
    return QDB_OK;
}

int32_t qdb_gb_export_partitioned(qdb_gb* gb, int32_t n_parts, uint64_t** out_keys, uint64_t** out_state,
                                  uint8_t** out_flags, int64_t* part_counts, void* stream) {
    if (!gb || !out_keys || !out_state || !out_flags || !part_counts)
        return fail(QDB_ERR_INVALID, "qdb_gb_export_partitioned: null argument");
    if (n_parts < 1 || n_parts > 4096) return fail(QDB_ERR_INVALID, "qdb_gb_export_partitioned: n_parts in [1, 4096]");
    *out_keys = nullptr;
    *out_state = nullptr;
    *out_flags = nullptr;
    cudaStream_t s = as_stream(stream);
    const SlotSpace sp = slot_space(gb);
    unsigned long long* counts = nullptr;
    int32_t rc = dev_alloc(reinterpret_cast<void**>(&counts), 2 * n_parts * sizeof(unsigned long long), s);
    if (rc != QDB_OK) return rc;
    QDB_CUDA_TRY(cudaMemsetAsync(counts, 0, 2 * n_parts * sizeof(unsigned long long), s));
    const DeviceInfo& di = device_info();
    uint64_t blocks = (sp.total + kExThreads - 1) / kExThreads;
    if (blocks > static_cast<uint64_t>(di.sm_count) * 8) blocks = static_cast<uint64_t>(di.sm_count) * 8;
    ex_hist_kernel<<<static_cast<unsigned>(blocks), kExThreads, n_parts * sizeof(unsigned int), s>>>(sp, n_parts,
                                                                                                        counts);
    note_launch();
    std::vector<unsigned long long> h(n_parts);
    cudaError_t e = cudaMemcpyAsync(h.data(), counts, n_parts * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        dev_free(counts, s);
        return cuda_fail(e, "qdb_gb_export_partitioned: histogram");
    }
    std::vector<unsigned long long> offs(n_parts);
    unsigned long long total = 0;
    for (int p = 0; p < n_parts; ++p) {
        offs[p] = total;
        total += h[p];
        part_counts[p] = static_cast<int64_t>(h[p]);
    }
    if (total == 0) {
        dev_free(counts, s);
        return QDB_OK;
    }
    const int sw = gb->L.W - 1;
    rc = dev_alloc(reinterpret_cast<void**>(out_keys), total * 8, s);
    if (rc == QDB_OK && sw > 0) rc = dev_alloc(reinterpret_cast<void**>(out_state), total * sw * 8, s);
    if (rc == QDB_OK) rc = dev_alloc(reinterpret_cast<void**>(out_flags), total, s);
    if (rc != QDB_OK) {
        dev_free(*out_keys, s);
        dev_free(*out_state, s);
        dev_free(*out_flags, s);
        *out_keys = nullptr;
        *out_state = nullptr;
        *out_flags = nullptr;
        dev_free(counts, s);
        return rc;
    }
    unsigned long long* cursors = counts + n_parts;
    QDB_CUDA_TRY(cudaMemcpyAsync(cursors, offs.data(), n_parts * sizeof(unsigned long long), cudaMemcpyHostToDevice, s));
    ex_scatter_kernel<<<static_cast<unsigned>(blocks), kExThreads, 0, s>>>(sp, n_parts, cursors, *out_keys, *out_state,
                                                                          *out_flags);
    note_launch();
    e = cudaGetLastError();
    // The host copy source `offs` must stay alive until the copy has run.
    cudaError_t e2 = cudaStreamSynchronize(s);
    dev_free(counts, s);
    if (e != cudaSuccess) return cuda_fail(e, "ex_scatter_kernel");
    if (e2 != cudaSuccess) return cuda_fail(e2, "qdb_gb_export_partitioned: scatter");
    return QDB_OK;
}

int32_t qdb_gb_merge_partial(qdb_gb* gb, const uint64_t* keys, const uint64_t* state, const uint8_t* flags, int64_t n,
                             void* stream) {
    if (!gb) return fail(QDB_ERR_INVALID, "qdb_gb_merge_partial: null table");
    if (n <= 0) return QDB_OK;
    if (!keys || !flags || (gb->L.W > 1 && !state)) return fail(QDB_ERR_INVALID, "qdb_gb_merge_partial: null buffers");
    cudaStream_t s = as_stream(stream);
    if (gb->n_key_cols == 2 && !gb->aux.slots) {
        int32_t rc = gb_init_region(gb, gb->aux, s);
        if (rc != QDB_OK) return rc;
    }
    const ValKind vk = val_kind(gb->val_type);
    const DeviceInfo& di = device_info();
    int64_t blocks = (n + kExThreads - 1) / kExThreads;
    if (blocks > di.sm_count * 8) blocks = di.sm_count * 8;
    merge_partial_kernel<<<static_cast<unsigned>(blocks), kExThreads, 0, s>>>(
        gb->main, gb->aux, gb->L, gb->L.sum >= 0, (gb->aggs & QDB_AGG_MIN) && gb->L.mn >= 0,
        (gb->aggs & QDB_AGG_MAX) && gb->L.mx >= 0, vk_is_32(vk), vk == VK_F32 || vk == VK_F64, keys, state, flags, n,
        gb->counters, static_cast<unsigned long long>(gb->capacity));
    note_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "merge_partial_kernel");
    return QDB_OK;
}

}  // extern "C"
