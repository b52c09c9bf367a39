// Result extraction of a GROUP BY table: the GetResults pass (qikkDB/QueryEngine/GPUCore/GPUGroupBy.cuh:478-587,
// GPUGroupByMultiKey.cuh:742-912).  The reference builds an occupancy mask, compacts keys with a CUB scan,
// folds 256 value replicas per slot, divides for AVG and compacts again.  Here the table has no replicas, so
// the pass is: count occupied slots per 4096-slot chunk, scan the chunk counts, and emit every output column
// (keys, key null bits, each requested aggregate with its null bits) in one kernel that finalises AVG and the
// NULL conventions on the fly.  Output order is slot order, like the reference's.
#include <limits>
#include <vector>

#include "groupby.cuh"

namespace qdb {

constexpr int kResThreads = 256;
constexpr int kResPerThread = 16;
constexpr int kResChunk = kResThreads * kResPerThread;

// Block-wide exclusive scan of one int per thread (kResThreads threads).
__device__ __forceinline__ int block_excl_scan(int x, int* total) {
    __shared__ int warp_sums[kResThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) warp_sums[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        int w = (lane < kResThreads / 32) ? warp_sums[lane] : 0;
        int wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += y;
        }
        if (lane < kResThreads / 32) warp_sums[lane] = wi - w;
        if (lane == 31) *total = wi;
    }
    __syncthreads();
    const int excl = warp_sums[wid] + inc - x;
    __syncthreads();
    return excl;
}

// A chunk's slots are walked warp by warp: warp w of the block takes the kResWarpSlots consecutive slots from
// chunk start + w kResWarpSlots, 32 at a time (one slot per lane), so every load of the key words is coalesced.
constexpr int kResWarpSlots = kResChunk / (kResThreads / 32);

__global__ void res_count_kernel(SlotSpace sp, int* chunk_counts) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint64_t wbase = static_cast<uint64_t>(blockIdx.x) * kResChunk + static_cast<uint64_t>(warp) * kResWarpSlots;
    int c = 0;
#pragma unroll 4
    for (int i = 0; i < kResWarpSlots; i += 32) c += present(sp, wbase + i + lane) ? 1 : 0;
    __shared__ int tot;
    block_excl_scan(c, &tot);
    if (threadIdx.x == 0) chunk_counts[blockIdx.x] = tot;
}

// Exclusive scan of the chunk counts in one block; total written to counts[nchunks].
__global__ void res_scan_kernel(int* counts, int64_t nchunks, long long* total_out) {
    __shared__ long long carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int64_t base = 0; base < nchunks; base += kResThreads) {
        const int64_t i = base + threadIdx.x;
        const int x = (i < nchunks) ? counts[i] : 0;
        int tot;
        __shared__ int tot_s;
        const int excl = block_excl_scan(x, &tot_s);
        tot = tot_s;
        if (i < nchunks) counts[i] = static_cast<int>(carry + excl);
        __syncthreads();
        if (threadIdx.x == 0) carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total_out = carry;
}

struct OutAgg {
    int32_t agg = 0;
    void* vals = nullptr;
    unsigned long long* nulls = nullptr;
};

struct EmitArgs {
    SlotSpace sp;
    Layout L;
    int32_t key_type = 0;
    int32_t composite = 0;
    int32_t vk = 0;
    void* keys0 = nullptr;
    void* keys1 = nullptr;
    unsigned long long* knull0 = nullptr;
    unsigned long long* knull1 = nullptr;
    int32_t n_out = 0;
    OutAgg out[5];
    const int* chunk_offsets = nullptr;
};

__device__ __forceinline__ void set_bit(unsigned long long* m, int64_t pos) {
    if (m) atomicOr(m + (pos >> 6), 1ull << (pos & 63));
}

template <typename V>
__device__ __forceinline__ void write_val(void* out, int64_t pos, V v) {
    static_cast<V*>(out)[pos] = v;
}

// Finalises one aggregate of a slot into the output type V.  `cnt` is the non-NULL value count.
template <typename V>
__device__ void emit_agg(const EmitArgs& a, const uint64_t* slot, uint64_t cnt, const OutAgg& o, int64_t pos) {
    const bool isnull = (cnt == 0);
    V v{};
    switch (o.agg) {
        case QDB_AGG_MIN:
        case QDB_AGG_MAX: {
            const bool mn = o.agg == QDB_AGG_MIN;
            if (isnull) {
                v = mn ? std::numeric_limits<V>::max() : std::numeric_limits<V>::lowest();
            } else if (a.L.packed) {
                const uint64_t w = slot[mn ? a.L.mn : a.L.mx];
                const int32_t e = static_cast<int32_t>(mn ? (w & 0xffffffffull) : (w >> 32));
                if constexpr (std::is_same<V, float>::value) v = fdec(e);
                else v = static_cast<V>(e);
            } else {
                const int64_t e = static_cast<int64_t>(slot[mn ? a.L.mn : a.L.mx]);
                if constexpr (std::is_same<V, double>::value) v = ddec(e);
                else v = static_cast<V>(e);
            }
            break;
        }
        case QDB_AGG_SUM: {
            if (isnull) v = V{0};
            else if constexpr (std::is_floating_point<V>::value) {
                double d;
                memcpy(&d, &slot[a.L.sum], 8);
                v = static_cast<V>(d);
            } else {
                v = static_cast<V>(static_cast<int64_t>(slot[a.L.sum]));
            }
            break;
        }
        case QDB_AGG_AVG: {
            if constexpr (std::is_floating_point<V>::value) {
                if (isnull) v = std::numeric_limits<V>::quiet_NaN();
                else {
                    double d;
                    memcpy(&d, &slot[a.L.sum], 8);
                    v = static_cast<V>(d / static_cast<double>(cnt));
                }
            } else {
                // Integer AVG truncates like GPUBinary<div, O, V*, int64_t*> (ArithmeticOperations.h div).
                if (isnull) v = std::numeric_limits<V>::min();
                else {
                    const V s = static_cast<V>(static_cast<int64_t>(slot[a.L.sum]));
                    v = static_cast<V>(static_cast<int64_t>(s) / static_cast<int64_t>(cnt));
                }
            }
            break;
        }
        default: break;
    }
    write_val<V>(o.vals, pos, v);
    if (isnull) set_bit(o.nulls, pos);
}

// Writes the result row `pos` of slot v: key columns, key NULL bits and every aggregate.
__device__ void res_emit_one(const EmitArgs& a, uint64_t v, int64_t pos) {
    const uint64_t per = a.sp.cap + 2;
    const uint64_t* slot = slot_at(a.sp, v);
    const uint64_t kw = slot[0];
    // Key columns and key NULL bits.
    if (a.composite) {
        int32_t k0, k1;
        bool n0 = false, n1 = false;
        if (v >= per) {  // composite key with NULL components
            const uint32_t pat = static_cast<uint32_t>(kw >> 32);
            const int32_t other = static_cast<int32_t>(kw & 0xffffffffull);
            n0 = pat & 1u;
            n1 = pat & 2u;
            k0 = n0 ? 0 : other;
            k1 = n1 ? 0 : other;
        } else if (v == per - 1) {  // the key equal to the empty marker
            k0 = std::numeric_limits<int32_t>::min();
            k1 = 0;
        } else {
            k0 = static_cast<int32_t>(kw >> 32);
            k1 = static_cast<int32_t>(kw & 0xffffffffull);
        }
        static_cast<int32_t*>(a.keys0)[pos] = k0;
        static_cast<int32_t*>(a.keys1)[pos] = k1;
        if (n0) set_bit(a.knull0, pos);
        if (n1) set_bit(a.knull1, pos);
    } else {
        const bool is_null = (v == per - 2);
        const bool is_escape = (v == per - 1);
        switch (a.key_type) {
            case QDB_INT32:
                static_cast<int32_t*>(a.keys0)[pos] = is_null ? 0 : static_cast<int32_t>(kw);
                break;
            case QDB_INT64:
                static_cast<int64_t*>(a.keys0)[pos] =
                    is_null ? 0 : (is_escape ? std::numeric_limits<int64_t>::min() : static_cast<int64_t>(kw));
                break;
            case QDB_FLOAT: {
                const uint32_t b = is_null ? 0u : static_cast<uint32_t>(kw);
                float f;
                memcpy(&f, &b, 4);
                static_cast<float*>(a.keys0)[pos] = f;
                break;
            }
            case QDB_DOUBLE: {
                const uint64_t b = is_null ? 0ull : kw;
                double d;
                memcpy(&d, &b, 8);
                static_cast<double*>(a.keys0)[pos] = d;
                break;
            }
            default: break;
        }
        if (is_null) set_bit(a.knull0, pos);
    }
    // Aggregates.
    const uint64_t cnt = (a.L.cnt >= 0) ? slot[a.L.cnt] : 0;
    for (int k = 0; k < a.n_out; ++k) {
        const OutAgg& o = a.out[k];
        if (!o.vals) continue;
        if (o.agg == QDB_AGG_COUNT) {
            static_cast<int64_t*>(o.vals)[pos] = static_cast<int64_t>(cnt);
            continue;
        }
        switch (a.vk) {
            case VK_I32: emit_agg<int32_t>(a, slot, cnt, o, pos); break;
            case VK_I64: emit_agg<int64_t>(a, slot, cnt, o, pos); break;
            case VK_F32: emit_agg<float>(a, slot, cnt, o, pos); break;
            case VK_F64: emit_agg<double>(a, slot, cnt, o, pos); break;
            default: break;
        }
    }
}

__global__ void res_emit_kernel(EmitArgs a) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint64_t wbase = static_cast<uint64_t>(blockIdx.x) * kResChunk + static_cast<uint64_t>(warp) * kResWarpSlots;
    // the warp's present slots, then its offset in the chunk (an exclusive scan of the warp counts)
    int c = 0;
#pragma unroll 4
    for (int i = 0; i < kResWarpSlots; i += 32) c += __popc(__ballot_sync(0xffffffffu, present(a.sp, wbase + i + lane)));
    __shared__ int tot;
    int64_t pos = a.chunk_offsets[blockIdx.x] + block_excl_scan(lane == 0 ? c : 0, &tot);
    pos = __shfl_sync(0xffffffffu, pos, 0);
    const unsigned lt = (1u << lane) - 1u;
    for (int i = 0; i < kResWarpSlots; i += 32) {
        const uint64_t v = wbase + i + lane;
        const bool pr = present(a.sp, v);
        const unsigned bal = __ballot_sync(0xffffffffu, pr);
        if (pr) res_emit_one(a, v, pos + __popc(bal & lt));
        pos += __popc(bal);
    }
}

static int agg_out_size(int32_t agg, ValKind vk) {
    if (agg == QDB_AGG_COUNT) return 8;
    return (vk == VK_I32 || vk == VK_F32) ? 4 : 8;
}

}  // namespace qdb

using namespace qdb;

extern "C" {

int32_t qdb_gb_results_multi(qdb_gb* gb, int32_t n_aggs, const int32_t* aggs, void** out_keys,
                             uint64_t** out_key_nulls, void** out_vals, uint64_t** out_val_nulls, int64_t* out_count,
                             void* stream) {
    if (!gb || !out_keys || !out_count) return fail(QDB_ERR_INVALID, "qdb_gb_results: null argument");
    if (n_aggs < 0 || n_aggs > 5 || (n_aggs > 0 && (!aggs || !out_vals)))
        return fail(QDB_ERR_INVALID, "qdb_gb_results: bad aggregate list");
    const ValKind vk = val_kind(gb->val_type);
    for (int i = 0; i < n_aggs; ++i) {
        const int32_t g = aggs[i];
        if (g != QDB_AGG_MIN && g != QDB_AGG_MAX && g != QDB_AGG_SUM && g != QDB_AGG_AVG && g != QDB_AGG_COUNT)
            return fail(QDB_UNKNOWN_AGG_FUN, "qdb_gb_results: unknown aggregate");
        if (!(gb->aggs & g)) return fail(QDB_UNKNOWN_AGG_FUN, "qdb_gb_results: aggregate not carried by this table");
    }
    const int nk = gb->n_key_cols;
    for (int c = 0; c < nk; ++c) {
        out_keys[c] = nullptr;
        if (out_key_nulls) out_key_nulls[c] = nullptr;
    }
    for (int i = 0; i < n_aggs; ++i) {
        out_vals[i] = nullptr;
        if (out_val_nulls) out_val_nulls[i] = nullptr;
    }
    *out_count = 0;
    cudaStream_t s = as_stream(stream);

    const SlotSpace sp = slot_space(gb);
    const int64_t nchunks = static_cast<int64_t>((sp.total + kResChunk - 1) / kResChunk);

    int* counts = nullptr;
    long long* d_total = nullptr;
    int32_t rc = dev_alloc(reinterpret_cast<void**>(&counts), (nchunks + 1) * sizeof(int), s);
    if (rc != QDB_OK) return rc;
    rc = dev_alloc(reinterpret_cast<void**>(&d_total), sizeof(long long), s);
    if (rc != QDB_OK) {
        dev_free(counts, s);
        return rc;
    }
    res_count_kernel<<<static_cast<unsigned>(nchunks), kResThreads, 0, s>>>(sp, counts);
    note_launch();
    res_scan_kernel<<<1, kResThreads, 0, s>>>(counts, nchunks, d_total);
    note_launch();
    long long total = 0;
    cudaError_t e = cudaMemcpyAsync(&total, d_total, sizeof(total), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        dev_free(counts, s);
        dev_free(d_total, s);
        return cuda_fail(e, "qdb_gb_results: count pass");
    }
    if (total == 0) {
        dev_free(counts, s);
        dev_free(d_total, s);
        return QDB_OK;
    }
    const size_t nwords = (static_cast<size_t>(total) + 63) / 64;
    const int ksize = (gb->n_key_cols == 2) ? 4 : type_size(gb->key_type);
    std::vector<void*> allocated;
    auto alloc = [&](void** p, size_t bytes) -> int32_t {
        int32_t r = dev_alloc(p, bytes, s);
        if (r == QDB_OK) allocated.push_back(*p);
        return r;
    };
    EmitArgs ea;
    ea.sp = sp;
    ea.L = gb->L;
    ea.key_type = gb->key_type;
    ea.composite = gb->n_key_cols == 2;
    ea.vk = vk;
    ea.chunk_offsets = counts;
    ea.n_out = n_aggs;
    for (int c = 0; c < nk && rc == QDB_OK; ++c) {
        rc = alloc(&out_keys[c], static_cast<size_t>(total) * ksize);
        if (rc == QDB_OK && out_key_nulls) rc = alloc(reinterpret_cast<void**>(&out_key_nulls[c]), nwords * 8);
    }
    for (int i = 0; i < n_aggs && rc == QDB_OK; ++i) {
        rc = alloc(&out_vals[i], static_cast<size_t>(total) * agg_out_size(aggs[i], vk));
        if (rc == QDB_OK && out_val_nulls) rc = alloc(reinterpret_cast<void**>(&out_val_nulls[i]), nwords * 8);
        ea.out[i].agg = aggs[i];
        ea.out[i].vals = out_vals[i];
        ea.out[i].nulls = out_val_nulls ? reinterpret_cast<unsigned long long*>(out_val_nulls[i]) : nullptr;
    }
    if (rc != QDB_OK) {
        for (void* p : allocated) dev_free(p, s);
        for (int c = 0; c < nk; ++c) {
            out_keys[c] = nullptr;
            if (out_key_nulls) out_key_nulls[c] = nullptr;
        }
        for (int i = 0; i < n_aggs; ++i) {
            out_vals[i] = nullptr;
            if (out_val_nulls) out_val_nulls[i] = nullptr;
        }
        dev_free(counts, s);
        dev_free(d_total, s);
        return rc;
    }
    ea.keys0 = out_keys[0];
    ea.keys1 = nk == 2 ? out_keys[1] : nullptr;
    if (out_key_nulls) {
        ea.knull0 = reinterpret_cast<unsigned long long*>(out_key_nulls[0]);
        ea.knull1 = nk == 2 ? reinterpret_cast<unsigned long long*>(out_key_nulls[1]) : nullptr;
        for (int c = 0; c < nk; ++c) cudaMemsetAsync(out_key_nulls[c], 0, nwords * 8, s);
    }
    if (out_val_nulls)
        for (int i = 0; i < n_aggs; ++i) cudaMemsetAsync(out_val_nulls[i], 0, nwords * 8, s);
    res_emit_kernel<<<static_cast<unsigned>(nchunks), kResThreads, 0, s>>>(ea);
    note_launch();
    e = cudaGetLastError();
    dev_free(counts, s);
    dev_free(d_total, s);
    if (e != cudaSuccess) return cuda_fail(e, "res_emit_kernel");
    *out_count = total;
    return QDB_OK;
}

int32_t qdb_gb_results(qdb_gb* gb, int32_t agg, void** out_keys, uint64_t** out_key_nulls, void** out_vals,
                       uint64_t** out_val_nulls, int64_t* out_count, void* stream) {
    if (agg == 0) {
        if (out_vals) *out_vals = nullptr;
        if (out_val_nulls) *out_val_nulls = nullptr;
        return qdb_gb_results_multi(gb, 0, nullptr, out_keys, out_key_nulls, nullptr, nullptr, out_count, stream);
    }
    if (!out_vals) return fail(QDB_ERR_INVALID, "qdb_gb_results: null out_vals");
    return qdb_gb_results_multi(gb, 1, &agg, out_keys, out_key_nulls, out_vals, out_val_nulls, out_count, stream);
}

}  // extern "C"
