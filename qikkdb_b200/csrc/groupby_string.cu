// GROUP BY over string keys: the replacement of GPUGroupBy<AGG, O, std::string, V>
// (qikkDB/QueryEngine/GPUCore/GPUGroupByString.cuh:39-169 and the class after it), whose kernel claims a slot by
// the row index of the string's first occurrence and re-reads input blocks to compare keys.
//
// Here a table owns its keys.  Input keys come in the reference's GPUString layout (all characters concatenated,
// and int64 end offsets: string i is chars[i ? ends[i - 1] : 0, ends[i])).  A row hashes its string (64-bit, our own
// word-at-a-time mixer) and probes linearly from the hash's home slot:
//   * an empty slot is claimed with a CAS of the hash into its header; the claimer copies the string into the
//     table's key arena (a bump allocator in device memory), writes its offset, and then publishes its length;
//   * a slot holding the same hash is compared byte for byte with the arena copy once its length is published
//     (a bounded wait: a claimer that never publishes ends the wait with QDB_ERR_TIMEOUT);
//   * the row's value then updates the slot's state words with global atomics: count, sum (two's complement or FP64),
//     min and max (order-preserving encodings), as the numeric table does.
// NULL keys form one group in a slot after the hashed ones.  New groups are counted per CTA and published once;
// more than max_groups distinct keys (or a full key arena) raise QDB_HASH_TABLE_FULL, as ProcessBlock does.
// Results compact the occupied slots into a GPUString of keys and one column per aggregate.
#include <climits>
#include <limits>
#include <vector>

#include "groupby_agg.cuh"

namespace qdb {

constexpr int kGbsThreads = 256;
constexpr uint64_t kLenPoison = ~0ull;      // a claimer that could not store its key
constexpr uint32_t kGbsWaitIters = 1u << 20; // bounded wait for a claimer to publish its key

struct GbsTable {
    uint64_t* header = nullptr;   // [cap + 1] 0: empty; else the key's hash (never 0); slot cap: the NULL key
    uint64_t* off = nullptr;      // [cap + 1] arena offset of the key
    uint64_t* len = nullptr;      // [cap + 1] 0: not published; else length + 1 (kLenPoison: no key stored)
    uint64_t* state = nullptr;    // [(cap + 1) * 4] count, sum bits, min enc, max enc
    char* arena = nullptr;
    uint64_t arena_bytes = 0;
    unsigned long long* arena_used = nullptr;
    unsigned long long* counters = nullptr;  // [0] groups, [1] status
    uint64_t cap = 0;             // hashed slots (power of two)
    unsigned long long capacity = 0;
};

__device__ __forceinline__ uint64_t gbs_hash(const char* s, int64_t n) {
    uint64_t h = 0x243F6A8885A308D3ull ^ static_cast<uint64_t>(n);
    int64_t i = 0;
    for (; i + 8 <= n; i += 8) {
        uint64_t w = 0;
#pragma unroll
        for (int b = 0; b < 8; ++b) w |= static_cast<uint64_t>(static_cast<unsigned char>(s[i + b])) << (8 * b);
        h = (h ^ (w * 0x9E3779B97F4A7C15ull)) * 0xBF58476D1CE4E5B9ull;
        h ^= h >> 29;
    }
    uint64_t w = 0;
    for (int b = 0; i + b < n; ++b) w |= static_cast<uint64_t>(static_cast<unsigned char>(s[i + b])) << (8 * b);
    h = (h ^ (w * 0x9E3779B97F4A7C15ull)) * 0xBF58476D1CE4E5B9ull;
    h = mix64(h);
    return h ? h : 1ull;
}

template <typename VT>
__device__ __forceinline__ void gbs_update(uint64_t* st, VT v) {
    atomicAdd(reinterpret_cast<unsigned long long*>(st), 1ull);
    if constexpr (std::is_floating_point<VT>::value) {
        atomicAdd(reinterpret_cast<double*>(st + 1), static_cast<double>(v));
        const long long e = std::is_same<VT, float>::value ? static_cast<long long>(fenc(static_cast<float>(v)))
                                                           : static_cast<long long>(denc(static_cast<double>(v)));
        atomicMin(reinterpret_cast<long long*>(st + 2), e);
        atomicMax(reinterpret_cast<long long*>(st + 3), e);
    } else {
        atomicAdd(reinterpret_cast<unsigned long long*>(st + 1), static_cast<unsigned long long>(static_cast<long long>(v)));
        atomicMin(reinterpret_cast<long long*>(st + 2), static_cast<long long>(v));
        atomicMax(reinterpret_cast<long long*>(st + 3), static_cast<long long>(v));
    }
}

// Finds or claims string (s, n) with hash h; returns its slot or -1 (table full, or a wait that gave up).
__device__ int64_t gbs_find(const GbsTable& t, const char* s, int64_t n, uint64_t h, unsigned* claims) {
    const uint64_t mask = t.cap - 1;
    uint64_t pos = __umul64hi(h, t.cap);
    for (uint64_t probe = 0; probe < t.cap; ++probe, pos = (pos + 1) & mask) {
        uint64_t cur = ld_volatile_u64(t.header + pos);
        if (cur == 0) {
            cur = atomicCAS(reinterpret_cast<unsigned long long*>(t.header + pos), 0ull, h);
            if (cur == 0) {  // claimed: store the key, then publish its length
                atomicAdd(claims, 1u);
                const unsigned long long o = atomicAdd(t.arena_used, static_cast<unsigned long long>(n));
                if (o + n > t.arena_bytes) {
                    atomicExch(reinterpret_cast<int*>(&t.counters[1]), static_cast<int>(QDB_HASH_TABLE_FULL));
                    atomicExch(reinterpret_cast<unsigned long long*>(t.len + pos), kLenPoison);
                    return -1;
                }
                for (int64_t b = 0; b < n; ++b) t.arena[o + b] = s[b];
                t.off[pos] = o;
                __threadfence();
                atomicExch(reinterpret_cast<unsigned long long*>(t.len + pos), static_cast<unsigned long long>(n) + 1ull);
                return static_cast<int64_t>(pos);
            }
        }
        if (cur != h) continue;
        // Same hash: wait for the key to be published, then compare it byte for byte.
        uint64_t l = ld_volatile_u64(t.len + pos);
        for (uint32_t it = 0; l == 0 && it < kGbsWaitIters; ++it) {
            __nanosleep(64);
            l = ld_volatile_u64(t.len + pos);
        }
        if (l == 0) {
            atomicExch(reinterpret_cast<int*>(&t.counters[1]), static_cast<int>(QDB_ERR_TIMEOUT));
            return -1;
        }
        if (l == kLenPoison || l != static_cast<uint64_t>(n) + 1ull) continue;
        __threadfence();
        // The arena is read around L1 (__ldcg): a line cached there for an earlier key can hold bytes of this key
        // from before they were written.
        const char* k = t.arena + ld_volatile_u64(t.off + pos);
        bool eq = true;
        for (int64_t b = 0; b < n && eq; ++b) eq = __ldcg(k + b) == s[b];
        if (eq) return static_cast<int64_t>(pos);
    }
    atomicExch(reinterpret_cast<int*>(&t.counters[1]), static_cast<int>(QDB_HASH_TABLE_FULL));
    return -1;
}

template <typename VT>
__global__ void __launch_bounds__(kGbsThreads) gbs_kernel(GbsTable t, const char* __restrict__ chars,
                                                          const int64_t* __restrict__ ends,
                                                          const uint64_t* __restrict__ knull, const VT* __restrict__ vals,
                                                          const uint64_t* __restrict__ vnull,
                                                          const int8_t* __restrict__ mask, int64_t n) {
    __shared__ unsigned s_claims;
    if (threadIdx.x == 0) s_claims = 0;
    __syncthreads();
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        if (mask && mask[i] == 0) continue;
        int64_t slot;
        if (knull && ((knull[i >> 6] >> (i & 63)) & 1ull)) {
            slot = static_cast<int64_t>(t.cap);
            if (ld_volatile_u64(t.header + slot) == 0)  // the NULL group is outside max_groups (keyBufferSize_ + 1)
                atomicCAS(reinterpret_cast<unsigned long long*>(t.header + slot), 0ull, 1ull);
        } else {
            const int64_t b = i ? ends[i - 1] : 0;
            const int64_t e = ends[i];
            const char* s = chars + b;
            slot = gbs_find(t, s, e - b, gbs_hash(s, e - b), &s_claims);
        }
        if (slot < 0) continue;
        if (!vals) atomicAdd(reinterpret_cast<unsigned long long*>(t.state + slot * 4), 1ull);  // COUNT of rows
        else if (!(vnull && ((vnull[i >> 6] >> (i & 63)) & 1ull))) gbs_update<VT>(t.state + slot * 4, vals[i]);
    }
    __syncthreads();
    if (threadIdx.x == 0 && s_claims) {
        if (atomicAdd(&t.counters[0], static_cast<unsigned long long>(s_claims)) + s_claims > t.capacity)
            atomicExch(reinterpret_cast<int*>(&t.counters[1]), static_cast<int>(QDB_HASH_TABLE_FULL));
    }
}

__global__ void gbs_init_kernel(GbsTable t) {
    for (uint64_t s = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; s <= t.cap;
         s += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        t.header[s] = 0;
        t.len[s] = 0;
        t.off[s] = 0;
        t.state[s * 4 + 0] = 0;
        t.state[s * 4 + 1] = 0;
        t.state[s * 4 + 2] = static_cast<uint64_t>(LLONG_MAX);
        t.state[s * 4 + 3] = static_cast<uint64_t>(LLONG_MIN);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *t.arena_used = 0;
        t.counters[0] = 0;
        t.counters[1] = 0;
    }
}

// Occupied slots and their key lengths, per slot: flag[s] (then its output row) and clen[s] (then its first char).
__global__ void gbs_occ_kernel(GbsTable t, long long* flag, long long* clen) {
    for (uint64_t s = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; s <= t.cap;
         s += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t l = t.len[s];
        const bool used = t.header[s] != 0 && (s == t.cap || (l != 0 && l != kLenPoison));
        flag[s] = used ? 1 : 0;
        clen[s] = (used && s != t.cap) ? static_cast<long long>(l - 1) : 0;
    }
}

// Exclusive scan of m int64 values in place by one block (chunks per thread, then the chunk sums).
__global__ void __launch_bounds__(1024) gbs_scan_kernel(long long* v, int64_t m, long long* total) {
    __shared__ long long part[1024];
    const int64_t per = (m + 1023) / 1024;
    const int64_t b = threadIdx.x * per;
    const int64_t e = min(m, b + per);
    long long sum = 0;
    for (int64_t i = b; i < e; ++i) sum += v[i];
    part[threadIdx.x] = sum;
    __syncthreads();
    for (int d = 1; d < 1024; d <<= 1) {
        const long long y = threadIdx.x >= d ? part[threadIdx.x - d] : 0;
        __syncthreads();
        part[threadIdx.x] += y;
        __syncthreads();
    }
    long long run = part[threadIdx.x] - sum;
    for (int64_t i = b; i < e; ++i) {
        const long long c = v[i];
        v[i] = run;
        run += c;
    }
    if (threadIdx.x == 1023) *total = part[1023];
}

// Finalises one aggregate of a slot into V.  A group without a non-NULL value gets the placeholders of the
// numeric operator: MIN max(V), MAX lowest(V), SUM 0, AVG NaN (floats) or min(V) (integers).
template <typename V>
__device__ V gbs_final(const uint64_t* st, int32_t agg) {
    const unsigned long long cnt = st[0];
    if (cnt == 0) {
        switch (agg) {
            case QDB_AGG_MIN: return std::numeric_limits<V>::max();
            case QDB_AGG_MAX: return std::numeric_limits<V>::lowest();
            case QDB_AGG_SUM: return V{0};
            default:
                if constexpr (std::is_floating_point<V>::value) return std::numeric_limits<V>::quiet_NaN();
                else return std::numeric_limits<V>::min();
        }
    }
    if (agg == QDB_AGG_MIN || agg == QDB_AGG_MAX) {
        const long long e = static_cast<long long>(st[agg == QDB_AGG_MIN ? 2 : 3]);
        if constexpr (std::is_same<V, float>::value) return fdec(static_cast<int32_t>(e));
        else if constexpr (std::is_same<V, double>::value) return ddec(e);
        else return static_cast<V>(e);
    }
    if constexpr (std::is_floating_point<V>::value) {
        double sum;
        memcpy(&sum, st + 1, 8);
        return static_cast<V>(agg == QDB_AGG_SUM ? sum : sum / static_cast<double>(cnt));
    } else {
        // the sum wraps in V; AVG divides the wrapped sum by the count, truncated
        const V wrapped = static_cast<V>(static_cast<long long>(st[1]));
        return agg == QDB_AGG_SUM ? wrapped : static_cast<V>(static_cast<long long>(wrapped) / static_cast<long long>(cnt));
    }
}

// One output row per occupied slot: key characters and end offset, key NULL bit, and every aggregate.
template <typename V>
__global__ void gbs_emit_kernel(GbsTable t, const long long* pos, const long long* cpos, const int32_t* aggs,
                                int32_t n_aggs, char* out_chars, int64_t* out_ends, unsigned long long* key_nulls,
                                void* const* out_vals, unsigned long long* const* val_nulls) {
    for (uint64_t s = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; s <= t.cap;
         s += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t l = t.len[s];
        const bool used = t.header[s] != 0 && (s == t.cap || (l != 0 && l != kLenPoison));
        if (!used) continue;
        const long long r = pos[s];
        const long long c0 = cpos[s];
        const long long n = s == t.cap ? 0 : static_cast<long long>(l - 1);
        const char* k = t.arena + t.off[s];
        for (long long b = 0; b < n; ++b) out_chars[c0 + b] = k[b];
        out_ends[r] = c0 + n;
        if (s == t.cap) atomicOr(key_nulls + (r >> 6), 1ull << (r & 63));
        const uint64_t* st = t.state + s * 4;
        for (int j = 0; j < n_aggs; ++j) {
            const int32_t a = aggs[j];
            if (a == QDB_AGG_COUNT) {
                static_cast<int64_t*>(out_vals[j])[r] = static_cast<int64_t>(st[0]);
                continue;
            }
            if (st[0] == 0 && val_nulls[j]) atomicOr(val_nulls[j] + (r >> 6), 1ull << (r & 63));
            static_cast<V*>(out_vals[j])[r] = gbs_final<V>(st, a);
        }
    }
}

static uint64_t gbs_pow2(uint64_t x) {
    uint64_t p = 16;
    while (p < x) p <<= 1;
    return p;
}

static int32_t gbs_zero(void* p, size_t bytes, cudaStream_t s) {
    const cudaError_t e = cudaMemsetAsync(p, 0, bytes, s);
    return e == cudaSuccess ? QDB_OK : cuda_fail(e, "cudaMemsetAsync");
}

static unsigned gbs_grid(uint64_t n) {
    const DeviceInfo& di = device_info();
    return static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, uint64_t(di.sm_count) * 16)));
}

}  // namespace qdb

struct qdb_gbs {
    int32_t aggs = 0;
    int32_t val_type = 0;
    int device = 0;
    int64_t max_groups = 0;
    qdb::GbsTable t;
};

using namespace qdb;

extern "C" {

int32_t qdb_gbs_create(qdb_gbs** out, int32_t agg_mask, int32_t val_type, int64_t max_groups, int64_t max_key_bytes,
                       void* stream) {
    if (!out) return fail(QDB_ERR_INVALID, "qdb_gbs_create: null out");
    *out = nullptr;
    if (agg_mask & ~(QDB_AGG_MIN | QDB_AGG_MAX | QDB_AGG_SUM | QDB_AGG_AVG | QDB_AGG_COUNT))
        return fail(QDB_UNKNOWN_AGG_FUN, "qdb_gbs_create: unknown aggregate bits");
    const bool vt_ok = val_type == QDB_INT32 || val_type == QDB_INT64 || val_type == QDB_FLOAT || val_type == QDB_DOUBLE;
    if ((val_type != 0 && !vt_ok) || ((agg_mask & ~QDB_AGG_COUNT) && !vt_ok))
        return fail(QDB_ERR_INVALID, "qdb_gbs_create: value type must be INT32, INT64, FLOAT or DOUBLE (0: COUNT of rows)");
    if (max_groups < 1) return fail(QDB_ERR_INVALID, "qdb_gbs_create: max_groups must be positive");
    max_groups = std::min<int64_t>(max_groups, int64_t(1) << 30);
    qdb_gbs* g = new qdb_gbs();
    g->aggs = agg_mask;
    g->val_type = val_type;
    g->max_groups = max_groups;
    cudaGetDevice(&g->device);
    GbsTable& t = g->t;
    t.cap = gbs_pow2(static_cast<uint64_t>(max_groups) + static_cast<uint64_t>(max_groups) / 2);
    t.capacity = static_cast<unsigned long long>(max_groups);
    t.arena_bytes = max_key_bytes > 0 ? static_cast<uint64_t>(max_key_bytes) : static_cast<uint64_t>(max_groups) * 32;
    cudaStream_t s = as_stream(stream);
    const uint64_t slots = t.cap + 1;
    int32_t rc = dev_alloc(reinterpret_cast<void**>(&t.header), slots * 8, s);
    if (rc == QDB_OK) rc = dev_alloc(reinterpret_cast<void**>(&t.off), slots * 8, s);
    if (rc == QDB_OK) rc = dev_alloc(reinterpret_cast<void**>(&t.len), slots * 8, s);
    if (rc == QDB_OK) rc = dev_alloc(reinterpret_cast<void**>(&t.state), slots * 32, s);
    if (rc == QDB_OK) rc = dev_alloc(reinterpret_cast<void**>(&t.arena), std::max<uint64_t>(t.arena_bytes, 8), s);
    if (rc == QDB_OK) rc = dev_alloc(reinterpret_cast<void**>(&t.arena_used), 8, s);
    if (rc == QDB_OK) rc = dev_alloc(reinterpret_cast<void**>(&t.counters), 16, s);
    if (rc == QDB_OK) rc = qdb_gbs_reset(g, stream);
    if (rc != QDB_OK) {
        qdb_gbs_destroy(g);
        return rc;
    }
    *out = g;
    return QDB_OK;
}

int32_t qdb_gbs_destroy(qdb_gbs* g) {
    if (!g) return QDB_OK;
    GbsTable& t = g->t;
    for (void* p : {static_cast<void*>(t.header), static_cast<void*>(t.off), static_cast<void*>(t.len),
                    static_cast<void*>(t.state), static_cast<void*>(t.arena), static_cast<void*>(t.arena_used),
                    static_cast<void*>(t.counters)})
        if (p) dev_free(p, nullptr);
    cudaStreamSynchronize(nullptr);
    delete g;
    return QDB_OK;
}

int32_t qdb_gbs_reset(qdb_gbs* g, void* stream) {
    if (!g) return fail(QDB_ERR_INVALID, "qdb_gbs_reset: null table");
    gbs_init_kernel<<<gbs_grid(g->t.cap + 1), 256, 0, as_stream(stream)>>>(g->t);
    note_launch();
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? QDB_OK : cuda_fail(e, "gbs_init_kernel");
}

int32_t qdb_gbs_process(qdb_gbs* g, const char* chars, const int64_t* ends, const uint64_t* key_nulls, const void* vals,
                        const uint64_t* val_nulls, const int8_t* mask, int64_t n, void* stream) {
    if (!g || n < 0) return fail(QDB_ERR_INVALID, "qdb_gbs_process: bad arguments");
    if (n == 0) return QDB_OK;
    // Without a value column a COUNT-only table counts rows (COUNT of the key column).
    if (!ends || (g->val_type && !vals && g->aggs != QDB_AGG_COUNT))
        return fail(QDB_ERR_INVALID, "qdb_gbs_process: null keys or values");
    cudaStream_t s = as_stream(stream);
    const unsigned grid = gbs_grid(static_cast<uint64_t>(n));
    const void* v = g->val_type ? vals : nullptr;
    const uint64_t* vn = g->val_type ? val_nulls : nullptr;
    switch (g->val_type) {
        case QDB_INT64: gbs_kernel<int64_t><<<grid, kGbsThreads, 0, s>>>(g->t, chars, ends, key_nulls, static_cast<const int64_t*>(v), vn, mask, n); break;
        case QDB_FLOAT: gbs_kernel<float><<<grid, kGbsThreads, 0, s>>>(g->t, chars, ends, key_nulls, static_cast<const float*>(v), vn, mask, n); break;
        case QDB_DOUBLE: gbs_kernel<double><<<grid, kGbsThreads, 0, s>>>(g->t, chars, ends, key_nulls, static_cast<const double*>(v), vn, mask, n); break;
        default: gbs_kernel<int32_t><<<grid, kGbsThreads, 0, s>>>(g->t, chars, ends, key_nulls, static_cast<const int32_t*>(v), vn, mask, n); break;
    }
    note_launch();
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? QDB_OK : cuda_fail(e, "gbs_kernel");
}

int32_t qdb_gbs_check(qdb_gbs* g, void* stream) {
    if (!g) return fail(QDB_ERR_INVALID, "qdb_gbs_check: null table");
    unsigned long long st = 0;
    QDB_CUDA_TRY(cudaMemcpyAsync(&st, g->t.counters + 1, 8, cudaMemcpyDeviceToHost, as_stream(stream)));
    QDB_CUDA_TRY(cudaStreamSynchronize(as_stream(stream)));
    const int32_t status = static_cast<int32_t>(st & 0xffffffffu);
    if (status == QDB_OK) return QDB_OK;
    QDB_CUDA_TRY(cudaMemsetAsync(g->t.counters + 1, 0, 8, as_stream(stream)));
    return fail(status, status == QDB_HASH_TABLE_FULL ? "string GROUP BY: more distinct keys than the table (or its key "
                                                        "arena) holds"
                                                      : "string GROUP BY: a wait for a key gave up");
}

int32_t qdb_gbs_results(qdb_gbs* g, int32_t n_aggs, const int32_t* aggs, char** out_chars, int64_t** out_ends,
                        uint64_t** out_key_nulls, void** out_vals, uint64_t** out_val_nulls, int64_t* out_count,
                        void* stream) {
    if (!g || !out_chars || !out_ends || !out_count || n_aggs < 0 || n_aggs > 5 || (n_aggs && (!aggs || !out_vals)))
        return fail(QDB_ERR_INVALID, "qdb_gbs_results: bad arguments");
    *out_chars = nullptr;
    *out_ends = nullptr;
    *out_count = 0;
    if (out_key_nulls) *out_key_nulls = nullptr;
    for (int j = 0; j < n_aggs; ++j) {
        out_vals[j] = nullptr;
        if (out_val_nulls) out_val_nulls[j] = nullptr;
        if (aggs[j] != QDB_AGG_COUNT && !(g->aggs & aggs[j])) return fail(QDB_ERR_INVALID, "qdb_gbs_results: aggregate not in the table");
    }
    cudaStream_t s = as_stream(stream);
    const GbsTable& t = g->t;
    const uint64_t slots = t.cap + 1;
    long long *flag = nullptr, *clen = nullptr, *tot = nullptr;
    int32_t rc = dev_alloc(reinterpret_cast<void**>(&flag), slots * 8, s);
    if (rc == QDB_OK) rc = dev_alloc(reinterpret_cast<void**>(&clen), slots * 8, s);
    if (rc == QDB_OK) rc = dev_alloc(reinterpret_cast<void**>(&tot), 16, s);
    long long h_tot[2] = {0, 0};
    if (rc == QDB_OK) {
        gbs_occ_kernel<<<gbs_grid(slots), 256, 0, s>>>(t, flag, clen);
        gbs_scan_kernel<<<1, 1024, 0, s>>>(flag, static_cast<int64_t>(slots), tot);
        gbs_scan_kernel<<<1, 1024, 0, s>>>(clen, static_cast<int64_t>(slots), tot + 1);
        note_launch();
        note_launch();
        note_launch();
        cudaError_t e = cudaMemcpyAsync(h_tot, tot, 16, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = cuda_fail(e, "qdb_gbs_results: count");
    }
    const int64_t groups = h_tot[0], nchars = h_tot[1];
    const size_t words = static_cast<size_t>((groups + 63) / 64);
    std::vector<void*> vals(5, nullptr);
    std::vector<unsigned long long*> vnulls(5, nullptr);
    unsigned long long* knull = nullptr;
    if (rc == QDB_OK && groups > 0) {
        rc = dev_alloc(reinterpret_cast<void**>(out_chars), static_cast<size_t>(std::max<int64_t>(nchars, 1)), s);
        if (rc == QDB_OK) rc = dev_alloc(reinterpret_cast<void**>(out_ends), static_cast<size_t>(groups) * 8, s);
        if (rc == QDB_OK) rc = dev_alloc(reinterpret_cast<void**>(&knull), words * 8, s);
        for (int j = 0; j < n_aggs && rc == QDB_OK; ++j) {
            const size_t w = aggs[j] == QDB_AGG_COUNT ? 8 : static_cast<size_t>(type_size(g->val_type));
            rc = dev_alloc(&vals[j], static_cast<size_t>(groups) * w, s);
            if (rc == QDB_OK) rc = dev_alloc(reinterpret_cast<void**>(&vnulls[j]), words * 8, s);
            if (rc == QDB_OK) rc = gbs_zero(vnulls[j], words * 8, s);
        }
        if (rc == QDB_OK) rc = gbs_zero(knull, words * 8, s);
        int32_t* daggs = nullptr;
        void** dvals = nullptr;
        unsigned long long** dvn = nullptr;
        if (rc == QDB_OK) rc = dev_alloc(reinterpret_cast<void**>(&daggs), 5 * 4, s);
        if (rc == QDB_OK) rc = dev_alloc(reinterpret_cast<void**>(&dvals), 5 * 8, s);
        if (rc == QDB_OK) rc = dev_alloc(reinterpret_cast<void**>(&dvn), 5 * 8, s);
        if (rc == QDB_OK) {
            int32_t ha[5] = {0, 0, 0, 0, 0};
            for (int j = 0; j < n_aggs; ++j) ha[j] = aggs[j];
            cudaError_t e = cudaMemcpyAsync(daggs, ha, sizeof(ha), cudaMemcpyHostToDevice, s);
            if (e == cudaSuccess) e = cudaMemcpyAsync(dvals, vals.data(), 5 * 8, cudaMemcpyHostToDevice, s);
            if (e == cudaSuccess) e = cudaMemcpyAsync(dvn, vnulls.data(), 5 * 8, cudaMemcpyHostToDevice, s);
            if (e == cudaSuccess) {
                const unsigned grid = gbs_grid(slots);
                switch (g->val_type) {
                    case QDB_INT64: gbs_emit_kernel<int64_t><<<grid, 256, 0, s>>>(t, flag, clen, daggs, n_aggs, *out_chars, *out_ends, knull, dvals, dvn); break;
                    case QDB_FLOAT: gbs_emit_kernel<float><<<grid, 256, 0, s>>>(t, flag, clen, daggs, n_aggs, *out_chars, *out_ends, knull, dvals, dvn); break;
                    case QDB_DOUBLE: gbs_emit_kernel<double><<<grid, 256, 0, s>>>(t, flag, clen, daggs, n_aggs, *out_chars, *out_ends, knull, dvals, dvn); break;
                    default: gbs_emit_kernel<int32_t><<<grid, 256, 0, s>>>(t, flag, clen, daggs, n_aggs, *out_chars, *out_ends, knull, dvals, dvn); break;
                }
                note_launch();
                e = cudaGetLastError();
            }
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // the host arrays copied above live on this frame
            if (e != cudaSuccess) rc = cuda_fail(e, "gbs_emit_kernel");
        }
        dev_free(daggs, s);
        dev_free(dvals, s);
        dev_free(dvn, s);
    }
    dev_free(flag, s);
    dev_free(clen, s);
    dev_free(tot, s);
    if (rc != QDB_OK) {
        dev_free(*out_chars, s);
        dev_free(*out_ends, s);
        dev_free(knull, s);
        for (int j = 0; j < 5; ++j) {
            dev_free(vals[j], s);
            dev_free(vnulls[j], s);
        }
        *out_chars = nullptr;
        *out_ends = nullptr;
        return rc;
    }
    *out_count = groups;
    if (out_key_nulls) *out_key_nulls = reinterpret_cast<uint64_t*>(knull);
    else dev_free(knull, s);
    for (int j = 0; j < n_aggs; ++j) {
        out_vals[j] = vals[j];
        if (out_val_nulls) out_val_nulls[j] = reinterpret_cast<uint64_t*>(vnulls[j]);
        else dev_free(vnulls[j], s);
    }
    return QDB_OK;
}

}  // extern "C"
