// ORDER BY over GROUP BY results: the permutation that sorts rows by several columns (each ascending or
// descending), and the gather that applies it with OFFSET / LIMIT.  The replacement of GPUOrderBy::OrderByColumn
// and ReOrderByIdx / ReOrderNullValuesByIdx (qikkDB/QueryEngine/GPUCore/GPUOrderBy.cuh:88-195), which the
// dispatcher runs over the result columns of a GROUP BY (a CUB radix sort per column, columns from the last to the
// first).
//
// The same order is produced here with our own stable LSD radix sort: every column, from the last to the first,
// re-sorts the current permutation by that column's key, so the first column ends up most significant and equal
// rows keep their input order.  A column's key is an order-preserving unsigned encoding of its value (integers:
// the sign bit flipped; IEEE values: all bits flipped when negative, else the sign bit set), inverted for a
// descending column; a NULL row takes the encoding of lowest(T), the value the reference writes into NULL rows
// before it sorts (TransformNullValsToSmallestVal).
//
// One radix pass over 8 bits = three kernels: a per-tile digit histogram, one scan of the (digit, tile) counts in
// digit-major order, and a stable scatter in which every warp ranks its rows per digit with __match_any_sync.
#include <climits>
#include <cfloat>
#include <vector>

#include "groupby.cuh"
#include "scan.cuh"

namespace qdb {

constexpr int kObThreads = 256;                      // 8 warps
constexpr int kObItems = 8;                          // rows per thread in a tile
constexpr int kObTile = kObThreads * kObItems;       // 2048 rows per tile
constexpr int kObWarps = kObThreads / 32;

// Order-preserving unsigned encodings (ascending order of the value = ascending unsigned order).
__device__ __forceinline__ uint32_t ob_enc(int32_t v) { return static_cast<uint32_t>(v) ^ 0x80000000u; }
__device__ __forceinline__ uint64_t ob_enc(int64_t v) { return static_cast<uint64_t>(v) ^ 0x8000000000000000ull; }
__device__ __forceinline__ uint32_t ob_enc(float v) {
    const uint32_t b = __float_as_uint(v);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ uint64_t ob_enc(double v) {
    const uint64_t b = static_cast<uint64_t>(__double_as_longlong(v));
    return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}

template <typename T>
__device__ __forceinline__ T ob_lowest() {
    if constexpr (std::is_same<T, int32_t>::value) return INT_MIN;
    else if constexpr (std::is_same<T, int64_t>::value) return LLONG_MIN;
    else if constexpr (std::is_same<T, float>::value) return -FLT_MAX;
    else return -DBL_MAX;
}

// keys[i] = the (possibly inverted) encoding of col[idx[i]] (idx == nullptr: row i), NULL rows as lowest(T).
template <typename T, typename K>
__global__ void ob_keys_kernel(const T* __restrict__ col, const uint64_t* __restrict__ nulls,
                               const int32_t* __restrict__ idx, int64_t n, int32_t desc, K* __restrict__ keys,
                               int32_t* __restrict__ idx_out) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t r = idx ? idx[i] : static_cast<int32_t>(i);
        T v = col[r];
        if (nulls && ((nulls[r >> 6] >> (r & 63)) & 1ull)) v = ob_lowest<T>();
        const K k = ob_enc(v);
        keys[i] = desc ? static_cast<K>(~k) : k;
        if (!idx) idx_out[i] = r;
    }
}

// Digit counts of every tile: hist[d * tiles + t].
template <typename K>
__global__ void __launch_bounds__(kObThreads) ob_hist_kernel(const K* __restrict__ keys, int64_t n, int shift,
                                                             int32_t* __restrict__ hist, int64_t tiles) {
    __shared__ int32_t cnt[256];
    cnt[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = blockIdx.x * static_cast<int64_t>(kObTile);
#pragma unroll
    for (int j = 0; j < kObItems; ++j) {
        const int64_t i = base + j * kObThreads + threadIdx.x;
        if (i < n) atomicAdd(&cnt[static_cast<uint32_t>(keys[i] >> shift) & 0xffu], 1);
    }
    __syncthreads();
    hist[static_cast<int64_t>(threadIdx.x) * tiles + blockIdx.x] = cnt[threadIdx.x];
}

// Stable scatter of one tile: row i of the tile (in row order: warp w holds rows [256 w, 256 w + 256), step j of
// the warp rows 32 j + lane) goes to offset[d][tile] + (rows of digit d in earlier warps of the tile) + (rows of
// digit d before it in its warp).
template <typename K>
__global__ void __launch_bounds__(kObThreads) ob_scatter_kernel(const K* __restrict__ keys_in,
                                                                const int32_t* __restrict__ idx_in, int64_t n,
                                                                int shift, const int32_t* __restrict__ offs,
                                                                int64_t tiles, K* __restrict__ keys_out,
                                                                int32_t* __restrict__ idx_out) {
    __shared__ int32_t wcnt[kObWarps][256];   // per warp and digit: rows so far, then the warp's offset
    __shared__ int32_t base[256];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < kObWarps * 256; i += kObThreads) (&wcnt[0][0])[i] = 0;
    base[threadIdx.x] = offs[static_cast<int64_t>(threadIdx.x) * tiles + blockIdx.x];
    __syncthreads();
    const int64_t w0 = blockIdx.x * static_cast<int64_t>(kObTile) + warp * (kObTile / kObWarps);
    const uint32_t lt = (1u << lane) - 1u;
    K key[kObItems];
    int32_t id[kObItems];
    int32_t rank[kObItems];
    uint32_t dig[kObItems];
#pragma unroll
    for (int j = 0; j < kObItems; ++j) {
        const int64_t i = w0 + 32 * j + lane;
        const bool in = i < n;
        key[j] = in ? keys_in[i] : K(0);
        id[j] = in ? idx_in[i] : 0;
        dig[j] = in ? (static_cast<uint32_t>(key[j] >> shift) & 0xffu) : 256u;  // 256: no row
        const unsigned peers = __match_any_sync(0xffffffffu, dig[j]);
        const int32_t before = wcnt[warp][dig[j] & 0xffu];
        rank[j] = before + __popc(peers & lt);
        __syncwarp();
        if (in && (peers & lt) == 0) wcnt[warp][dig[j]] = before + __popc(peers);  // the first lane of the group
        __syncwarp();
    }
    __syncthreads();
    {  // per digit (one thread each): exclusive scan of the warps' counts
        int32_t run = 0;
        for (int w = 0; w < kObWarps; ++w) {
            const int32_t c = wcnt[w][threadIdx.x];
            wcnt[w][threadIdx.x] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kObItems; ++j) {
        if (dig[j] < 256u) {
            const int64_t pos = static_cast<int64_t>(base[dig[j]]) + wcnt[warp][dig[j]] + rank[j];
            keys_out[pos] = key[j];
            idx_out[pos] = id[j];
        }
    }
}

// out[i] = in[idx[offset + i]] for i < count.
template <typename T>
__global__ void ob_gather_kernel(const T* __restrict__ in, const int32_t* __restrict__ idx, int64_t offset,
                                 int64_t count, T* __restrict__ out) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < count;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        out[i] = in[idx[offset + i]];
}

// Null bits gathered the same way: word w of out holds the bits of rows 64 w .. 64 w + 63.
__global__ void ob_gather_nulls_kernel(const uint64_t* __restrict__ in, const int32_t* __restrict__ idx,
                                       int64_t offset, int64_t count, uint64_t* __restrict__ out) {
    for (int64_t w = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; w < (count + 63) / 64;
         w += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        uint64_t bits = 0;
        for (int b = 0; b < 64 && 64 * w + b < count; ++b) {
            const int32_t r = idx[offset + 64 * w + b];
            bits |= ((in[r >> 6] >> (r & 63)) & 1ull) << b;
        }
        out[w] = bits;
    }
}

static unsigned ob_grid(int64_t n, int threads) {
    const DeviceInfo& di = device_info();
    return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads,
                                                                        int64_t(di.sm_count) * 16)));
}

// Sorts (keys, idx) by key, stable, ping-ponging between the a and b buffers; the result ends in a.
template <typename K>
static int32_t ob_radix(K* ka, int32_t* ia, K* kb, int32_t* ib, int64_t n, int32_t* hist, cudaStream_t s) {
    const int64_t tiles = (n + kObTile - 1) / kObTile;
    for (int shift = 0; shift < static_cast<int>(8 * sizeof(K)); shift += 8) {
        ob_hist_kernel<K><<<static_cast<unsigned>(tiles), kObThreads, 0, s>>>(ka, n, shift, hist, tiles);
        note_launch();
        const int32_t rc = exclusive_scan<int32_t>(hist, 256 * tiles, nullptr, s);
        if (rc != QDB_OK) return rc;
        ob_scatter_kernel<K><<<static_cast<unsigned>(tiles), kObThreads, 0, s>>>(ka, ia, n, shift, hist, tiles, kb, ib);
        note_launch();
        std::swap(ka, kb);
        std::swap(ia, ib);
    }
    // 4 or 8 passes: an even count, so the sorted data is back in the a buffers.
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? QDB_OK : cuda_fail(e, "ORDER BY radix pass");
}

template <typename T>
static int32_t ob_column(const void* col, const uint64_t* nulls, int32_t desc, int64_t n, bool first, int32_t* idx,
                         int32_t* idx2, void* keys, void* keys2, int32_t* hist, cudaStream_t s) {
    using K = typename std::conditional<sizeof(T) == 4, uint32_t, uint64_t>::type;
    // The first column sorted (the last in the ORDER BY list) starts from the identity permutation.
    ob_keys_kernel<T, K><<<ob_grid(n, 256), 256, 0, s>>>(static_cast<const T*>(col), nulls, first ? nullptr : idx, n,
                                                         desc, static_cast<K*>(keys), idx);
    note_launch();
    return ob_radix<K>(static_cast<K*>(keys), idx, static_cast<K*>(keys2), idx2, n, hist, s);
}

}  // namespace qdb

using namespace qdb;

extern "C" {

int32_t qdb_order_by_column(int32_t type, const void* col, const uint64_t* nulls, int32_t descending, int64_t n,
                            int32_t first, int32_t* indices, void* stream) {
    if (n < 0) return fail(QDB_ERR_INVALID, "qdb_order_by_column: negative row count");
    if (n > INT32_MAX) return fail(QDB_ERR_TOO_LARGE, "qdb_order_by_column: at most 2^31 - 1 rows");
    if (type != QDB_INT32 && type != QDB_INT64 && type != QDB_FLOAT && type != QDB_DOUBLE)
        return fail(QDB_ERR_INVALID, "qdb_order_by_column: column type must be INT32, INT64, FLOAT or DOUBLE");
    if (n == 0) return QDB_OK;
    if (!col || !indices) return fail(QDB_ERR_INVALID, "qdb_order_by_column: null column or indices");
    cudaStream_t s = as_stream(stream);
    const int64_t tiles = (n + kObTile - 1) / kObTile;
    void* keys = nullptr;
    void* keys2 = nullptr;
    int32_t* idx2 = nullptr;
    int32_t* hist = nullptr;
    int32_t rc = dev_alloc(&keys, static_cast<size_t>(n) * 8, s);
    if (rc == QDB_OK) rc = dev_alloc(&keys2, static_cast<size_t>(n) * 8, s);
    if (rc == QDB_OK) rc = dev_alloc(reinterpret_cast<void**>(&idx2), static_cast<size_t>(n) * 4, s);
    if (rc == QDB_OK) rc = dev_alloc(reinterpret_cast<void**>(&hist), static_cast<size_t>(256 * tiles) * 4, s);
    if (rc == QDB_OK) {
        const bool f = first != 0;
        switch (type) {
            case QDB_INT32: rc = ob_column<int32_t>(col, nulls, descending, n, f, indices, idx2, keys, keys2, hist, s); break;
            case QDB_INT64: rc = ob_column<int64_t>(col, nulls, descending, n, f, indices, idx2, keys, keys2, hist, s); break;
            case QDB_FLOAT: rc = ob_column<float>(col, nulls, descending, n, f, indices, idx2, keys, keys2, hist, s); break;
            default: rc = ob_column<double>(col, nulls, descending, n, f, indices, idx2, keys, keys2, hist, s); break;
        }
    }
    dev_free(keys, s);
    dev_free(keys2, s);
    dev_free(idx2, s);
    dev_free(hist, s);
    return rc;
}

int32_t qdb_order_by(int32_t n_cols, const int32_t* types, const void* const* cols, const uint64_t* const* nulls,
                     const int32_t* descending, int64_t n, int32_t* out_indices, void* stream) {
    if (n_cols < 1 || !types || !cols || n < 0) return fail(QDB_ERR_INVALID, "qdb_order_by: bad arguments");
    for (int c = n_cols - 1; c >= 0; --c) {
        const int32_t rc = qdb_order_by_column(types[c], cols[c], nulls ? nulls[c] : nullptr,
                                               descending ? descending[c] : 0, n, c == n_cols - 1, out_indices, stream);
        if (rc != QDB_OK) return rc;
    }
    return QDB_OK;
}

int32_t qdb_reorder(int32_t elem_bytes, const void* in, const int32_t* indices, int64_t offset, int64_t count,
                    void* out, void* stream) {
    if (count < 0 || offset < 0 || (count > 0 && (!in || !indices || !out)))
        return fail(QDB_ERR_INVALID, "qdb_reorder: bad arguments");
    if (count == 0) return QDB_OK;
    cudaStream_t s = as_stream(stream);
    const unsigned g = ob_grid(count, 256);
    switch (elem_bytes) {
        case 1: ob_gather_kernel<uint8_t><<<g, 256, 0, s>>>(static_cast<const uint8_t*>(in), indices, offset, count, static_cast<uint8_t*>(out)); break;
        case 2: ob_gather_kernel<uint16_t><<<g, 256, 0, s>>>(static_cast<const uint16_t*>(in), indices, offset, count, static_cast<uint16_t*>(out)); break;
        case 4: ob_gather_kernel<uint32_t><<<g, 256, 0, s>>>(static_cast<const uint32_t*>(in), indices, offset, count, static_cast<uint32_t*>(out)); break;
        case 8: ob_gather_kernel<uint64_t><<<g, 256, 0, s>>>(static_cast<const uint64_t*>(in), indices, offset, count, static_cast<uint64_t*>(out)); break;
        default: return fail(QDB_ERR_INVALID, "qdb_reorder: elem_bytes must be 1, 2, 4 or 8");
    }
    note_launch();
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? QDB_OK : cuda_fail(e, "ob_gather_kernel");
}

int32_t qdb_reorder_nulls(const uint64_t* in, const int32_t* indices, int64_t offset, int64_t count, uint64_t* out,
                          void* stream) {
    if (count < 0 || offset < 0 || (count > 0 && (!in || !indices || !out)))
        return fail(QDB_ERR_INVALID, "qdb_reorder_nulls: bad arguments");
    if (count == 0) return QDB_OK;
    cudaStream_t s = as_stream(stream);
    ob_gather_nulls_kernel<<<ob_grid((count + 63) / 64, 256), 256, 0, s>>>(in, indices, offset, count, out);
    note_launch();
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? QDB_OK : cuda_fail(e, "ob_gather_nulls_kernel");
}

}  // extern "C"
