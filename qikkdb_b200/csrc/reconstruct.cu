// Stream compaction: GPUReconstruct (qikkDB/QueryEngine/GPUCore/GPUReconstruct.cuh:204-355 reconstructCol /
// reconstructColKeep, :487-566 GenerateIndexes(Keep), :573-583 PrefixSum, GPUReconstruct.cu:8-43 and
// :756-764 null-mask reconstruction and CompressNullMask).
//
// The reference runs a CUB InclusiveSum of the int8 mask into an int32 array (4 B/row written and read
// back), reads the count back, allocates, and scatters with kernel_reconstruct_col.  Here a pass counts
// the selected rows of every 4096-row tile (1 B/row read), one block scans the tile counts, and the
// scatter pass recomputes each thread's offset inside its tile from the mask (a block scan in registers
// and shared memory), so no per-row prefix array touches HBM.  No pass waits on another CTA.
#include <mutex>
#include <string>
#include <vector>

#include "qdb_common.cuh"

namespace qdb {

constexpr int kRcThreads = 256;
constexpr int kRcPerThread = 16;
constexpr int kRcTile = kRcThreads * kRcPerThread;  // 4096 rows

__device__ __forceinline__ int rc_block_excl_scan(int x, int* total) {
    __shared__ int warp_sums[kRcThreads / 32];
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
        const int w = (lane < kRcThreads / 32) ? warp_sums[lane] : 0;
        int wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += y;
        }
        if (lane < kRcThreads / 32) warp_sums[lane] = wi - w;
        if (lane == 31) *total = wi;
    }
    __syncthreads();
    const int excl = warp_sums[wid] + inc - x;
    __syncthreads();
    return excl;
}

// The 16 mask bytes of this thread as a bit set (bit e = row base+e selected).
__device__ __forceinline__ uint32_t mask_bits(const int8_t* __restrict__ mask, int64_t base, int64_t n, bool vec) {
    uint32_t bits = 0;
    if (vec && base + kRcPerThread <= n) {
        const int4 q = __ldcs(reinterpret_cast<const int4*>(mask + base));
        const uint32_t w[4] = {static_cast<uint32_t>(q.x), static_cast<uint32_t>(q.y), static_cast<uint32_t>(q.z),
                               static_cast<uint32_t>(q.w)};
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int e = 0; e < 4; ++e) bits |= (((w[k] >> (8 * e)) & 0xffu) ? 1u : 0u) << (4 * k + e);
    } else {
        for (int e = 0; e < kRcPerThread; ++e)
            if (base + e < n && mask[base + e]) bits |= 1u << e;
    }
    return bits;
}

__global__ void rc_count_kernel(const int8_t* __restrict__ mask, int64_t n, int vec, long long* tile_counts) {
    const int64_t base = static_cast<int64_t>(blockIdx.x) * kRcTile + threadIdx.x * kRcPerThread;
    const int c = (base < n) ? __popc(mask_bits(mask, base, n, vec)) : 0;
    __shared__ int tot;
    rc_block_excl_scan(c, &tot);
    if (threadIdx.x == 0) tile_counts[blockIdx.x] = tot;
}

// Exclusive scan of tile counts in one block; tile_counts[ntiles] receives the total.
__global__ void rc_scan_kernel(long long* tile_counts, int64_t ntiles) {
    __shared__ long long carry;
    __shared__ long long wsum[kRcThreads / 32];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int64_t base = 0; base < ntiles; base += kRcThreads) {
        const int64_t i = base + threadIdx.x;
        const long long x = (i < ntiles) ? tile_counts[i] : 0;
        long long inc = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        if (lane == 31) wsum[wid] = inc;
        __syncthreads();
        long long before = 0, all = 0;
        for (int w = 0; w < kRcThreads / 32; ++w) {
            if (w < wid) before += wsum[w];
            all += wsum[w];
        }
        if (i < ntiles) tile_counts[i] = carry + before + inc - x;
        __syncthreads();
        if (threadIdx.x == 0) carry += all;
        __syncthreads();
    }
    if (threadIdx.x == 0) tile_counts[ntiles] = carry;
}

template <typename T>
__global__ void rc_scatter_kernel(const T* __restrict__ in, const int8_t* __restrict__ mask, int64_t n, int vec,
                                  const long long* __restrict__ tile_offsets, T* __restrict__ out,
                                  const uint64_t* __restrict__ null_in, unsigned long long* null_out) {
    const int64_t base = static_cast<int64_t>(blockIdx.x) * kRcTile + threadIdx.x * kRcPerThread;
    const uint32_t bits = (base < n) ? mask_bits(mask, base, n, vec) : 0u;
    __shared__ int tot;
    long long pos = tile_offsets[blockIdx.x] + rc_block_excl_scan(__popc(bits), &tot);
    for (int e = 0; e < kRcPerThread; ++e) {
        if (!((bits >> e) & 1u)) continue;
        const int64_t r = base + e;
        out[pos] = in[r];
        if (null_out && null_bit(null_in, r)) atomicOr(null_out + (pos >> 6), 1ull << (pos & 63));
        ++pos;
    }
}

// Row indices (int32) of the selected rows (kernel_generate_indexes, GPUReconstruct.cuh:56-71).
__global__ void rc_indexes_kernel(const int8_t* __restrict__ mask, int64_t n, int vec,
                                  const long long* __restrict__ tile_offsets, int32_t* __restrict__ out) {
    const int64_t base = static_cast<int64_t>(blockIdx.x) * kRcTile + threadIdx.x * kRcPerThread;
    const uint32_t bits = (base < n) ? mask_bits(mask, base, n, vec) : 0u;
    __shared__ int tot;
    long long pos = tile_offsets[blockIdx.x] + rc_block_excl_scan(__popc(bits), &tot);
    for (int e = 0; e < kRcPerThread; ++e)
        if ((bits >> e) & 1u) out[pos++] = static_cast<int32_t>(base + e);
}

// Inclusive prefix sum of the mask (PrefixSum<int32_t,int8_t>).  Like CUB's InclusiveSum over int8 input
// accumulated in int32, every non-zero byte counts its value; the reference's masks hold 0/1.
__global__ void rc_prefix_kernel(const int8_t* __restrict__ mask, int64_t n, const long long* __restrict__ tile_offsets,
                                 int32_t* __restrict__ out) {
    const int64_t base = static_cast<int64_t>(blockIdx.x) * kRcTile + threadIdx.x * kRcPerThread;
    int vals[kRcPerThread];
    int c = 0;
#pragma unroll
    for (int e = 0; e < kRcPerThread; ++e) {
        vals[e] = (base + e < n) ? static_cast<int>(mask[base + e]) : 0;
        c += vals[e];
    }
    __shared__ int tot;
    long long run = tile_offsets[blockIdx.x] + rc_block_excl_scan(c, &tot);
#pragma unroll
    for (int e = 0; e < kRcPerThread; ++e) {
        run += vals[e];
        if (base + e < n) out[base + e] = static_cast<int32_t>(run);
    }
}

// Tile sums of the mask values (for the prefix sum, which counts values, not non-zero bytes).
__global__ void rc_sum_kernel(const int8_t* __restrict__ mask, int64_t n, long long* tile_counts) {
    const int64_t base = static_cast<int64_t>(blockIdx.x) * kRcTile + threadIdx.x * kRcPerThread;
    int c = 0;
    for (int e = 0; e < kRcPerThread; ++e) c += (base + e < n) ? static_cast<int>(mask[base + e]) : 0;
    __shared__ int tot;
    rc_block_excl_scan(c, &tot);
    if (threadIdx.x == 0) tile_counts[blockIdx.x] = tot;
}

// uint8 null array -> bit-packed mask via warp ballots (kernel_compress_null_mask, GPUReconstruct.cu:31-43).
__global__ void rc_compress_kernel(const uint8_t* __restrict__ in, int64_t n, uint32_t* __restrict__ out32) {
    const int64_t nwarps = (n + 31) / 32;
    const int lane = threadIdx.x & 31;
    for (int64_t w = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) / 32; w < nwarps;
         w += (static_cast<int64_t>(gridDim.x) * blockDim.x) / 32) {
        const int64_t i = w * 32 + lane;
        const bool bit = (i < n) && (in[i] & 1u);
        const uint32_t b = __ballot_sync(0xffffffffu, bit);
        if (lane == 0) out32[w] = b;
    }
}

// Counts the selected rows per tile and scans the counts; returns the device offsets (ntiles + 1 entries,
// the last one the total) and the total on the host.
static int32_t count_and_scan(const int8_t* mask, int64_t n, bool sum_values, long long** offsets, long long* total,
                              cudaStream_t s) {
    const int64_t ntiles = (n + kRcTile - 1) / kRcTile;
    int32_t rc = dev_alloc(reinterpret_cast<void**>(offsets), (ntiles + 1) * sizeof(long long), s);
    if (rc != QDB_OK) return rc;
    const int vec = (reinterpret_cast<uintptr_t>(mask) & 15u) == 0;
    if (sum_values) rc_sum_kernel<<<static_cast<unsigned>(ntiles), kRcThreads, 0, s>>>(mask, n, *offsets);
    else rc_count_kernel<<<static_cast<unsigned>(ntiles), kRcThreads, 0, s>>>(mask, n, vec, *offsets);
    note_launch();
    rc_scan_kernel<<<1, kRcThreads, 0, s>>>(*offsets, ntiles);
    note_launch();
    if (total) {
        cudaError_t e = cudaMemcpyAsync(total, *offsets + ntiles, sizeof(long long), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            dev_free(*offsets, s);
            *offsets = nullptr;
            return cuda_fail(e, "compaction count pass");
        }
    } else {
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(e, "compaction count pass");
    }
    return QDB_OK;
}

template <typename T>
static void launch_scatter(const void* in, const int8_t* mask, int64_t n, const long long* offs, void* out,
                           const uint64_t* null_in, unsigned long long* null_out, cudaStream_t s) {
    const int64_t ntiles = (n + kRcTile - 1) / kRcTile;
    const int vec = (reinterpret_cast<uintptr_t>(mask) & 15u) == 0;
    rc_scatter_kernel<T><<<static_cast<unsigned>(ntiles), kRcThreads, 0, s>>>(
        static_cast<const T*>(in), mask, n, vec, offs, static_cast<T*>(out), null_in, null_out);
    note_launch();
}

}  // namespace qdb

using namespace qdb;

extern "C" {

int32_t qdb_reconstruct_keep(int32_t elem_bytes, const void* in, const int8_t* mask, int64_t n, void** out,
                             int64_t* out_count, const uint64_t* null_in, uint64_t** out_null_mask, void* stream) {
    if (!out || !out_count) return fail(QDB_ERR_INVALID, "qdb_reconstruct_keep: null out arguments");
    if (elem_bytes != 1 && elem_bytes != 2 && elem_bytes != 4 && elem_bytes != 8)
        return fail(QDB_ERR_INVALID, "qdb_reconstruct_keep: elem_bytes must be 1, 2, 4 or 8");
    *out = nullptr;
    *out_count = 0;
    if (out_null_mask) *out_null_mask = nullptr;
    if (n <= 0) return QDB_OK;
    if (!in) return fail(QDB_ERR_INVALID, "qdb_reconstruct_keep: null input");
    if (!mask) {
        // Without a mask the input is returned as is (GPUReconstruct.cuh:320-327).
        *out = const_cast<void*>(in);
        *out_count = n;
        if (out_null_mask) *out_null_mask = const_cast<uint64_t*>(null_in);
        return QDB_OK;
    }
    cudaStream_t s = as_stream(stream);
    long long* offs = nullptr;
    long long total = 0;
    int32_t rc = count_and_scan(mask, n, false, &offs, &total, s);
    if (rc != QDB_OK) return rc;
    if (total == 0) {
        dev_free(offs, s);
        return QDB_OK;
    }
    rc = dev_alloc(out, static_cast<size_t>(total) * elem_bytes, s);
    unsigned long long* nout = nullptr;
    const size_t nwords = (static_cast<size_t>(total) + 63) / 64;
    if (rc == QDB_OK && null_in && out_null_mask) {
        rc = dev_alloc(reinterpret_cast<void**>(&nout), nwords * 8, s);
        if (rc == QDB_OK && cudaMemsetAsync(nout, 0, nwords * 8, s) != cudaSuccess)
            rc = cuda_fail(cudaGetLastError(), "cudaMemsetAsync(null mask)");
    }
    if (rc != QDB_OK) {
        dev_free(*out, s);
        dev_free(nout, s);
        dev_free(offs, s);
        *out = nullptr;
        return rc;
    }
    switch (elem_bytes) {
        case 1: launch_scatter<uint8_t>(in, mask, n, offs, *out, null_in, nout, s); break;
        case 2: launch_scatter<uint16_t>(in, mask, n, offs, *out, null_in, nout, s); break;
        case 4: launch_scatter<uint32_t>(in, mask, n, offs, *out, null_in, nout, s); break;
        default: launch_scatter<uint64_t>(in, mask, n, offs, *out, null_in, nout, s); break;
    }
    cudaError_t e = cudaGetLastError();
    dev_free(offs, s);
    if (e != cudaSuccess) return cuda_fail(e, "rc_scatter_kernel");
    *out_count = total;
    if (out_null_mask) *out_null_mask = reinterpret_cast<uint64_t*>(nout);
    return QDB_OK;
}

int32_t qdb_generate_indexes(const int8_t* mask, int64_t n, int32_t** out, int64_t* out_count, void* stream) {
    if (!out || !out_count) return fail(QDB_ERR_INVALID, "qdb_generate_indexes: null out arguments");
    *out = nullptr;
    *out_count = 0;
    if (!mask) return fail(QDB_ERROR, "inMask cannot be nullptr in GenerateIndexes");
    if (n <= 0) return QDB_OK;
    cudaStream_t s = as_stream(stream);
    long long* offs = nullptr;
    long long total = 0;
    int32_t rc = count_and_scan(mask, n, false, &offs, &total, s);
    if (rc != QDB_OK) return rc;
    if (total > 0) {
        rc = dev_alloc(reinterpret_cast<void**>(out), static_cast<size_t>(total) * 4, s);
        if (rc == QDB_OK) {
            const int64_t ntiles = (n + kRcTile - 1) / kRcTile;
            const int vec = (reinterpret_cast<uintptr_t>(mask) & 15u) == 0;
            rc_indexes_kernel<<<static_cast<unsigned>(ntiles), kRcThreads, 0, s>>>(mask, n, vec, offs, *out);
            note_launch();
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) rc = cuda_fail(e, "rc_indexes_kernel");
        }
    }
    dev_free(offs, s);
    if (rc == QDB_OK) *out_count = total;
    return rc;
}

int32_t qdb_prefix_sum(const int8_t* mask, int64_t n, int32_t* out, void* stream) {
    if (n <= 0) return QDB_OK;
    if (!mask || !out) return fail(QDB_ERR_INVALID, "qdb_prefix_sum: null argument");
    cudaStream_t s = as_stream(stream);
    long long* offs = nullptr;
    int32_t rc = count_and_scan(mask, n, true, &offs, nullptr, s);
    if (rc != QDB_OK) return rc;
    const int64_t ntiles = (n + kRcTile - 1) / kRcTile;
    rc_prefix_kernel<<<static_cast<unsigned>(ntiles), kRcThreads, 0, s>>>(mask, n, offs, out);
    note_launch();
    cudaError_t e = cudaGetLastError();
    dev_free(offs, s);
    if (e != cudaSuccess) return cuda_fail(e, "rc_prefix_kernel");
    return QDB_OK;
}

int32_t qdb_compress_null_mask(const uint8_t* in, int64_t n, uint64_t** out, void* stream) {
    if (!out) return fail(QDB_ERR_INVALID, "qdb_compress_null_mask: null out");
    *out = nullptr;
    if (n <= 0) return QDB_OK;
    if (!in) return fail(QDB_ERR_INVALID, "qdb_compress_null_mask: null input");
    cudaStream_t s = as_stream(stream);
    const size_t nwords = (static_cast<size_t>(n) + 63) / 64;
    int32_t rc = dev_alloc(reinterpret_cast<void**>(out), nwords * 8, s);
    if (rc != QDB_OK) return rc;
    QDB_CUDA_TRY(cudaMemsetAsync(*out, 0, nwords * 8, s));
    const DeviceInfo& di = device_info();
    int64_t blocks = ((n + 31) / 32 * 32 + 255) / 256;
    if (blocks > static_cast<int64_t>(di.sm_count) * 16) blocks = static_cast<int64_t>(di.sm_count) * 16;
    rc_compress_kernel<<<static_cast<unsigned>(blocks), 256, 0, s>>>(in, n, reinterpret_cast<uint32_t*>(*out));
    note_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "rc_compress_kernel");
    return QDB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Compaction without any allocation, for callers that may not allocate device memory.
//
// Some callers own every byte of device memory themselves: a database buffer pool that accounts all
// HBM, or a serving loop that admits queries against a fixed HBM budget.  They cannot let a library
// call cudaMalloc behind their back: the allocation can fail in the middle of a query under their
// memory pressure, escapes their accounting, and cudaFree synchronises the whole device.  This entry
// point therefore works only in memory the caller passes in plus one fixed scratch array that the
// library holds for the life of the process on every GPU that loads it.
// ---------------------------------------------------------------------------------------------
namespace qdb {

// Largest input the no-allocation compaction accepts: kNoAllocMaxTiles tiles of kRcTile rows (2^28 rows).
constexpr int64_t kNoAllocMaxTiles = 65536;
constexpr int64_t kNoAllocMaxRows = kNoAllocMaxTiles * kRcTile;

// Per-tile counts and offsets (+ the total in the last entry): 512 KiB + 8 bytes per GPU, allocated when
// the library is loaded and kept until the process exits.  Shared by every call on the device.
static __device__ __align__(256) long long g_noalloc_tile_offsets[kNoAllocMaxTiles + 1];

// Device address of g_noalloc_tile_offsets on each device.  In host code the symbol is only a host-side
// stand-in, so the address must be looked up with the device current.
static std::mutex g_noalloc_mu;
static std::vector<long long*> g_noalloc_ptr;

static int32_t noalloc_scratch(long long** out) {
    int dev = 0;
    QDB_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (static_cast<int>(g_noalloc_ptr.size()) <= dev) g_noalloc_ptr.resize(dev + 1, nullptr);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_tile_offsets);
        if (e != cudaSuccess || !p) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_tile_offsets)");
        g_noalloc_ptr[dev] = static_cast<long long*>(p);
    }
    *out = g_noalloc_ptr[dev];
    return QDB_OK;
}

}  // namespace qdb

extern "C" int32_t qdb_reconstruct_keep_noalloc(int32_t elem_bytes, const void* in, const int8_t* mask, int64_t n,
                                                void* out, int64_t out_capacity, int64_t* out_count,
                                                const uint64_t* null_in, uint64_t* out_null_mask, void* stream) {
    if (!out_count) return fail(QDB_ERR_INVALID, "qdb_reconstruct_keep_noalloc: null out_count");
    *out_count = 0;
    if (elem_bytes != 1 && elem_bytes != 2 && elem_bytes != 4 && elem_bytes != 8)
        return fail(QDB_ERR_INVALID, "qdb_reconstruct_keep_noalloc: elem_bytes must be 1, 2, 4 or 8");
    if (n < 0) return fail(QDB_ERR_INVALID, "qdb_reconstruct_keep_noalloc: negative row count");
    if (n > kNoAllocMaxRows)
        return fail(QDB_ERR_TOO_LARGE, "qdb_reconstruct_keep_noalloc: at most 268435456 rows per call (n = " +
                                           std::to_string(n) + ")");
    if (n == 0) return QDB_OK;
    if (!in || !mask || (!out && out_capacity > 0))
        return fail(QDB_ERR_INVALID, "qdb_reconstruct_keep_noalloc: null input, mask or output");
    long long* offs = nullptr;
    int32_t rc = noalloc_scratch(&offs);
    if (rc != QDB_OK) return rc;
    cudaStream_t s = as_stream(stream);
    const int64_t ntiles = (n + kRcTile - 1) / kRcTile;
    const int vec = (reinterpret_cast<uintptr_t>(mask) & 15u) == 0;
    // Every entry the scan reads is written by the count pass first, so the scratch needs no clearing.
    rc_count_kernel<<<static_cast<unsigned>(ntiles), kRcThreads, 0, s>>>(mask, n, vec, offs);
    note_launch();
    rc_scan_kernel<<<1, kRcThreads, 0, s>>>(offs, ntiles);
    note_launch();
    long long total = 0;
    cudaError_t e = cudaMemcpyAsync(&total, offs + ntiles, sizeof(long long), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "qdb_reconstruct_keep_noalloc: count pass");
    if (total > out_capacity)
        return fail(QDB_ERR_TOO_LARGE, "qdb_reconstruct_keep_noalloc: " + std::to_string(total) +
                                           " selected rows exceed out_capacity " + std::to_string(out_capacity));
    if (total == 0) return QDB_OK;
    unsigned long long* nout = nullptr;
    if (null_in && out_null_mask) {
        nout = reinterpret_cast<unsigned long long*>(out_null_mask);
        QDB_CUDA_TRY(cudaMemsetAsync(nout, 0, ((static_cast<size_t>(total) + 63) / 64) * 8, s));
    }
    switch (elem_bytes) {
        case 1: launch_scatter<uint8_t>(in, mask, n, offs, out, null_in, nout, s); break;
        case 2: launch_scatter<uint16_t>(in, mask, n, offs, out, null_in, nout, s); break;
        case 4: launch_scatter<uint32_t>(in, mask, n, offs, out, null_in, nout, s); break;
        default: launch_scatter<uint64_t>(in, mask, n, offs, out, null_in, nout, s); break;
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "rc_scatter_kernel (no-allocation form)");
    *out_count = total;
    return QDB_OK;
}
