// Exclusive prefix sum of a device array in three launches: the sums of 4096-element tiles, one block's scan of the
// tile sums, and each tile's scan offset by its tile's prefix.  Used where a single block's scan of millions of
// counts would serialise: the key lengths of string GROUP BY results and the digit counts of ORDER BY's radix passes.
#pragma once

#include "qdb_common.cuh"

namespace qdb {

constexpr int kScanThreads = 512;
constexpr int kScanPer = 8;
constexpr int kScanTile = kScanThreads * kScanPer;

template <typename T>
__device__ __forceinline__ T scan_block_exclusive(T x, T* warp_sums, T* total) {
    // exclusive scan of one value per thread over the block; *total (shared) receives the block's sum
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T inc = x;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const T y = __shfl_up_sync(0xffffffffu, inc, d);
        if (lane >= d) inc += y;
    }
    if (lane == 31) warp_sums[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        constexpr int NW = kScanThreads / 32;
        T ws = lane < NW ? warp_sums[lane] : T(0);
        T wi = ws;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const T y = __shfl_up_sync(0xffffffffu, wi, d);
            if (lane >= d) wi += y;
        }
        if (lane < NW) warp_sums[lane] = wi - ws;
        if (lane == NW - 1) *total = wi;
    }
    __syncthreads();
    return inc - x + warp_sums[warp];
}

template <typename T>
__global__ void __launch_bounds__(kScanThreads) scan_sums_kernel(const T* __restrict__ v, int64_t m, T* __restrict__ sums) {
    __shared__ T ws[kScanThreads / 32];
    __shared__ T tot;
    const int64_t base = static_cast<int64_t>(blockIdx.x) * kScanTile + static_cast<int64_t>(threadIdx.x) * kScanPer;
    T s = 0;
#pragma unroll
    for (int j = 0; j < kScanPer; ++j)
        if (base + j < m) s += v[base + j];
    scan_block_exclusive<T>(s, ws, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// One block: exclusive scan of m values in place (chunks per thread, then the chunk sums); *total (optional)
// receives the sum.
template <typename T>
__global__ void __launch_bounds__(kScanThreads) scan_one_block_kernel(T* v, int64_t m, T* total) {
    __shared__ T ws[kScanThreads / 32];
    __shared__ T tot;
    const int64_t per = (m + kScanThreads - 1) / kScanThreads;
    const int64_t b = threadIdx.x * per;
    const int64_t e = min(m, b + per);
    T s = 0;
    for (int64_t i = b; i < e; ++i) s += v[i];
    T run = scan_block_exclusive<T>(s, ws, &tot);
    for (int64_t i = b; i < e; ++i) {
        const T c = v[i];
        v[i] = run;
        run += c;
    }
    if (threadIdx.x == 0 && total) *total = tot;
}

template <typename T>
__global__ void __launch_bounds__(kScanThreads) scan_tiles_kernel(T* __restrict__ v, int64_t m, const T* __restrict__ offs) {
    __shared__ T ws[kScanThreads / 32];
    __shared__ T tot;
    const int64_t base = static_cast<int64_t>(blockIdx.x) * kScanTile + static_cast<int64_t>(threadIdx.x) * kScanPer;
    T x[kScanPer];
    T s = 0;
#pragma unroll
    for (int j = 0; j < kScanPer; ++j) {
        x[j] = base + j < m ? v[base + j] : T(0);
        s += x[j];
    }
    T run = scan_block_exclusive<T>(s, ws, &tot) + offs[blockIdx.x];
#pragma unroll
    for (int j = 0; j < kScanPer; ++j) {
        if (base + j < m) v[base + j] = run;
        run += x[j];
    }
}

// Exclusive scan of v[0, m) in place on `s`; *total (device, optional) receives the sum.  Allocates the tile sums
// from the stream-ordered pool.
template <typename T>
int32_t exclusive_scan(T* v, int64_t m, T* total, cudaStream_t s) {
    if (m <= 0) {
        if (total) {
            const cudaError_t e = cudaMemsetAsync(total, 0, sizeof(T), s);
            if (e != cudaSuccess) return cuda_fail(e, "exclusive_scan");
        }
        return QDB_OK;
    }
    const int64_t tiles = (m + kScanTile - 1) / kScanTile;
    if (tiles == 1) {
        scan_one_block_kernel<T><<<1, kScanThreads, 0, s>>>(v, m, total);
        note_launch();
        const cudaError_t e = cudaGetLastError();
        return e == cudaSuccess ? QDB_OK : cuda_fail(e, "scan_one_block_kernel");
    }
    T* sums = nullptr;
    int32_t rc = dev_alloc(reinterpret_cast<void**>(&sums), static_cast<size_t>(tiles) * sizeof(T), s);
    if (rc != QDB_OK) return rc;
    scan_sums_kernel<T><<<static_cast<unsigned>(tiles), kScanThreads, 0, s>>>(v, m, sums);
    scan_one_block_kernel<T><<<1, kScanThreads, 0, s>>>(sums, tiles, total);
    scan_tiles_kernel<T><<<static_cast<unsigned>(tiles), kScanThreads, 0, s>>>(v, m, sums);
    note_launch(3);
    const cudaError_t e = cudaGetLastError();
    dev_free(sums, s);
    return e == cudaSuccess ? QDB_OK : cuda_fail(e, "exclusive_scan");
}

}  // namespace qdb
