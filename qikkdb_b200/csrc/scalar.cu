// Scalar aggregation (an aggregate without GROUP BY) over a WHERE-filtered column, and the dispatcher's block
// skipping by column min/max.  The replacement of GPUAggregation::col<AGG, OUT, IN>
// (qikkDB/QueryEngine/GPUCore/GPUAggregation.cuh:15-37, a CUB DeviceReduce per aggregate over the compacted block,
// AggregationFunctions.cuh:92-356) and of the CPU WHERE evaluation that skips a block whose min/max cannot satisfy
// the predicate (GpuSqlDispatcher::WhereEvaluation, qikkDB/GpuSqlParser/GpuSqlDispatcher.cpp:1116-1125, over the
// block statistics of qikkDB/BlockBase.h:190-200).
//
// One fused pass per block of rows: the predicate (the same [lo, hi] / invert interval as the GROUP BY pass) and
// the NULL masks select rows, every thread accumulates COUNT, SUM (a 64-bit two's-complement word for integers, FP64
// for floats), MIN and MAX (order-preserving integer encodings) over a grid-stride slice, a warp and then a block
// reduce the partials, and one set of global atomics per block folds them into the accumulator, which carries over
// the calls of a query's blocks.  Results follow the GROUP BY operator's types: V for MIN/MAX/SUM/AVG (an integer SUM
// wraps in V, an integer AVG truncates), int64 for COUNT; MIN/MAX/SUM/AVG over no row are NULL.
#include <climits>
#include <limits>

#include "groupby_agg.cuh"

namespace qdb {

struct ScalarState {            // device accumulator of one scalar query
    unsigned long long count;   // selected non-NULL values
    unsigned long long isum;    // integer sum (two's complement, wraps)
    double fsum;                // float sum
    long long mn, mx;           // order-preserving encodings of MIN and MAX
};

constexpr int kScThreads = 256;

// Order-preserving encoding of a value in the narrowest integer that holds it (32 bits for 4-byte types).
template <typename VT>
using EncT = typename std::conditional<sizeof(VT) == 4, int32_t, long long>::type;

template <typename VT>
__device__ __forceinline__ EncT<VT> sc_enc(VT v) {
    if constexpr (std::is_same<VT, float>::value) return fenc(v);
    else if constexpr (std::is_same<VT, double>::value) return denc(v);
    else return static_cast<EncT<VT>>(v);
}

// Four consecutive elements from a 16-byte aligned address (streaming loads: read once).
template <typename T>
__device__ __forceinline__ void load4(const T* p, T (&o)[4]) {
    const uint4* q = reinterpret_cast<const uint4*>(p);
    if constexpr (sizeof(T) == 4) {
        const uint4 a = __ldcs(q);
        memcpy(o, &a, 16);
    } else {
        const uint4 a = __ldcs(q), b = __ldcs(q + 1);
        memcpy(o, &a, 16);
        memcpy(o + 2, &b, 16);
    }
}

// VEC: the value and predicate columns start on 16-byte boundaries, so each thread takes four consecutive rows per
// step with vector loads (two steps in flight); otherwise four rows strided by the grid per step.
template <typename VT, typename PT, bool VEC>
__global__ void __launch_bounds__(kScThreads, 6) scalar_kernel(const VT* __restrict__ vals, const uint64_t* __restrict__ vnull,
                                                            int64_t n, const PT* __restrict__ pcol,
                                                            const uint64_t* __restrict__ pnull, PredInterval pi,
                                                            const int8_t* __restrict__ mask, ScalarState* st) {
    constexpr bool HAS_PRED = !std::is_same<PT, NoPred>::value;
    constexpr bool VFLOAT = std::is_floating_point<VT>::value;
    using PL = typename std::conditional<HAS_PRED, PT, int32_t>::type;
    using ET = EncT<VT>;
    // An int32 sum is kept mod 2^32 per thread: the result wraps in the value type.
    using ST = typename std::conditional<sizeof(VT) == 4, unsigned int, unsigned long long>::type;
    const PL plo = HAS_PRED ? from_bits<PL>(pi.lo) : PL{};
    const PL phi = HAS_PRED ? from_bits<PL>(pi.hi) : PL{};
    unsigned int cnt = 0;
    ST isum = 0;
    double fsum = 0.0;
    ET mn = std::numeric_limits<ET>::max(), mx = std::numeric_limits<ET>::min();
    auto take = [&](VT v) {
        ++cnt;
        if constexpr (VFLOAT) fsum += static_cast<double>(v);
        else isum += static_cast<ST>(v);
        const ET e = sc_enc(v);
        mn = min(mn, e);
        mx = max(mx, e);
    };
    auto row = [&](int64_t i, PL x, VT v) {
        bool keep = true;
        if constexpr (HAS_PRED) {
            keep = ((x >= plo) & (x <= phi)) != (pi.invert != 0);
            if (pnull) keep = keep && !((pnull[i >> 6] >> (i & 63)) & 1ull);
        }
        if (mask) keep = keep && mask[i] != 0;
        if (vnull) keep = keep && !((vnull[i >> 6] >> (i & 63)) & 1ull);
        if (keep) take(v);
    };
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    const int64_t tid = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if constexpr (VEC) {
        const int64_t chunks = n >> 2;
        auto chunk = [&](int64_t c, const VT (&v)[4], const PL (&x)[4]) {
            const int64_t i = c << 2;
            // the four rows' NULL and mask flags as bits 0..3
            unsigned drop = 0;
            if (pnull) drop |= static_cast<unsigned>(pnull[i >> 6] >> (i & 63)) & 15u;
            if (vnull) drop |= static_cast<unsigned>(vnull[i >> 6] >> (i & 63)) & 15u;
            if (mask)
#pragma unroll
                for (int u = 0; u < 4; ++u) drop |= (mask[i + u] == 0 ? 1u : 0u) << u;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                bool keep = !((drop >> u) & 1u);
                if constexpr (HAS_PRED) keep = keep && (((x[u] >= plo) & (x[u] <= phi)) != (pi.invert != 0));
                if (keep) take(v[u]);
            }
        };
        int64_t c = tid;
        for (; c + stride < chunks; c += 2 * stride) {
            VT v0[4], v1[4];
            PL x0[4], x1[4];
            load4(vals + (c << 2), v0);
            load4(vals + ((c + stride) << 2), v1);
            if constexpr (HAS_PRED) {
                load4(reinterpret_cast<const PL*>(pcol) + (c << 2), x0);
                load4(reinterpret_cast<const PL*>(pcol) + ((c + stride) << 2), x1);
            }
            chunk(c, v0, x0);
            chunk(c + stride, v1, x1);
        }
        for (; c < chunks; c += stride) {
            VT v0[4];
            PL x0[4];
            load4(vals + (c << 2), v0);
            if constexpr (HAS_PRED) load4(reinterpret_cast<const PL*>(pcol) + (c << 2), x0);
            chunk(c, v0, x0);
        }
        for (int64_t i = (chunks << 2) + tid; i < n; i += stride)
            row(i, HAS_PRED ? reinterpret_cast<const PL*>(pcol)[i] : PL{}, vals[i]);
    } else {
        int64_t i = tid;
        // Four rows per thread and step, all loads issued before any is used, so that enough bytes are in flight per
        // SM to cover the memory latency at full bandwidth.
        constexpr int U = 4;
        for (; i + (U - 1) * stride < n; i += U * stride) {
            PL x[U];
            VT v[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                x[u] = HAS_PRED ? __ldcs(reinterpret_cast<const PL*>(pcol) + i + u * stride) : PL{};
                v[u] = __ldcs(vals + i + u * stride);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) row(i + u * stride, x[u], v[u]);
        }
        for (; i < n; i += stride) row(i, HAS_PRED ? reinterpret_cast<const PL*>(pcol)[i] : PL{}, vals[i]);
    }
    // warp, then block reduce
    unsigned long long c64 = cnt, s64 = isum;
    long long mn64 = mn, mx64 = mx;
    if (cnt == 0) {
        mn64 = LLONG_MAX;
        mx64 = LLONG_MIN;
    }
    for (int d = 16; d > 0; d >>= 1) {
        c64 += __shfl_down_sync(0xffffffffu, c64, d);
        s64 += __shfl_down_sync(0xffffffffu, s64, d);
        fsum += __shfl_down_sync(0xffffffffu, fsum, d);
        mn64 = min(mn64, __shfl_down_sync(0xffffffffu, mn64, d));
        mx64 = max(mx64, __shfl_down_sync(0xffffffffu, mx64, d));
    }
    __shared__ unsigned long long s_cnt[kScThreads / 32], s_isum[kScThreads / 32];
    __shared__ double s_fsum[kScThreads / 32];
    __shared__ long long s_mn[kScThreads / 32], s_mx[kScThreads / 32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        s_cnt[warp] = c64;
        s_isum[warp] = s64;
        s_fsum[warp] = fsum;
        s_mn[warp] = mn64;
        s_mx[warp] = mx64;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kScThreads / 32; ++w) {
            c64 += s_cnt[w];
            s64 += s_isum[w];
            fsum += s_fsum[w];
            mn64 = min(mn64, s_mn[w]);
            mx64 = max(mx64, s_mx[w]);
        }
        if (c64) {
            atomicAdd(&st->count, c64);
            if (VFLOAT) atomicAdd(&st->fsum, fsum);
            else atomicAdd(&st->isum, s64);
            atomicMin(&st->mn, mn64);
            atomicMax(&st->mx, mx64);
        }
    }
}

template <typename VT, typename PT>
static void scalar_launch(const void* vals, const uint64_t* vnull, int64_t n, const void* pcol, const uint64_t* pnull,
                          const PredInterval& pi, const int8_t* mask, ScalarState* st, cudaStream_t s) {
    const DeviceInfo& di = device_info();
    const bool vec = (reinterpret_cast<uintptr_t>(vals) & 15u) == 0 && (reinterpret_cast<uintptr_t>(pcol) & 15u) == 0;
    auto kern = vec ? scalar_kernel<VT, PT, true> : scalar_kernel<VT, PT, false>;
    // One wave: as many blocks as are resident on every SM at once.
    static int per_sm[2] = {0, 0};
    if (per_sm[vec] == 0) {
        int b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern, kScThreads, 0) != cudaSuccess || b < 1) b = 4;
        per_sm[vec] = b;
    }
    const unsigned grid = static_cast<unsigned>(std::max<int64_t>(
        1, std::min<int64_t>((n + kScThreads - 1) / kScThreads, int64_t(di.sm_count) * per_sm[vec])));
    kern<<<grid, kScThreads, 0, s>>>(static_cast<const VT*>(vals), vnull, n, static_cast<const PT*>(pcol), pnull, pi,
                                     mask, st);
    note_launch();
}

template <typename VT>
static void scalar_launch_p(int32_t ptype, const void* vals, const uint64_t* vnull, int64_t n, const void* pcol,
                            const uint64_t* pnull, const PredInterval& pi, const int8_t* mask, ScalarState* st,
                            cudaStream_t s) {
    switch (ptype) {
        case QDB_INT32: scalar_launch<VT, int32_t>(vals, vnull, n, pcol, pnull, pi, mask, st, s); break;
        case QDB_INT64: scalar_launch<VT, int64_t>(vals, vnull, n, pcol, pnull, pi, mask, st, s); break;
        case QDB_FLOAT: scalar_launch<VT, float>(vals, vnull, n, pcol, pnull, pi, mask, st, s); break;
        case QDB_DOUBLE: scalar_launch<VT, double>(vals, vnull, n, pcol, pnull, pi, mask, st, s); break;
        default: scalar_launch<VT, NoPred>(vals, vnull, n, pcol, pnull, pi, mask, st, s); break;
    }
}

template <typename T>
static bool block_may_pass(const PredInterval& pi, const void* bmin, const void* bmax) {
    const T lo = from_bits<T>(pi.lo), hi = from_bits<T>(pi.hi);
    const T mn = *static_cast<const T*>(bmin), mx = *static_cast<const T*>(bmax);
    if (pi.invert) return !(mn >= lo && mx <= hi);  // some value outside [lo, hi] (unordered min/max: kept)
    if (!(lo <= hi)) return false;                  // an empty interval: no value passes
    return !(hi < mn || lo > mx);                   // [lo, hi] meets [min, max] (unordered min/max: kept)
}

}  // namespace qdb

struct qdb_scalar {
    int32_t val_type = 0;
    int device = 0;
    qdb::ScalarState* st = nullptr;
};

using namespace qdb;

extern "C" {

int32_t qdb_scalar_create(qdb_scalar** out, int32_t val_type, void* stream) {
    if (!out) return fail(QDB_ERR_INVALID, "qdb_scalar_create: null out");
    *out = nullptr;
    if (val_type != QDB_INT32 && val_type != QDB_INT64 && val_type != QDB_FLOAT && val_type != QDB_DOUBLE)
        return fail(QDB_ERR_INVALID, "qdb_scalar_create: value type must be INT32, INT64, FLOAT or DOUBLE");
    qdb_scalar* q = new qdb_scalar();
    q->val_type = val_type;
    cudaGetDevice(&q->device);
    int32_t rc = dev_alloc(reinterpret_cast<void**>(&q->st), sizeof(ScalarState), as_stream(stream));
    if (rc == QDB_OK) rc = qdb_scalar_reset(q, stream);
    if (rc != QDB_OK) {
        qdb_scalar_destroy(q);
        return rc;
    }
    *out = q;
    return QDB_OK;
}

int32_t qdb_scalar_destroy(qdb_scalar* q) {
    if (!q) return QDB_OK;
    if (q->st) {
        dev_free(q->st, nullptr);
        cudaStreamSynchronize(nullptr);
    }
    delete q;
    return QDB_OK;
}

int32_t qdb_scalar_reset(qdb_scalar* q, void* stream) {
    if (!q) return fail(QDB_ERR_INVALID, "qdb_scalar_reset: null accumulator");
    const ScalarState init{0ull, 0ull, 0.0, LLONG_MAX, LLONG_MIN};
    QDB_CUDA_TRY(cudaMemcpyAsync(q->st, &init, sizeof(init), cudaMemcpyHostToDevice, as_stream(stream)));
    QDB_CUDA_TRY(cudaStreamSynchronize(as_stream(stream)));  // `init` lives on this stack frame
    return QDB_OK;
}

int32_t qdb_scalar_process(qdb_scalar* q, const void* vals, const uint64_t* val_nulls, int64_t n, const qdb_pred* pred,
                           const int8_t* mask, void* stream) {
    if (!q || n < 0 || (n > 0 && !vals)) return fail(QDB_ERR_INVALID, "qdb_scalar_process: bad arguments");
    if (n == 0) return QDB_OK;
    PredInterval pi;
    int32_t ptype = 0;
    if (pred) {
        if (!pred->col) return fail(QDB_ERR_INVALID, "qdb_scalar_process: predicate without a column");
        if (pred->op < QDB_GREATER || pred->op > QDB_NOT_EQUAL)
            return fail(QDB_ERR_INVALID, "qdb_scalar_process: the predicate must be a comparison");
        pi = pred_interval(*pred);
        ptype = pred->type;
    }
    cudaStream_t s = as_stream(stream);
    const void* pc = pred ? pred->col : nullptr;
    const uint64_t* pn = pred ? pred->nulls : nullptr;
    switch (q->val_type) {
        case QDB_INT32: scalar_launch_p<int32_t>(ptype, vals, val_nulls, n, pc, pn, pi, mask, q->st, s); break;
        case QDB_INT64: scalar_launch_p<int64_t>(ptype, vals, val_nulls, n, pc, pn, pi, mask, q->st, s); break;
        case QDB_FLOAT: scalar_launch_p<float>(ptype, vals, val_nulls, n, pc, pn, pi, mask, q->st, s); break;
        default: scalar_launch_p<double>(ptype, vals, val_nulls, n, pc, pn, pi, mask, q->st, s); break;
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? QDB_OK : cuda_fail(e, "scalar_kernel");
}

int32_t qdb_scalar_result(qdb_scalar* q, int32_t agg, void* out_value, int32_t* out_is_null, void* stream) {
    if (!q || !out_value) return fail(QDB_ERR_INVALID, "qdb_scalar_result: bad arguments");
    ScalarState h{};
    QDB_CUDA_TRY(cudaMemcpyAsync(&h, q->st, sizeof(h), cudaMemcpyDeviceToHost, as_stream(stream)));
    QDB_CUDA_TRY(cudaStreamSynchronize(as_stream(stream)));
    const bool empty = h.count == 0;
    if (out_is_null) *out_is_null = (agg != QDB_AGG_COUNT && empty) ? 1 : 0;
    if (agg == QDB_AGG_COUNT) {
        *static_cast<int64_t*>(out_value) = static_cast<int64_t>(h.count);
        return QDB_OK;
    }
    if (agg != QDB_AGG_MIN && agg != QDB_AGG_MAX && agg != QDB_AGG_SUM && agg != QDB_AGG_AVG)
        return fail(QDB_UNKNOWN_AGG_FUN, "qdb_scalar_result: unknown aggregate");
    const int t = q->val_type;
    const bool fl = t == QDB_FLOAT || t == QDB_DOUBLE;
    if (empty) {
        memset(out_value, 0, t == QDB_INT32 || t == QDB_FLOAT ? 4 : 8);
        return QDB_OK;
    }
    long long iv = 0;
    double fv = 0.0;
    if (agg == QDB_AGG_MIN || agg == QDB_AGG_MAX) {
        const long long e = agg == QDB_AGG_MIN ? h.mn : h.mx;
        if (t == QDB_FLOAT) fv = fdec(static_cast<int32_t>(e));
        else if (t == QDB_DOUBLE) fv = ddec(e);
        else iv = e;
    } else if (fl) {
        fv = agg == QDB_AGG_SUM ? h.fsum : h.fsum / static_cast<double>(h.count);
    } else {
        // integer SUM wraps in the value type; AVG divides the wrapped sum by the count, truncated
        const long long wrapped = t == QDB_INT32 ? static_cast<long long>(static_cast<int32_t>(static_cast<uint32_t>(h.isum)))
                                                 : static_cast<long long>(h.isum);
        iv = agg == QDB_AGG_SUM ? wrapped : wrapped / static_cast<long long>(h.count);
    }
    switch (t) {
        case QDB_INT32: *static_cast<int32_t*>(out_value) = static_cast<int32_t>(iv); break;
        case QDB_INT64: *static_cast<int64_t*>(out_value) = iv; break;
        case QDB_FLOAT: *static_cast<float*>(out_value) = static_cast<float>(fv); break;
        default: *static_cast<double*>(out_value) = fv; break;
    }
    return QDB_OK;
}

int32_t qdb_pred_block_may_pass(const qdb_pred* pred, const void* block_min, const void* block_max, int32_t* may_pass) {
    if (!pred || !block_min || !block_max || !may_pass) return fail(QDB_ERR_INVALID, "qdb_pred_block_may_pass: null argument");
    if (pred->op < QDB_GREATER || pred->op > QDB_NOT_EQUAL)
        return fail(QDB_ERR_INVALID, "qdb_pred_block_may_pass: the predicate must be a comparison");
    const PredInterval pi = pred_interval(*pred);
    bool m = true;
    switch (pred->type) {
        case QDB_INT32: m = block_may_pass<int32_t>(pi, block_min, block_max); break;
        case QDB_INT64: m = block_may_pass<int64_t>(pi, block_min, block_max); break;
        case QDB_FLOAT: m = block_may_pass<float>(pi, block_min, block_max); break;
        case QDB_DOUBLE: m = block_may_pass<double>(pi, block_min, block_max); break;
        default: return fail(QDB_ERR_INVALID, "qdb_pred_block_may_pass: column type must be INT32, INT64, FLOAT or DOUBLE");
    }
    *may_pass = m ? 1 : 0;
    return QDB_OK;
}

}  // extern "C"
