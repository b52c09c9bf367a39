// Filter: `mask[i] = OP(a[i] | a, b[i] | b) && !null(i)` into an int8 mask, the standalone form of
// GPUBinary<FilterConditions::OP, int8_t, L, R>::Binary (qikkDB/QueryEngine/GPUCore/GPUBinary.cuh:555-579)
// and kernel_filter (qikkDB/QueryEngine/GPUCore/GPUFilter.cuh:22-44).  The aggregation pass evaluates its
// predicate itself; this kernel serves callers that want the mask (and the reference's filter tests).
// Each thread handles 4 consecutive rows with 128-bit loads and one 32-bit store.
#include "groupby_agg.cuh"

namespace qdb {

constexpr int kFilterThreads = 256;

template <typename A, typename B, bool ACOL, bool BCOL>
__global__ void filter_kernel(int32_t op, const A* __restrict__ a, A ac, const B* __restrict__ b, B bc,
                              const uint64_t* __restrict__ nulls, int8_t* __restrict__ out, int64_t n, int vec_ok) {
    const int64_t groups = (n + 3) / 4;
    for (int64_t g = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; g < groups;
         g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t r0 = g * 4;
        const bool full = vec_ok && r0 + 4 <= n;
        A av[4];
        B bv[4];
        if constexpr (ACOL) load4<A>(a, r0, n, full, av);
        else
#pragma unroll
            for (int e = 0; e < 4; ++e) av[e] = ac;
        if constexpr (BCOL) load4<B>(b, r0, n, full, bv);
        else
#pragma unroll
            for (int e = 0; e < 4; ++e) bv[e] = bc;
        uint32_t word = 0;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const bool r = cmp_op(op, av[e], bv[e]) && !null_bit(nulls, r0 + e);
            word |= (r ? 1u : 0u) << (8 * e);
        }
        if (full) {
            *reinterpret_cast<uint32_t*>(out + r0) = word;
        } else {
#pragma unroll
            for (int e = 0; e < 4; ++e)
                if (r0 + e < n) out[r0 + e] = static_cast<int8_t>((word >> (8 * e)) & 1u);
        }
    }
}

template <typename T>
static T host_value(const void* p) {
    T v;
    memcpy(&v, p, sizeof(T));
    return v;
}

template <typename A, typename B>
static int32_t launch_filter_ab(int32_t op, int a_col, const void* a, int b_col, const void* b, const uint64_t* nulls,
                                int8_t* out, int64_t n, cudaStream_t s) {
    const bool vec_ok = (!a_col || (reinterpret_cast<uintptr_t>(a) & 15u) == 0) &&
                        (!b_col || (reinterpret_cast<uintptr_t>(b) & 15u) == 0) &&
                        (reinterpret_cast<uintptr_t>(out) & 3u) == 0;
    const DeviceInfo& di = device_info();
    int64_t groups = (n + 3) / 4;
    int64_t blocks = (groups + kFilterThreads - 1) / kFilterThreads;
    if (blocks > static_cast<int64_t>(di.sm_count) * 16) blocks = static_cast<int64_t>(di.sm_count) * 16;
    const unsigned grid = static_cast<unsigned>(blocks);
    if (a_col && b_col)
        filter_kernel<A, B, true, true><<<grid, kFilterThreads, 0, s>>>(op, static_cast<const A*>(a), A{},
                                                                        static_cast<const B*>(b), B{}, nulls, out, n,
                                                                        vec_ok);
    else if (a_col)
        filter_kernel<A, B, true, false><<<grid, kFilterThreads, 0, s>>>(
            op, static_cast<const A*>(a), A{}, nullptr, host_value<B>(b), nulls, out, n, vec_ok);
    else
        filter_kernel<A, B, false, true><<<grid, kFilterThreads, 0, s>>>(
            op, nullptr, host_value<A>(a), static_cast<const B*>(b), B{}, nulls, out, n, vec_ok);
    note_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "filter_kernel");
    return QDB_OK;
}

template <typename A>
static int32_t launch_filter_a(int32_t op, int a_col, const void* a, int32_t b_type, int b_col, const void* b,
                               const uint64_t* nulls, int8_t* out, int64_t n, cudaStream_t s) {
    switch (b_type) {
        case QDB_INT8: return launch_filter_ab<A, int8_t>(op, a_col, a, b_col, b, nulls, out, n, s);
        case QDB_INT32: return launch_filter_ab<A, int32_t>(op, a_col, a, b_col, b, nulls, out, n, s);
        case QDB_INT64: return launch_filter_ab<A, int64_t>(op, a_col, a, b_col, b, nulls, out, n, s);
        case QDB_FLOAT: return launch_filter_ab<A, float>(op, a_col, a, b_col, b, nulls, out, n, s);
        case QDB_DOUBLE: return launch_filter_ab<A, double>(op, a_col, a, b_col, b, nulls, out, n, s);
        default: return fail(QDB_ERR_INVALID, "qdb_filter: unsupported right operand type");
    }
}

template <typename A, typename B>
static bool host_cmp(int32_t op, const void* a, const void* b) {
    const A x = host_value<A>(a);
    const B y = host_value<B>(b);
    switch (op) {
        case QDB_GREATER: return x > y;
        case QDB_GREATER_EQUAL: return x >= y;
        case QDB_LESS: return x < y;
        case QDB_LESS_EQUAL: return x <= y;
        case QDB_EQUAL: return x == y;
        case QDB_NOT_EQUAL: return x != y;
        case QDB_LOGICAL_AND: return x && y;
        case QDB_LOGICAL_OR: return x || y;
        default: return false;
    }
}

template <typename A>
static int host_cmp_a(int32_t op, const void* a, int32_t b_type, const void* b) {
    switch (b_type) {
        case QDB_INT8: return host_cmp<A, int8_t>(op, a, b);
        case QDB_INT32: return host_cmp<A, int32_t>(op, a, b);
        case QDB_INT64: return host_cmp<A, int64_t>(op, a, b);
        case QDB_FLOAT: return host_cmp<A, float>(op, a, b);
        case QDB_DOUBLE: return host_cmp<A, double>(op, a, b);
        default: return -1;
    }
}

}  // namespace qdb

using namespace qdb;

extern "C" int32_t qdb_filter(int32_t op, int32_t a_type, int32_t a_is_col, const void* a, int32_t b_type,
                              int32_t b_is_col, const void* b, const uint64_t* null_mask, int8_t* out_mask, int64_t n,
                              void* stream) {
    if (op < QDB_GREATER || op > QDB_LOGICAL_OR) return fail(QDB_ERR_INVALID, "qdb_filter: unknown operator");
    if (n < 0 || !a || !b || (n > 0 && !out_mask)) return fail(QDB_ERR_INVALID, "qdb_filter: bad arguments");
    if (n == 0) return QDB_OK;
    cudaStream_t s = as_stream(stream);
    if (!a_is_col && !b_is_col) {
        // Constant-constant: the whole mask is one value (GPUBinary.cuh:573-575).
        int r;
        switch (a_type) {
            case QDB_INT8: r = host_cmp_a<int8_t>(op, a, b_type, b); break;
            case QDB_INT32: r = host_cmp_a<int32_t>(op, a, b_type, b); break;
            case QDB_INT64: r = host_cmp_a<int64_t>(op, a, b_type, b); break;
            case QDB_FLOAT: r = host_cmp_a<float>(op, a, b_type, b); break;
            case QDB_DOUBLE: r = host_cmp_a<double>(op, a, b_type, b); break;
            default: r = -1;
        }
        if (r < 0) return fail(QDB_ERR_INVALID, "qdb_filter: unsupported operand type");
        QDB_CUDA_TRY(cudaMemsetAsync(out_mask, r, n, s));
        return QDB_OK;
    }
    switch (a_type) {
        case QDB_INT8: return launch_filter_a<int8_t>(op, a_is_col, a, b_type, b_is_col, b, null_mask, out_mask, n, s);
        case QDB_INT32: return launch_filter_a<int32_t>(op, a_is_col, a, b_type, b_is_col, b, null_mask, out_mask, n, s);
        case QDB_INT64: return launch_filter_a<int64_t>(op, a_is_col, a, b_type, b_is_col, b, null_mask, out_mask, n, s);
        case QDB_FLOAT: return launch_filter_a<float>(op, a_is_col, a, b_type, b_is_col, b, null_mask, out_mask, n, s);
        case QDB_DOUBLE: return launch_filter_a<double>(op, a_is_col, a, b_type, b_is_col, b, null_mask, out_mask, n, s);
        default: return fail(QDB_ERR_INVALID, "qdb_filter: unsupported left operand type");
    }
}

namespace qdb {

// out[i] = in[i] % m (the C++ remainder): the expression column `key % m` that the dispatcher materialises with
// GPUBinary<ArithmeticOperations::mod, T, T*, T> before a GROUP BY over it (GPUBinary.cuh:145-166).
// The remainder uses the multiply-high form of the division by the invariant |m| (mod_signed, qdb_common.cuh);
// a % m == a % |m| for C++'s truncating division.
template <typename T, typename O = T>
__global__ void mod_kernel(const T* __restrict__ in, ModMagic mm, O* __restrict__ out, int64_t n) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        out[i] = static_cast<O>(mod_signed(static_cast<int64_t>(in[i]), mm.d, mm.m, mm.s1, mm.s2));
}

// Four consecutive elements through 16-byte accesses (the pointer is 16-byte aligned).
__device__ __forceinline__ void ld4(const int32_t* p, int64_t (&x)[4]) {
    const int4 v = __ldcs(reinterpret_cast<const int4*>(p));
    x[0] = v.x;
    x[1] = v.y;
    x[2] = v.z;
    x[3] = v.w;
}
__device__ __forceinline__ void ld4(const int64_t* p, int64_t (&x)[4]) {
    const longlong2 a = __ldcs(reinterpret_cast<const longlong2*>(p));
    const longlong2 b = __ldcs(reinterpret_cast<const longlong2*>(p) + 1);
    x[0] = a.x;
    x[1] = a.y;
    x[2] = b.x;
    x[3] = b.y;
}
__device__ __forceinline__ void st4(int32_t* p, const int64_t (&y)[4]) {
    *reinterpret_cast<int4*>(p) = make_int4(static_cast<int>(y[0]), static_cast<int>(y[1]), static_cast<int>(y[2]),
                                            static_cast<int>(y[3]));
}
__device__ __forceinline__ void st4(int64_t* p, const int64_t (&y)[4]) {
    reinterpret_cast<longlong2*>(p)[0] = make_longlong2(y[0], y[1]);
    reinterpret_cast<longlong2*>(p)[1] = make_longlong2(y[2], y[3]);
}

// The same remainder, four rows per thread and step with 16-byte loads and stores (both columns 16-byte aligned);
// block 0 takes the last n % 4 rows.
template <typename T, typename O>
__global__ void mod4_kernel(const T* __restrict__ in, ModMagic mm, O* __restrict__ out, int64_t n) {
    const int64_t n4 = n >> 2;
    for (int64_t g = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; g < n4;
         g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        int64_t x[4];
        ld4(in + 4 * g, x);
#pragma unroll
        for (int j = 0; j < 4; ++j) x[j] = mod_signed(x[j], mm.d, mm.m, mm.s1, mm.s2);
        st4(out + 4 * g, x);
    }
    if (blockIdx.x == 0 && threadIdx.x < static_cast<unsigned>(n & 3)) {
        const int64_t i = 4 * n4 + threadIdx.x;
        out[i] = static_cast<O>(mod_signed(static_cast<int64_t>(in[i]), mm.d, mm.m, mm.s1, mm.s2));
    }
}

// in % m into out: the vector form when both columns are 16-byte aligned, the scalar one otherwise.
template <typename T, typename O>
static int32_t launch_mod(const T* in, const ModMagic& mm, O* out, int64_t n, cudaStream_t s) {
    const DeviceInfo& di = device_info();
    const bool vec = ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15u) == 0;
    const int64_t units = vec ? std::max<int64_t>(1, n / 4) : n;
    const unsigned grid = static_cast<unsigned>(std::min<int64_t>((units + 255) / 256, int64_t(di.sm_count) * 16));
    if (vec) mod4_kernel<T, O><<<grid, 256, 0, s>>>(in, mm, out, n);
    else mod_kernel<T, O><<<grid, 256, 0, s>>>(in, mm, out, n);
    note_launch();
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? QDB_OK : cuda_fail(e, "mod_kernel");
}

}  // namespace qdb

extern "C" int32_t qdb_arith_mod(int32_t type, const void* in, int64_t modulus, void* out, int64_t n, void* stream) {
    using namespace qdb;
    if (n < 0 || (n > 0 && (!in || !out))) return fail(QDB_ERR_INVALID, "qdb_arith_mod: bad arguments");
    if (modulus == 0) return fail(QDB_DIVISION_BY_ZERO, "qdb_arith_mod: modulo by zero");
    if (n == 0) return QDB_OK;
    cudaStream_t s = as_stream(stream);
    if (modulus == INT64_MIN) return fail(QDB_ERR_INVALID, "qdb_arith_mod: modulus out of range");
    const ModMagic mm = mod_magic(static_cast<uint64_t>(modulus < 0 ? -modulus : modulus));
    if (type == QDB_INT32) {
        if (modulus > INT32_MAX || modulus < INT32_MIN)
            return fail(QDB_ERR_INVALID, "qdb_arith_mod: modulus out of int32 range");
        return launch_mod<int32_t, int32_t>(static_cast<const int32_t*>(in), mm, static_cast<int32_t*>(out), n, s);
    }
    if (type == QDB_INT64)
        return launch_mod<int64_t, int64_t>(static_cast<const int64_t*>(in), mm, static_cast<int64_t*>(out), n, s);
    return fail(QDB_ERR_INVALID, "qdb_arith_mod: column must be INT32 or INT64");
}
