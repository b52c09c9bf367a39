// Shared device/host helpers of the B200 GROUP BY path: status handling, key canonicalisation,
// hashing, value encodings and streaming loads.
#pragma once

#include <cstdint>
#include <cstring>
#include <type_traits>
#include <string>
#include <cuda_runtime.h>

#include "../../include/qdb_gb.h"

namespace qdb {

// ---------------------------------------------------------------------------------------------
// Error plumbing (host).  The C ABI returns codes; the message of the last failure is kept per
// thread so that a caller can fetch it with qdb_last_error().
// ---------------------------------------------------------------------------------------------
void set_last_error(const std::string& msg);
int32_t fail(int32_t code, const std::string& msg);
int32_t cuda_fail(cudaError_t err, const char* what);

#define QDB_CUDA_TRY(expr)                                   \
    do {                                                     \
        cudaError_t _e = (expr);                             \
        if (_e != cudaSuccess) return ::qdb::cuda_fail(_e, #expr); \
    } while (0)

// Device properties of the current device (cached per device ordinal).
struct DeviceInfo {
    int device = -1;
    int sm_count = 148;
    int max_smem_optin = 227 * 1024;
    int l2_bytes = 126 * 1024 * 1024;
};
const DeviceInfo& device_info();

// Counts this library's kernel launches (reported by qdb_launch_count()).
void note_launch(int64_t n = 1);

// Stream-ordered allocation helpers (the pool keeps freed blocks for reuse).
int32_t dev_alloc(void** p, size_t bytes, cudaStream_t s);
void dev_free(void* p, cudaStream_t s);

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

inline int type_size(int32_t t) {
    switch (t) {
        case QDB_INT32: return 4;
        case QDB_INT64: return 8;
        case QDB_FLOAT: return 4;
        case QDB_DOUBLE: return 8;
        case QDB_INT8: return 1;
        default: return 0;
    }
}

// ---------------------------------------------------------------------------------------------
// Table key words.  Every key is held as one 64-bit word.  kEmpty marks a free slot; the one real
// key that collides with it (INT64_MIN, or the composite (INT32_MIN, 0)) is routed to a dedicated
// "escape" slot, so every key value is representable (the reference reserves lowest(K) as its empty
// marker and cannot store that key, qikkDB/QueryEngine/GPUCore/GPUGroupBy.cuh:24-30).
// ---------------------------------------------------------------------------------------------
constexpr uint64_t kEmpty = 0x8000000000000000ull;

// Canonical key words.  Floating-point keys use their bit pattern with -0.0 folded onto +0.0 and every
// NaN folded onto one quiet NaN, so keys that compare equal share one group.
__host__ __device__ __forceinline__ uint64_t key_word(int32_t k) {
    return static_cast<uint64_t>(static_cast<int64_t>(k));
}
__host__ __device__ __forceinline__ uint64_t key_word(int64_t k) { return static_cast<uint64_t>(k); }
__host__ __device__ __forceinline__ uint64_t key_word(float k) {
    uint32_t b;
    memcpy(&b, &k, 4);
    if ((b & 0x7fffffffu) == 0u) b = 0u;
    else if ((b & 0x7f800000u) == 0x7f800000u && (b & 0x007fffffu)) b = 0x7fc00000u;
    return static_cast<uint64_t>(b);
}
__host__ __device__ __forceinline__ uint64_t key_word(double k) {
    uint64_t b;
    memcpy(&b, &k, 8);
    if ((b & 0x7fffffffffffffffull) == 0ull) b = 0ull;
    else if ((b & 0x7ff0000000000000ull) == 0x7ff0000000000000ull && (b & 0x000fffffffffffffull))
        b = 0x7ff8000000000000ull;
    return b;
}
__host__ __device__ __forceinline__ uint64_t composite_word(int32_t a, int32_t b) {
    return (static_cast<uint64_t>(static_cast<uint32_t>(a)) << 32) | static_cast<uint32_t>(b);
}

// 64-bit finaliser of MurmurHash3 (Austin Appleby, public domain): a bijective avalanche mix.
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return k;
}

// ---------------------------------------------------------------------------------------------
// Remainder by an invariant divisor with one multiply-high: the unsigned division of Granlund and Montgomery,
// "Division by Invariant Integers using Multiplication" (PLDI 1994), Figure 4.1 with N = 64.  For a divisor
// 1 <= d < 2^63: l = ceil(log2 d), m = floor(2^64 (2^l - d) / d) + 1, and for every n < 2^64
// q = (t + ((n - t) >> min(l, 1))) >> max(l - 1, 0) with t = mulhi(m, n).  The signed remainder follows C++
// (the sign of the dividend), as GPUBinary's `a % b`.
// ---------------------------------------------------------------------------------------------
struct ModMagic {
    uint64_t d = 1;
    uint64_t m = 1;
    int32_t s1 = 0;
    int32_t s2 = 0;
};

inline ModMagic mod_magic(uint64_t d) {
    ModMagic mm;
    mm.d = d;
    int l = 0;
    while (l < 63 && (uint64_t(1) << l) < d) ++l;
    const unsigned __int128 num = static_cast<unsigned __int128>((uint64_t(1) << l) - d) << 64;
    mm.m = static_cast<uint64_t>(num / d) + 1;
    mm.s1 = l < 1 ? l : 1;
    mm.s2 = l > 1 ? l - 1 : 0;
    return mm;
}

__host__ __device__ __forceinline__ uint64_t mulhi_u64(uint64_t a, uint64_t b) {
#ifdef __CUDA_ARCH__
    return __umul64hi(a, b);
#else
    return static_cast<uint64_t>((static_cast<unsigned __int128>(a) * b) >> 64);
#endif
}

__host__ __device__ __forceinline__ int64_t mod_signed(int64_t k, uint64_t d, uint64_t m, int s1, int s2) {
    const uint64_t u = k >= 0 ? static_cast<uint64_t>(k) : 0ull - static_cast<uint64_t>(k);
    const uint64_t t = mulhi_u64(m, u);
    const uint64_t q = (t + ((u - t) >> s1)) >> s2;
    const uint64_t r = u - q * d;
    return k >= 0 ? static_cast<int64_t>(r) : -static_cast<int64_t>(r);
}

// ---------------------------------------------------------------------------------------------
// Order-preserving integer encodings of IEEE floats, so MIN/MAX use native signed-integer atomics.
// enc(x) < enc(y) iff x < y for non-NaN x, y (with -0.0 < +0.0).  The map is an involution.
// ---------------------------------------------------------------------------------------------
__host__ __device__ __forceinline__ int32_t fenc(float x) {
    int32_t b;
    memcpy(&b, &x, 4);
    return b ^ ((b >> 31) & 0x7fffffff);
}
__host__ __device__ __forceinline__ float fdec(int32_t e) {
    int32_t b = e ^ ((e >> 31) & 0x7fffffff);
    float x;
    memcpy(&x, &b, 4);
    return x;
}
__host__ __device__ __forceinline__ int64_t denc(double x) {
    int64_t b;
    memcpy(&b, &x, 8);
    return b ^ ((b >> 63) & 0x7fffffffffffffffll);
}
__host__ __device__ __forceinline__ double ddec(int64_t e) {
    int64_t b = e ^ ((e >> 63) & 0x7fffffffffffffffll);
    double x;
    memcpy(&x, &b, 8);
    return x;
}

// ---------------------------------------------------------------------------------------------
// Streaming loads: evict-first so that the column stream does not push the hash table out of L2.
// ---------------------------------------------------------------------------------------------
#ifdef __CUDACC__
__device__ __forceinline__ int4 ld_stream16(const void* p) { return __ldcs(reinterpret_cast<const int4*>(p)); }
__device__ __forceinline__ uint32_t ld_stream4(const void* p) {
    return static_cast<uint32_t>(__ldcs(reinterpret_cast<const int*>(p)));
}
__device__ __forceinline__ uint64_t ld_volatile_u64(const uint64_t* p) {
    return *reinterpret_cast<const volatile uint64_t*>(p);
}
__device__ __forceinline__ int32_t ld_volatile_i32(const int32_t* p) {
    return *reinterpret_cast<const volatile int32_t*>(p);
}
__device__ __forceinline__ bool null_bit(const uint64_t* mask, int64_t i) {
    return mask != nullptr && ((__ldg(reinterpret_cast<const unsigned long long*>(mask) + (i >> 6)) >> (i & 63)) & 1ull);
}
#endif

}  // namespace qdb
