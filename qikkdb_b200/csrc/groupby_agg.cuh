// The fused filter + hash-aggregate pass (the B200 replacement of kernel_filter ->
// reconstructColKeep -> group_by_kernel, qikkDB/QueryEngine/GPUCore/GPUFilter.cuh:22-44,
// GPUReconstruct.cuh:29-45 and :272-355, GPUGroupBy.cuh:68-196).
//
// One persistent CTA per SM, warp-specialised:
//   * a producer warp streams the CTA's tiles of every input column (keys, values, predicate column,
//     mask, null words) from HBM into a ring of shared-memory stages with bulk asynchronous copies
//     (cp.async.bulk, executed by the TMA engine) that complete on per-stage mbarriers;
//   * 30 consumer warps take the stages in order.  For every row they evaluate the predicate as an
//     interval test in the column's own type (the host turns `col OP constant` into [lo, hi] plus an
//     invert flag, so the test is two compares and no branch), read the key, and insert it
//       - first into a per-CTA shared-memory table (bounded linear probe, shared-memory atomics), which
//         absorbs low-cardinality and skewed (Zipf) key streams,
//       - on a miss, into the global open-addressing table (bounded linear probe, 64-bit atomicCAS on the
//         key word, fire-and-forget reductions on the state words).  Misses are queued per warp and
//         inserted 32 at a time with every lane active, so 32 probe loads of a warp are in flight together;
//     then release the stage to the producer.  No mask or compacted column is written to HBM.
// A warp that sees a low shared-memory hit rate after its first tiles stops probing shared memory.
// At the end each CTA merges its shared-memory table into the global table.
// Every wait on an mbarrier is bounded; a wait that gives up records QDB_ERR_TIMEOUT in the table status.
#pragma once

#include <climits>

#include "groupby.cuh"

namespace qdb {

constexpr int kConsumerWarps = 30;
constexpr int kConsumerThreads = kConsumerWarps * 32;     // 960
constexpr int kAggThreads = kConsumerThreads + 32;         // + one producer warp: 992 threads
constexpr int kRowsPerWarpUnit = 64;                       // a tile is kConsumerWarps * R rows, R a multiple of 64
constexpr int kQueueCap = 64;                              // per-warp queue of shared-memory misses
constexpr int kDecideTile = 3;                             // tile index at which a warp judges its hit rate
constexpr uint32_t kMaxWaitIters = 1u << 24;               // bounded mbarrier waits (seconds, then give up)

// `col OP constant` as an interval of the column type: keep = (lo <= x && x <= hi) != invert.
struct PredInterval {
    int64_t lo = 0;     // bit pattern of the bound in the column type (floats: the IEEE bits)
    int64_t hi = 0;
    int32_t invert = 0;
};

// Byte offsets of the columns inside one shared-memory stage (-1 = absent).
struct StageLayout {
    int32_t key0 = -1, key1 = -1, val = -1, pred = -1, mask = -1;
    int32_t knull0 = -1, knull1 = -1, vnull = -1, pnull = -1;
    int32_t bytes = 0;  // stage size (multiple of 128)
};

struct AggArgs {
    const void* key0 = nullptr;
    const void* key1 = nullptr;
    const uint64_t* knull0 = nullptr;
    const uint64_t* knull1 = nullptr;
    const void* vals = nullptr;
    const uint64_t* vnull = nullptr;
    const void* pcol = nullptr;
    const uint64_t* pnull = nullptr;
    PredInterval pi;
    const int8_t* mask = nullptr;
    int64_t n = 0;
    int32_t T = 1920;        // rows per tile: kConsumerWarps * R with R a multiple of 64
    int32_t NS = 3;          // stages in the ring
    int64_t tiles = 0;       // all tiles, the last one possibly partial
    int64_t full_tiles = 0;  // tiles with T rows
    int32_t staged = 0;      // 1: full tiles arrive by bulk copy; 0: every tile is read directly from HBM
    StageLayout sl;
    Region main;
    Region aux;
    Layout L;
    int32_t has_sum = 0;
    int32_t has_min = 0;
    int32_t has_max = 0;
    unsigned long long* counters = nullptr;  // [0] groups, [1] status
    unsigned long long capacity = 0;
    int32_t S = 0;       // shared-memory hash slots (power of two) or 0 for a global-only pass
    int32_t probe = 0;   // shared-memory probe limit
    // byte offsets inside dynamic shared memory
    int32_t so_stage = 0, so_bar = 0, so_list = 0, so_queue = 0;
    int32_t so_sum = 0, so_mn = 0, so_mx = 0, so_cnt = 0;  // hash arrays (keys at offset 0), S + 2 entries each
};

template <typename A, typename B>
__host__ __device__ __forceinline__ bool cmp_op(int32_t op, A a, B b) {
    switch (op) {
        case QDB_GREATER: return a > b;
        case QDB_GREATER_EQUAL: return a >= b;
        case QDB_LESS: return a < b;
        case QDB_LESS_EQUAL: return a <= b;
        case QDB_EQUAL: return a == b;
        case QDB_NOT_EQUAL: return a != b;
        case QDB_LOGICAL_AND: return a && b;
        case QDB_LOGICAL_OR: return a || b;
        default: return false;
    }
}

struct NoPred {};

template <typename T>
__host__ __device__ __forceinline__ T from_bits(int64_t b) {
    T v;
    if constexpr (sizeof(T) == 4) {
        const int32_t w = static_cast<int32_t>(b);
        memcpy(&v, &w, 4);
    } else {
        memcpy(&v, &b, 8);
    }
    return v;
}

// 4-row vector loads (used by the standalone filter kernel).  Row r0 is a multiple of 4; `full` means
// rows r0..r0+3 are all < n and the pointer is 16-byte aligned.
template <typename T>
__device__ __forceinline__ void load4(const T* __restrict__ p, int64_t r0, int64_t n, bool full, T (&out)[4]) {
    if (full) {
        if constexpr (sizeof(T) == 4) {
            int4 q = ld_stream16(p + r0);
            memcpy(&out[0], &q.x, 4);
            memcpy(&out[1], &q.y, 4);
            memcpy(&out[2], &q.z, 4);
            memcpy(&out[3], &q.w, 4);
        } else if constexpr (sizeof(T) == 8) {
            int4 q0 = ld_stream16(p + r0);
            int4 q1 = ld_stream16(p + r0 + 2);
            memcpy(&out[0], &q0.x, 8);
            memcpy(&out[1], &q0.z, 8);
            memcpy(&out[2], &q1.x, 8);
            memcpy(&out[3], &q1.z, 8);
        } else {
            uint32_t q = ld_stream4(p + r0);
            memcpy(&out[0], &q, 4);
        }
    } else {
#pragma unroll
        for (int e = 0; e < 4; ++e) out[e] = (r0 + e < n) ? p[r0 + e] : T{};
    }
}

// ---------------------------------------------------------------------------------------------
// mbarrier and bulk-copy primitives (PTX ISA: mbarrier, cp.async.bulk).
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Waits for phase `parity` of `bar`; gives up after kMaxWaitIters tries and records QDB_ERR_TIMEOUT.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, unsigned long long* counters) {
    for (uint32_t it = 0; it < kMaxWaitIters; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if (it >= 16) __nanosleep(128);
    }
    atomicExch(reinterpret_cast<int*>(&counters[1]), static_cast<int>(QDB_ERR_TIMEOUT));
    return false;
}
// L2 policy for data read once: evict first, so the column stream does not push the hash table out of L2.
__device__ __forceinline__ uint64_t l2_evict_first_policy() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar, uint64_t pol) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::
            "r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(pol)
        : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// ---------------------------------------------------------------------------------------------
// Value state updates.
// ---------------------------------------------------------------------------------------------
template <typename VT>
__device__ __forceinline__ int32_t enc32(VT v) {
    if constexpr (std::is_same<VT, float>::value) return fenc(v);
    else return static_cast<int32_t>(v);
}
template <typename VT>
__device__ __forceinline__ long long enc64(VT v) {
    if constexpr (std::is_same<VT, double>::value) return static_cast<long long>(denc(v));
    else return static_cast<long long>(v);
}

// New groups are counted in a per-CTA shared-memory counter (a single global counter hit by every new
// key would serialise in L2); each CTA publishes its count once with publish_claims, which raises
// HASH_TABLE_FULL when the total passes the capacity.
__device__ __forceinline__ void claim_counted(unsigned long long* claims) { atomicAdd(claims, 1ull); }

__device__ __forceinline__ void publish_claims(unsigned long long* counters, unsigned long long capacity,
                                               unsigned long long claims) {
    if (claims == 0) return;
    if (atomicAdd(&counters[0], claims) + claims > capacity)
        atomicExch(reinterpret_cast<int*>(&counters[1]), static_cast<int>(QDB_HASH_TABLE_FULL));
}

__device__ __forceinline__ bool table_full(const unsigned long long* counters) {
    return ld_volatile_i32(reinterpret_cast<const int32_t*>(&counters[1])) == QDB_HASH_TABLE_FULL;
}

// Finds or claims `key` in region R starting at slot s whose key word `cur` was already loaded.
// The probe visits at most every slot once, so it always ends; it gives up (returns nullptr) when the
// region is full or another thread has already reported HASH_TABLE_FULL.
__device__ __forceinline__ uint64_t* g_find_from(const Region& R, int W, uint64_t key, uint64_t s, uint64_t cur,
                                                 unsigned long long* counters, unsigned long long* claims) {
    for (uint64_t i = 0; i <= R.mask; ++i) {
        uint64_t* slot = R.slots + s * W;
        if (i > 0) cur = ld_volatile_u64(slot);
        if (cur == key) return slot;
        if (cur == kEmpty) {
            unsigned long long prev = atomicCAS(reinterpret_cast<unsigned long long*>(slot), kEmpty, key);
            if (prev == kEmpty) {
                claim_counted(claims);
                return slot;
            }
            if (prev == key) return slot;
        }
        s = (s + 1) & R.mask;
        if ((i & 63) == 63 && table_full(counters)) return nullptr;
    }
    atomicExch(reinterpret_cast<int*>(&counters[1]), static_cast<int>(QDB_HASH_TABLE_FULL));
    return nullptr;
}

__device__ __forceinline__ uint64_t* g_find(const Region& R, int W, uint64_t key, uint64_t h,
                                            unsigned long long* counters, unsigned long long* claims) {
    const uint64_t s = h & R.mask;
    return g_find_from(R, W, key, s, ld_volatile_u64(R.slots + s * W), counters, claims);
}

// Special slot `which` (0: NULL key, 1: the key equal to kEmpty) of the main region.
__device__ __forceinline__ uint64_t* g_special(const Region& R, int W, int which, unsigned long long* claims) {
    uint64_t* slot = R.slots + (R.mask + 1 + which) * W;
    if (ld_volatile_u64(slot) == kEmpty) {
        unsigned long long prev = atomicCAS(reinterpret_cast<unsigned long long*>(slot), kEmpty, 0ull);
        if (prev == kEmpty && which == 1) claim_counted(claims);
    }
    return slot;
}

// One row's value into a global slot.
template <typename VT>
__device__ __forceinline__ void g_acc_row(uint64_t* slot, const AggArgs& a, VT v) {
    atomicAdd(reinterpret_cast<unsigned long long*>(slot + a.L.cnt), 1ull);
    if (a.has_sum) {
        if constexpr (std::is_floating_point<VT>::value)
            atomicAdd(reinterpret_cast<double*>(slot + a.L.sum), static_cast<double>(v));
        else
            atomicAdd(reinterpret_cast<unsigned long long*>(slot + a.L.sum),
                      static_cast<unsigned long long>(static_cast<long long>(v)));
    }
    if constexpr (sizeof(VT) == 4) {
        const int32_t e = enc32(v);
        if (a.has_min) atomicMin(reinterpret_cast<int*>(slot + a.L.mn), e);
        if (a.has_max) atomicMax(reinterpret_cast<int*>(slot + a.L.mx) + 1, e);
    } else {
        const long long e = enc64(v);
        if (a.has_min) atomicMin(reinterpret_cast<long long*>(slot + a.L.mn), e);
        if (a.has_max) atomicMax(reinterpret_cast<long long*>(slot + a.L.mx), e);
    }
}

// A row of a table without a value column: only the row count.
__device__ __forceinline__ void g_count_row(uint64_t* slot, const Layout& L) {
    if (L.cnt >= 0) atomicAdd(reinterpret_cast<unsigned long long*>(slot + L.cnt), 1ull);
}

// Merges a partial state (cnt, sum bits, encoded min, encoded max) into a global slot.
__device__ __forceinline__ void g_merge(uint64_t* slot, const Layout& L, bool has_sum, bool has_min, bool has_max,
                                        bool v32, bool vfloat, unsigned long long c, uint64_t sumbits,
                                        long long mn, long long mx) {
    if (c == 0 || L.cnt < 0) return;
    atomicAdd(reinterpret_cast<unsigned long long*>(slot + L.cnt), c);
    if (has_sum) {
        if (vfloat) {
            double d;
            memcpy(&d, &sumbits, 8);
            atomicAdd(reinterpret_cast<double*>(slot + L.sum), d);
        } else {
            atomicAdd(reinterpret_cast<unsigned long long*>(slot + L.sum), static_cast<unsigned long long>(sumbits));
        }
    }
    if (v32) {
        if (has_min) atomicMin(reinterpret_cast<int*>(slot + L.mn), static_cast<int>(mn));
        if (has_max) atomicMax(reinterpret_cast<int*>(slot + L.mx) + 1, static_cast<int>(mx));
    } else {
        if (has_min) atomicMin(reinterpret_cast<long long*>(slot + L.mn), mn);
        if (has_max) atomicMax(reinterpret_cast<long long*>(slot + L.mx), mx);
    }
}

// Slot index hash of the shared-memory table: Fibonacci hashing of the folded 64-bit key word
// (multiplicative hashing, Knuth TAOCP vol. 3, 6.4), keeping the top log2(S) bits.
__device__ __forceinline__ uint32_t smem_hash(uint64_t kw, int shift) {
    const uint32_t f = static_cast<uint32_t>(kw) ^ static_cast<uint32_t>(kw >> 32);
    return (f * 0x9e3779b1u) >> shift;
}

// Shared-memory probe.  Returns the slot, or -1 after `P` probes.  *found is set when the key was
// already present (a reuse rather than a first claim).
__device__ __forceinline__ int s_find(uint64_t* skey, int S, int P, uint64_t key, uint32_t h, bool* found) {
    uint32_t s = h & static_cast<uint32_t>(S - 1);
    for (int p = 0; p < P; ++p) {
        const uint64_t cur = *reinterpret_cast<volatile uint64_t*>(&skey[s]);
        if (cur == key) {
            *found = true;
            return static_cast<int>(s);
        }
        if (cur == kEmpty) {
            const unsigned long long prev =
                atomicCAS(reinterpret_cast<unsigned long long*>(&skey[s]), kEmpty, key);
            if (prev == kEmpty) return static_cast<int>(s);
            if (prev == key) {
                *found = true;
                return static_cast<int>(s);
            }
        }
        s = (s + 1) & static_cast<uint32_t>(S - 1);
    }
    return -1;
}

template <typename VT>
__device__ __forceinline__ void s_acc_row(unsigned char* sm, const AggArgs& a, int s, VT v, bool has_val) {
    atomicAdd(reinterpret_cast<unsigned int*>(sm + a.so_cnt) + s, 1u);
    if (!has_val) return;
    if (a.has_sum) {
        if constexpr (std::is_floating_point<VT>::value)
            atomicAdd(reinterpret_cast<double*>(sm + a.so_sum) + s, static_cast<double>(v));
        else
            atomicAdd(reinterpret_cast<unsigned long long*>(sm + a.so_sum) + s,
                      static_cast<unsigned long long>(static_cast<long long>(v)));
    }
    if constexpr (sizeof(VT) == 4) {
        const int32_t e = enc32(v);
        if (a.has_min) atomicMin(reinterpret_cast<int*>(sm + a.so_mn) + 2 * s, e);
        if (a.has_max) atomicMax(reinterpret_cast<int*>(sm + a.so_mx) + 2 * s + 1, e);
    } else {
        const long long e = enc64(v);
        if (a.has_min) atomicMin(reinterpret_cast<long long*>(sm + a.so_mn) + s, e);
        if (a.has_max) atomicMax(reinterpret_cast<long long*>(sm + a.so_mx) + s, e);
    }
}

// Register accumulation helpers: the running sum of a group of rows (FP64 for float values, wrapping int64 for
// integer values) and the order-preserving MIN/MAX encoding.
template <typename VT>
using AccOf = typename std::conditional<std::is_floating_point<VT>::value, double, long long>::type;

template <typename VT>
__device__ __forceinline__ AccOf<VT> to_acc(VT v) {
    return static_cast<AccOf<VT>>(v);
}

template <typename VT>
__device__ __forceinline__ long long enc_any(VT v) {
    if constexpr (sizeof(VT) == 4) return enc32(v);
    else return enc64(v);
}

// Merges c rows with sum `acc` and encoded min/max into shared slot s.
template <typename VT>
__device__ __forceinline__ void s_merge_acc(unsigned char* sm, const AggArgs& a, int s, unsigned c, AccOf<VT> acc,
                                            long long mn, long long mx, bool has_val) {
    atomicAdd(reinterpret_cast<unsigned int*>(sm + a.so_cnt) + s, c);
    if (!has_val) return;
    if (a.has_sum) {
        if constexpr (std::is_floating_point<VT>::value)
            atomicAdd(reinterpret_cast<double*>(sm + a.so_sum) + s, acc);
        else
            atomicAdd(reinterpret_cast<unsigned long long*>(sm + a.so_sum) + s, static_cast<unsigned long long>(acc));
    }
    if constexpr (sizeof(VT) == 4) {
        if (a.has_min) atomicMin(reinterpret_cast<int*>(sm + a.so_mn) + 2 * s, static_cast<int>(mn));
        if (a.has_max) atomicMax(reinterpret_cast<int*>(sm + a.so_mx) + 2 * s + 1, static_cast<int>(mx));
    } else {
        if (a.has_min) atomicMin(reinterpret_cast<long long*>(sm + a.so_mn) + s, mn);
        if (a.has_max) atomicMax(reinterpret_cast<long long*>(sm + a.so_mx) + s, mx);
    }
}

// ---------------------------------------------------------------------------------------------
// The aggregation kernel.  KT: key column type; COMP: composite (int32, int32) key; VT: value type
// (int32_t when the table has no value column); PT: predicate column type or NoPred; NULLS: some null
// mask (key, value or predicate) is present.
// ---------------------------------------------------------------------------------------------
template <typename KT, bool COMP, typename VT, typename PT, bool NULLS>
__global__ void __launch_bounds__(kAggThreads, 1) gb_agg_kernel(const AggArgs a) {
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ unsigned long long s_claims;
    constexpr bool HAS_PRED = !std::is_same<PT, NoPred>::value;
    using PL = typename std::conditional<HAS_PRED, PT, int32_t>::type;
    using AccT = AccOf<VT>;

    const int S = a.S;
    const int S2 = S ? S + 2 : 0;
    uint64_t* skey = reinterpret_cast<uint64_t*>(sm);
    uint64_t* full_bar = reinterpret_cast<uint64_t*>(sm + a.so_bar);
    uint64_t* empty_bar = full_bar + a.NS;
    const bool has_mm = a.has_min || a.has_max;
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;

    for (int i = threadIdx.x; i < S2; i += blockDim.x) {
        skey[i] = kEmpty;
        reinterpret_cast<unsigned int*>(sm + a.so_cnt)[i] = 0u;
        if (a.has_sum) reinterpret_cast<unsigned long long*>(sm + a.so_sum)[i] = 0ull;
        if (has_mm) {
            if (sizeof(VT) == 4) {
                reinterpret_cast<unsigned long long*>(sm + a.so_mn)[i] = kPackedMinMaxInit;
            } else {
                reinterpret_cast<unsigned long long*>(sm + a.so_mn)[i] = kMinInit64;
                reinterpret_cast<unsigned long long*>(sm + a.so_mx)[i] = kMaxInit64;
            }
        }
    }
    if (threadIdx.x == 0) s_claims = 0;
    if (threadIdx.x == 0 && a.staged) {
        for (int s = 0; s < a.NS; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], kConsumerWarps);
        }
        mbar_fence_init();
    }
    __syncthreads();

    const int64_t my_tiles =
        (a.tiles > static_cast<int64_t>(blockIdx.x)) ? (a.tiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
    const int W = a.L.W;
    const int T = a.T;

    if (warp == kConsumerWarps) {
        // ---------------- producer warp: one elected lane issues the bulk copies ----------------
        if (lane == 0 && a.staged) {
            const StageLayout& sl = a.sl;
            const uint64_t pol = l2_evict_first_policy();
            int64_t q = 0;
            for (; q < my_tiles; ++q) {
                const int64_t tile = blockIdx.x + q * static_cast<int64_t>(gridDim.x);
                if (tile >= a.full_tiles) break;  // the partial last tile is read directly
                const int s = static_cast<int>(q % a.NS);
                if (q >= a.NS && !mbar_wait(&empty_bar[s], static_cast<uint32_t>((q / a.NS - 1) & 1), a.counters))
                    break;
                unsigned char* st = sm + a.so_stage + static_cast<size_t>(s) * sl.bytes;
                const int64_t r0 = tile * T;
                const uint32_t words = static_cast<uint32_t>(T / 64) * 8u;
                uint32_t tx = static_cast<uint32_t>(T) * sizeof(KT) * (COMP ? 2 : 1);
                if (sl.val >= 0) tx += static_cast<uint32_t>(T) * sizeof(VT);
                if (sl.pred >= 0) tx += static_cast<uint32_t>(T) * sizeof(PL);
                if (sl.mask >= 0) tx += static_cast<uint32_t>(T);
                tx += words * ((sl.knull0 >= 0) + (sl.knull1 >= 0) + (sl.vnull >= 0) + (sl.pnull >= 0));
                fence_proxy_async_smem();
                mbar_arrive_expect_tx(&full_bar[s], tx);
                bulk_g2s(st + sl.key0, static_cast<const KT*>(a.key0) + r0, T * sizeof(KT), &full_bar[s], pol);
                if (COMP) bulk_g2s(st + sl.key1, static_cast<const KT*>(a.key1) + r0, T * sizeof(KT), &full_bar[s], pol);
                if (sl.val >= 0) bulk_g2s(st + sl.val, static_cast<const VT*>(a.vals) + r0, T * sizeof(VT), &full_bar[s], pol);
                if (sl.pred >= 0) bulk_g2s(st + sl.pred, static_cast<const PL*>(a.pcol) + r0, T * sizeof(PL), &full_bar[s], pol);
                if (sl.mask >= 0) bulk_g2s(st + sl.mask, a.mask + r0, T, &full_bar[s], pol);
                if (sl.knull0 >= 0) bulk_g2s(st + sl.knull0, a.knull0 + r0 / 64, words, &full_bar[s], pol);
                if (sl.knull1 >= 0) bulk_g2s(st + sl.knull1, a.knull1 + r0 / 64, words, &full_bar[s], pol);
                if (sl.vnull >= 0) bulk_g2s(st + sl.vnull, a.vnull + r0 / 64, words, &full_bar[s], pol);
                if (sl.pnull >= 0) bulk_g2s(st + sl.pnull, a.pnull + r0 / 64, words, &full_bar[s], pol);
            }
            // Drain: every issued stage must have been consumed (so no copy is still in flight) before exit.
            for (int64_t d = (q > a.NS ? q - a.NS : 0); d < q; ++d) {
                const int s = static_cast<int>(d % a.NS);
                if (!mbar_wait(&empty_bar[s], static_cast<uint32_t>((d / a.NS) & 1), a.counters)) break;
            }
        }
    } else {
        // ---------------- consumer warps ----------------
        // Warp w owns rows [w*R, (w+1)*R) of every tile (R = T / kConsumerWarps).  Phase A evaluates the
        // predicate and mask for all of them and compacts the passing row indices into a per-warp list;
        // phase B inserts the passing rows with every lane busy.
        const bool has_vals = a.vals != nullptr;
        const PL plo = HAS_PRED ? from_bits<PL>(a.pi.lo) : PL{};
        const PL phi = HAS_PRED ? from_bits<PL>(a.pi.hi) : PL{};
        const bool pinv = a.pi.invert != 0;
        bool use_smem = S > 0;
        unsigned my_hits = 0, my_tries = 0;
        const int R = T / kConsumerWarps;
        uint16_t* list = reinterpret_cast<uint16_t*>(sm + a.so_list) + warp * R;
        const uint32_t lt_mask = (1u << lane) - 1u;
        const int smem_shift = 32 - (31 - __clz(S > 0 ? S : 1));
        // Per-warp queue of shared-memory misses (raw rows: key word, value bits, kind | agg flag).
        uint64_t* qkw = reinterpret_cast<uint64_t*>(sm + a.so_queue) + warp * kQueueCap;
        uint64_t* qval = reinterpret_cast<uint64_t*>(sm + a.so_queue) + (kConsumerWarps + warp) * kQueueCap;
        uint32_t* qmeta = reinterpret_cast<uint32_t*>(reinterpret_cast<uint64_t*>(sm + a.so_queue) +
                                                      2 * kConsumerWarps * kQueueCap) + warp * kQueueCap;
        int qn = 0;
        // Two hot keys per warp (the CTA's most frequent shared slots after the first tiles) with per-lane
        // register accumulators.  64-bit shared atomics serialise when many warps update one slot, so a skewed
        // key stream would otherwise queue on its hottest slots.
        uint64_t hk0 = kEmpty, hk1 = kEmpty;  // kEmpty never equals a NORMAL key word
        unsigned hc0 = 0, hc1 = 0;
        AccT ha0 = AccT{}, ha1 = AccT{};
        long long hmn0 = LLONG_MAX, hmx0 = LLONG_MIN, hmn1 = LLONG_MAX, hmx1 = LLONG_MIN;
        auto pick_hot_keys = [&]() {
            // warp-wide argmax of the shared slot counts, twice; only keys with a real share of the rows
            const unsigned* cnt = reinterpret_cast<const unsigned*>(sm + a.so_cnt);
            unsigned total = 0, b0 = 0, b1 = 0;
            for (int i = lane; i < S; i += 32) {
                const unsigned c = cnt[i];
                total += c;
                const unsigned key = (min(c, 0x7ffffu) << 13) | static_cast<unsigned>(i & 0x1fff);
                if (key > b0) {
                    b1 = b0;
                    b0 = key;
                } else if (key > b1) {
                    b1 = key;
                }
            }
            total = __reduce_add_sync(0xffffffffu, total);
            const unsigned w0 = __reduce_max_sync(0xffffffffu, b0);
            const unsigned c0 = (b0 == w0) ? b1 : b0;  // the owner of the first pick offers its runner-up
            const unsigned w1 = __reduce_max_sync(0xffffffffu, c0);
            if (S <= 8192 && w0 && (w0 >> 13) * 32u >= total) hk0 = skey[w0 & 0x1fffu];
            if (S <= 8192 && w1 && (w1 >> 13) * 32u >= total) hk1 = skey[w1 & 0x1fffu];
            if (hk0 == kEmpty) hk1 = kEmpty;
        };
        // Reduces a hot key's per-lane partials over the warp and merges them into the key's shared slot.
        auto flush_hot = [&](uint64_t hk, unsigned c, AccT acc, long long mn, long long mx) {
            if (hk == kEmpty) return;
            for (int o = 16; o > 0; o >>= 1) {
                c += __shfl_xor_sync(0xffffffffu, c, o);
                acc += __shfl_xor_sync(0xffffffffu, acc, o);
                mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
                mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            }
            if (lane == 0 && c) {
                bool found = false;
                const int s = s_find(skey, S, S, hk, smem_hash(hk, smem_shift), &found);
                if (s >= 0) s_merge_acc<VT>(sm, a, s, c, acc, mn, mx, has_vals);
            }
        };
        // Global inserts of queued misses: `issue` pops queue entry e into this lane's registers and issues the
        // first probe load; `complete` finishes the probe and applies the reductions.  A whole warp drains 32
        // entries at once, so 32 probe loads are in flight together.  (Deferring `complete` by one batch to
        // overlap the round trip with the next tile measured slower.)
        bool pf = false;
        uint64_t pf_kw = 0, pf_val = 0, pf_word = 0, pf_s = 0;
        uint32_t pf_meta = 0;
        auto issue = [&](int e) {
            pf_kw = qkw[e];
            pf_val = qval[e];
            pf_meta = qmeta[e];
            pf = true;
            const int kind = static_cast<int>(pf_meta & 3u);
            if (kind == KK_NORMAL || kind == KK_AUX) {
                const Region& Rg = (kind == KK_AUX) ? a.aux : a.main;
                pf_s = mix64(pf_kw) & Rg.mask;
                pf_word = ld_volatile_u64(Rg.slots + pf_s * W);
            }
        };
        auto complete = [&]() {
            if (!pf) return;
            pf = false;
            const int kind = static_cast<int>(pf_meta & 3u);
            uint64_t* slot;
            if (kind == KK_NORMAL || kind == KK_AUX) {
                const Region& Rg = (kind == KK_AUX) ? a.aux : a.main;
                slot = g_find_from(Rg, W, pf_kw, pf_s, pf_word, a.counters, &s_claims);
            } else {
                slot = g_special(a.main, W, kind == KK_ESCAPE ? 1 : 0, &s_claims);
            }
            if (slot && (pf_meta & 4u)) {
                if (has_vals) {
                    VT v;
                    memcpy(&v, &pf_val, sizeof(VT));
                    g_acc_row<VT>(slot, a, v);
                } else {
                    g_count_row(slot, a.L);
                }
            }
        };
        for (int64_t q = 0; q < my_tiles; ++q) {
            const int64_t tile = blockIdx.x + q * static_cast<int64_t>(gridDim.x);
            const bool staged = a.staged && tile < a.full_tiles;
            const int s = static_cast<int>(q % a.NS);
            if (staged && !mbar_wait(&full_bar[s], static_cast<uint32_t>((q / a.NS) & 1), a.counters)) break;
            const unsigned char* st = sm + a.so_stage + static_cast<size_t>(s) * a.sl.bytes;
            const int64_t base = tile * T;
            const bool skip = ((q & 15) == 0) && __any_sync(0xffffffffu, table_full(a.counters));
            // Phase A: filter and compact.
            int count = 0;
            for (int j = 0; j < R && !skip; j += 32) {
                const int i = warp * R + j + lane;
                const int64_t r = base + i;
                bool keep = r < a.n;
                if (keep) {
                    if (a.mask) keep = (staged ? reinterpret_cast<const int8_t*>(st + a.sl.mask)[i] : a.mask[r]) != 0;
                    if constexpr (HAS_PRED) {
                        const PL pv = staged ? reinterpret_cast<const PL*>(st + a.sl.pred)[i]
                                             : static_cast<const PL*>(a.pcol)[r];
                        keep = keep && (((pv >= plo) && (pv <= phi)) != pinv);
                        if constexpr (NULLS) {
                            if (a.pnull) {
                                const bool pn = staged ? ((reinterpret_cast<const uint64_t*>(st + a.sl.pnull)[i >> 6] >> (i & 63)) & 1)
                                                       : null_bit(a.pnull, r);
                                keep = keep && !pn;
                            }
                        }
                    }
                }
                const uint32_t b = __ballot_sync(0xffffffffu, keep);
                if (keep) list[count + __popc(b & lt_mask)] = static_cast<uint16_t>(i);
                count += __popc(b);
            }
            __syncwarp();
            // Phase B: insert the passing rows into the shared-memory table; rows that miss it are queued
            // and inserted into the global table 32 at a time, so the L2 round trips of a warp overlap.
            for (int e0 = 0; e0 < count; e0 += 32) {
                const int e = e0 + lane;
                const bool act = e < count;
                uint64_t kw = 0;
                int kind = KK_NORMAL;
                bool agg_it = false;
                VT v = VT{};
                if (act) {
                    const int i = list[e];
                    const int64_t r = base + i;
                    KT k0, k1 = KT{};
                    bool kn0 = false, kn1 = false, vn = false;
                    if (staged) {
                        k0 = reinterpret_cast<const KT*>(st + a.sl.key0)[i];
                        if constexpr (COMP) k1 = reinterpret_cast<const KT*>(st + a.sl.key1)[i];
                        if (has_vals) v = reinterpret_cast<const VT*>(st + a.sl.val)[i];
                        if constexpr (NULLS) {
                            const int wi = i >> 6, bb = i & 63;
                            if (a.sl.knull0 >= 0) kn0 = (reinterpret_cast<const uint64_t*>(st + a.sl.knull0)[wi] >> bb) & 1;
                            if (a.sl.knull1 >= 0) kn1 = (reinterpret_cast<const uint64_t*>(st + a.sl.knull1)[wi] >> bb) & 1;
                            if (a.sl.vnull >= 0) vn = (reinterpret_cast<const uint64_t*>(st + a.sl.vnull)[wi] >> bb) & 1;
                        }
                    } else {
                        k0 = static_cast<const KT*>(a.key0)[r];
                        if constexpr (COMP) k1 = static_cast<const KT*>(a.key1)[r];
                        if (has_vals) v = static_cast<const VT*>(a.vals)[r];
                        if constexpr (NULLS) {
                            kn0 = null_bit(a.knull0, r);
                            kn1 = null_bit(a.knull1, r);
                            vn = null_bit(a.vnull, r);
                        }
                    }
                    if constexpr (COMP) {
                        if (kn0 || kn1) {
                            kind = KK_AUX;
                            const uint32_t other =
                                kn0 ? (kn1 ? 0u : static_cast<uint32_t>(k1)) : static_cast<uint32_t>(k0);
                            kw = (static_cast<uint64_t>((kn0 ? 1u : 0u) | (kn1 ? 2u : 0u)) << 32) | other;
                        } else {
                            kw = composite_word(static_cast<int32_t>(k0), static_cast<int32_t>(k1));
                            kind = (kw == kEmpty) ? KK_ESCAPE : KK_NORMAL;
                        }
                    } else {
                        if (kn0) {
                            kind = KK_NULL;
                        } else {
                            kw = key_word(k0);
                            kind = (kw == kEmpty) ? KK_ESCAPE : KK_NORMAL;
                        }
                    }
                    agg_it = !has_vals || !vn;
                }
                bool miss = act;
                // Rows of the warp's hot keys accumulate in this lane's registers: no probe, no atomic.
                if (act && kind == KK_NORMAL && (kw == hk0 || kw == hk1)) {
                    miss = false;
                    if (agg_it) {
                        const int j = (kw == hk0) ? 0 : 1;
                        const AccT x = has_vals ? to_acc<VT>(v) : AccT{};
                        const long long e = has_vals ? enc_any<VT>(v) : 0;
                        if (j == 0) {
                            hc0 += 1;
                            ha0 += x;
                            hmn0 = min(hmn0, e);
                            hmx0 = max(hmx0, e);
                        } else {
                            hc1 += 1;
                            ha1 += x;
                            hmn1 = min(hmn1, e);
                            hmx1 = max(hmx1, e);
                        }
                    }
                } else if (act && use_smem && kind != KK_AUX) {
                    int slot_s;
                    if (kind == KK_NORMAL) {
                        bool found = false;
                        slot_s = s_find(skey, S, a.probe, kw, smem_hash(kw, smem_shift), &found);
                        ++my_tries;
                        my_hits += found ? 1u : 0u;
                    } else {
                        slot_s = S + (kind == KK_ESCAPE ? 1 : 0);
                        if (*reinterpret_cast<volatile uint64_t*>(&skey[slot_s]) == kEmpty)
                            atomicCAS(reinterpret_cast<unsigned long long*>(&skey[slot_s]), kEmpty, 0ull);
                    }
                    if (slot_s >= 0) {
                        miss = false;
                        if (agg_it) s_acc_row<VT>(sm, a, slot_s, v, has_vals);
                    }
                }
                const uint32_t mb = __ballot_sync(0xffffffffu, miss);
                if (miss) {
                    const int pos = qn + __popc(mb & lt_mask);
                    qkw[pos] = kw;
                    uint64_t vb = 0;
                    memcpy(&vb, &v, sizeof(VT));
                    qval[pos] = vb;
                    qmeta[pos] = static_cast<uint32_t>(kind) | (agg_it ? 4u : 0u);
                }
                qn += __popc(mb);
                if (qn >= 32) {
                    __syncwarp();
                    qn -= 32;
                    issue(qn + lane);
                    complete();
                    __syncwarp();
                }
            }
            if (staged) {
                __syncwarp();
                if (lane == 0) mbar_arrive(&empty_bar[s]);
            }
            if (q == kDecideTile && use_smem) {
                const unsigned hits = __reduce_add_sync(0xffffffffu, my_hits);
                const unsigned tries = __reduce_add_sync(0xffffffffu, my_tries);
                if (tries >= 256 && hits * 8u < tries) use_smem = false;
                else pick_hot_keys();
            }
            __syncwarp();
        }
        flush_hot(hk0, hc0, ha0, hmn0, hmx0);
        flush_hot(hk1, hc1, ha1, hmn1, hmx1);
        __syncwarp();
        complete();
        if (lane < qn) {
            issue(lane);
            complete();
        }
        __syncwarp();
    }

    // Merge this CTA's shared-memory table into the global table.
    __syncthreads();
    if (S) {
        const bool v32 = sizeof(VT) == 4;
        const bool vfloat = std::is_floating_point<VT>::value;
        for (int i = threadIdx.x; i < S2; i += blockDim.x) {
            const uint64_t key = skey[i];
            if (key == kEmpty) continue;
            uint64_t* slot = (i < S) ? g_find(a.main, W, key, mix64(key), a.counters, &s_claims)
                                     : g_special(a.main, W, i - S, &s_claims);
            if (!slot) continue;
            const unsigned long long c = reinterpret_cast<unsigned int*>(sm + a.so_cnt)[i];
            const uint64_t sumbits = a.has_sum ? reinterpret_cast<unsigned long long*>(sm + a.so_sum)[i] : 0ull;
            long long mn = 0, mx = 0;
            if (has_mm) {
                if (v32) {
                    const int* w = reinterpret_cast<const int*>(sm + a.so_mn) + 2 * i;
                    mn = w[0];
                    mx = w[1];
                } else {
                    mn = reinterpret_cast<long long*>(sm + a.so_mn)[i];
                    mx = reinterpret_cast<long long*>(sm + a.so_mx)[i];
                }
            }
            g_merge(slot, a.L, a.has_sum, a.has_min, a.has_max, v32, vfloat, c, sumbits, mn, mx);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) publish_claims(a.counters, a.capacity, s_claims);
}

// Launches the kernel for one type combination: one persistent CTA per SM.
template <typename KT, bool COMP, typename VT, typename PT, bool NULLS>
int32_t launch_agg_t(const AggArgs& a, size_t smem, cudaStream_t st) {
    auto kern = gb_agg_kernel<KT, COMP, VT, PT, NULLS>;
    const DeviceInfo& di = device_info();
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(gb_agg_kernel)");
    }
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kAggThreads, smem);
    if (e != cudaSuccess) return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    if (per_sm < 1) return fail(QDB_ERROR, "gb_agg_kernel: launch configuration does not fit an SM");
    int64_t grid = static_cast<int64_t>(di.sm_count) * per_sm;
    if (grid > a.tiles) grid = a.tiles;
    if (grid < 1) return QDB_OK;
    kern<<<static_cast<unsigned>(grid), kAggThreads, smem, st>>>(a);
    note_launch();
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "gb_agg_kernel launch");
    return QDB_OK;
}

template <typename KT, bool COMP, typename VT, typename PT>
int32_t launch_agg_n(const AggArgs& a, bool nulls, size_t smem, cudaStream_t st) {
    return nulls ? launch_agg_t<KT, COMP, VT, PT, true>(a, smem, st) : launch_agg_t<KT, COMP, VT, PT, false>(a, smem, st);
}

template <typename KT, bool COMP, typename VT>
int32_t launch_agg_p(const AggArgs& a, int32_t ptype, bool nulls, size_t smem, cudaStream_t st) {
    switch (ptype) {
        case 0: return launch_agg_n<KT, COMP, VT, NoPred>(a, nulls, smem, st);
        case QDB_INT32: return launch_agg_n<KT, COMP, VT, int32_t>(a, nulls, smem, st);
        case QDB_INT64: return launch_agg_n<KT, COMP, VT, int64_t>(a, nulls, smem, st);
        case QDB_FLOAT: return launch_agg_n<KT, COMP, VT, float>(a, nulls, smem, st);
        case QDB_DOUBLE: return launch_agg_n<KT, COMP, VT, double>(a, nulls, smem, st);
        default: return fail(QDB_ERR_INVALID, "unsupported predicate column type");
    }
}

template <typename KT, bool COMP>
int32_t launch_agg_k(const AggArgs& a, ValKind vk, int32_t ptype, bool nulls, size_t smem, cudaStream_t st) {
    switch (vk) {
        case VK_NONE:
        case VK_I32: return launch_agg_p<KT, COMP, int32_t>(a, ptype, nulls, smem, st);
        case VK_I64: return launch_agg_p<KT, COMP, int64_t>(a, ptype, nulls, smem, st);
        case VK_F32: return launch_agg_p<KT, COMP, float>(a, ptype, nulls, smem, st);
        case VK_F64: return launch_agg_p<KT, COMP, double>(a, ptype, nulls, smem, st);
        default: return fail(QDB_ERR_INVALID, "unsupported value type");
    }
}

// Slot layout of a table carrying `aggs` over values of kind vk (groupby.cu).
Layout make_layout(int32_t aggs, ValKind vk);
// `col OP constant` as an interval of the column type (groupby.cu).
PredInterval pred_interval(const qdb_pred& p);

// Per-key-type entry points, each instantiated in its own translation unit.
int32_t launch_agg_i32(const AggArgs& a, ValKind vk, int32_t ptype, bool nulls, size_t smem, cudaStream_t st);
int32_t launch_agg_i64(const AggArgs& a, ValKind vk, int32_t ptype, bool nulls, size_t smem, cudaStream_t st);
int32_t launch_agg_f32(const AggArgs& a, ValKind vk, int32_t ptype, bool nulls, size_t smem, cudaStream_t st);
int32_t launch_agg_f64(const AggArgs& a, ValKind vk, int32_t ptype, bool nulls, size_t smem, cudaStream_t st);
int32_t launch_agg_comp(const AggArgs& a, ValKind vk, int32_t ptype, bool nulls, size_t smem, cudaStream_t st);

}  // namespace qdb
