// The fused filter + hash-aggregate pass (the B200 replacement of kernel_filter ->
// reconstructColKeep -> group_by_kernel, qikkDB/QueryEngine/GPUCore/GPUFilter.cuh:22-44,
// GPUReconstruct.cuh:29-45 and :272-355, GPUGroupBy.cuh:68-196).
//
// One persistent CTA per SM, warp-specialised:
//   * a producer warp streams the CTA's tiles of every input column (keys, values, predicate column,
//     mask, null words) from HBM into a ring of shared-memory stages with bulk asynchronous copies
//     (cp.async.bulk, executed by the TMA engine) that complete on per-stage mbarriers;
//   * 16 consumer warps take the stages in order.  For every row they evaluate the predicate as an
//     interval test in the column's own type (the host turns `col OP constant` into [lo, hi] plus an
//     invert flag, so the test is two compares and no branch), compact the passing rows per warp, read
//     the key, and insert it into a per-CTA shared-memory table (bounded linear probe) whose state is
//     updated with 32-bit shared-memory atomics only (exact multi-limb sums), so skewed (Zipf) key
//     streams do not serialise on hot slots.  A row whose key misses the table goes
//       - to a hash-partitioned spill area in HBM when the table's group bound is larger than the
//         shared table (gb_spill_kernel aggregates each partition in shared memory afterwards), or
//       - to the global open-addressing table (bounded linear probe, 64-bit atomicCAS on the key word,
//         fire-and-forget reductions), queued per warp and inserted 32 at a time after the stage has
//         been released;
//     no mask or compacted column is written to HBM.
// At the end each CTA merges its shared-memory table into the global table.
// Every wait on an mbarrier or a spill chunk is bounded; an mbarrier wait that gives up records
// QDB_ERR_TIMEOUT in the table status, a chunk wait that gives up sends its row to the global table.
#pragma once

#include <climits>

#include "groupby.cuh"

namespace qdb {

constexpr int kConsumerWarps = 16;
constexpr int kConsumerThreads = kConsumerWarps * 32;     // 512
constexpr int kAggThreads = kConsumerThreads + 32;         // + one producer warp: 544 threads
constexpr int kRowsPerWarpUnit = 64;                       // a tile is kConsumerWarps * R rows, R a multiple of 64
constexpr int kQueueCap = 64;                              // per-warp queue of shared-table misses
constexpr int kSpillThreads = 512;                         // threads of a spill-pass CTA
constexpr int kSeenWords = 1024;                           // 32768-bit filter of keys seen once (spilling tables)
constexpr int kCountTile = 4;                              // from this tile on a warp counts its shared-table hits
constexpr int kDecideTile = 12;                            // tile index at which a warp judges its hit rate
constexpr uint32_t kMaxWaitIters = 1u << 18;               // bounded mbarrier waits (seconds, then give up)

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
    int32_t T = 2048;        // rows per tile: kConsumerWarps * R with R a multiple of 64
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
    int32_t so_stage = 0, so_bar = 0, so_list = 0, so_queue = 0, so_spill = 0;
    // shared table arrays (keys at offset 0, S + 2 entries each): counts, sum limbs, min/max
    int32_t so_cnt = 0, so_l0 = 0, so_l1 = 0, so_l2 = 0, so_mn = 0;
    // hash-partitioned spill of shared-table misses (spill_keys == nullptr: misses go to the global table).
    // Cell (c, p), the rows CTA c spills into partition p, holds spill_cell rows at (p * spill_ctas + c) * spill_cell.
    uint64_t* spill_keys = nullptr;  // key words
    void* spill_vals = nullptr;      // values (absent without a value column)
    uint32_t* spill_fill = nullptr;  // [partitions * spill_ctas] rows written per cell
    int64_t spill_cell = 0;          // rows per cell
    int32_t spill_bits = 0;          // log2 of the partition count
    int32_t spill_ctas = 0;          // CTAs of the aggregation pass (its grid)
    // Bucketed table of the fast pass (groupby_fast.cuh): NB buckets of four slots, one 64-bit tag word per
    // bucket at so_tags, key words at so_keys; counts, sum limbs and min/max at so_cnt, so_l0, so_l1, so_mn.
    int32_t NB = 0;
    int32_t so_tags = 0, so_keys = 0;
    int32_t fits = 0;      // 1: every group fits the table: a key may overflow into the next probe_b - 1 buckets
    int32_t probe_b = 1;   // buckets a claim may visit
    int32_t dedup = 2;     // warp aggregation of equal keys: 0 off, 1 on, 2 decided per warp from its first batches
    int32_t pred_float = 0;  // the fast pass compares IEEE predicate values as order-preserving integers
    int32_t flush_rounds = 16;  // lock-step probe rounds of a shared table's merge into the global table
    // Second spill level (fast pass, tables with more partitions than one pass writes well): the spill pass over the
    // first level sends the rows its table cannot take to cell p * 2^spill2_bits + q of this area, q the next
    // spill2_bits bits of the key's hash, and a third pass aggregates those cells.
    uint64_t* spill2_keys = nullptr;
    uint32_t* spill2_fill = nullptr;  // [2^(spill_bits + spill2_bits)] rows per cell, then the next pass's work counter
    int64_t spill2_cell = 0;
    int32_t spill2_bits = 0;
    int32_t so_spill2 = 0;            // shared-memory offset of the spill pass's second-level fill counters
    // AAFL-compressed key column (fast pass, single key): key0 is unused; the consumer warps unpack their rows' keys
    // from the groups' packed words (kz_words, kz_len of them; group g at kz_pos[g] with kz_bits[g] bits per value)
    // into the ring and add kz_off back.
    int32_t kz = 0;
    const void* kz_words = nullptr;
    const uint64_t* kz_pos = nullptr;
    const uint8_t* kz_bits = nullptr;
    uint64_t kz_off = 0;
    int64_t kz_len = 0;
    // Fused key % m (fast pass, a single integer key): each key is replaced by its C++ remainder by the modulus whose
    // multiply-high constants these are (mod_signed) as it is read, before it is hashed.
    int32_t kmod = 0;
    int32_t km_s1 = 0, km_s2 = 0;
    uint64_t km_d = 1, km_m = 1;
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
// try_wait with a suspend-time hint: the warp sleeps in hardware until the phase completes or about `ns` pass,
// so a waiting warp issues no instructions while it waits.
__device__ __forceinline__ bool mbar_try_wait_for(uint64_t* bar, uint32_t parity, uint32_t ns) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(ns)
        : "memory");
    return ok != 0;
}
// Waits for phase `parity` of `bar`; gives up after kMaxWaitIters tries (each suspends up to 10 us, so about
// 2.6 s in all) and records QDB_ERR_TIMEOUT.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, unsigned long long* counters) {
    for (uint32_t it = 0; it < kMaxWaitIters; ++it)
        if (mbar_try_wait_for(bar, parity, 10000u)) return true;
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
// A CTA claims fewer than 2^32 groups per launch, so the count lives in the low 32-bit word of its 64-bit counter
// and a native 32-bit shared atomic updates it: a 64-bit shared atomic is a retry loop, which collapses when a
// thousand threads claim new groups at once (the spill pass merging a partition of new keys).
__device__ __forceinline__ void claim_counted(unsigned long long* claims) {
    atomicAdd(reinterpret_cast<unsigned int*>(claims), 1u);
}

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

// Home slot of a key whose mix64 hash is h: the top log2(cap) bits of h (a multiply-high, no power-of-two mask).
__device__ __forceinline__ uint64_t home_slot(const Region& R, uint64_t h) { return __umul64hi(h, R.mask + 1); }

__device__ __forceinline__ uint64_t* g_find(const Region& R, int W, uint64_t key, uint64_t h,
                                            unsigned long long* counters, unsigned long long* claims) {
    const uint64_t s = home_slot(R, h);
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

// Shared-memory accesses by 32-bit shared-window address (PTX ld/atom/red .shared), so the table code does its
// address arithmetic in 32 bits.  Keys are never removed from a table, so a weak read of a key word can only be
// stale by showing an empty slot, which the claiming CAS then corrects.
__device__ __forceinline__ uint64_t lds64(uint32_t a) {
    uint64_t v;
    asm volatile("ld.shared.u64 %0, [%1];" : "=l"(v) : "r"(a) : "memory");
    return v;
}
__device__ __forceinline__ int32_t lds32(uint32_t a) {
    int32_t v;
    asm volatile("ld.shared.s32 %0, [%1];" : "=r"(v) : "r"(a) : "memory");
    return v;
}
__device__ __forceinline__ int64_t lds64s(uint32_t a) {
    int64_t v;
    asm volatile("ld.shared.s64 %0, [%1];" : "=l"(v) : "r"(a) : "memory");
    return v;
}
__device__ __forceinline__ unsigned atoms_add(uint32_t a, unsigned x) {
    unsigned old;
    asm volatile("atom.shared.add.u32 %0, [%1], %2;" : "=r"(old) : "r"(a), "r"(x) : "memory");
    return old;
}
__device__ __forceinline__ void reds_add(uint32_t a, unsigned x) {
    asm volatile("red.shared.add.u32 [%0], %1;" ::"r"(a), "r"(x) : "memory");
}
__device__ __forceinline__ void reds_min32(uint32_t a, int32_t x) {
    asm volatile("red.shared.min.s32 [%0], %1;" ::"r"(a), "r"(x) : "memory");
}
__device__ __forceinline__ void reds_max32(uint32_t a, int32_t x) {
    asm volatile("red.shared.max.s32 [%0], %1;" ::"r"(a), "r"(x) : "memory");
}
__device__ __forceinline__ void reds_min64(uint32_t a, int64_t x) {
    asm volatile("red.shared.min.s64 [%0], %1;" ::"r"(a), "l"(x) : "memory");
}
__device__ __forceinline__ void reds_max64(uint32_t a, int64_t x) {
    asm volatile("red.shared.max.s64 [%0], %1;" ::"r"(a), "l"(x) : "memory");
}
__device__ __forceinline__ uint64_t atoms_cas64(uint32_t a, uint64_t cmp, uint64_t val) {
    uint64_t old;
    asm volatile("atom.shared.cas.b64 %0, [%1], %2, %3;" : "=l"(old) : "r"(a), "l"(cmp), "l"(val) : "memory");
    return old;
}

// Shared-memory probe by address: table key words at `keys` (S slots, S a power of two), starting at slot h.
// Returns the slot, or -1 after P probes; *found is set when the key was already present.
__device__ __forceinline__ int s_find32(uint32_t keys, int S, int P, uint64_t key, uint32_t h, bool* found) {
    uint32_t s = h;
    for (int p = 0; p < P; ++p) {
        const uint64_t cur = lds64(keys + s * 8u);
        if (cur == key) {
            *found = true;
            return static_cast<int>(s);
        }
        if (cur == kEmpty) {
            const uint64_t prev = atoms_cas64(keys + s * 8u, kEmpty, key);
            if (prev == kEmpty) return static_cast<int>(s);
            if (prev == key) {
                *found = true;
                return static_cast<int>(s);
            }
        }
        s = (s + 1u) & static_cast<uint32_t>(S - 1);
    }
    return -1;
}

// The table is read as 4-way buckets: a key's home is slot 4 * bucket, and a bounded linear probe that starts
// there (the generic path, and the claim of a new key) visits the bucket's four slots first.  The common case
// reads the whole bucket with two 16-byte loads and compares the four key words without a loop.
__device__ __forceinline__ uint32_t bucket_home(uint64_t kw, int smem_shift) { return smem_hash(kw, smem_shift + 2) * 4u; }

// Returns the slot of kw in the bucket at slot h4 (or -1); *has_empty tells whether the bucket has a free slot.
__device__ __forceinline__ int probe4(uint32_t keys, uint32_t h4, uint64_t kw, bool* has_empty) {
    uint4 w0, w1;
    asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(w0.x), "=r"(w0.y), "=r"(w0.z), "=r"(w0.w) : "r"(keys + h4 * 8u) : "memory");
    asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(w1.x), "=r"(w1.y), "=r"(w1.z), "=r"(w1.w) : "r"(keys + h4 * 8u + 16u) : "memory");
    const uint64_t k0 = (static_cast<uint64_t>(w0.y) << 32) | w0.x, k1 = (static_cast<uint64_t>(w0.w) << 32) | w0.z;
    const uint64_t k2 = (static_cast<uint64_t>(w1.y) << 32) | w1.x, k3 = (static_cast<uint64_t>(w1.w) << 32) | w1.z;
    *has_empty = (k0 == kEmpty) | (k1 == kEmpty) | (k2 == kEmpty) | (k3 == kEmpty);
    return (k0 == kw) ? static_cast<int>(h4) : (k1 == kw) ? static_cast<int>(h4 + 1) :
           (k2 == kw) ? static_cast<int>(h4 + 2) : (k3 == kw) ? static_cast<int>(h4 + 3) : -1;
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

// ---------------------------------------------------------------------------------------------
// Shared-memory slot state.  Every update is a 32-bit shared-memory atomic: those are resolved by the
// shared-memory atomic unit even when many lanes and warps hit one address (a skewed key stream), while
// 64-bit shared-memory atomics (CAS loops) serialise on hot slots.
//   count : u32 per slot (the rows one CTA adds to one slot fit 32 bits).
//   sum   : integer values: a 64-bit two's-complement accumulator kept as two u32 limbs; the carry out of
//           the low limb is detected from the value the atomic returns and added to the high limb, so the
//           sum is exact and wraps like the reference's 64-bit integer atomicAdd.
//           float/double values: a 96-bit fixed-point accumulator (three u32 limbs) of q = round(v * 2^F),
//           F chosen per CTA from the magnitudes of its first tile (fix_scale).  Values outside the window
//           where q keeps at least 24 significant bits and |q| < 2^63 (and NaN/Inf) take the global FP64 path.
//   min/max : order-preserving encodings; 32-bit atomics for 32-bit values, 64-bit ones for 64-bit values,
//           both issued only when the value improves on the slot's current bound.
// ---------------------------------------------------------------------------------------------
struct FixScale {
    double scale = 1.0;  // 2^F
    double inv = 1.0;    // 2^-F
    double lo = 0.0;     // smallest magnitude kept in fixed point
    double hi = 0.0;     // magnitudes at or above this take the FP64 path
    int sh0 = 0;         // float values: q = mantissa << (biased exponent - sh0), kept when 1 <= shift <= 39
};

// emax: the largest binary exponent e (|v| < 2^e) seen in the CTA's first tile.
__device__ __forceinline__ FixScale fix_scale(int emax) {
    emax = max(-960, min(960, emax));
    FixScale f;
    f.scale = ldexp(1.0, 48 - emax);
    f.inv = ldexp(1.0, emax - 48);
    f.lo = ldexp(1.0, emax - 24);
    f.hi = ldexp(1.0, emax + 15);
    f.sh0 = emax + 102;
    return f;
}

// Binary exponent e with |v| < 2^e for a finite non-zero value, INT_MIN otherwise.
template <typename VT>
__device__ __forceinline__ int value_exp(VT v) {
    if constexpr (std::is_same<VT, float>::value) {
        const uint32_t b = __float_as_uint(v);
        const int e = static_cast<int>((b >> 23) & 0xffu);
        return (e == 0 || e == 0xff) ? INT_MIN : e - 126;
    } else if constexpr (std::is_same<VT, double>::value) {
        const uint64_t b = static_cast<uint64_t>(__double_as_longlong(v));
        const int e = static_cast<int>((b >> 52) & 0x7ffu);
        return (e == 0 || e == 0x7ff) ? INT_MIN : e - 1022;
    } else {
        return INT_MIN;
    }
}

// The fixed-point (or exact integer) addend of one value; ok is false when the value must take the FP64 path.
template <typename VT>
__device__ __forceinline__ long long sum_addend(VT v, const FixScale& f, bool* ok) {
    if constexpr (std::is_same<VT, float>::value) {
        // integer-only: v = +-m * 2^(e - 150) with m the 24-bit significand, so q = +-m << (e - sh0) exactly
        const uint32_t b = __float_as_uint(v);
        const int e = static_cast<int>((b >> 23) & 0xffu);
        const uint32_t fr = b & 0x7fffffu;
        const int sh = e - f.sh0;
        const bool inw = e != 0 && e != 0xff && sh >= 1 && sh <= 39;
        *ok = inw || (b & 0x7fffffffu) == 0u;  // zero is exact; subnormals, NaN and Inf take the FP64 path
        const long long q = inw ? static_cast<long long>(static_cast<uint64_t>(fr | 0x800000u) << sh) : 0ll;
        return (b >> 31) ? -q : q;
    } else if constexpr (std::is_floating_point<VT>::value) {
        const double d = static_cast<double>(v);
        const double m = fabs(d);
        *ok = (m == 0.0) || (m >= f.lo && m < f.hi);  // false for NaN and Inf
        return *ok ? __double2ll_rn(d * f.scale) : 0ll;
    } else {
        *ok = true;
        return static_cast<long long>(v);
    }
}

struct STable {
    uint64_t* key;
    unsigned* cnt;
    unsigned* l0;
    unsigned* l1;
    unsigned* l2;
    unsigned char* mm;  // min/max region
    // the same arrays as 32-bit shared-window addresses
    uint32_t ak, ac, a0, a1, a2, am;
};

__device__ __forceinline__ STable stable(unsigned char* sm, const AggArgs& a) {
    STable t;
    t.key = reinterpret_cast<uint64_t*>(sm);
    t.cnt = reinterpret_cast<unsigned*>(sm + a.so_cnt);
    t.l0 = reinterpret_cast<unsigned*>(sm + a.so_l0);
    t.l1 = reinterpret_cast<unsigned*>(sm + a.so_l1);
    t.l2 = reinterpret_cast<unsigned*>(sm + a.so_l2);
    t.mm = sm + a.so_mn;
    t.ak = smem_u32(t.key);
    t.ac = smem_u32(t.cnt);
    t.a0 = smem_u32(t.l0);
    t.a1 = smem_u32(t.l1);
    t.a2 = smem_u32(t.l2);
    t.am = smem_u32(t.mm);
    return t;
}

// Adds the sign-extended 64-bit addend q to slot s's limbs (2 limbs: 64-bit wrap; 3 limbs: 96-bit).
template <int LIMBS>
__device__ __forceinline__ void limbs_add(const STable& t, int s, long long q) {
    const unsigned long long uq = static_cast<unsigned long long>(q);
    const unsigned x0 = static_cast<unsigned>(uq);
    const unsigned x1 = static_cast<unsigned>(uq >> 32);
    const uint32_t o = static_cast<uint32_t>(s) * 4u;
    const unsigned old0 = atoms_add(t.a0 + o, x0);
    const unsigned c = (old0 + x0 < old0) ? 1u : 0u;
    if constexpr (LIMBS == 2) {
        reds_add(t.a1 + o, x1 + c);  // the top limb wraps: the sum is exact modulo 2^64
    } else {
        const unsigned long long y1 = static_cast<unsigned long long>(x1) + c;
        const unsigned y1l = static_cast<unsigned>(y1);
        const unsigned old1 = atoms_add(t.a1 + o, y1l);
        const unsigned c1 = static_cast<unsigned>(y1 >> 32) + ((old1 + y1l < old1) ? 1u : 0u);
        const unsigned y2 = (q < 0 ? 0xffffffffu : 0u) + c1;
        if (y2) reds_add(t.a2 + o, y2);
    }
}

// The 96-bit fixed-point accumulator of a slot as a double (before scaling): |error| <= 2 ulp.
__device__ __forceinline__ double limbs96_to_double(unsigned l0, unsigned l1, unsigned l2) {
    unsigned long long lo = (static_cast<unsigned long long>(l1) << 32) | l0;
    unsigned hi = l2;
    const bool neg = (hi & 0x80000000u) != 0;
    if (neg) {  // two's-complement negation of the 96-bit value
        lo = ~lo + 1ull;
        hi = ~hi + (lo == 0ull ? 1u : 0u);
    }
    const double m = static_cast<double>(hi) * 18446744073709551616.0 + static_cast<double>(lo);
    return neg ? -m : m;
}

// One row's value into shared slot s (q: the precomputed sum addend).
template <typename VT>
__device__ __forceinline__ void s_add(const STable& t, const AggArgs& a, int s, VT v, long long q, bool has_val) {
    reds_add(t.ac + static_cast<uint32_t>(s) * 4u, 1u);
    if (!has_val) return;
    if (a.has_sum) {
        if constexpr (std::is_floating_point<VT>::value) limbs_add<3>(t, s, q);
        else limbs_add<2>(t, s, q);
    }
    if (a.has_min || a.has_max) {
        if constexpr (sizeof(VT) == 4) {
            const int32_t e = enc32(v);
            const uint32_t w = t.am + static_cast<uint32_t>(s) * 8u;
            if (a.has_min && e < lds32(w)) reds_min32(w, e);
            if (a.has_max && e > lds32(w + 4u)) reds_max32(w + 4u, e);
        } else {
            const long long e = enc64(v);
            const uint32_t w = t.am + static_cast<uint32_t>(s) * 16u;
            if (a.has_min && e < lds64s(w)) reds_min64(w, e);
            if (a.has_max && e > lds64s(w + 8u)) reds_max64(w + 8u, e);
        }
    }
}

// Initialises S2 slots of a shared table.
template <typename VT>
__device__ __forceinline__ void s_init(const STable& t, const AggArgs& a, int S2) {
    const bool has_mm = a.has_min || a.has_max;
    for (int i = threadIdx.x; i < S2; i += blockDim.x) {
        t.key[i] = kEmpty;
        t.cnt[i] = 0u;
        if (a.has_sum) {
            t.l0[i] = 0u;
            t.l1[i] = 0u;
            if (std::is_floating_point<VT>::value) t.l2[i] = 0u;
        }
        if (has_mm) {
            if (sizeof(VT) == 4) {
                reinterpret_cast<unsigned long long*>(t.mm)[i] = kPackedMinMaxInit;
            } else {
                reinterpret_cast<unsigned long long*>(t.mm)[2 * i] = kMinInit64;
                reinterpret_cast<unsigned long long*>(t.mm)[2 * i + 1] = kMaxInit64;
            }
        }
    }
}

// Merges every occupied slot of a shared table into the global table (whole CTA).
// Merges one occupied shared slot i into global slot g.
template <typename VT>
__device__ __forceinline__ void s_merge_slot(const STable& t, const AggArgs& a, int i, uint64_t* g, const FixScale& fs) {
    const bool has_mm = a.has_min || a.has_max;
    const bool v32 = sizeof(VT) == 4;
    const bool vfloat = std::is_floating_point<VT>::value;
    const unsigned long long c = t.cnt[i];
    uint64_t sumbits = 0;
    if (a.has_sum) {
        if (vfloat) {
            const double d = limbs96_to_double(t.l0[i], t.l1[i], t.l2[i]) * fs.inv;
            memcpy(&sumbits, &d, 8);
        } else {
            sumbits = (static_cast<uint64_t>(t.l1[i]) << 32) | t.l0[i];
        }
    }
    long long mn = 0, mx = 0;
    if (has_mm) {
        if (v32) {
            const int* w = reinterpret_cast<const int*>(t.mm) + 2 * i;
            mn = w[0];
            mx = w[1];
        } else {
            const long long* w = reinterpret_cast<const long long*>(t.mm) + 2 * i;
            mn = w[0];
            mx = w[1];
        }
    }
    g_merge(g, a.L, a.has_sum, a.has_min, a.has_max, v32, vfloat, c, sumbits, mn, mx);
}

// Merges every occupied slot of a shared table into the global table (whole CTA).  Each thread takes four
// slots at a time and issues the four home-slot loads of the global table before resolving any of them, so
// the L2 round trips overlap.
template <typename VT>
__device__ __forceinline__ void s_flush(const STable& t, const AggArgs& a, int S, const FixScale& fs,
                                        unsigned long long* claims) {
    const int W = a.L.W;
    constexpr int U = 4;
    for (int i0 = threadIdx.x; i0 < S; i0 += U * blockDim.x) {
        uint64_t key[U], pos[U], cur[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int i = i0 + u * blockDim.x;
            key[u] = (i < S) ? t.key[i] : kEmpty;
            pos[u] = home_slot(a.main, mix64(key[u]));
        }
#pragma unroll
        for (int u = 0; u < U; ++u) cur[u] = (key[u] != kEmpty) ? ld_volatile_u64(a.main.slots + pos[u] * W) : 0ull;
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (key[u] == kEmpty) continue;
            uint64_t* g = g_find_from(a.main, W, key[u], pos[u], cur[u], a.counters, claims);
            if (g) s_merge_slot<VT>(t, a, i0 + u * blockDim.x, g, fs);
        }
    }
    if (threadIdx.x < 2 && t.key[S + threadIdx.x] != kEmpty) {  // the NULL-key and escaped-key slots
        uint64_t* g = g_special(a.main, W, static_cast<int>(threadIdx.x), claims);
        if (g) s_merge_slot<VT>(t, a, S + threadIdx.x, g, fs);
    }
}

// ---------------------------------------------------------------------------------------------
// Hash-partitioned spill of shared-memory misses.  A row whose key is not in the CTA's shared table is
// appended to partition p = (top bits of its key hash) of a spill area in HBM instead of being inserted
// into the global table with L2 atomics; gb_spill_kernel then aggregates each partition in shared memory
// (a partition holds a bounded share of the distinct keys) and merges it into the global table.
// Every CTA owns one cell of every partition, so an append is one 32-bit shared-memory atomic on the cell's
// fill counter and two plain stores; a row that finds its cell full takes the global path instead.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ bool spill_keys_on(const AggArgs& a) { return a.spill_keys != nullptr; }

// ---------------------------------------------------------------------------------------------
// The aggregation kernel.  KT: key column type; COMP: composite (int32, int32) key; VT: value type
// (int32_t when the table has no value column); PT: predicate column type or NoPred; NULLS: some null
// mask (key, value or predicate) is present.
// ---------------------------------------------------------------------------------------------
template <typename KT, bool COMP, typename VT, typename PT, bool NULLS>
__global__ void __launch_bounds__(kAggThreads, 1) gb_agg_kernel(const AggArgs a) {
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ unsigned long long s_claims;
    __shared__ int s_emax;
    constexpr bool HAS_PRED = !std::is_same<PT, NoPred>::value;
    constexpr bool VFLOAT = std::is_floating_point<VT>::value;
    constexpr bool FASTROW = !COMP && !NULLS;
    using PL = typename std::conditional<HAS_PRED, PT, int32_t>::type;

    const int S = a.S;
    const STable tab = stable(sm, a);
    uint64_t* full_bar = reinterpret_cast<uint64_t*>(sm + a.so_bar);
    uint64_t* empty_bar = full_bar + a.NS;
    unsigned* sfill = reinterpret_cast<unsigned*>(sm + a.so_spill);
    unsigned* seen = sfill + (spill_keys_on(a) ? (1 << a.spill_bits) : 0);
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const bool spill_on = a.spill_keys != nullptr;

    if (S) s_init<VT>(tab, a, S + 2);
    if (spill_on)
        for (int i = threadIdx.x; i < (1 << a.spill_bits) + kSeenWords; i += blockDim.x) sfill[i] = 0u;
    if (threadIdx.x == 0) {
        s_claims = 0;
        s_emax = INT_MIN;
    }
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
    FixScale fs;

    if (warp == kConsumerWarps) {
        // ---------------- producer warp: one elected lane issues the bulk copies ----------------
        if (lane == 0 && a.staged) {
            const StageLayout& sl = a.sl;
            const uint64_t pol = l2_evict_first_policy();
            int64_t q = 0;
            int s = 0;
            uint32_t ph = 0;  // phase of stage s's current round
            for (; q < my_tiles; ++q) {
                const int64_t tile = blockIdx.x + q * static_cast<int64_t>(gridDim.x);
                if (tile >= a.full_tiles) break;  // the partial last tile is read directly
                if (q >= a.NS && !mbar_wait(&empty_bar[s], ph ^ 1u, a.counters)) break;
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
                if (++s == a.NS) {
                    s = 0;
                    ph ^= 1u;
                }
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
        const int R = T / kConsumerWarps;
        uint16_t* list = reinterpret_cast<uint16_t*>(sm + a.so_list) + warp * R;
        const uint32_t lt_mask = (1u << lane) - 1u;

        // Fixed-point scale of float sums: the largest exponent of this CTA's first tile of values.
        if (VFLOAT && a.has_sum && has_vals && my_tiles > 0) {
            const int64_t tile = blockIdx.x;
            const bool staged = a.staged && tile < a.full_tiles;
            bool ok = true;
            if (staged) ok = mbar_wait(&full_bar[0], 0u, a.counters);
            int e = INT_MIN;
            if (ok) {
                const unsigned char* st = sm + a.so_stage;
                for (int j = lane; j < R; j += 32) {
                    const int i = warp * R + j;
                    const int64_t r = tile * T + i;
                    if (r < a.n) {
                        const VT v = staged ? reinterpret_cast<const VT*>(st + a.sl.val)[i] : static_cast<const VT*>(a.vals)[r];
                        e = max(e, value_exp<VT>(v));
                    }
                }
            }
            e = __reduce_max_sync(0xffffffffu, e);
            if (lane == 0 && e != INT_MIN) atomicMax(&s_emax, e);
        }
        asm volatile("bar.sync 1, %0;" ::"r"(kConsumerThreads) : "memory");
        fs = fix_scale(s_emax == INT_MIN ? 0 : s_emax);

        bool use_smem = S > 0;
        unsigned my_hits = 0, my_tries = 0;
        bool spill_ok = spill_on;  // cleared, with use_smem, when this warp's shared-table hit rate is low
        const int smem_shift = 32 - (31 - __clz(S > 0 ? S : 1));
        // Per-warp queue of rows for the global table (raw rows: key word, value bits, kind | agg flag).
        uint64_t* qkw = reinterpret_cast<uint64_t*>(sm + a.so_queue) + warp * kQueueCap;
        uint64_t* qval = reinterpret_cast<uint64_t*>(sm + a.so_queue) + (kConsumerWarps + warp) * kQueueCap;
        uint32_t* qmeta = reinterpret_cast<uint32_t*>(reinterpret_cast<uint64_t*>(sm + a.so_queue) +
                                                      2 * kConsumerWarps * kQueueCap) + warp * kQueueCap;
        int qn = 0;
        // Global inserts of queued rows, 32 at a time with every lane active, so the warp's 32 probe loads
        // are in flight together.
        // Spill cell addressing of this CTA: row pos of partition p is at p * pstride + cell_off + pos.
        const int64_t pstride = spill_on ? static_cast<int64_t>(a.spill_ctas) * a.spill_cell : 0;
        const int64_t cell_off = spill_on ? static_cast<int64_t>(blockIdx.x) * a.spill_cell : 0;
        const unsigned cell_cap = spill_on ? static_cast<unsigned>(a.spill_cell) : 0u;
        VT* const spill_v = static_cast<VT*>(a.spill_vals);
        const uint32_t sfill_a = smem_u32(sfill);
        // Rows of the warp's queue, lanes < nvalid taking entries first + lane: a spillable row (meta bit 8) is
        // appended to its partition's cell, every other row (and a row whose cell is full) is inserted into the
        // global table.  A whole warp handles the queue at once, so the spill stores and the global probe loads of
        // up to 32 rows are in flight together.
        auto drain = [&](int first, int nvalid) {
            if (lane >= nvalid) return;
            const int e = first + lane;
            const uint64_t kw = qkw[e];
            const uint64_t vb = qval[e];
            const uint32_t meta = qmeta[e];
            VT v;
            memcpy(&v, &vb, sizeof(VT));
            if (meta & 8u) {
                const int p = a.spill_bits ? static_cast<int>((kw * 0x9e3779b97f4a7c15ull) >> (64 - a.spill_bits)) : 0;
                const unsigned pos = atoms_add(sfill_a + static_cast<uint32_t>(p) * 4u, 1u);
                if (pos < cell_cap) {
                    const int64_t idx = p * pstride + cell_off + pos;
                    a.spill_keys[idx] = kw;
                    if (has_vals) spill_v[idx] = v;
                    return;
                }
            }
            const int kind = static_cast<int>(meta & 3u);
            uint64_t* slot;
            if (kind == KK_NORMAL || kind == KK_AUX) {
                const Region& Rg = (kind == KK_AUX) ? a.aux : a.main;
                slot = g_find(Rg, W, kw, mix64(kw), a.counters, &s_claims);
            } else {
                slot = g_special(a.main, W, kind == KK_ESCAPE ? 1 : 0, &s_claims);
            }
            if (slot && (meta & 4u)) {
                if (has_vals) g_acc_row<VT>(slot, a, v);
                else g_count_row(slot, a.L);
            }
        };
        auto drain32 = [&](int first) { drain(first, 32); };
        const int K = R >> 5;  // rows per lane in phase A
        // One passing row (list entry e): probe the shared table, update the slot, or spill; returns true when the
        // row must go to the warp's queue of global inserts.
        auto insert_row = [&](int e, const unsigned char* st, bool staged, int64_t base, uint64_t& kw_out,
                              VT& v_out, uint32_t& meta_out) -> bool {
            const int i = list[e];
            KT k0, k1 = KT{};
            bool kn0 = false, kn1 = false, vn = false;
            VT v = VT{};
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
                const int64_t r = base + i;
                k0 = static_cast<const KT*>(a.key0)[r];
                if constexpr (COMP) k1 = static_cast<const KT*>(a.key1)[r];
                if (has_vals) v = static_cast<const VT*>(a.vals)[r];
                if constexpr (NULLS) {
                    kn0 = null_bit(a.knull0, r);
                    kn1 = null_bit(a.knull1, r);
                    vn = null_bit(a.vnull, r);
                }
            }
            uint64_t kw = 0;
            int kind = KK_NORMAL;
            if constexpr (COMP) {
                if (kn0 || kn1) {
                    kind = KK_AUX;
                    const uint32_t other = kn0 ? (kn1 ? 0u : static_cast<uint32_t>(k1)) : static_cast<uint32_t>(k0);
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
            const bool agg_it = !has_vals || !vn;
            bool inwin = true;
            long long qv = 0;
            if (agg_it && has_vals && a.has_sum) qv = sum_addend<VT>(v, fs, &inwin);
            kw_out = kw;
            v_out = v;
            meta_out = static_cast<uint32_t>(kind) | (agg_it ? 4u : 0u);
            if (!use_smem || kind == KK_AUX || !inwin) return true;
            int slot_s;
            if (kind == KK_NORMAL) {
                const uint32_t h = bucket_home(kw, smem_shift);
                bool found = false;
                slot_s = s_find(tab.key, S, a.probe, kw, h, &found);
                ++my_tries;
                my_hits += slot_s >= 0 ? 1u : 0u;
            } else {
                slot_s = S + (kind == KK_ESCAPE ? 1 : 0);
                if (*reinterpret_cast<volatile uint64_t*>(&tab.key[slot_s]) == kEmpty)
                    atomicCAS(reinterpret_cast<unsigned long long*>(&tab.key[slot_s]), kEmpty, 0ull);
            }
            if (slot_s >= 0) {
                if (agg_it) s_add<VT>(tab, a, slot_s, v, qv, has_vals);
                return false;
            }
            if (spill_ok && kind == KK_NORMAL && agg_it) meta_out |= 8u;  // the queue drain spills it
            return true;
        };
        // Queues row (kw, v, meta) of a lane whose `miss` is set; drains 32 rows when the queue is nearly full.
        auto enqueue = [&](bool miss, uint64_t kw, VT v, uint32_t meta) {
            const uint32_t mb = __ballot_sync(0xffffffffu, miss);
            if (mb == 0u) return;
            if (miss) {
                const int pos = qn + __popc(mb & lt_mask);
                qkw[pos] = kw;
                uint64_t vb = 0;
                memcpy(&vb, &v, sizeof(VT));
                qval[pos] = vb;
                qmeta[pos] = meta;
            }
            qn += __popc(mb);
            if (qn > kQueueCap - 32) {  // keep room for the next batch
                __syncwarp();
                qn -= 32;
                drain32(qn);
                __syncwarp();
            }
        };
        // The common case (one key column, no NULL masks, a staged tile) with few divergent regions per batch:
        // every lane loads its row and probes the key's home slot; only lanes that did not find their key there
        // run the full probe, only missing lanes take the spill / queue path.
        auto fast_row = [&](int e0, const unsigned char* st, int count) {
            const int e = e0 + lane;
            const bool act = e < count;
            const int i = list[act ? e : e0];
            const uint64_t kw = key_word(reinterpret_cast<const KT*>(st + a.sl.key0)[i]);
            const VT v = has_vals ? reinterpret_cast<const VT*>(st + a.sl.val)[i] : VT{};
            bool inwin = true;
            long long qv = 0;
            if (a.has_sum) qv = sum_addend<VT>(v, fs, &inwin);
            const bool normal = kw != kEmpty;
            const uint32_t h0 = use_smem ? bucket_home(kw, smem_shift) : 0u;
            const bool ok = act && normal && inwin && use_smem;
            bool has_empty = false;
            int slot = ok ? probe4(tab.ak, h0, kw, &has_empty) : -1;
            bool hit = slot >= 0;
            const bool need = ok && !hit && (has_empty || a.probe > 4);
            if (__any_sync(0xffffffffu, need)) {
                // While the table fills, a spilling table admits a key on its second occurrence only (a bit
                // filter of keys seen once), so the slots go to keys that recur rather than to the first comers.
                bool admit = need;
                if (need && spill_on) {
                    const uint32_t hb = static_cast<uint32_t>((kw * 0xd6e8feb86659fd93ull) >> 49);
                    const unsigned bit = 1u << (hb & 31u);
                    admit = (atomicOr(&seen[hb >> 5], bit) & bit) != 0u;
                }
                if (admit) {
                    bool found = false;
                    slot = s_find32(tab.ak, S, a.probe, kw, h0, &found);
                    hit = slot >= 0;
                }
            }
            my_tries += ok ? 1u : 0u;
            my_hits += hit ? 1u : 0u;
            if (hit) s_add<VT>(tab, a, slot, v, qv, has_vals);
            const bool miss = act && !hit;
            const uint32_t spillable = (spill_ok && normal && inwin) ? 8u : 0u;
            enqueue(miss, kw, v, static_cast<uint32_t>(normal ? KK_NORMAL : KK_ESCAPE) | 4u | spillable);
        };
        int s = 0;
        uint32_t ph = 0;
        bool skip = false;
        int64_t tile = blockIdx.x;
        for (int64_t q = 0; q < my_tiles; ++q, tile += gridDim.x) {
            const bool staged = a.staged && tile < a.full_tiles;
            if (staged && !mbar_wait(&full_bar[s], ph, a.counters)) break;
            const unsigned char* st = sm + a.so_stage + static_cast<size_t>(s) * a.sl.bytes;
            const int64_t base = tile * T;
            if ((q & 127) == 0) skip = __any_sync(0xffffffffu, table_full(a.counters));  // an L2 round trip: rarely
            // Phase A: filter and compact.  Lane l evaluates the K = R/32 consecutive rows [l*K, (l+1)*K) of the
            // warp's slice (vector loads from the stage); one ballot per row position ranks the passing rows into
            // the warp's list.
            int count = 0;
            if (!skip) {
                const int i0 = warp * R + lane * K;
                uint32_t bits = 0;
                if (staged && HAS_PRED && !a.mask && !NULLS) {
                    const PL* pp = reinterpret_cast<const PL*>(st + a.sl.pred) + i0;
                    if constexpr (sizeof(PL) == 4) {
                        if (K == 2) {
                            const int2 w2 = *reinterpret_cast<const int2*>(pp);
                            const PL p0 = from_bits<PL>(w2.x), p1 = from_bits<PL>(w2.y);
                            bits = ((((p0 >= plo) && (p0 <= phi)) != pinv) ? 1u : 0u) |
                                   ((((p1 >= plo) && (p1 <= phi)) != pinv) ? 2u : 0u);
                        }
                        for (int j = 0; K >= 4 && j < K; j += 4) {
                            const int4 w4 = *reinterpret_cast<const int4*>(pp + j);
                            const int32_t wv[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
                            for (int u = 0; u < 4; ++u) {
                                const PL pv = from_bits<PL>(wv[u]);
                                bits |= (((pv >= plo) && (pv <= phi)) != pinv ? 1u : 0u) << (j + u);
                            }
                        }
                    } else {
                        for (int j = 0; j < K; j += 2) {
                            const int4 w4 = *reinterpret_cast<const int4*>(pp + j);
                            const int64_t wv[2] = {(static_cast<int64_t>(static_cast<uint32_t>(w4.y)) << 32) | static_cast<uint32_t>(w4.x),
                                                   (static_cast<int64_t>(static_cast<uint32_t>(w4.w)) << 32) | static_cast<uint32_t>(w4.z)};
#pragma unroll
                            for (int u = 0; u < 2; ++u) {
                                const PL pv = from_bits<PL>(wv[u]);
                                bits |= (((pv >= plo) && (pv <= phi)) != pinv ? 1u : 0u) << (j + u);
                            }
                        }
                    }
                } else if (staged && !HAS_PRED && !a.mask) {
                    bits = (K >= 32) ? 0xffffffffu : ((1u << K) - 1u);
                } else {
                    for (int j = 0; j < K; ++j) {
                        const int i = i0 + j;
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
                        bits |= (keep ? 1u : 0u) << j;
                    }
                }
                for (int j = 0; j < K; ++j) {
                    const bool kj = (bits >> j) & 1u;
                    const uint32_t bj = __ballot_sync(0xffffffffu, kj);
                    if (kj) list[count + __popc(bj & lt_mask)] = static_cast<uint16_t>(i0 + j);
                    count += __popc(bj);
                }
            }
            __syncwarp();
            // Phase B: two passing rows per lane per step (their loads and probes overlap); a row whose key misses
            // the shared table goes to the spill area or, without one, to this warp's queue of global inserts.
            if (FASTROW && staged) {
                for (int e0 = 0; e0 < count; e0 += 32) fast_row(e0, st, count);
            } else {
                for (int e0 = 0; e0 < count; e0 += 64) {
                    const int ea = e0 + lane, eb = e0 + 32 + lane;
                    uint64_t kwa = 0, kwb = 0;
                    VT va = VT{}, vb = VT{};
                    uint32_t ma = 0, mbm = 0;
                    const bool missa = ea < count && insert_row(ea, st, staged, base, kwa, va, ma);
                    const bool missb = eb < count && insert_row(eb, st, staged, base, kwb, vb, mbm);
                    enqueue(missa, kwa, va, ma);
                    enqueue(missb, kwb, vb, mbm);
                }
            }
            if (staged) {
                __syncwarp();
                if (lane == 0) mbar_arrive(&empty_bar[s]);
            }
            // Global inserts after the stage is released, so a slow L2 round trip does not hold the ring.
            while (qn >= 32) {
                __syncwarp();
                qn -= 32;
                drain32(qn);
                __syncwarp();
            }
            // After the table's fill phase a warp judges its shared-table hit rate.  Below 1/2 (keys spread evenly
            // over many more groups than the table holds) the spill would carry most rows through HBM twice and
            // through the spill pass, which measured slower than inserting them into the global table directly:
            // misses go to the global table.  Below 1/8 the warp also stops probing the shared table.
            if (q + 1 == kCountTile) my_hits = my_tries = 0;
            if (q == kDecideTile && use_smem) {
                const unsigned hits = __reduce_add_sync(0xffffffffu, my_hits);
                const unsigned tries = __reduce_add_sync(0xffffffffu, my_tries);
                if (tries >= 256 && hits * 2u < tries) spill_ok = false;
                if (tries >= 256 && hits * 8u < tries) use_smem = false;
            }
            if (++s == a.NS) {
                s = 0;
                ph ^= 1u;
            }
            __syncwarp();
        }
        __syncwarp();
        drain(0, qn);  // the last partial batch: lanes >= qn idle
        __syncwarp();
    }

    // Merge this CTA's shared-memory table into the global table; publish the spill cell fills.
    __syncthreads();
    fs = fix_scale(s_emax == INT_MIN ? 0 : s_emax);  // the producer warp's threads merge slots too
    if (S) s_flush<VT>(tab, a, S, fs, &s_claims);
    if (spill_on)
        for (int i = threadIdx.x; i < (1 << a.spill_bits); i += blockDim.x)
            a.spill_fill[static_cast<int64_t>(i) * a.spill_ctas + blockIdx.x] = min(sfill[i], static_cast<unsigned>(a.spill_cell));
    __syncthreads();
    if (threadIdx.x == 0) publish_claims(a.counters, a.capacity, s_claims);
}

// ---------------------------------------------------------------------------------------------
// Second pass over the spill: CTA (p, j) aggregates cells j, j + slices, ... of partition p in a shared-memory
// table (each warp walks whole cells, 64 rows per step with both loads issued first), sends the rows its table
// cannot hold to the global table directly, and merges the table into the global table.
// ---------------------------------------------------------------------------------------------
// One spilled row per lane (act: the lane has a row): home-slot probe, full probe only for lanes that need it,
// slot update, and the global table for rows the shared table cannot take.
template <typename VT>
__device__ __forceinline__ void spill_rows(const STable& tab, const AggArgs& a, const FixScale& fs, int S, int shift,
                                           bool act, uint64_t kw, VT v, bool has_vals, unsigned long long* claims) {
    bool inwin = true;
    long long qv = 0;
    if (has_vals && a.has_sum) qv = sum_addend<VT>(v, fs, &inwin);
    const uint32_t h0 = bucket_home(kw, shift);
    const bool ok = act && inwin;
    bool has_empty = false;
    int slot = ok ? probe4(tab.ak, h0, kw, &has_empty) : -1;
    bool hit = slot >= 0;
    const bool need = ok && !hit && (has_empty || a.probe > 4);
    if (__any_sync(0xffffffffu, need)) {
        if (need) {
            bool found = false;
            slot = s_find32(tab.ak, S, a.probe, kw, h0, &found);
            hit = slot >= 0;
        }
    }
    if (hit) s_add<VT>(tab, a, slot, v, qv, has_vals);
    const bool miss = act && !hit;
    if (__any_sync(0xffffffffu, miss)) {
        if (miss) {
            uint64_t* g = g_find(a.main, a.L.W, kw, mix64(kw), a.counters, claims);
            if (g) {
                if (has_vals) g_acc_row<VT>(g, a, v);
                else g_count_row(g, a.L);
            }
        }
    }
}

template <typename VT>
__global__ void __launch_bounds__(kSpillThreads) gb_spill_kernel(const AggArgs a) {
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ unsigned long long s_claims;
    __shared__ int s_emax;
    __shared__ int s_next_cell;
    constexpr bool VFLOAT = std::is_floating_point<VT>::value;
    const int S = a.S;
    const STable tab = stable(sm, a);
    const int parts = 1 << a.spill_bits;
    const int p = static_cast<int>(blockIdx.x % parts);
    const int j = static_cast<int>(blockIdx.x / parts);
    const int slices = static_cast<int>(gridDim.x / parts);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool has_vals = a.spill_vals != nullptr;
    s_init<VT>(tab, a, S + 2);
    if (threadIdx.x == 0) {
        s_claims = 0;
        s_emax = INT_MIN;
        s_next_cell = 0;
    }
    __syncthreads();
    const int64_t cell0 = static_cast<int64_t>(p) * a.spill_ctas;
    const int ncells = (a.spill_ctas - j + slices - 1) / slices;  // cells j, j + slices, ... of this partition
    if (VFLOAT && a.has_sum && has_vals) {  // scale from the first rows of each warp's first cell
        int e = INT_MIN;
        const int c = j + slices * warp;
        if (c < a.spill_ctas) {
            const int f = static_cast<int>(a.spill_fill[cell0 + c]);
            if (lane < f) e = value_exp<VT>(static_cast<const VT*>(a.spill_vals)[(cell0 + c) * a.spill_cell + lane]);
        }
        e = __reduce_max_sync(0xffffffffu, e);
        if (lane == 0 && e != INT_MIN) atomicMax(&s_emax, e);
    }
    __syncthreads();
    const FixScale fs = fix_scale(s_emax == INT_MIN ? 0 : s_emax);
    const int shift = 32 - (31 - __clz(S));
    for (;;) {  // warps take the next cell from a shared counter, so uneven cells do not leave warps idle
        int t = 0;
        if (lane == 0) t = atomicAdd(&s_next_cell, 1);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= ncells) break;
        const int c = j + slices * t;
        const int f = static_cast<int>(a.spill_fill[cell0 + c]);
        const int64_t base = (cell0 + c) * a.spill_cell;
        const uint64_t* keys = a.spill_keys + base;
        const VT* vals = has_vals ? static_cast<const VT*>(a.spill_vals) + base : nullptr;
        for (int r0 = 0; r0 < f; r0 += 128) {  // four rows per lane: all their loads are issued first
            uint64_t k[4];
            VT v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int r = r0 + 32 * u + lane;
                k[u] = r < f ? keys[r] : 0ull;
                v[u] = (has_vals && r < f) ? vals[r] : VT{};
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (r0 + 32 * u < f) spill_rows<VT>(tab, a, fs, S, shift, r0 + 32 * u + lane < f, k[u], v[u], has_vals, &s_claims);
        }
    }
    __syncthreads();
    s_flush<VT>(tab, a, S, fs, &s_claims);
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
    if (a.spill_keys) {  // the spill cells are laid out for exactly spill_ctas CTAs
        if (a.spill_ctas > grid) return fail(QDB_ERROR, "gb_agg_kernel: spill plan needs more CTAs than fit");
        grid = a.spill_ctas;
    }
    kern<<<static_cast<unsigned>(grid), kAggThreads, smem, st>>>(a);
    note_launch();
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "gb_agg_kernel launch");
    return QDB_OK;
}

// Launches the spill pass (grid = partitions x slices).
template <typename VT>
int32_t launch_spill_t(const AggArgs& a, size_t smem, int64_t grid, cudaStream_t st) {
    auto kern = gb_spill_kernel<VT>;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(gb_spill_kernel)");
    }
    kern<<<static_cast<unsigned>(grid), kSpillThreads, smem, st>>>(a);
    note_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "gb_spill_kernel launch");
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
