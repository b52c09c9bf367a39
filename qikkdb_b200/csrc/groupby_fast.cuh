// The fast form of the fused filter + hash-aggregate pass, for the common call: no NULL masks, no precomputed
// mask, 16-byte aligned columns (the replacement of kernel_filter -> reconstructColKeep -> group_by_kernel,
// qikkDB/QueryEngine/GPUCore/GPUFilter.cuh:22-44, GPUReconstruct.cuh:272-355, GPUGroupBy.cuh:68-196, and of the
// multi-key kernel_group_by_multi_key, GPUGroupByMultiKey.cuh:156-259, for (int32, int32) keys).
//
// One persistent CTA per SM: a producer warp streams 2048-row tiles of the key, value and predicate columns into a
// ring of shared-memory stages with cp.async.bulk (TMA engine, mbarrier completion, evict-first L2 policy); 16
// consumer warps take the stages in order.  Warp w owns rows [128 w, 128 (w + 1)) of a tile and reads them as four
// 32-row segments (lane l: rows 32 j + l), so the predicate loads are conflict-free and the ballot of segment j lists
// its passing rows in row order.  The passing rows are then processed 32 at a time:
//   * the key's bucket (four slots) holds four 15-bit tags in one 64-bit word: one 8-byte shared load and a
//     zero-halfword test find the slot whose tag matches, one more load confirms the key; a key absent from a full
//     bucket is a miss after that single load;
//   * a hit updates the slot with 32-bit shared atomics only: a u32 count, a 64-bit sum kept as two u32 limbs (the
//     carry out of the low limb is read from the value the atomic returns) and min/max issued only when the value
//     improves on the slot's bound.  Integer sums wrap like the reference's 64-bit atomicAdd; float and double
//     values are added in fixed point (q = v * 2^F, F from the CTA's first tile and its row count, so that no sum
//     can overflow), exactly for float values; values outside that window take the FP64 global path;
//   * when equal keys are common within a warp (few groups, or heavy skew), lanes holding one slot are combined
//     first (__match_any_sync on the slot, then full-warp __reduce_*_sync of the group's count, sum pieces and
//     min/max, one round per group of four or more lanes), and one lane updates the slot;
//   * a miss is appended to its partition's cell of the hash-partitioned spill area (gb_fspill_kernel aggregates
//     each partition in shared memory afterwards) or, without one, inserted into the global table.
// At the end every CTA merges its table into the global open-addressing table.
#pragma once

#include "groupby_agg.cuh"

namespace qdb {

constexpr int kFastWarps = 16;                      // consumer warps
constexpr int kFastThreads = (kFastWarps + 1) * 32; // + one producer warp
constexpr int kFastSeg = 4;                         // 32-row segments per warp and tile
constexpr int kFastR = 32 * kFastSeg;               // rows per warp and tile
constexpr int kFastT = kFastWarps * kFastR;         // rows per tile (2048)
constexpr int kDedupTrial = 4;                      // steps a warp runs with warp aggregation before deciding
constexpr int kDedupGroup = 4;                      // lanes sharing a slot that are combined before the update
constexpr int kMaxSpillBits = 13;                   // partitions the aggregation pass writes: at most 8192
constexpr int kMaxSpill2Bits = 6;                   // second-level partitions per first-level one: at most 64
constexpr uint64_t kHashMul = 0x9E3779B97F4A7C15ull;

__device__ __forceinline__ uint32_t atoms_or(uint32_t a, uint32_t x) {
    uint32_t old;
    asm volatile("atom.shared.or.b32 %0, [%1], %2;" : "=r"(old) : "r"(a), "r"(x) : "memory");
    return old;
}
__device__ __forceinline__ void lds128(uint32_t a, uint64_t& k0, uint64_t& k1) {
    asm volatile("ld.shared.v2.u64 {%0, %1}, [%2];" : "=l"(k0), "=l"(k1) : "r"(a) : "memory");
}

// Shared-window addresses of the bucketed table's arrays.  A bucket is two slots whose key words sit side by side
// (keys[2 b + j]); the slot's state lives in position-major arrays at index s = j NB + b, so that the states of
// different buckets' first positions fall in consecutive banks.
struct FTab {
    uint32_t keys, cnt, l0, l1, mm;
    uint32_t NB;
};

__device__ __forceinline__ FTab ftab(unsigned char* sm, const AggArgs& a) {
    FTab t;
    t.keys = smem_u32(sm + a.so_keys);
    t.cnt = smem_u32(sm + a.so_cnt);
    t.l0 = smem_u32(sm + a.so_l0);
    t.l1 = smem_u32(sm + a.so_l1);
    t.mm = smem_u32(sm + a.so_mn);
    t.NB = static_cast<uint32_t>(a.NB);
    return t;
}

// Hash of a key word for the shared tables and the spill: one 64-bit multiply (Fibonacci hashing, Knuth TAOCP vol. 3,
// 6.4).  Its top bits pick the spill partition, the 32 bits below bit `shift` (32 - partition bits) the bucket (so
// a partition's rows spread over every bucket of the spill pass's table), and bits 32..46 the bit of the seen-once
// filter.  The global table hashes with the independent mix64.
__device__ __forceinline__ uint64_t fhash(uint64_t kw) { return kw * kHashMul; }
__device__ __forceinline__ uint32_t fbucket(uint64_t m, int shift, uint32_t NB) {
    const uint32_t x = __funnelshift_rc(static_cast<uint32_t>(m), static_cast<uint32_t>(m >> 32), shift);
    return __umulhi(x, NB);
}

// Looks kw up in bucket b: returns its slot or -1; empty: the bucket has a free position.
__device__ __forceinline__ int fprobe(const FTab& t, uint32_t b, uint64_t kw, bool& empty) {
    uint64_t k0, k1;
    lds128(t.keys + b * 16u, k0, k1);
    empty = (k0 == kEmpty) | (k1 == kEmpty);
    return (k0 == kw) ? static_cast<int>(b) : ((k1 == kw) ? static_cast<int>(t.NB + b) : -1);
}

// Finds or claims kw in buckets b, b + 1, ... (nb buckets at most): a new key is claimed with a CAS on its key word.
// Returns the slot or -1.
static __device__ __noinline__ int fclaim(const FTab t, uint32_t b, uint64_t kw, int nb) {
    uint32_t bb = b;
    for (int k = 0; k < nb; ++k) {
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const uint32_t ka = t.keys + (bb * 2u + j) * 8u;
            const uint64_t cur = lds64(ka);
            if (cur == kw) return static_cast<int>(j * t.NB + bb);
            if (cur == kEmpty) {
                const uint64_t prev = atoms_cas64(ka, kEmpty, kw);
                if (prev == kEmpty || prev == kw) return static_cast<int>(j * t.NB + bb);
            }
        }
        bb = (bb + 1u == t.NB) ? 0u : bb + 1u;
    }
    return -1;
}

// ---------------------------------------------------------------------------------------------
// 64-bit fixed-point sum addends.  A CTA that may add up to 2^hb - 1 values into one slot keeps every addend below
// 2^(63 - hb) in magnitude, so the slot's two's-complement sum cannot overflow.  emax is the largest binary exponent
// (|v| < 2^emax) of the CTA's first tile; values up to 2^(emax + 2) are kept.
//   float: q = m24 << sh with sh = biased exponent - sh0 in [0, 39 - hb]: exact.
//   double: q = round(v * 2^F) for |v| in [lo, hi): every kept value has at least 24 significant bits.
// ---------------------------------------------------------------------------------------------
struct FixQ {
    int sh0 = 0;
    int shmax = 0;
    double scale = 1.0;  // 2^F
    double inv = 1.0;    // 2^-F
    double lo = 0.0;
    double hi = 0.0;
};

template <typename VT>
__device__ __forceinline__ FixQ fixq(int emax, int hb) {
    FixQ f;
    emax = max(-900, min(900, emax));
    const int g = 2;
    f.shmax = max(0, 39 - hb);
    if constexpr (std::is_same<VT, float>::value) {
        // A value of exponent emax + g would take sh = shmax.  sh0 stays in [1, 254 - shmax], so the biased exponents
        // 0 (zero, subnormals) and 255 (Inf, NaN) always fall outside [sh0, sh0 + shmax].
        f.sh0 = max(1, min(254 - f.shmax, emax + 126 + g - f.shmax));
        f.scale = ldexp(1.0, 150 - f.sh0);         // q = v * 2^(150 - sh0)
        f.inv = ldexp(1.0, f.sh0 - 150);
    } else {
        const int F = 63 - hb - emax - g;          // |v| < 2^(emax + g) gives |q| < 2^(63 - hb)
        f.scale = ldexp(1.0, F);
        f.inv = ldexp(1.0, -F);
        f.hi = ldexp(1.0, emax + g);
        f.lo = ldexp(1.0, emax + g - f.shmax - 1);
    }
    return f;
}

template <typename VT>
__device__ __forceinline__ long long addq(VT v, const FixQ& f, bool& ok) {
    if constexpr (std::is_same<VT, float>::value) {
        const uint32_t b = __float_as_uint(v);
        const uint32_t sh = ((b >> 23) & 0xffu) - static_cast<uint32_t>(f.sh0);  // below sh0: wraps to a large value
        const bool inw = sh <= static_cast<uint32_t>(f.shmax);
        ok = inw | ((b << 1) == 0u);  // zero is exact; subnormals, NaN and Inf take the FP64 path
        const uint64_t mag = inw ? static_cast<uint64_t>((b & 0x7fffffu) | 0x800000u) << sh : 0ull;
        const uint64_t sg = static_cast<uint64_t>(static_cast<int64_t>(static_cast<int32_t>(b) >> 31));
        return static_cast<long long>((mag ^ sg) - sg);
    } else if constexpr (std::is_same<VT, double>::value) {
        const double m = fabs(v);
        ok = (m == 0.0) | ((m >= f.lo) & (m < f.hi));  // false for NaN and Inf
        return ok ? __double2ll_rn(v * f.scale) : 0ll;
    } else {
        ok = true;
        return static_cast<long long>(v);
    }
}

// Largest binary exponent of a finite non-zero value, INT_MIN otherwise (integers: INT_MIN).
template <typename VT>
__device__ __forceinline__ int fexp(VT v) { return value_exp<VT>(v); }

// ---------------------------------------------------------------------------------------------
// Table initialisation and merge into the global table.
// ---------------------------------------------------------------------------------------------
template <typename VT>
__device__ __forceinline__ void ftab_init(unsigned char* sm, const AggArgs& a, int tid, int nthreads) {
    const int S = a.NB * 2;
    uint64_t* keys = reinterpret_cast<uint64_t*>(sm + a.so_keys);
    unsigned* cnt = reinterpret_cast<unsigned*>(sm + a.so_cnt);
    unsigned* l0 = reinterpret_cast<unsigned*>(sm + a.so_l0);
    unsigned* l1 = reinterpret_cast<unsigned*>(sm + a.so_l1);
    unsigned long long* mm = reinterpret_cast<unsigned long long*>(sm + a.so_mn);
    const bool has_mm = a.has_min || a.has_max;
    for (int i = tid; i < S; i += nthreads) {
        keys[i] = kEmpty;
        cnt[i] = 0u;
        if (a.has_sum) {
            l0[i] = 0u;
            l1[i] = 0u;
        }
        if (has_mm) {
            if (sizeof(VT) == 4) {
                mm[i] = kPackedMinMaxInit;
            } else {
                mm[2 * i] = kMinInit64;
                mm[2 * i + 1] = kMaxInit64;
            }
        }
    }
}

// Merges every occupied slot into the global table (whole CTA).  Each thread takes U slots at a time and finds their
// global slots in lock-step rounds: a round issues the pending probe loads, or the claims (CAS) of keys that met an
// empty slot, of all U before it looks at any result, so their L2/DRAM round trips overlap.  A key still unresolved
// after a.flush_rounds rounds (a long probe run) finishes with the one-key search, which bounds the probe and reports
// a full table.

template <typename VT>
__device__ __forceinline__ void ftab_flush(unsigned char* sm, const AggArgs& a, const FixQ& fq,
                                           unsigned long long* claims) {
    constexpr bool V32 = sizeof(VT) == 4;
    constexpr bool VFLOAT = std::is_floating_point<VT>::value;
    const int S = a.NB * 2;
    const int W = a.L.W;
    const uint64_t* keys = reinterpret_cast<const uint64_t*>(sm + a.so_keys);
    const unsigned* cnt = reinterpret_cast<const unsigned*>(sm + a.so_cnt);
    const unsigned* l0 = reinterpret_cast<const unsigned*>(sm + a.so_l0);
    const unsigned* l1 = reinterpret_cast<const unsigned*>(sm + a.so_l1);
    const unsigned char* mm = sm + a.so_mn;
    const uint64_t mask = a.main.mask;
    constexpr int U = 4;
    for (int i0 = threadIdx.x; i0 < S; i0 += U * blockDim.x) {
        uint64_t key[U], pos[U], cur[U];
        uint64_t* g[U];
        bool pend[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int ki = i0 + u * blockDim.x;
            key[u] = (ki < S) ? keys[ki] : kEmpty;
            g[u] = nullptr;
            pend[u] = key[u] != kEmpty && cnt[(ki & 1) * a.NB + (ki >> 1)] != 0u;  // key index 2 b + j -> state j NB + b
            pos[u] = pend[u] ? home_slot(a.main, mix64(key[u])) : 0ull;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) cur[u] = pend[u] ? ld_volatile_u64(a.main.slots + pos[u] * W) : 0ull;
        for (int r = 0; r < a.flush_rounds && (pend[0] | pend[1] | pend[2] | pend[3]); ++r) {
            unsigned long long prev[U];
#pragma unroll
            for (int u = 0; u < U; ++u)  // claims of keys that met an empty slot, all issued before any is read
                prev[u] = (pend[u] && cur[u] == kEmpty)
                              ? atomicCAS(reinterpret_cast<unsigned long long*>(a.main.slots + pos[u] * W), kEmpty, key[u])
                              : cur[u];
            bool load[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                load[u] = false;
                if (!pend[u]) continue;
                if (prev[u] == key[u] || (cur[u] == kEmpty && prev[u] == kEmpty)) {
                    if (cur[u] == kEmpty && prev[u] == kEmpty) claim_counted(claims);
                    g[u] = a.main.slots + pos[u] * W;
                    pend[u] = false;
                } else {  // the slot holds another key: probe the next one
                    pos[u] = (pos[u] + 1) & mask;
                    load[u] = true;
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (load[u]) cur[u] = ld_volatile_u64(a.main.slots + pos[u] * W);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (pend[u]) g[u] = g_find_from(a.main, W, key[u], pos[u], cur[u], a.counters, claims);
            if (!g[u]) continue;
            const int ki = i0 + u * blockDim.x;
            const int i = (ki & 1) * a.NB + (ki >> 1);
            const unsigned long long c = cnt[i];
            uint64_t sumbits = 0;
            if (a.has_sum) {
                const uint64_t s = (static_cast<uint64_t>(l1[i]) << 32) | l0[i];
                if (VFLOAT) {
                    const double d = static_cast<double>(static_cast<long long>(s)) * fq.inv;
                    memcpy(&sumbits, &d, 8);
                } else {
                    sumbits = s;
                }
            }
            long long mn = 0, mx = 0;
            if (a.has_min || a.has_max) {
                if (V32) {
                    const int* w = reinterpret_cast<const int*>(mm) + 2 * i;
                    mn = w[0];
                    mx = w[1];
                } else {
                    const long long* w = reinterpret_cast<const long long*>(mm) + 2 * i;
                    mn = w[0];
                    mx = w[1];
                }
            }
            g_merge(g[u], a.L, a.has_sum, a.has_min, a.has_max, V32, VFLOAT, c, sumbits, mn, mx);
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Rows of one step: two rows per lane (64 per warp), each row's table lookup, slot update and the fate of its miss.
// MODE bits: FM_SUM (a 64-bit sum), FM_MM (min and/or max), FM_VALS (a value column is read); without FM_VALS only
// the row count is kept.
// ---------------------------------------------------------------------------------------------
constexpr int FM_SUM = 1;
constexpr int FM_MM = 2;
constexpr int FM_VALS = 4;
constexpr int FM_KZ = 8;  // the key column is an AAFL-compressed block (single key, not DOUBLE)
constexpr int FM_KMOD = 16;  // keys are replaced by key % m as they are read (single INT32 or INT64 key)

template <typename VT, int MODE>
struct FastWarp {
    static constexpr bool SUM = (MODE & FM_SUM) != 0;
    static constexpr bool MM = (MODE & FM_MM) != 0;
    static constexpr bool VALS = (MODE & FM_VALS) != 0;
    const AggArgs& a;
    FTab t;
    FixQ fq;
    unsigned long long* claims;
    int bshift = 32;       // bucket bits start at this bit of the hash
    int probe_b = 1;       // buckets a claim may visit
    bool fits = false;
    bool use_smem = true;  // probe the shared table at all
    bool spill_ok = false; // append misses to the spill area
    bool dedup = false;
    bool counting = true;  // count lookups and hits (until the warp has judged its hit rate)
    int trial = 0;         // steps run so far in the warp-aggregation trial
    unsigned trial_hits = 0, trial_leaders = 0;  // warp totals over the trial
    unsigned hits = 0, tries = 0;
    // Where a miss goes: partition q = (fhash(key) >> part_shift) & part_mask, appended to cell cell_base + q cell_mul
    // of spill_out (records of 16 bytes, or 8 for a count-only table) at the position its shared fill counter
    // sfill[q] hands out; a full cell sends the row to the global table.
    uint32_t sfill = 0;    // shared-window address of the per-partition fill counters
    uint32_t seen = 0;     // shared-window address of the seen-once filter (0: admit every key)
    unsigned cell_cap = 0;
    int part_shift = 64;
    uint32_t part_mask = 0;
    int64_t cell_base = 0;
    int64_t cell_mul = 0;
    uint64_t* spill_out = nullptr;

    __device__ __forceinline__ FastWarp(const AggArgs& args, const FTab& tab, const FixQ& f, unsigned long long* c)
        : a(args), t(tab), fq(f), claims(c) {}

    __device__ __forceinline__ void global_row(uint64_t kw, VT v) {
        uint64_t* slot = (kw == kEmpty) ? g_special(a.main, a.L.W, 1, claims)
                                        : g_find(a.main, a.L.W, kw, mix64(kw), a.counters, claims);
        if (slot) {
            if (VALS) g_acc_row<VT>(slot, a, v);
            else g_count_row(slot, a.L);
        }
    }

    // Adds (n rows, sum addend q, encoded min e_mn and max e_mx) to slot s.
    __device__ __forceinline__ void update(uint32_t s, unsigned n, long long q, long long e_mn, long long e_mx) {
        reds_add(t.cnt + s * 4u, n);
        if constexpr (SUM) {
            const unsigned long long uq = static_cast<unsigned long long>(q);
            const unsigned x0 = static_cast<unsigned>(uq);
            const unsigned old0 = atoms_add(t.l0 + s * 4u, x0);
            const unsigned c = (old0 + x0 < old0) ? 1u : 0u;
            reds_add(t.l1 + s * 4u, static_cast<unsigned>(uq >> 32) + c);
        }
        if constexpr (MM) {
            if constexpr (sizeof(VT) == 4) {
                const uint32_t w = t.mm + s * 8u;
                const uint64_t cur = lds64(w);
                if (a.has_min && static_cast<int32_t>(e_mn) < static_cast<int32_t>(cur)) reds_min32(w, static_cast<int32_t>(e_mn));
                if (a.has_max && static_cast<int32_t>(e_mx) > static_cast<int32_t>(cur >> 32)) reds_max32(w + 4u, static_cast<int32_t>(e_mx));
            } else {
                const uint32_t w = t.mm + s * 16u;
                if (a.has_min && e_mn < lds64s(w)) reds_min64(w, e_mn);
                if (a.has_max && e_mx > lds64s(w + 8u)) reds_max64(w + 8u, e_mx);
            }
        }
    }

    __device__ __forceinline__ long long encv(VT v) const {
        if constexpr (sizeof(VT) == 4) return enc32(v);
        else return enc64(v);
    }

    // Warp aggregation of one row per lane: lanes holding one slot in groups of kDedupGroup or more are combined with
    // full-warp reductions (one round per such group) and one lane updates the slot; other hit lanes update directly.
    __device__ __forceinline__ void dedup_rows(bool hit, int slot, long long q, VT v, unsigned lane) {
        const long long e = MM ? encv(v) : 0;
        const unsigned peers = __match_any_sync(0xffffffffu, hit ? static_cast<unsigned>(slot) : (0x80000000u | lane));
        const bool big = hit && __popc(peers) >= kDedupGroup;
        unsigned bigmask = __ballot_sync(0xffffffffu, big);
        if (trial < kDedupTrial) {
            trial_hits += __popc(__ballot_sync(0xffffffffu, hit));
            trial_leaders += __popc(__ballot_sync(0xffffffffu, hit && (__ffs(peers) - 1 == static_cast<int>(lane))));
        }
        while (bigmask) {
            const int leader = __ffs(bigmask) - 1;
            const unsigned grp = __shfl_sync(0xffffffffu, peers, leader);
            const bool in = (grp >> lane) & 1u;
            long long qs = 0;
            if constexpr (SUM) {
                const unsigned uq0 = in ? static_cast<unsigned>(q) : 0u;
                const unsigned s_lo = __reduce_add_sync(0xffffffffu, uq0 & 0xffffu);
                const unsigned s_mid = __reduce_add_sync(0xffffffffu, uq0 >> 16);
                const unsigned s_hi = __reduce_add_sync(
                    0xffffffffu, in ? static_cast<unsigned>(static_cast<unsigned long long>(q) >> 32) : 0u);
                qs = static_cast<long long>((static_cast<unsigned long long>(s_hi) << 32) +
                                            (static_cast<unsigned long long>(s_mid) << 16) + s_lo);
            }
            long long g_mn = 0, g_mx = 0;
            if constexpr (MM) {
                if constexpr (sizeof(VT) == 4) {
                    if (a.has_min) g_mn = __reduce_min_sync(0xffffffffu, in ? static_cast<int>(e) : INT_MAX);
                    if (a.has_max) g_mx = __reduce_max_sync(0xffffffffu, in ? static_cast<int>(e) : INT_MIN);
                } else {
                    if (a.has_min) {
                        const int h = __reduce_min_sync(0xffffffffu, in ? static_cast<int>(e >> 32) : INT_MAX);
                        const unsigned l = __reduce_min_sync(
                            0xffffffffu, (in && static_cast<int>(e >> 32) == h) ? static_cast<unsigned>(e) : 0xffffffffu);
                        g_mn = static_cast<long long>((static_cast<unsigned long long>(static_cast<unsigned>(h)) << 32) | l);
                    }
                    if (a.has_max) {
                        const int h = __reduce_max_sync(0xffffffffu, in ? static_cast<int>(e >> 32) : INT_MIN);
                        const unsigned l = __reduce_max_sync(
                            0xffffffffu, (in && static_cast<int>(e >> 32) == h) ? static_cast<unsigned>(e) : 0u);
                        g_mx = static_cast<long long>((static_cast<unsigned long long>(static_cast<unsigned>(h)) << 32) | l);
                    }
                }
            }
            if (lane == static_cast<unsigned>(leader)) update(static_cast<uint32_t>(slot), __popc(grp), qs, g_mn, g_mx);
            bigmask &= ~grp;
        }
        if (hit && !big) update(static_cast<uint32_t>(slot), 1u, q, e, e);
    }

    // Stores a spilled row as one record (key word, value bits: a single 8- or 16-byte store) at position pos of its
    // partition's cell.
    __device__ __forceinline__ void spill_store(uint64_t kw, VT v, uint32_t p, unsigned pos) {
        const uint64_t idx = static_cast<uint64_t>(cell_base + static_cast<int64_t>(p) * cell_mul) * cell_cap + pos;
        if constexpr (VALS) {
            uint64_t vb = 0;
            memcpy(&vb, &v, sizeof(VT));
            reinterpret_cast<ulonglong2*>(spill_out)[idx] = make_ulonglong2(kw, vb);
        } else {
            spill_out[idx] = kw;
        }
    }

    // Two rows per lane: (act[u], kw[u], v[u]) for u = 0, 1.  The two rows' loads and arithmetic are independent, so
    // their latencies overlap; the rare paths (claims, next-bucket probes, misses) run under warp votes.
    __device__ __forceinline__ void rows2(const bool (&act)[2], const uint64_t (&kw)[2], const VT (&v)[2], unsigned lane) {
        long long q[2];
        bool inwin[2], look[2], hit[2], empty[2];
        uint64_t m[2], k0[2], k1[2];
        uint32_t b[2];
        int slot[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            inwin[u] = true;
            q[u] = 0;
            if constexpr (SUM) q[u] = addq<VT>(v[u], fq, inwin[u]);
            m[u] = fhash(kw[u]);
            look[u] = act[u] & (kw[u] != kEmpty) & inwin[u] & use_smem;
            b[u] = fbucket(m[u], bshift, t.NB);
            k0[u] = k1[u] = kEmpty;
        }
#pragma unroll
        for (int u = 0; u < 2; ++u)
            if (look[u]) lds128(t.keys + b[u] * 16u, k0[u], k1[u]);
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const bool h0 = k0[u] == kw[u];
            hit[u] = look[u] & (h0 | (k1[u] == kw[u]));
            slot[u] = hit[u] ? static_cast<int>(h0 ? b[u] : t.NB + b[u]) : -1;
            empty[u] = (k0[u] == kEmpty) | (k1[u] == kEmpty);
        }
        if (fits) {
            // A table sized for every group places a key whose home bucket is full in a later bucket, almost always
            // the next one: look there before the claim path.
            bool nx[2];
#pragma unroll
            for (int u = 0; u < 2; ++u) nx[u] = look[u] & !hit[u] & !empty[u];
            if (__any_sync(0xffffffffu, nx[0] | nx[1])) {
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    if (nx[u]) {
                        bool e2 = false;
                        const int s2 = fprobe(t, (b[u] + 1u == t.NB) ? 0u : b[u] + 1u, kw[u], e2);
                        if (s2 >= 0) {
                            slot[u] = s2;
                            hit[u] = true;
                        }
                    }
                }
            }
        }
        // Claim path: a new key with room in its bucket or (a table sized for every group) any key not found so far.
        bool need[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) need[u] = look[u] & !hit[u] & (empty[u] | fits);
        if (__any_sync(0xffffffffu, need[0] | need[1])) {
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                bool go = need[u];
                if (go && seen) {
                    // While a spilling table fills, a key is admitted on its second occurrence only, so that the
                    // slots go to keys that recur rather than to the first comers.
                    const uint32_t hb = static_cast<uint32_t>(m[u] >> 32) & 0x7fffu;
                    const uint32_t bit = 1u << (hb & 31u);
                    go = (atoms_or(seen + (hb >> 5) * 4u, bit) & bit) != 0u;
                }
                if (go) {
                    slot[u] = fclaim(t, b[u], kw[u], fits ? probe_b : 1);
                    hit[u] = slot[u] >= 0;
                }
            }
        }
        if (counting) {
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                tries += look[u] ? 1u : 0u;
                hits += hit[u] ? 1u : 0u;
            }
        }
        if (dedup) {
#pragma unroll
            for (int u = 0; u < 2; ++u) dedup_rows(hit[u], slot[u], q[u], v[u], lane);
            if (trial < kDedupTrial && ++trial == kDedupTrial && a.dedup == 2) {
                const unsigned th = __reduce_add_sync(0xffffffffu, lane == 0 ? trial_hits : 0u);
                const unsigned tl = __reduce_add_sync(0xffffffffu, lane == 0 ? trial_leaders : 0u);
                dedup = th > 0 && (th - tl) * 2u >= th;  // keep it when half the hits share a slot with another lane
            }
        } else {
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                if (hit[u]) {
                    const long long e = MM ? encv(v[u]) : 0;
                    update(static_cast<uint32_t>(slot[u]), 1u, q[u], e, e);
                }
            }
        }
        bool miss[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) miss[u] = act[u] & !hit[u];
        if (__any_sync(0xffffffffu, miss[0] | miss[1])) {
            // Both rows' spill positions are claimed before either record is stored, so the two shared-atomic round
            // trips overlap; rows that cannot spill (or whose cell is full) go to the global table.
            bool sp[2];
            unsigned pos[2];
            uint32_t part[2];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                sp[u] = miss[u] & spill_ok & (kw[u] != kEmpty) & inwin[u];
                part[u] = (sp[u] && part_shift < 64) ? static_cast<uint32_t>(m[u] >> part_shift) & part_mask : 0u;
            }
#pragma unroll
            for (int u = 0; u < 2; ++u) pos[u] = sp[u] ? atoms_add(sfill + part[u] * 4u, 1u) : 0u;
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                if (sp[u] && pos[u] < cell_cap) {
                    spill_store(kw[u], v[u], part[u], pos[u]);
                } else if (miss[u]) {
                    global_row(kw[u], v[u]);
                }
            }
        }
    }
};

// Key of row R of an AAFL-compressed key column (the block layout of qikkDB's GPUCompression.cu / feathergpu AAFL):
// rows come in groups of 32 W (W = bits of the key type); row R is lane R % 32, value i = (R % 32W) / 32 of its group,
// and occupies bits [i b, (i + 1) b) of the lane's stream, whose word k is words[pos[g] + lane + 32 k], least
// significant bit first.  Lanes of a warp that hold consecutive rows read consecutive words.  A word index past the
// packed words (a malformed block) latches QDB_ERR_INVALID and yields the offset.
template <typename KT>
__device__ __forceinline__ KT kz_key(const AggArgs& a, int64_t R) {
    using WT = typename std::conditional<sizeof(KT) == 8, unsigned long long, unsigned int>::type;
    constexpr int W = sizeof(KT) * 8;
    const int64_t g = R / (32 * W);
    const int i = static_cast<int>((R % (32 * W)) >> 5);
    const int l = static_cast<int>(R & 31);
    const int b = a.kz_bits[g];
    WT x = 0;
    if (b) {
        const int o = i * b;
        const int k = o / W;
        const int p = o % W;
        const int64_t i0 = static_cast<int64_t>(a.kz_pos[g]) + l + 32 * k;
        const bool two = p + b > W;
        if (i0 >= 0 && i0 + (two ? 32 : 0) < a.kz_len) {
            const WT* w = static_cast<const WT*>(a.kz_words);
            x = w[i0] >> p;
            if (two) x |= w[i0 + 32] << (W - p);
            if (b < W) x &= (WT(1) << b) - WT(1);
        } else {
            atomicExch(reinterpret_cast<int*>(&a.counters[1]), static_cast<int>(QDB_ERR_INVALID));
        }
    }
    const WT v = static_cast<WT>(x + static_cast<WT>(a.kz_off));
    KT out;
    memcpy(&out, &v, sizeof(KT));
    return out;
}

// Compressed keys in the ring: stage s's key region holds the tile's groups (one of 64-bit words, two of 32-bit),
// group gi at byte gi kzSlot<KT>() of the region, each copied from the 16-byte boundary at or below its first word:
// the words start `lead` bytes into the slot.  kzb[4 s + 2 gi] is the group's bit length, kzb[4 s + 2 gi + 1] its lead.
template <typename KT>
constexpr uint32_t kzSlot() { return 32u * sizeof(KT) * 8u * sizeof(KT) + 32u; }
template <typename KT>
constexpr uint32_t kzStage() { return static_cast<uint32_t>(kFastT) * sizeof(KT) + 64u; }

template <typename KT>
__device__ __forceinline__ KT kz_ring(const unsigned char* keys, const uint8_t* kzb, int g, uint64_t off) {
    using WT = typename std::conditional<sizeof(KT) == 8, unsigned long long, unsigned int>::type;
    constexpr int W = sizeof(KT) * 8;
    constexpr int GW = 32 * W;
    const int s = g / kFastT;
    const int r = g % kFastT;
    const int gi = r / GW;
    const int i = (r % GW) >> 5;
    const int l = r & 31;
    const int b = kzb[4 * s + 2 * gi];
    WT x = 0;
    if (b) {
        const WT* w = reinterpret_cast<const WT*>(keys + static_cast<size_t>(s) * kzStage<KT>() + gi * kzSlot<KT>() +
                                                  kzb[4 * s + 2 * gi + 1]) + l;
        const int o = i * b;
        const int k = o / W;
        const int p = o % W;
        x = w[32 * k] >> p;
        if (p + b > W) x |= w[32 * (k + 1)] << (W - p);
        if (b < W) x &= (WT(1) << b) - WT(1);
    }
    const WT v = static_cast<WT>(x + static_cast<WT>(off));
    KT out;
    memcpy(&out, &v, sizeof(KT));
    return out;
}

// ---------------------------------------------------------------------------------------------
// The aggregation kernel.  KT: key column type; COMP: composite (int32, int32) key; VT: value type (int32_t for a
// count-only table); PT: predicate column type or NoPred; MODE: FM_* bits.
//
// The ring holds NS stages column by column: column c of stage s, row i is at so_stage + off_c + (s T + i) * size_c,
// so a list entry g = s T + i addresses a row of any stage.  With three or more stages, the passing rows a warp has not
// processed when a tile ends (fewer than 64) stay in its list and its hold on that stage continues until the next
// tile's first step has taken them, so every step but the last has 64 rows.
// ---------------------------------------------------------------------------------------------
constexpr int kListCap = 192;  // list entries per warp: fewer than 64 carried plus a tile's 128

// A key's C++ remainder by the call's modulus (the fused key % m variant).
template <typename KT>
__device__ __forceinline__ KT kmod_key(const AggArgs& a, KT k) {
    return static_cast<KT>(mod_signed(static_cast<int64_t>(k), a.km_d, a.km_m, a.km_s1, a.km_s2));
}

template <typename KT, bool COMP, typename VT, typename PT, int MODE>
__global__ void __launch_bounds__(kFastThreads, 1) gb_fast_kernel(const AggArgs a) {
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ unsigned long long s_claims;
    __shared__ int s_emax;
    constexpr bool HAS_PRED = !std::is_same<PT, NoPred>::value;
    constexpr bool VFLOAT = std::is_floating_point<VT>::value;
    constexpr bool VALS = (MODE & FM_VALS) != 0;
    constexpr bool KZ = !COMP && (MODE & FM_KZ) != 0;
    constexpr bool KMOD = !COMP && !KZ && (MODE & FM_KMOD) != 0 && std::is_integral<KT>::value;
    using PL = typename std::conditional<HAS_PRED, PT, int32_t>::type;
    constexpr int PW = sizeof(PL);

    const FTab tab = ftab(sm, a);
    uint64_t* full_bar = reinterpret_cast<uint64_t*>(sm + a.so_bar);
    uint64_t* empty_bar = full_bar + a.NS;
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const bool spill_on = a.spill_keys != nullptr;
    const int parts = spill_on ? (1 << a.spill_bits) : 0;
    unsigned* sfill = reinterpret_cast<unsigned*>(sm + a.so_spill);
    unsigned char* ring = sm + a.so_stage;
    const StageLayout& sl = a.sl;

    ftab_init<VT>(sm, a, threadIdx.x, blockDim.x);
    if (spill_on) {
        for (int i = threadIdx.x; i < parts + kSeenWords; i += blockDim.x) sfill[i] = 0u;
        if (blockIdx.x == 0 && threadIdx.x == 0) a.spill_fill[static_cast<int64_t>(parts) * a.spill_ctas] = 0u;  // spill-pass work counter
    }
    if (threadIdx.x == 0) {
        s_claims = 0;
        s_emax = INT_MIN;
        for (int s = 0; s < a.NS; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], kFastWarps);
        }
        mbar_fence_init();
    }
    __syncthreads();

    const int64_t my_tiles =
        (a.tiles > static_cast<int64_t>(blockIdx.x)) ? (a.tiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
    // Headroom of the fixed-point sums: a slot of this CTA receives fewer than 2^hb values.
    const int hb = max(1, 64 - __clzll(static_cast<long long>(my_tiles * kFastT)));
    FixQ fq;

    if (warp == kFastWarps) {
        // ---------------- producer warp: one elected lane issues the bulk copies ----------------
        if (lane == 0) {
            const uint64_t pol = l2_evict_first_policy();
            int64_t q = 0;
            int s = 0;
            uint32_t ph = 0;
            uint32_t tx = static_cast<uint32_t>(kFastT) * sizeof(KT) * ((COMP ? 2 : 1) - (KZ ? 1 : 0));
            if (VALS) tx += static_cast<uint32_t>(kFastT) * sizeof(VT);
            if (HAS_PRED) tx += static_cast<uint32_t>(kFastT) * PW;
            for (; q < my_tiles; ++q) {
                const int64_t tile = blockIdx.x + q * static_cast<int64_t>(gridDim.x);
                if (tile >= a.full_tiles) break;  // the partial last tile is read directly
                if (q >= a.NS && !mbar_wait(&empty_bar[s], ph ^ 1u, a.counters)) break;
                const int64_t r0 = tile * kFastT;
                const size_t so = static_cast<size_t>(s) * kFastT;
                // Compressed keys: the tile's groups (one of 64-bit words, two of 32-bit) arrive as their packed words,
                // each copied from the 16-byte boundary at or below its first word through the 16-byte chunk that holds
                // its last (a chunk that holds a byte of the block lies in a page the block uses).
                constexpr int KZ_GW = 32 * static_cast<int>(sizeof(KT)) * 8;
                constexpr int KZ_NG = COMP ? 1 : kFastT / KZ_GW;
                uint32_t kz_bytes[2] = {0u, 0u};
                uint64_t kz_src[2] = {0ull, 0ull};
                if constexpr (KZ) {
                    uint8_t* kzb = reinterpret_cast<uint8_t*>(sm + a.so_bar + 96) + 4 * s;
#pragma unroll
                    for (int gi = 0; gi < KZ_NG; ++gi) {
                        const int64_t g = tile * KZ_NG + gi;
                        int b = a.kz_bits[g];
                        const uint64_t pos = a.kz_pos[g];
                        const uint64_t words = 32ull * static_cast<uint64_t>(b);
                        if (b > static_cast<int>(sizeof(KT)) * 8 || pos + words > static_cast<uint64_t>(a.kz_len)) {
                            if (b) atomicExch(reinterpret_cast<int*>(&a.counters[1]), static_cast<int>(QDB_ERR_INVALID));
                            b = 0;
                        }
                        const uint64_t src = reinterpret_cast<uint64_t>(a.kz_words) + pos * sizeof(KT);
                        const uint32_t lead = static_cast<uint32_t>(src & 15u);
                        kzb[2 * gi] = static_cast<uint8_t>(b);
                        kzb[2 * gi + 1] = static_cast<uint8_t>(lead);
                        kz_bytes[gi] = b ? ((lead + static_cast<uint32_t>(words * sizeof(KT)) + 15u) & ~15u) : 0u;
                        kz_src[gi] = src - lead;
                    }
                }
                fence_proxy_async_smem();
                mbar_arrive_expect_tx(&full_bar[s], tx + kz_bytes[0] + kz_bytes[1]);
#pragma unroll
                for (int gi = 0; gi < KZ_NG; ++gi)
                    if (kz_bytes[gi])
                        bulk_g2s(ring + sl.key0 + static_cast<size_t>(s) * kzStage<KT>() + gi * kzSlot<KT>(),
                                 reinterpret_cast<const void*>(kz_src[gi]), kz_bytes[gi], &full_bar[s], pol);
                if constexpr (!KZ) bulk_g2s(ring + sl.key0 + so * sizeof(KT), static_cast<const KT*>(a.key0) + r0, kFastT * sizeof(KT), &full_bar[s], pol);
                if (COMP) bulk_g2s(ring + sl.key1 + so * sizeof(KT), static_cast<const KT*>(a.key1) + r0, kFastT * sizeof(KT), &full_bar[s], pol);
                if (VALS) bulk_g2s(ring + sl.val + so * sizeof(VT), static_cast<const VT*>(a.vals) + r0, kFastT * sizeof(VT), &full_bar[s], pol);
                if (HAS_PRED) bulk_g2s(ring + sl.pred + so * PW, static_cast<const PL*>(a.pcol) + r0, kFastT * PW, &full_bar[s], pol);
                if (++s == a.NS) {
                    s = 0;
                    ph ^= 1u;
                }
            }
            // Drain: every issued stage must have been consumed (so no copy is still in flight) before exit.
            for (int64_t d = (q > a.NS ? q - a.NS : 0); d < q; ++d) {
                const int sd = static_cast<int>(d % a.NS);
                if (!mbar_wait(&empty_bar[sd], static_cast<uint32_t>((d / a.NS) & 1), a.counters)) break;
            }
        }
    } else {
        // ---------------- consumer warps ----------------
        const PL plo = HAS_PRED ? from_bits<PL>(a.pi.lo) : PL{};
        const PL phi = HAS_PRED ? from_bits<PL>(a.pi.hi) : PL{};
        const bool pinv = a.pi.invert != 0;
        uint16_t* list = reinterpret_cast<uint16_t*>(sm + a.so_list) + warp * kListCap;
        const uint32_t lt_mask = (1u << lane) - 1u;
        const KT* rk0 = reinterpret_cast<const KT*>(ring + sl.key0);
        const KT* rk1 = reinterpret_cast<const KT*>(ring + sl.key1);
        const VT* rv = reinterpret_cast<const VT*>(ring + sl.val);
        const PL* rp = reinterpret_cast<const PL*>(ring + sl.pred);

        // Fixed-point scale of float sums: the largest exponent of this CTA's first tile of values.
        if (VFLOAT && (MODE & FM_SUM) && my_tiles > 0) {
            const int64_t tile = blockIdx.x;
            const bool staged = tile < a.full_tiles;
            bool ok = true;
            if (staged) ok = mbar_wait(&full_bar[0], 0u, a.counters);
            int e = INT_MIN;
            if (ok) {
                for (int j = lane; j < kFastR; j += 32) {
                    const int i = warp * kFastR + j;
                    const int64_t r = tile * kFastT + i;
                    if (r < a.n) e = max(e, fexp<VT>(staged ? rv[i] : static_cast<const VT*>(a.vals)[r]));
                }
            }
            e = __reduce_max_sync(0xffffffffu, e);
            if (lane == 0 && e != INT_MIN) atomicMax(&s_emax, e);
        }
        asm volatile("bar.sync 1, %0;" ::"r"(kFastWarps * 32) : "memory");
        fq = fixq<VT>(s_emax == INT_MIN ? 0 : s_emax, hb);

        FastWarp<VT, MODE> fw(a, tab, fq, &s_claims);
        fw.bshift = 32;
        fw.fits = a.fits != 0;
        fw.probe_b = a.probe_b;
        fw.spill_ok = spill_on;
        // Warp aggregation pays only when lanes often share a slot: tried on tables sized for every group.
        fw.dedup = a.dedup == 1 || (a.dedup == 2 && a.fits != 0);
        if (spill_on) {
            fw.sfill = smem_u32(sfill);
            fw.seen = smem_u32(sfill + parts);
            fw.cell_cap = static_cast<unsigned>(a.spill_cell);
            fw.part_shift = 64 - a.spill_bits;
            fw.part_mask = static_cast<uint32_t>(parts - 1);
            fw.cell_base = blockIdx.x;
            fw.cell_mul = a.spill_ctas;
            fw.spill_out = a.spill_keys;
        }
        auto pass = [&](PL x) -> bool { return ((x >= plo) & (x <= phi)) != pinv; };
        const uint8_t* kzb = reinterpret_cast<const uint8_t*>(sm + a.so_bar + 96);
        auto ring_row = [&](int g, uint64_t& kw, VT& v) {
            if constexpr (COMP) kw = composite_word(static_cast<int32_t>(rk0[g]), static_cast<int32_t>(rk1[g]));
            else if constexpr (KZ) kw = key_word(kz_ring<KT>(ring + sl.key0, kzb, g, a.kz_off));
            else kw = key_word(rk0[g]);
            if constexpr (VALS) v = rv[g];
            else v = VT{};
        };
        // Steps over list entries [e0, e1): full 64-row steps, and the remainder when `flush`.  Returns the entries taken.
        auto steps = [&](int total, bool flush) -> int {
            int e0 = 0;
            for (; e0 + 64 <= total || (flush && e0 < total); e0 += 64) {
                bool act[2];
                uint64_t kw[2];
                VT v[2];
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int e = e0 + 32 * u + lane;
                    act[u] = e < total;
                    int g;
                    if constexpr (HAS_PRED) g = list[act[u] ? e : e0];
                    else g = list[0] + (act[u] ? e : e0);  // list[0]: the first row of the warp's slice
                    ring_row(g, kw[u], v[u]);
                }
                fw.rows2(act, kw, v, static_cast<unsigned>(lane));
            }
            return e0 < total ? e0 : total;
        };

        int s = 0;
        uint32_t ph = 0;
        int lc = 0;     // entries carried at the front of the list
        int held = -1;  // the stage those entries live in
        const bool carry = a.NS >= 3;
        int64_t tile = blockIdx.x;
        for (int64_t q = 0; q < my_tiles; ++q, tile += gridDim.x) {
            const bool staged = tile < a.full_tiles;
            if (!staged) {
                // The last, partial tile of the input: read directly from HBM, one step per 64 rows.
                const int64_t base = tile * kFastT;
                const int64_t lim = a.n - base;
                const int w0 = warp * kFastR;
                const KT* k0p = static_cast<const KT*>(a.key0) + base;
                const KT* k1p = static_cast<const KT*>(a.key1) + base;
                const VT* vp = static_cast<const VT*>(a.vals) + base;
                int count = 0;
                if constexpr (HAS_PRED) {
                    const PL* pp = static_cast<const PL*>(a.pcol) + base;
#pragma unroll
                    for (int j = 0; j < kFastSeg; ++j) {
                        const int i = w0 + 32 * j + lane;
                        const bool keep = i < lim && pass(pp[i]);
                        const uint32_t bj = __ballot_sync(0xffffffffu, keep);
                        if (keep) list[count + __popc(bj & lt_mask)] = static_cast<uint16_t>(i);
                        count += __popc(bj);
                    }
                } else {
                    count = static_cast<int>(lim - w0 < 0 ? 0 : (lim - w0 > kFastR ? kFastR : lim - w0));
                }
                __syncwarp();
                for (int e0 = 0; e0 < count; e0 += 64) {
                    bool act[2];
                    uint64_t kw[2];
                    VT v[2];
#pragma unroll
                    for (int u = 0; u < 2; ++u) {
                        const int e = e0 + 32 * u + lane;
                        act[u] = e < count;
                        const int i = HAS_PRED ? list[act[u] ? e : e0] : w0 + (act[u] ? e : e0);
                        if constexpr (COMP) kw[u] = composite_word(static_cast<int32_t>(k0p[i]), static_cast<int32_t>(k1p[i]));
                        else if constexpr (KZ) kw[u] = key_word(kz_key<KT>(a, base + i));
                        else if constexpr (KMOD) kw[u] = key_word(kmod_key<KT>(a, k0p[i]));
                        else kw[u] = key_word(k0p[i]);
                        if constexpr (VALS) v[u] = vp[i];
                        else v[u] = VT{};
                    }
                    fw.rows2(act, kw, v, static_cast<unsigned>(lane));
                }
                __syncwarp();
                continue;
            }
            if (!mbar_wait(&full_bar[s], ph, a.counters)) break;
            const bool full = (q & 127) == 0 && __any_sync(0xffffffffu, table_full(a.counters));
            // The next tile of this CTA is staged too: rows left over may wait for it.
            const bool keep_going = carry && !full && q + 1 < my_tiles && tile + gridDim.x < a.full_tiles;
            const int g0 = s * kFastT + warp * kFastR;  // ring index of the warp's first row in this stage
            if constexpr (KMOD) {
                if (!full) {
                    // Fused key % m: the warp replaces its own rows' keys in the stage by their remainders (no other
                    // warp reads them), then fences its writes against the producer's next copy into the stage.
                    KT* wk = const_cast<KT*>(rk0);
#pragma unroll
                    for (int j = 0; j < kFastSeg; ++j) {
                        const int g = g0 + 32 * j + lane;
                        wk[g] = static_cast<KT>(mod_signed(static_cast<int64_t>(wk[g]), a.km_d, a.km_m, a.km_s1, a.km_s2));
                    }
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    __syncwarp();
                }
            }
            int total = lc;
            if (!full) {
                if constexpr (HAS_PRED) {
                    // Filter: segment j of the warp's slice is rows 32 j + lane; its ballot lists the passing rows in
                    // row order behind the carried entries.
#pragma unroll
                    for (int j = 0; j < kFastSeg; ++j) {
                        const int g = g0 + 32 * j + lane;
                        const bool keep = pass(rp[g]);
                        const uint32_t bj = __ballot_sync(0xffffffffu, keep);
                        if (keep) list[total + __popc(bj & lt_mask)] = static_cast<uint16_t>(g);
                        total += __popc(bj);
                    }
                } else {
                    if (lane == 0) list[0] = static_cast<uint16_t>(g0);
                    total = kFastR;
                }
                __syncwarp();
            }
            int taken = full ? total : steps(total, !keep_going);
            if (held >= 0 && taken == 0) taken = steps(total, true);  // never hold two stages into the next tile
            __syncwarp();
            if (held >= 0 && lane == 0) mbar_arrive(&empty_bar[held]);  // its rows were the first lc entries
            held = -1;
            const int rem = total - taken;
            if (rem > 0) {
                // Move the leftover entries to the front (source at 64 or beyond, so the ranges do not overlap).
                const uint16_t t0 = lane < rem ? list[taken + lane] : 0;
                const uint16_t t1 = lane + 32 < rem ? list[taken + 32 + lane] : 0;
                __syncwarp();
                if (lane < rem) list[lane] = t0;
                if (lane + 32 < rem) list[32 + lane] = t1;
                __syncwarp();
                held = s;
            } else if (lane == 0) {
                mbar_arrive(&empty_bar[s]);
            }
            lc = rem;
            if (++s == a.NS) {
                s = 0;
                ph ^= 1u;
            }
            // After the table's fill phase a warp judges its hit rate: below 1/8 (keys spread evenly over many more
            // groups than the table holds) it stops probing the table and sends every row to the spill, which the
            // spill pass aggregates partition by partition in shared memory.
            if (q + 1 == kCountTile) fw.hits = fw.tries = 0;
            if (q == kDecideTile && fw.use_smem) {
                const unsigned h = __reduce_add_sync(0xffffffffu, fw.hits);
                const unsigned t = __reduce_add_sync(0xffffffffu, fw.tries);
                if (t >= 256 && h * 8u < t) fw.use_smem = false;
                fw.counting = false;
            }
            __syncwarp();
        }
        if (held >= 0) {  // a wait that gave up left rows behind: release the stage all the same
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty_bar[held]);
        }
    }

    __syncthreads();
    fq = fixq<VT>(s_emax == INT_MIN ? 0 : s_emax, hb);  // the producer warp's threads merge slots too
    ftab_flush<VT>(sm, a, fq, &s_claims);
    if (spill_on)
        for (int i = threadIdx.x; i < parts; i += blockDim.x)
            a.spill_fill[static_cast<int64_t>(i) * a.spill_ctas + blockIdx.x] = min(sfill[i], static_cast<unsigned>(a.spill_cell));
    __syncthreads();
    if (threadIdx.x == 0) publish_claims(a.counters, a.capacity, s_claims);
}

// ---------------------------------------------------------------------------------------------
// Second pass over the spill.  Work item i is partition p = i % parts, slice j = i / parts: the cells j, j + slices, ...
// of p (one per aggregation-pass CTA).  One persistent CTA per SM takes items from a counter in global memory,
// aggregates the item's rows in a bucketed shared table as large as shared memory allows and merges it into the
// global table.  The item's cells are read as one stream (a prefix of their fill counts maps a stream row to its
// cell): warp w takes the contiguous stream range [total w / W, total (w + 1) / W), finds the cell of its first row
// once and then moves its cell cursor forward step by step, so every step but the last takes 64 rows however small
// the cells are, and each warp loads its next step's records before it processes the current one.
// ---------------------------------------------------------------------------------------------
constexpr int kFSpillThreads = 1024;

template <typename VT, int MODE>
__global__ void __launch_bounds__(kFSpillThreads, 1) gb_fspill_kernel(const AggArgs a, int32_t slices) {
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ unsigned long long s_claims;
    __shared__ int s_emax;
    __shared__ int s_item;
    constexpr bool VFLOAT = std::is_floating_point<VT>::value;
    constexpr bool VALS = (MODE & FM_VALS) != 0;
    constexpr int kWarps = kFSpillThreads / 32;
    const FTab tab = ftab(sm, a);
    const int parts = 1 << a.spill_bits;
    const int items = parts * slices;
    unsigned* work = a.spill_fill + static_cast<int64_t>(parts) * a.spill_ctas;  // zeroed by the aggregation pass
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int* pre = reinterpret_cast<int*>(sm + a.so_spill);  // pre[t]: rows of the item's cells before its t-th cell
    // First level of a two-level spill: the rows this pass's table cannot take go to the second level.
    const bool level2 = a.spill2_keys != nullptr;
    const int parts2 = level2 ? (1 << a.spill2_bits) : 0;
    unsigned* fill2 = reinterpret_cast<unsigned*>(sm + a.so_spill2);
    if (threadIdx.x == 0) s_claims = 0;
    if (level2 && blockIdx.x == 0 && threadIdx.x == 0)
        a.spill2_fill[static_cast<int64_t>(parts) * parts2] = 0u;  // the next pass's work counter
    for (;;) {
        if (threadIdx.x == 0) {
            s_item = static_cast<int>(atomicAdd(work, 1u));
            s_emax = INT_MIN;
            pre[0] = 0;
        }
        for (int i = threadIdx.x; i < parts2; i += blockDim.x) fill2[i] = 0u;
        ftab_init<VT>(sm, a, threadIdx.x, blockDim.x);
        __syncthreads();
        const int item = s_item;
        if (item >= items) break;
        const int p = item % parts;
        const int j = item / parts;
        const int64_t cell0 = static_cast<int64_t>(p) * a.spill_ctas;
        const int ncells = (a.spill_ctas - j + slices - 1) / slices;
        for (int t = threadIdx.x; t < ncells; t += blockDim.x)
            pre[t + 1] = min(static_cast<int>(a.spill_fill[cell0 + j + slices * t]), static_cast<int>(a.spill_cell));
        __syncthreads();
        if (warp == 0) {  // inclusive scan of pre[1..ncells]: a chunk per lane, then a warp scan of the chunk sums
            const int per = (ncells + 31) / 32;
            const int t0 = 1 + lane * per;
            int sum = 0;
            for (int t = t0; t < t0 + per && t <= ncells; ++t) sum += pre[t];
            int incl = sum;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, d);
                if (lane >= d) incl += y;
            }
            int run = incl - sum;
            for (int t = t0; t < t0 + per && t <= ncells; ++t) {
                run += pre[t];
                pre[t] = run;
            }
        }
        __syncthreads();
        const int total = pre[ncells];
        const int r_end = static_cast<int>(static_cast<int64_t>(total) * (warp + 1) / kWarps);
        int r0 = static_cast<int>(static_cast<int64_t>(total) * warp / kWarps);
        // The warp's cell cursor: the largest t with pre[t] <= r0 (pre[0] = 0 <= r0; empty cells share a prefix).
        int tw = 0;
        {
            int lo = 0, hi = ncells;
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (pre[mid] <= r0) lo = mid;
                else hi = mid;
            }
            tw = lo;
        }
        // The step starting at stream row s0 (two rows per lane, s0 + lane and s0 + 32 + lane): moves the cursor to
        // the cell of s0, then each lane walks forward to the cell of its own rows and loads their records.
        auto load = [&](int s0, bool (&act)[2], uint64_t (&kw)[2], VT (&v)[2]) {
            while (tw + 1 < ncells && pre[tw + 1] <= s0) ++tw;
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int r = s0 + 32 * u + lane;
                act[u] = r < r_end;
                kw[u] = 0ull;
                v[u] = VT{};
                if (act[u]) {
                    int t = tw;
                    while (t + 1 < ncells && pre[t + 1] <= r) ++t;
                    const int64_t ri = (cell0 + j + static_cast<int64_t>(slices) * t) * a.spill_cell + (r - pre[t]);
                    if constexpr (VALS) {
                        const ulonglong2 x = reinterpret_cast<const ulonglong2*>(a.spill_keys)[ri];
                        kw[u] = x.x;
                        memcpy(&v[u], &x.y, sizeof(VT));
                    } else {
                        kw[u] = a.spill_keys[ri];
                    }
                }
            }
        };
        bool act[2], nact[2];
        uint64_t kw[2], nkw[2];
        VT v[2], nv[2];
        if (r0 < r_end) load(r0, act, kw, v);
        else act[0] = act[1] = false;
        if (VFLOAT && (MODE & FM_SUM)) {  // fixed-point scale from every warp's first rows
            int e = max(act[0] ? fexp<VT>(v[0]) : INT_MIN, act[1] ? fexp<VT>(v[1]) : INT_MIN);
            e = __reduce_max_sync(0xffffffffu, e);
            if (lane == 0 && e != INT_MIN) atomicMax(&s_emax, e);
        }
        __syncthreads();
        const int hb = max(1, 64 - __clzll(static_cast<long long>(total)));
        const FixQ fq = fixq<VT>(s_emax == INT_MIN ? 0 : s_emax, hb);
        FastWarp<VT, MODE> fw(a, tab, fq, &s_claims);
        fw.bshift = 32 - a.spill_bits;
        fw.fits = a.fits != 0;
        fw.probe_b = a.probe_b;
        fw.dedup = a.dedup != 0;
        if (level2) {
            fw.spill_ok = true;
            fw.sfill = smem_u32(fill2);
            fw.cell_cap = static_cast<unsigned>(a.spill2_cell);
            fw.part_shift = 64 - a.spill_bits - a.spill2_bits;
            fw.part_mask = static_cast<uint32_t>(parts2 - 1);
            fw.cell_base = static_cast<int64_t>(p) * parts2;
            fw.cell_mul = 1;
            fw.spill_out = a.spill2_keys;
        }
        for (; r0 < r_end; r0 += 64) {
            const int n0 = r0 + 64;
            if (n0 < r_end) load(n0, nact, nkw, nv);
            fw.rows2(act, kw, v, static_cast<unsigned>(lane));
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                act[u] = nact[u];
                kw[u] = nkw[u];
                v[u] = nv[u];
            }
        }
        __syncthreads();
        for (int i = threadIdx.x; i < parts2; i += blockDim.x)
            a.spill2_fill[static_cast<int64_t>(p) * parts2 + i] = min(fill2[i], static_cast<unsigned>(a.spill2_cell));
        ftab_flush<VT>(sm, a, fq, &s_claims);
        __syncthreads();
    }
    if (threadIdx.x == 0) publish_claims(a.counters, a.capacity, s_claims);
}

// Launches the fast aggregation pass: one persistent CTA per SM (exactly spill_ctas CTAs when spilling).
template <typename KT, bool COMP, typename VT, typename PT, int MODE>
int32_t launch_fast_t(const AggArgs& a, size_t smem, cudaStream_t st) {
    auto kern = gb_fast_kernel<KT, COMP, VT, PT, MODE>;
    const DeviceInfo& di = device_info();
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(gb_fast_kernel)");
    int64_t grid = std::min<int64_t>(di.sm_count, a.tiles);
    if (a.spill_keys) {
        if (a.spill_ctas > grid) return fail(QDB_ERROR, "gb_fast_kernel: spill plan needs more CTAs than fit");
        grid = a.spill_ctas;
    }
    if (grid < 1) return QDB_OK;
    kern<<<static_cast<unsigned>(grid), kFastThreads, smem, st>>>(a);
    note_launch();
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "gb_fast_kernel launch");
    return QDB_OK;
}

template <typename VT, int MODE>
int32_t launch_fspill_t(const AggArgs& a, size_t smem, int64_t grid, int32_t slices, cudaStream_t st) {
    auto kern = gb_fspill_kernel<VT, MODE>;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(gb_fspill_kernel)");
    }
    kern<<<static_cast<unsigned>(grid), kFSpillThreads, smem, st>>>(a, slices);
    note_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "gb_fspill_kernel launch");
    return QDB_OK;
}

// Mode of a table for the fast pass: FM_VALS only when some aggregate reads the values.
inline int fast_mode(const AggArgs& a) {
    const int mm = (a.has_min || a.has_max) ? FM_MM : 0;
    const int sum = a.has_sum ? FM_SUM : 0;
    return (mm | sum) ? (FM_VALS | mm | sum) : 0;
}

// The compressed-key variant exists for single keys other than DOUBLE; plain keys run the kernel without it.  KM
// selects the fused key % m variant (instantiated in its own translation units, fast_i32_mod.cu and fast_i64_mod.cu).
template <typename KT, bool COMP, typename VT, typename PT, int MODE, bool KM>
int32_t launch_fast_z(const AggArgs& a, size_t smem, cudaStream_t st) {
    if constexpr (KM) {
        return launch_fast_t<KT, COMP, VT, PT, MODE | FM_KMOD>(a, smem, st);
    } else {
        if constexpr (!COMP && !std::is_same<KT, double>::value) {
            if (a.kz) return launch_fast_t<KT, COMP, VT, PT, MODE | FM_KZ>(a, smem, st);
        }
        if (a.kz) return fail(QDB_ERR_INVALID, "gb_fast_kernel: compressed keys need a single INT32, INT64 or FLOAT key");
        return launch_fast_t<KT, COMP, VT, PT, MODE>(a, smem, st);
    }
}

template <typename KT, bool COMP, typename VT, typename PT, bool KM>
int32_t launch_fast_m(const AggArgs& a, size_t smem, cudaStream_t st) {
    switch (fast_mode(a)) {
        case FM_VALS | FM_SUM: return launch_fast_z<KT, COMP, VT, PT, FM_VALS | FM_SUM, KM>(a, smem, st);
        case FM_VALS | FM_MM: return launch_fast_z<KT, COMP, VT, PT, FM_VALS | FM_MM, KM>(a, smem, st);
        case FM_VALS | FM_SUM | FM_MM: return launch_fast_z<KT, COMP, VT, PT, FM_VALS | FM_SUM | FM_MM, KM>(a, smem, st);
        default: return fail(QDB_ERR_INVALID, "gb_fast_kernel: unsupported aggregate set");
    }
}

template <typename KT, bool COMP, typename PT, bool KM>
int32_t launch_fast_v(const AggArgs& a, ValKind vk, size_t smem, cudaStream_t st) {
    if (fast_mode(a) == 0) return launch_fast_z<KT, COMP, int32_t, PT, 0, KM>(a, smem, st);
    switch (vk) {
        case VK_I32: return launch_fast_m<KT, COMP, int32_t, PT, KM>(a, smem, st);
        case VK_I64: return launch_fast_m<KT, COMP, int64_t, PT, KM>(a, smem, st);
        case VK_F32: return launch_fast_m<KT, COMP, float, PT, KM>(a, smem, st);
        case VK_F64: return launch_fast_m<KT, COMP, double, PT, KM>(a, smem, st);
        default: return fail(QDB_ERR_INVALID, "unsupported value type");
    }
}

template <typename KT, bool COMP, bool KM = false>
int32_t launch_fast_k(const AggArgs& a, ValKind vk, int32_t ptype, size_t smem, cudaStream_t st) {
    switch (ptype) {
        case 0: return launch_fast_v<KT, COMP, NoPred, KM>(a, vk, smem, st);
        case QDB_INT32: return launch_fast_v<KT, COMP, int32_t, KM>(a, vk, smem, st);
        case QDB_INT64: return launch_fast_v<KT, COMP, int64_t, KM>(a, vk, smem, st);
        case QDB_FLOAT: return launch_fast_v<KT, COMP, float, KM>(a, vk, smem, st);
        case QDB_DOUBLE: return launch_fast_v<KT, COMP, double, KM>(a, vk, smem, st);
        default: return fail(QDB_ERR_INVALID, "unsupported predicate column type");
    }
}

template <typename VT>
int32_t launch_fspill_m(const AggArgs& a, size_t smem, int64_t grid, int32_t slices, cudaStream_t st) {
    switch (fast_mode(a)) {
        case FM_VALS | FM_SUM: return launch_fspill_t<VT, FM_VALS | FM_SUM>(a, smem, grid, slices, st);
        case FM_VALS | FM_MM: return launch_fspill_t<VT, FM_VALS | FM_MM>(a, smem, grid, slices, st);
        case FM_VALS | FM_SUM | FM_MM: return launch_fspill_t<VT, FM_VALS | FM_SUM | FM_MM>(a, smem, grid, slices, st);
        default: return fail(QDB_ERR_INVALID, "gb_fspill_kernel: unsupported aggregate set");
    }
}

// Per-key-type entry points of the fast pass, each instantiated in its key type's translation unit.
int32_t launch_fast_i32(const AggArgs& a, ValKind vk, int32_t ptype, size_t smem, cudaStream_t st);
int32_t launch_fast_i64(const AggArgs& a, ValKind vk, int32_t ptype, size_t smem, cudaStream_t st);
int32_t launch_fast_i32_mod(const AggArgs& a, ValKind vk, int32_t ptype, size_t smem, cudaStream_t st);
int32_t launch_fast_i64_mod(const AggArgs& a, ValKind vk, int32_t ptype, size_t smem, cudaStream_t st);
int32_t launch_fast_f32(const AggArgs& a, ValKind vk, int32_t ptype, size_t smem, cudaStream_t st);
int32_t launch_fast_f64(const AggArgs& a, ValKind vk, int32_t ptype, size_t smem, cudaStream_t st);
int32_t launch_fast_comp(const AggArgs& a, ValKind vk, int32_t ptype, size_t smem, cudaStream_t st);

}  // namespace qdb
