// The fused filter + hash-aggregate pass (the B200 replacement of kernel_filter ->
// reconstructColKeep -> group_by_kernel, qikkDB/QueryEngine/GPUCore/GPUFilter.cuh:22-44,
// GPUReconstruct.cuh:29-45 and :272-355, GPUGroupBy.cuh:68-196).
//
// One persistent CTA per SM walks 4096-row tiles of the input columns with 128-bit evict-first
// loads, prefetching the next tile into registers while it works on the current one.  For every row
// it evaluates the predicate and the optional mask in registers (no mask or compacted column is
// written to HBM), then inserts the key:
//   * first into a per-CTA shared-memory table (bounded linear probe, shared-memory atomics), which
//     absorbs low-cardinality and skewed (Zipf) key streams;
//   * on a shared-memory miss, into the global open-addressing table (bounded linear probe with a
//     64-bit atomicCAS on the key word, fire-and-forget reductions on the state words).  The first
//     probe loads of a thread's misses are issued together so their L2 latencies overlap.
// A warp that sees a low shared-memory hit rate after its first tiles stops probing shared memory.
// At the end each CTA merges its shared-memory table into the global table.
#pragma once

#include "groupby.cuh"

namespace qdb {

constexpr int kAggThreads = 512;
constexpr int kItems = 8;                         // rows per thread per tile (two 4-row vectors)
constexpr int kTileRows = kAggThreads * kItems;   // 4096
constexpr int kDecideTile = 3;                    // tile index at which a warp judges its hit rate

struct PredConst {
    int32_t op = -1;     // qdb_cmp, -1 = no predicate
    int32_t ctype = 0;   // qdb_type of the constant
    int64_t ci = 0;
    double cf = 0.0;
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
    PredConst pc;
    const int8_t* mask = nullptr;
    int64_t n = 0;
    int64_t tiles = 0;
    Region main;
    Region aux;
    Layout L;
    int32_t has_sum = 0;
    int32_t has_min = 0;
    int32_t has_max = 0;
    unsigned long long* counters = nullptr;  // [0] groups, [1] status
    unsigned long long capacity = 0;
    int32_t S = 0;       // shared-memory slots (power of two) or 0 for a global-only pass
    int32_t probe = 0;   // shared-memory probe limit
    int32_t vec_ok = 0;  // all column pointers 16-byte aligned
    // byte offsets of the shared-memory arrays (S + 2 entries each)
    int32_t so_sum = 0, so_mn = 0, so_mx = 0, so_cnt = 0;
};

// ---------------------------------------------------------------------------------------------
// Predicate: `col OP constant` in the C++ common type of (column type, constant type), exactly as
// kernel_filter evaluates OP{}(a, b) on typed operands (GPUFilterConditions.cuh:9-120).
// ---------------------------------------------------------------------------------------------
template <typename A, typename B>
__device__ __forceinline__ bool cmp_op(int32_t op, A a, B b) {
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

template <typename PT>
__device__ __forceinline__ bool eval_pred(const PredConst& pc, PT a) {
    switch (pc.ctype) {
        case QDB_INT32: return cmp_op(pc.op, a, static_cast<int32_t>(pc.ci));
        case QDB_INT64: return cmp_op(pc.op, a, static_cast<int64_t>(pc.ci));
        case QDB_FLOAT: return cmp_op(pc.op, a, static_cast<float>(pc.cf));
        case QDB_DOUBLE: return cmp_op(pc.op, a, pc.cf);
        case QDB_INT8: return cmp_op(pc.op, a, static_cast<int8_t>(pc.ci));
        default: return false;
    }
}

struct NoPred {};

// ---------------------------------------------------------------------------------------------
// 4-row vector loads.  Row r0 is a multiple of 4; `full` means rows r0..r0+3 are all < n and the
// pointer is 16-byte aligned.
// ---------------------------------------------------------------------------------------------
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

__device__ __forceinline__ void claim_counted(unsigned long long* counters, unsigned long long capacity) {
    if (atomicAdd(&counters[0], 1ull) >= capacity)
        atomicExch(reinterpret_cast<int*>(&counters[1]), static_cast<int>(QDB_HASH_TABLE_FULL));
}

__device__ __forceinline__ bool table_full(const unsigned long long* counters) {
    return ld_volatile_i32(reinterpret_cast<const int32_t*>(&counters[1])) == QDB_HASH_TABLE_FULL;
}

// Finds or claims `key` in region R starting at slot s whose key word `cur` was already loaded.
// The probe visits at most every slot once, so it always ends; it gives up (returns nullptr) when the
// region is full or another thread has already reported HASH_TABLE_FULL.
__device__ __forceinline__ uint64_t* g_find_from(const Region& R, int W, uint64_t key, uint64_t s, uint64_t cur,
                                                 unsigned long long* counters, unsigned long long capacity) {
    for (uint64_t i = 0; i <= R.mask; ++i) {
        uint64_t* slot = R.slots + s * W;
        if (i > 0) cur = ld_volatile_u64(slot);
        if (cur == key) return slot;
        if (cur == kEmpty) {
            unsigned long long prev = atomicCAS(reinterpret_cast<unsigned long long*>(slot), kEmpty, key);
            if (prev == kEmpty) {
                claim_counted(counters, capacity);
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
                                            unsigned long long* counters, unsigned long long capacity) {
    const uint64_t s = h & R.mask;
    return g_find_from(R, W, key, s, ld_volatile_u64(R.slots + s * W), counters, capacity);
}

// Special slot `which` (0: NULL key, 1: the key equal to kEmpty) of the main region.
__device__ __forceinline__ uint64_t* g_special(const Region& R, int W, int which, unsigned long long* counters,
                                               unsigned long long capacity) {
    uint64_t* slot = R.slots + (R.mask + 1 + which) * W;
    if (ld_volatile_u64(slot) == kEmpty) {
        unsigned long long prev = atomicCAS(reinterpret_cast<unsigned long long*>(slot), kEmpty, 0ull);
        if (prev == kEmpty && which == 1) claim_counted(counters, capacity);
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

// Shared-memory probe.  Returns the slot, or -1 after `P` probes.  *found is set when the key was
// already present (a reuse rather than a first claim).
__device__ __forceinline__ int s_find(uint64_t* skey, int S, int P, uint64_t key, uint64_t h, bool* found) {
    uint32_t s = static_cast<uint32_t>(h >> 40) & static_cast<uint32_t>(S - 1);
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

// ---------------------------------------------------------------------------------------------
// The aggregation kernel.  KT: key column type; COMP: composite (int32, int32) key; VT: value type
// (int32_t when the table has no value column); PT: predicate column type or NoPred.
// ---------------------------------------------------------------------------------------------
template <typename KT, bool COMP, typename VT, typename PT>
__global__ void __launch_bounds__(kAggThreads, 1) gb_agg_kernel(const AggArgs a) {
    extern __shared__ __align__(16) unsigned char sm[];
    constexpr bool HAS_PRED = !std::is_same<PT, NoPred>::value;
    using PL = typename std::conditional<HAS_PRED, PT, int8_t>::type;  // storage type for predicate lanes

    const int S = a.S;
    const int S2 = S ? S + 2 : 0;
    uint64_t* skey = reinterpret_cast<uint64_t*>(sm);
    const bool has_mm = a.has_min || a.has_max;

    if (S) {
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
    }
    __syncthreads();

    const bool has_vals = a.vals != nullptr;
    const KT* __restrict__ k0p = static_cast<const KT*>(a.key0);
    const KT* __restrict__ k1p = static_cast<const KT*>(a.key1);
    const VT* __restrict__ vp = static_cast<const VT*>(a.vals);
    const PL* __restrict__ pp = static_cast<const PL*>(a.pcol);
    const int W = a.L.W;

    bool use_smem = S > 0;
    unsigned my_hits = 0, my_tries = 0;

    // Register fragments of the current and the next tile.
    KT ck0[2][4], ck1[2][4], nk0[2][4], nk1[2][4];
    VT cv[2][4], nv[2][4];
    PL cp[2][4], np[2][4];
    uint32_t cm[2], nm[2];  // 4 mask bytes per vector

    auto row0 = [&](int64_t tile, int j) -> int64_t {
        return tile * kTileRows + (static_cast<int64_t>(j) * kAggThreads + threadIdx.x) * 4;
    };
    auto load_tile = [&](int64_t tile, KT (&k0)[2][4], KT (&k1)[2][4], VT (&v)[2][4], PL (&p)[2][4],
                         uint32_t (&m)[2]) {
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int64_t r0 = row0(tile, j);
            const bool full = a.vec_ok && (r0 + 4 <= a.n);
            if (r0 >= a.n) continue;
            load4<KT>(k0p, r0, a.n, full, k0[j]);
            if constexpr (COMP) load4<KT>(k1p, r0, a.n, full, k1[j]);
            if (has_vals) load4<VT>(vp, r0, a.n, full, v[j]);
            if constexpr (HAS_PRED) load4<PL>(pp, r0, a.n, full, p[j]);
            if (a.mask) {
                int8_t mb[4];
                load4<int8_t>(a.mask, r0, a.n, full, mb);
                memcpy(&m[j], mb, 4);
            }
        }
    };

    int64_t tile = blockIdx.x;
    if (tile < a.tiles) load_tile(tile, ck0, ck1, cv, cp, cm);

    for (int it = 0; tile < a.tiles; ++it, tile += gridDim.x) {
        const int64_t next = tile + gridDim.x;
        if (next < a.tiles) load_tile(next, nk0, nk1, nv, np, nm);

        // Pass 1: predicate, key word and the shared-memory table.
        uint64_t kw[8];
        uint32_t kinds = 0;  // 2 bits per item
        uint32_t pend = 0;   // items still to insert into the global table
        uint32_t cntit = 0;  // items whose value is aggregated (non-NULL value, or no value column)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int64_t r0 = row0(tile, j);
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int i = j * 4 + e;
                const int64_t r = r0 + e;
                kw[i] = 0;
                int kind = KK_NORMAL;
                if (r >= a.n) continue;
                bool keep = true;
                if constexpr (HAS_PRED) keep = eval_pred<PT>(a.pc, cp[j][e]) && !null_bit(a.pnull, r);
                if (a.mask) keep = keep && (((cm[j] >> (8 * e)) & 0xffu) != 0u);
                if (!keep) continue;
                if constexpr (COMP) {
                    const bool n0 = null_bit(a.knull0, r);
                    const bool n1 = null_bit(a.knull1, r);
                    if (n0 || n1) {
                        kind = KK_AUX;
                        const uint32_t other = n0 ? (n1 ? 0u : static_cast<uint32_t>(ck1[j][e]))
                                                  : static_cast<uint32_t>(ck0[j][e]);
                        kw[i] = (static_cast<uint64_t>((n0 ? 1u : 0u) | (n1 ? 2u : 0u)) << 32) | other;
                    } else {
                        kw[i] = composite_word(static_cast<int32_t>(ck0[j][e]), static_cast<int32_t>(ck1[j][e]));
                        kind = (kw[i] == kEmpty) ? KK_ESCAPE : KK_NORMAL;
                    }
                } else {
                    if (null_bit(a.knull0, r)) {
                        kind = KK_NULL;
                    } else {
                        kw[i] = key_word(ck0[j][e]);
                        kind = (kw[i] == kEmpty) ? KK_ESCAPE : KK_NORMAL;
                    }
                }
                kinds |= static_cast<uint32_t>(kind) << (2 * i);
                const bool agg_it = !has_vals || !null_bit(a.vnull, r);
                if (agg_it) cntit |= 1u << i;
                int s = -1;
                if (use_smem && kind != KK_AUX) {
                    if (kind == KK_NORMAL) {
                        bool found = false;
                        s = s_find(skey, S, a.probe, kw[i], mix64(kw[i]), &found);
                        ++my_tries;
                        my_hits += found ? 1u : 0u;
                    } else {
                        s = S + (kind == KK_ESCAPE ? 1 : 0);
                        if (*reinterpret_cast<volatile uint64_t*>(&skey[s]) == kEmpty)
                            atomicCAS(reinterpret_cast<unsigned long long*>(&skey[s]), kEmpty, 0ull);
                    }
                }
                if (s >= 0) {
                    if (agg_it) s_acc_row<VT>(sm, a, s, has_vals ? cv[j][e] : VT{}, has_vals);
                } else {
                    pend |= 1u << i;
                }
            }
        }

        // Pass 2: global table for the shared-memory misses; first probes issued together.
        if (pend) {
            uint64_t first[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                first[i] = 0;
                const int kind = (kinds >> (2 * i)) & 3;
                if (((pend >> i) & 1u) && (kind == KK_NORMAL || kind == KK_AUX)) {
                    const Region& R = (kind == KK_AUX) ? a.aux : a.main;
                    first[i] = ld_volatile_u64(R.slots + (mix64(kw[i]) & R.mask) * W);
                }
            }
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                if (!((pend >> i) & 1u)) continue;
                const int kind = (kinds >> (2 * i)) & 3;
                uint64_t* slot;
                if (kind == KK_NORMAL || kind == KK_AUX) {
                    const Region& R = (kind == KK_AUX) ? a.aux : a.main;
                    slot = g_find_from(R, W, kw[i], mix64(kw[i]) & R.mask, first[i], a.counters, a.capacity);
                } else {
                    slot = g_special(a.main, W, kind == KK_ESCAPE ? 1 : 0, a.counters, a.capacity);
                }
                if (slot && ((cntit >> i) & 1u)) {
                    if (has_vals) g_acc_row<VT>(slot, a, cv[i >> 2][i & 3]);
                    else g_count_row(slot, a.L);
                }
            }
        }

        // Warp-uniform control: stop on a full table; judge the shared-memory hit rate once.
        if (__any_sync(0xffffffffu, table_full(a.counters))) break;
        if (it == kDecideTile && use_smem) {
            const unsigned hits = __reduce_add_sync(0xffffffffu, my_hits);
            const unsigned tries = __reduce_add_sync(0xffffffffu, my_tries);
            if (tries >= 256 && hits * 8u < tries) use_smem = false;
        }

        if (next < a.tiles) {
#pragma unroll
            for (int j = 0; j < 2; ++j)
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    ck0[j][e] = nk0[j][e];
                    if constexpr (COMP) ck1[j][e] = nk1[j][e];
                    cv[j][e] = nv[j][e];
                    cp[j][e] = np[j][e];
                }
#pragma unroll
            for (int j = 0; j < 2; ++j) cm[j] = nm[j];
        }
    }

    // Merge this CTA's shared-memory table into the global table.
    __syncthreads();
    if (S) {
        const bool v32 = sizeof(VT) == 4;
        const bool vfloat = std::is_floating_point<VT>::value;
        for (int i = threadIdx.x; i < S2; i += blockDim.x) {
            const uint64_t key = skey[i];
            if (key == kEmpty) continue;
            uint64_t* slot = (i < S) ? g_find(a.main, W, key, mix64(key), a.counters, a.capacity)
                                     : g_special(a.main, W, i - S, a.counters, a.capacity);
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
}

// Launches the kernel for one (key, value, predicate) type combination.
template <typename KT, bool COMP, typename VT, typename PT>
int32_t launch_agg_t(const AggArgs& a, size_t smem, cudaStream_t st) {
    auto kern = gb_agg_kernel<KT, COMP, VT, PT>;
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
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "gb_agg_kernel launch");
    return QDB_OK;
}

template <typename KT, bool COMP, typename VT>
int32_t launch_agg_p(const AggArgs& a, int32_t ptype, size_t smem, cudaStream_t st) {
    switch (ptype) {
        case 0: return launch_agg_t<KT, COMP, VT, NoPred>(a, smem, st);
        case QDB_INT32: return launch_agg_t<KT, COMP, VT, int32_t>(a, smem, st);
        case QDB_INT64: return launch_agg_t<KT, COMP, VT, int64_t>(a, smem, st);
        case QDB_FLOAT: return launch_agg_t<KT, COMP, VT, float>(a, smem, st);
        case QDB_DOUBLE: return launch_agg_t<KT, COMP, VT, double>(a, smem, st);
        default: return fail(QDB_ERR_INVALID, "unsupported predicate column type");
    }
}

template <typename KT, bool COMP>
int32_t launch_agg_k(const AggArgs& a, ValKind vk, int32_t ptype, size_t smem, cudaStream_t st) {
    switch (vk) {
        case VK_NONE:
        case VK_I32: return launch_agg_p<KT, COMP, int32_t>(a, ptype, smem, st);
        case VK_I64: return launch_agg_p<KT, COMP, int64_t>(a, ptype, smem, st);
        case VK_F32: return launch_agg_p<KT, COMP, float>(a, ptype, smem, st);
        case VK_F64: return launch_agg_p<KT, COMP, double>(a, ptype, smem, st);
        default: return fail(QDB_ERR_INVALID, "unsupported value type");
    }
}

// Per-key-type entry points, each instantiated in its own translation unit.
int32_t launch_agg_i32(const AggArgs& a, ValKind vk, int32_t ptype, size_t smem, cudaStream_t st);
int32_t launch_agg_i64(const AggArgs& a, ValKind vk, int32_t ptype, size_t smem, cudaStream_t st);
int32_t launch_agg_f32(const AggArgs& a, ValKind vk, int32_t ptype, size_t smem, cudaStream_t st);
int32_t launch_agg_f64(const AggArgs& a, ValKind vk, int32_t ptype, size_t smem, cudaStream_t st);
int32_t launch_agg_comp(const AggArgs& a, ValKind vk, int32_t ptype, size_t smem, cudaStream_t st);

}  // namespace qdb
