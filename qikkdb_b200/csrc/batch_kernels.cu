// Kernels of the batched GROUP BY: table initialisation, the persistent work-queue aggregation kernel and the
// result kernel.  The reference runs group_by_kernel once per query and block (GPUGroupBy.cuh:68-196,
// :395-410) and one GetResults per query (:478-587); here every query of a batch is a set of work items in
// one launch.
//
// Aggregation kernel: one CTA per SM of 12 consumer warps and 4 producer warps.  The CTA drains three work queues
// in turn; in queue q it is split into 2^q warp groups (12, 6 or 3 consumer warps plus one producer warp), each
// with its own share of shared memory, so that small queries do not hold a whole SM.  A work item is a row range
// of a scan group: up to kBMaxMembers queries over the same columns.  Per group:
//   * the producer warp takes items from the queue and streams their column tiles (keys, values, predicate
//     column) into a ring of shared-memory stages with bulk asynchronous copies (cp.async.bulk, TMA engine)
//     completing on per-stage mbarriers; the copies of the next item overlap the merge of the current one;
//   * the consumer warps take the stages in order and apply every member query to the tile: WHERE interval,
//     key modulus, then the insert
//       - shared placement: into one of the query's R shared-memory tables (warp w uses table w % R, so
//         low-cardinality queries spread their same-key atomics over R copies); after the item's last tile every
//         occupied shared slot is merged into the query's global table;
//       - global placement: straight into the query's global table, each lane issuing the probe loads of all
//         its rows of the tile before completing any of them.
// Rows whose shared-memory probe fails (a cardinality estimate that was too low) go to the global table.
// All waits (ring stages, consumer-group syncs) are mbarrier waits with an iteration limit; a wait that gives up
// records QDB_ERR_TIMEOUT, which the result kernel reports for every query.  Every item is timed with the global
// timer for the autotuner.
#include <climits>

#include "batch.cuh"

namespace qdb {

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Bounded wait on phase `parity`; gives up after kMaxWaitIters tries (each suspends up to 10 us) and records
// QDB_ERR_TIMEOUT in *err.
__device__ __forceinline__ bool b_wait(uint64_t* bar, uint32_t parity, int32_t* err) {
    for (uint32_t it = 0; it < kMaxWaitIters; ++it)
        if (mbar_try_wait_for(bar, parity, 10000u)) return true;
    atomicExch(err, static_cast<int>(QDB_ERR_TIMEOUT));
    return false;
}

// ---------------------------------------------------------------------------------------------
// Table initialisation (only after a new plan: the result kernel cleans every slot it reads).
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) gb_batch_init_kernel(const BatchArgs ba) {
    if (blockIdx.x == 0 && threadIdx.x == 0) ba.hdr->error = 0;
    if (!ba.hdr->init_needed) return;
    const int i = blockIdx.x;
    if (i >= ba.hdr->n_inst) return;
    const BInst& I = ba.inst[i];
    const int W = I.L.W;
    const uint64_t words = (I.main.mask + 3) * static_cast<uint64_t>(W);
    for (uint64_t w = threadIdx.x; w < words; w += blockDim.x) {
        const int r = static_cast<int>(w % W);
        uint64_t v = 0;
        if (r == 0) v = kEmpty;
        else if (r == I.L.mn && I.L.packed) v = kPackedMinMaxInit;
        else if (r == I.L.mn) v = kMinInit64;
        else if (r == I.L.mx) v = kMaxInit64;
        I.main.slots[w] = v;
    }
    if (threadIdx.x == 0) {
        I.counters[0] = 0;
        I.counters[1] = 0;
    }
}

// ---------------------------------------------------------------------------------------------
// State updates with explicit layouts (shared and global).
// ---------------------------------------------------------------------------------------------
struct BSmem {
    uint64_t* key;
    unsigned long long* sum;
    unsigned char* mn;
    unsigned char* mx;
    unsigned int* cnt;
};

// float SUM in a shared slot: a 64-bit two's-complement fixed-point accumulator of q = v * 2^F in the slot's sum
// word, F = 31 - e with e the largest exponent (|v| < 2^e) of the item's first tile.  A value is kept when its
// shift e_v - sh0 lies in [-1, 15], so q is in [2^22, 2^39): exact, or rounded to 23 significant bits when the
// shift is -1, and the at most 2^24 rows of an item cannot overflow the word.  Other values (and NaN, Inf,
// subnormals) take the global FP64 path.
struct BFix {
    int sh0 = 119;     // emax + 119
    double inv = 0.0;  // 2^-F
};

__device__ __forceinline__ BFix b_fix(int emax) {
    emax = max(-100, min(100, emax));
    BFix f;
    f.sh0 = emax + 119;
    f.inv = ldexp(1.0, emax - 31);
    return f;
}

__device__ __forceinline__ long long b_addend(float v, const BFix& f, bool* ok) {
    const uint32_t b = __float_as_uint(v);
    const int e = static_cast<int>((b >> 23) & 0xffu);
    const uint32_t fr = b & 0x7fffffu;
    if (e == 0) {
        *ok = fr == 0u;
        return 0ll;
    }
    const int sh = e - f.sh0;
    *ok = e != 0xff && sh >= -1 && sh <= 15;
    if (!*ok) return 0ll;
    const uint32_t m = fr | 0x800000u;
    const long long q = sh >= 0 ? static_cast<long long>(static_cast<uint64_t>(m) << sh)
                                : static_cast<long long>((m + (1u << (-sh - 1))) >> (-sh));
    return (b >> 31) ? -q : q;
}

// q: the integer value, or the fixed-point addend of a float value.
template <typename VT>
__device__ __forceinline__ void b_s_acc(const BSmem& t, int s, VT v, long long q, bool has_vals, bool has_sum,
                                        bool has_min, bool has_max) {
    atomicAdd(t.cnt + s, 1u);
    if (!has_vals) return;
    if (has_sum) {
        if constexpr (std::is_same<VT, double>::value) {
            atomicAdd(reinterpret_cast<double*>(t.sum) + s, v);
        } else {
            // The 64-bit two's-complement add as two 32-bit shared atomics on the halves of the word (the carry out
            // of the low half is read from the value its atomic returns): the same word as a 64-bit atomicAdd,
            // without the 64-bit CAS loop that serialises when many lanes hit one slot.
            const unsigned long long u = static_cast<unsigned long long>(q);
            unsigned* w = reinterpret_cast<unsigned*>(t.sum + s);
            const unsigned x0 = static_cast<unsigned>(u), x1 = static_cast<unsigned>(u >> 32);
            const unsigned old = atomicAdd(w, x0);
            const unsigned hi = x1 + ((old + x0 < old) ? 1u : 0u);
            if (hi) atomicAdd(w + 1, hi);
        }
    }
    // min/max: an atomic only when the value improves on the slot's current bound
    if constexpr (sizeof(VT) == 4) {
        const int32_t e = enc32(v);
        int* mn = reinterpret_cast<int*>(t.mn) + 2 * s;
        int* mx = reinterpret_cast<int*>(t.mx) + 2 * s + 1;
        if (has_min && e < *reinterpret_cast<volatile int*>(mn)) atomicMin(mn, e);
        if (has_max && e > *reinterpret_cast<volatile int*>(mx)) atomicMax(mx, e);
    } else {
        const long long e = enc64(v);
        long long* mn = reinterpret_cast<long long*>(t.mn) + s;
        long long* mx = reinterpret_cast<long long*>(t.mx) + s;
        if (has_min && e < *reinterpret_cast<volatile long long*>(mn)) atomicMin(mn, e);
        if (has_max && e > *reinterpret_cast<volatile long long*>(mx)) atomicMax(mx, e);
    }
}

template <typename VT>
__device__ __forceinline__ void b_g_acc(uint64_t* slot, const Layout& L, VT v, bool has_vals, bool has_sum,
                                        bool has_min, bool has_max) {
    if (L.cnt >= 0) atomicAdd(reinterpret_cast<unsigned long long*>(slot + L.cnt), 1ull);
    if (!has_vals) return;
    if (has_sum) {
        if constexpr (std::is_floating_point<VT>::value)
            atomicAdd(reinterpret_cast<double*>(slot + L.sum), static_cast<double>(v));
        else
            atomicAdd(reinterpret_cast<unsigned long long*>(slot + L.sum),
                      static_cast<unsigned long long>(static_cast<long long>(v)));
    }
    if constexpr (sizeof(VT) == 4) {
        const int32_t e = enc32(v);
        if (has_min) atomicMin(reinterpret_cast<int*>(slot + L.mn), e);
        if (has_max) atomicMax(reinterpret_cast<int*>(slot + L.mx) + 1, e);
    } else {
        const long long e = enc64(v);
        if (has_min) atomicMin(reinterpret_cast<long long*>(slot + L.mn), e);
        if (has_max) atomicMax(reinterpret_cast<long long*>(slot + L.mx), e);
    }
}

// Ordinal of a predicate column value (order-preserving for IEEE values, identity for integers).
__device__ __forceinline__ int64_t pred_ord32(int32_t b, bool is_float) {
    return is_float ? static_cast<int64_t>(b ^ ((b >> 31) & 0x7fffffff)) : static_cast<int64_t>(b);
}
__device__ __forceinline__ int64_t pred_ord64(int64_t b, bool is_float) {
    return is_float ? (b ^ ((b >> 63) & 0x7fffffffffffffffll)) : b;
}


// ---------------------------------------------------------------------------------------------
// Warp-group plumbing.
// ---------------------------------------------------------------------------------------------
constexpr int kMetaFirst = 1;  // first tile of its item
constexpr int kMetaLast = 2;   // last tile of its item
constexpr int kMetaDone = 4;   // the queue is exhausted

struct BStageMeta {
    int32_t item;
    int32_t flags;
    int64_t r0;
    int32_t nrows;
    int32_t pad;
};

// The header of a warp group's shared memory.
struct BGroupSmem {
    uint64_t full[kBStages];
    uint64_t empty[kBStages];
    uint64_t csync;
    uint64_t pad;
    BStageMeta meta[kBStages];
    int32_t emax;  // largest value exponent of the current item's first tile (float values)
    int32_t pad2;
};
static_assert(sizeof(BGroupSmem) <= kBHeaderBytes, "group header");

// Column offsets inside one stage tile of `rows` rows.
__device__ __forceinline__ int b_align128(int x) { return (x + 127) & ~127; }

// Sync of the consumer warps of one group (mbarrier with one arrival per warp; bounded wait).
__device__ __forceinline__ void b_csync(uint64_t* bar, uint32_t& parity, int32_t* err) {
    __syncwarp();
    if ((threadIdx.x & 31) == 0) mbar_arrive(bar);
    b_wait(bar, parity, err);
    parity ^= 1u;
    __syncwarp();
}

// Shared-memory arrays of one query's tables inside the group's table region.
__device__ __forceinline__ BSmem b_tables(unsigned char* base, const BInst& I, bool v32) {
    const int RS = I.S * I.R;
    const bool has_mm = I.has_min || I.has_max;
    unsigned char* t0 = base + I.so_table;
    BSmem t;
    t.key = reinterpret_cast<uint64_t*>(t0);
    size_t off = static_cast<size_t>(RS) * 8;
    t.sum = reinterpret_cast<unsigned long long*>(t0 + off);
    if (I.has_sum) off += static_cast<size_t>(RS) * 8;
    t.mn = t0 + off;
    t.mx = t0 + off;
    if (has_mm) {
        off += static_cast<size_t>(RS) * 8;
        if (!v32) {
            t.mx = t0 + off;
            off += static_cast<size_t>(RS) * 8;
        }
    }
    t.cnt = reinterpret_cast<unsigned int*>(t0 + off);
    return t;
}

template <typename VT>
__device__ void b_clear(unsigned char* base, const BInst& I, int ctid, int cthreads) {
    constexpr bool V32 = sizeof(VT) == 4;
    const int RS = I.S * I.R;
    if (RS == 0) return;
    const BSmem t = b_tables(base, I, V32);
    const bool has_sum = I.has_sum, has_mm = I.has_min || I.has_max;
    for (int i = ctid; i < RS; i += cthreads) {
        t.key[i] = kEmpty;
        t.cnt[i] = 0u;
        if (has_sum) t.sum[i] = 0ull;
        if (has_mm) {
            if (V32) {
                reinterpret_cast<unsigned long long*>(t.mn)[i] = kPackedMinMaxInit;
            } else {
                reinterpret_cast<unsigned long long*>(t.mn)[i] = kMinInit64;
                reinterpret_cast<unsigned long long*>(t.mx)[i] = kMaxInit64;
            }
        }
    }
}

// Merges one query's shared tables into its global table.
template <typename VT>
__device__ void b_flush(unsigned char* base, const BInst& I, int ctid, int cthreads, unsigned long long* claims,
                        const BFix& fx) {
    constexpr bool V32 = sizeof(VT) == 4;
    const int RS = I.S * I.R;
    if (RS == 0) return;
    const BSmem t = b_tables(base, I, V32);
    const bool has_vals = I.vk != VK_NONE;
    const bool has_sum = I.has_sum, has_min = I.has_min, has_max = I.has_max, has_mm = has_min || has_max;
    const bool vfloat = std::is_floating_point<VT>::value;
    const Layout L = I.L;
    const Region main = I.main;
    for (int i = ctid; i < RS; i += cthreads) {
        const uint64_t key = t.key[i];
        if (key == kEmpty) continue;
        uint64_t* slot = g_find(main, L.W, key, mix64(key), I.counters, claims);
        if (!slot) continue;
        const unsigned long long c = t.cnt[i];
        uint64_t sumbits = has_sum ? t.sum[i] : 0ull;
        if (has_sum && std::is_same<VT, float>::value) {  // fixed point -> FP64
            const double d = static_cast<double>(static_cast<long long>(sumbits)) * fx.inv;
            memcpy(&sumbits, &d, 8);
        }
        long long mn = 0, mx = 0;
        if (has_mm) {
            if (V32) {
                const int* w = reinterpret_cast<const int*>(t.mn) + 2 * i;
                mn = w[0];
                mx = w[1];
            } else {
                mn = reinterpret_cast<const long long*>(t.mn)[i];
                mx = reinterpret_cast<const long long*>(t.mx)[i];
            }
        }
        if (has_vals) g_merge(slot, L, has_sum, has_min, has_max, V32, vfloat, c, sumbits, mn, mx);
        else if (L.cnt >= 0) atomicAdd(reinterpret_cast<unsigned long long*>(slot + L.cnt), c);
    }
}

// Shared-memory probe of a table of any S slots: the 32-bit multiplicative hash of the folded key is mapped to
// [0, S) by a multiply-high (Lemire's range reduction), then linear probing with wrap-around.  Returns the slot or
// -1 after P probes.
__device__ __forceinline__ int b_s_find(uint64_t* skey, int S, int P, uint64_t key) {
    const uint32_t f = static_cast<uint32_t>(key) ^ static_cast<uint32_t>(key >> 32);
    int s = static_cast<int>(__umulhi(f * 0x9e3779b1u, static_cast<uint32_t>(S)));
    for (int p = 0; p < P; ++p) {
        const uint64_t cur = *reinterpret_cast<volatile uint64_t*>(&skey[s]);
        if (cur == key) return s;
        if (cur == kEmpty) {
            const unsigned long long prev = atomicCAS(reinterpret_cast<unsigned long long*>(&skey[s]), kEmpty, key);
            if (prev == kEmpty || prev == key) return s;
        }
        s = (s + 1 == S) ? 0 : s + 1;
    }
    return -1;
}

// Probe rounds a lane runs for its rows together before it falls back to the full (sequential) probe.
constexpr int kProbeRounds = 4;

// Applies one query to one staged tile of nrows rows.  Consumer warp wig of the group takes a contiguous share of
// the tile's rows.  Phase A evaluates the WHERE interval and compacts the passing rows' indices into the warp's
// list with ballots (so rows that fail cost nothing later); phase B walks the list in steps of RPT rows per lane:
// key (and key modulus), value, insert.  In the global placement the RPT probe sequences of a step advance in
// rounds, every round issuing the next probe load of all unresolved rows together, so a lane waits for the longest
// sequence rather than the sum of them.
template <typename VT, int RPT>
__device__ void b_tile(const BInst& I, const unsigned char* st, int koff, int voff, int poff, int nrows,
                       unsigned char* tbase, int wig, int cw, uint16_t* list, unsigned long long* claims,
                       const BFix& fx) {
    constexpr bool V32 = sizeof(VT) == 4;
    const int lane = threadIdx.x & 31;
    const int per_warp = (((nrows + cw - 1) / cw) + 31) & ~31;
    const int r0 = wig * per_warp;
    const int r1 = min(nrows, r0 + per_warp);
    if (r0 >= r1) return;
    const int S = I.S;
    const bool has_vals = I.vk != VK_NONE;
    const bool has_sum = I.has_sum, has_min = I.has_min, has_max = I.has_max;
    const Layout L = I.L;
    const int W = L.W;
    const Region main = I.main;
    const bool k32 = I.kt == 4;
    const bool kmod = I.key_mod > 0;
    const uint64_t md = static_cast<uint64_t>(I.key_mod), mm = I.mod_m;
    const int ms1 = I.mod_s1, ms2 = I.mod_s2;
    const int pbytes = I.pbytes;

    // ---- phase A: compact the rows passing the WHERE interval
    int count = r1 - r0;
    if (pbytes) {
        const bool pfloat = I.pfloat != 0, pinv = I.pinv != 0;
        const int64_t plo = I.plo, phi = I.phi;
        const uint32_t lt = (1u << lane) - 1u;
        count = 0;
        for (int j0 = r0; j0 < r1; j0 += 32) {
            const int j = j0 + lane;
            bool keep = j < r1;
            if (keep) {
                int64_t o;
                if (pbytes == 4) {
                    const int32_t b = reinterpret_cast<const int32_t*>(st + poff)[j];
                    o = pfloat ? static_cast<int64_t>(b ^ ((b >> 31) & 0x7fffffff)) : static_cast<int64_t>(b);
                } else {
                    const int64_t b = reinterpret_cast<const int64_t*>(st + poff)[j];
                    o = pfloat ? (b ^ ((b >> 63) & 0x7fffffffffffffffll)) : b;
                }
                keep = ((o >= plo) && (o <= phi)) != pinv;
            }
            const uint32_t bal = __ballot_sync(0xffffffffu, keep);
            if (keep) list[count + __popc(bal & lt)] = static_cast<uint16_t>(j);
            count += __popc(bal);
        }
        __syncwarp();
    }

    BSmem t{};
    int probe = 0;
    if (S > 0) {
        t = b_tables(tbase, I, V32);
        const int tb = (I.R > 1) ? (wig % I.R) * S : 0;
        t.key += tb;
        t.sum += tb;
        t.cnt += tb;
        t.mn += static_cast<size_t>(tb) * 8;
        t.mx += static_cast<size_t>(tb) * 8;
        probe = I.probe;
    }
    // ---- phase B: the passing rows, RPT per lane per step
    for (int e0 = 0; e0 < count; e0 += RPT * 32) {
        uint64_t kw[RPT];
        VT v[RPT];
        bool ok[RPT];
#pragma unroll
        for (int u = 0; u < RPT; ++u) {
            const int e = e0 + u * 32 + lane;
            ok[u] = e < count;
            kw[u] = 0;
            v[u] = VT{};
            if (!ok[u]) continue;
            const int j = pbytes ? static_cast<int>(list[e]) : r0 + e;
            int64_t k = k32 ? static_cast<int64_t>(reinterpret_cast<const int32_t*>(st + koff)[j])
                            : reinterpret_cast<const int64_t*>(st + koff)[j];
            if (kmod) k = mod_signed(k, md, mm, ms1, ms2);
            kw[u] = k32 ? key_word(static_cast<int32_t>(k)) : key_word(k);
            if (has_vals) v[u] = reinterpret_cast<const VT*>(st + voff)[j];
        }
        if (S > 0) {
#pragma unroll
            for (int u = 0; u < RPT; ++u) {
                if (!ok[u]) continue;
                bool inwin = true;
                long long q = 0;
                if constexpr (std::is_same<VT, float>::value) {
                    if (has_sum) q = b_addend(v[u], fx, &inwin);
                } else if constexpr (!std::is_floating_point<VT>::value) {
                    q = static_cast<long long>(v[u]);
                }
                const int s = (kw[u] != kEmpty && inwin) ? b_s_find(t.key, S, probe, kw[u]) : -1;
                if (s >= 0) {
                    b_s_acc<VT>(t, s, v[u], q, has_vals, has_sum, has_min, has_max);
                } else {
                    uint64_t* slot = (kw[u] == kEmpty) ? g_special(main, W, 1, claims)
                                                       : g_find(main, W, kw[u], mix64(kw[u]), I.counters, claims);
                    if (slot) b_g_acc<VT>(slot, L, v[u], has_vals, has_sum, has_min, has_max);
                }
            }
        } else {
            uint64_t pos[RPT], cur[RPT];
            uint64_t* slot[RPT];
            bool pend[RPT];
#pragma unroll
            for (int u = 0; u < RPT; ++u) {
                pos[u] = home_slot(main, mix64(kw[u]));
                pend[u] = ok[u] && kw[u] != kEmpty;
                slot[u] = nullptr;
                cur[u] = pend[u] ? ld_volatile_u64(main.slots + pos[u] * W) : 0ull;
            }
            for (int round = 0; round < kProbeRounds; ++round) {
                bool any = false;
#pragma unroll
                for (int u = 0; u < RPT; ++u) {
                    if (!pend[u]) continue;
                    uint64_t* sp = main.slots + pos[u] * W;
                    if (cur[u] == kw[u]) {
                        slot[u] = sp;
                        pend[u] = false;
                    } else if (cur[u] == kEmpty) {
                        const unsigned long long prev =
                            atomicCAS(reinterpret_cast<unsigned long long*>(sp), kEmpty, kw[u]);
                        if (prev == kEmpty || prev == kw[u]) {
                            if (prev == kEmpty) claim_counted(claims);
                            slot[u] = sp;
                            pend[u] = false;
                        }
                    }
                    if (pend[u]) {
                        pos[u] = (pos[u] + 1) & main.mask;
                        any = true;
                    }
                }
                if (!any) break;
#pragma unroll
                for (int u = 0; u < RPT; ++u)
                    if (pend[u]) cur[u] = ld_volatile_u64(main.slots + pos[u] * W);
            }
#pragma unroll
            for (int u = 0; u < RPT; ++u) {
                if (!ok[u]) continue;
                if (kw[u] == kEmpty) slot[u] = g_special(main, W, 1, claims);
                else if (pend[u]) slot[u] = g_find_from(main, W, kw[u], pos[u], cur[u], I.counters, claims);
                if (slot[u]) b_g_acc<VT>(slot[u], L, v[u], has_vals, has_sum, has_min, has_max);
            }
        }
    }
    __syncwarp();  // the list is reused by the next query of the scan group
}

template <typename VT>
__device__ __forceinline__ void b_members_tile(const BGroup& grp, const BInst* desc, const unsigned char* st,
                                               int koff, int voff, int poff, int nrows, unsigned char* tbase,
                                               int wig, int cw, uint16_t* list, int rpt, unsigned long long* claims,
                                               const BFix& fx) {
    for (int k = 0; k < grp.n_members; ++k) {
        switch (rpt) {
            case 1: b_tile<VT, 1>(desc[k], st, koff, voff, poff, nrows, tbase, wig, cw, list, claims + k, fx); break;
            case 2: b_tile<VT, 2>(desc[k], st, koff, voff, poff, nrows, tbase, wig, cw, list, claims + k, fx); break;
            default: b_tile<VT, 4>(desc[k], st, koff, voff, poff, nrows, tbase, wig, cw, list, claims + k, fx); break;
        }
    }
}

template <typename VT>
__device__ __forceinline__ void b_members_clear(const BGroup& grp, const BInst* desc, unsigned char* tbase, int ctid,
                                                int cthreads) {
    for (int k = 0; k < grp.n_members; ++k) b_clear<VT>(tbase, desc[k], ctid, cthreads);
}

template <typename VT>
__device__ __forceinline__ void b_members_flush(const BGroup& grp, const BInst* desc, unsigned char* tbase, int ctid,
                                                int cthreads, unsigned long long* claims, const BFix& fx) {
    for (int k = 0; k < grp.n_members; ++k) b_flush<VT>(tbase, desc[k], ctid, cthreads, claims + k, fx);
}

// Copies the rows of [r, r + nrows) of one column that a bulk copy cannot move (the final < 16 bytes of an
// unaligned tail) with plain loads; returns the bytes the bulk copy moves.
__device__ __forceinline__ uint32_t b_tail(unsigned char* dst, const void* col, int elem, int64_t r, int nrows, int lane) {
    const uint32_t bytes = static_cast<uint32_t>(nrows) * elem;
    const uint32_t bulk = bytes & ~15u;
    for (int j = static_cast<int>(bulk / elem) + lane; j < nrows; j += 32) {
        if (elem == 4) reinterpret_cast<int32_t*>(dst)[j] = static_cast<const int32_t*>(col)[r + j];
        else reinterpret_cast<int64_t*>(dst)[j] = static_cast<const int64_t*>(col)[r + j];
    }
    return bulk;
}

__global__ void __launch_bounds__(kBThreads, 1) gb_batch_agg_kernel(const BatchArgs ba) {
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ unsigned long long s_claims[4][kBMaxMembers];
    __shared__ __align__(16) BInst s_desc[4][kBMaxMembers];  // member descriptors of every group's current item
    __shared__ uint16_t s_list[kBCons][kBListRows];          // per consumer warp: passing rows of the tile
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    int32_t* err = &ba.hdr->error;
    for (int q = 0; q < kBQueues; ++q) {
        const int qb = ba.hdr->q_begin[q];
        const int qe = ba.hdr->q_begin[q + 1];
        if (qb >= qe) continue;
        const int G = 1 << q;
        const int cw = kBCons >> q;
        const size_t gbytes = (static_cast<size_t>(ba.dyn_bytes) >> q) & ~static_cast<size_t>(127);
        const int SB = b_stage_bytes(q);
        // barriers of every group of this phase
        if (threadIdx.x == 0) {
            for (int g = 0; g < G; ++g) {
                BGroupSmem* h = reinterpret_cast<BGroupSmem*>(sm + g * gbytes);
                for (int s = 0; s < kBStages; ++s) {
                    mbar_init(&h->full[s], 1);
                    mbar_init(&h->empty[s], cw);
                }
                mbar_init(&h->csync, cw);
            }
            mbar_fence_init();
        }
        if (threadIdx.x < 4 * kBMaxMembers) s_claims[threadIdx.x / kBMaxMembers][threadIdx.x % kBMaxMembers] = 0;
        __syncthreads();

        if (warp >= kBCons) {
            // ---------------- producer warp of group g ----------------
            const int g = warp - kBCons;
            if (g < G) {
                unsigned char* gsm = sm + g * gbytes;
                BGroupSmem* h = reinterpret_cast<BGroupSmem*>(gsm);
                unsigned char* ring = gsm + gbytes - b_ring_bytes(q);
                const uint64_t pol = l2_evict_first_policy();
                uint32_t seq = 0;
                bool alive = true;
                while (alive) {
                    int idx = 0;
                    if (lane == 0) idx = qb + static_cast<int>(atomicAdd(&ba.hdr->heads[q], 1ull));
                    idx = __shfl_sync(0xffffffffu, idx, 0);
                    if (idx >= qe) {
                        const int s = static_cast<int>(seq % kBStages);
                        if (seq >= kBStages && !b_wait(&h->empty[s], ((seq / kBStages) - 1) & 1u, err)) break;
                        if (lane == 0) {
                            h->meta[s].flags = kMetaDone;
                            mbar_arrive(&h->full[s]);
                        }
                        break;
                    }
                    const BItem it = ba.items[idx];
                    const BGroup& grp = ba.groups[it.group];
                    const int T = grp.stage_rows;
                    const int kt = grp.kt, vb = grp.vbytes, pb = grp.pbytes;
                    const int koff = 0, voff = b_align128(T * kt), poff = voff + b_align128(T * vb);
                    const void* kcol = grp.keys;
                    const void* vcol = grp.vals;
                    const void* pcol = grp.pcol;
                    for (int64_t r = it.r0; r < it.r1; r += T) {
                        const int s = static_cast<int>(seq % kBStages);
                        if (seq >= kBStages && !b_wait(&h->empty[s], ((seq / kBStages) - 1) & 1u, err)) {
                            alive = false;
                            break;
                        }
                        const int nrows = static_cast<int>(min(static_cast<int64_t>(T), it.r1 - r));
                        unsigned char* st = ring + s * SB;
                        const uint32_t kbulk = b_tail(st + koff, kcol, kt, r, nrows, lane);
                        const uint32_t vbulk = vb ? b_tail(st + voff, vcol, vb, r, nrows, lane) : 0u;
                        const uint32_t pbulk = pb ? b_tail(st + poff, pcol, pb, r, nrows, lane) : 0u;
                        __syncwarp();
                        if (lane == 0) {
                            BStageMeta& m = h->meta[s];
                            m.item = idx;
                            m.r0 = r;
                            m.nrows = nrows;
                            m.flags = (r == it.r0 ? kMetaFirst : 0) | (r + T >= it.r1 ? kMetaLast : 0);
                            fence_proxy_async_smem();
                            mbar_arrive_expect_tx(&h->full[s], kbulk + vbulk + pbulk);
                            if (kbulk) bulk_g2s(st + koff, static_cast<const unsigned char*>(kcol) + r * kt, kbulk, &h->full[s], pol);
                            if (vbulk) bulk_g2s(st + voff, static_cast<const unsigned char*>(vcol) + r * vb, vbulk, &h->full[s], pol);
                            if (pbulk) bulk_g2s(st + poff, static_cast<const unsigned char*>(pcol) + r * pb, pbulk, &h->full[s], pol);
                        }
                        __syncwarp();
                        ++seq;
                    }
                }
                // Every issued stage must be consumed (no copy in flight) before the phase ends.
                for (uint32_t d = (seq > kBStages ? seq - kBStages : 0); d < seq; ++d)
                    if (!b_wait(&h->empty[d % kBStages], (d / kBStages) & 1u, err)) break;
            }
        } else {
            // ---------------- consumer warps of group g ----------------
            const int g = warp / cw;
            const int wig = warp - g * cw;
            const int cthreads = cw * 32;
            const int ctid = threadIdx.x - g * cthreads;
            unsigned char* gsm = sm + g * gbytes;
            BGroupSmem* h = reinterpret_cast<BGroupSmem*>(gsm);
            unsigned char* tbase = gsm + kBHeaderBytes;
            const unsigned char* ring = gsm + gbytes - b_ring_bytes(q);
            unsigned long long* claims = s_claims[g];
            uint32_t seq = 0, cpar = 0;
            unsigned long long t0 = 0;
            BFix fx;  // the current item's fixed-point scale (float values)
            for (;;) {
                const int s = static_cast<int>(seq % kBStages);
                if (!b_wait(&h->full[s], (seq / kBStages) & 1u, err)) break;
                const BStageMeta m = h->meta[s];
                if (m.flags & kMetaDone) break;
                const BItem it = ba.items[m.item];
                const BGroup& grp = ba.groups[it.group];
                const int T = grp.stage_rows;
                const int koff = 0, voff = b_align128(T * grp.kt), poff = voff + b_align128(T * grp.vbytes);
                const unsigned char* st = ring + s * SB;
                const int vk = grp.vk;
                BInst* desc = s_desc[g];
                if (m.flags & kMetaFirst) {
                    b_csync(&h->csync, cpar, err);  // the previous item's claims are published
                    if (ctid == 0) t0 = global_ns();
                    constexpr int kWords = static_cast<int>(sizeof(BInst) / 8);
                    for (int w = ctid; w < grp.n_members * kWords; w += cthreads)
                        reinterpret_cast<uint64_t*>(desc)[w] =
                            reinterpret_cast<const uint64_t*>(ba.inst + grp.members[w / kWords])[w % kWords];
                    if (ctid == 0) h->emax = INT_MIN;
                    b_csync(&h->csync, cpar, err);
                    switch (vk) {
                        case VK_I64: b_members_clear<int64_t>(grp, desc, tbase, ctid, cthreads); break;
                        case VK_F32: b_members_clear<float>(grp, desc, tbase, ctid, cthreads); break;
                        case VK_F64: b_members_clear<double>(grp, desc, tbase, ctid, cthreads); break;
                        default: b_members_clear<int32_t>(grp, desc, tbase, ctid, cthreads); break;
                    }
                    if (vk == VK_F32) {  // the fixed-point scale of this item's float sums
                        int e = INT_MIN;
                        const float* vals = reinterpret_cast<const float*>(st + voff);
                        for (int j = ctid; j < m.nrows; j += cthreads) {
                            const uint32_t b = __float_as_uint(vals[j]);
                            const int be = static_cast<int>((b >> 23) & 0xffu);
                            if (be != 0 && be != 0xff) e = max(e, be - 126);
                        }
                        e = __reduce_max_sync(0xffffffffu, e);
                        if (lane == 0 && e != INT_MIN) atomicMax(&h->emax, e);
                    }
                    b_csync(&h->csync, cpar, err);
                    fx = b_fix(h->emax == INT_MIN ? 0 : h->emax);
                }
                const int rpt = grp.rpt;
                switch (vk) {
                    case VK_I64: b_members_tile<int64_t>(grp, desc, st, koff, voff, poff, m.nrows, tbase, wig, cw, s_list[warp], rpt, claims, fx); break;
                    case VK_F32: b_members_tile<float>(grp, desc, st, koff, voff, poff, m.nrows, tbase, wig, cw, s_list[warp], rpt, claims, fx); break;
                    case VK_F64: b_members_tile<double>(grp, desc, st, koff, voff, poff, m.nrows, tbase, wig, cw, s_list[warp], rpt, claims, fx); break;
                    default: b_members_tile<int32_t>(grp, desc, st, koff, voff, poff, m.nrows, tbase, wig, cw, s_list[warp], rpt, claims, fx); break;
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(&h->empty[s]);
                if (m.flags & kMetaLast) {
                    b_csync(&h->csync, cpar, err);
                    switch (vk) {
                        case VK_I64: b_members_flush<int64_t>(grp, desc, tbase, ctid, cthreads, claims, fx); break;
                        case VK_F32: b_members_flush<float>(grp, desc, tbase, ctid, cthreads, claims, fx); break;
                        case VK_F64: b_members_flush<double>(grp, desc, tbase, ctid, cthreads, claims, fx); break;
                        default: b_members_flush<int32_t>(grp, desc, tbase, ctid, cthreads, claims, fx); break;
                    }
                    b_csync(&h->csync, cpar, err);
                    if (ctid == 0) {
                        for (int k = 0; k < grp.n_members; ++k) {
                            const BInst& I = desc[k];
                            publish_claims(I.counters, static_cast<unsigned long long>(I.capacity), claims[k]);
                            claims[k] = 0;
                        }
                        ba.item_ns[m.item] = static_cast<long long>(global_ns() - t0);
                    }
                }
                ++seq;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int g = 0; g < G; ++g) {
                BGroupSmem* h = reinterpret_cast<BGroupSmem*>(sm + g * gbytes);
                for (int s = 0; s < kBStages; ++s) {
                    mbar_inval(&h->full[s]);
                    mbar_inval(&h->empty[s]);
                }
                mbar_inval(&h->csync);
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------
// Results: one CTA per query walks its table in slot order, writes keys and finalised aggregates into the
// query's result region and resets every slot it read to the empty state.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ int b_block_scan(int x, int* total) {
    __shared__ int warp_sums[kBResThreads / 32];
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
        const int w = (lane < kBResThreads / 32) ? warp_sums[lane] : 0;
        int wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += y;
        }
        if (lane < kBResThreads / 32) warp_sums[lane] = wi - w;
        if (lane == 31) *total = wi;
    }
    __syncthreads();
    const int excl = warp_sums[wid] + inc - x;
    __syncthreads();
    return excl;
}

__device__ __forceinline__ uint64_t dbits(double d) {
    uint64_t b;
    memcpy(&b, &d, 8);
    return b;
}

// The 8-byte output word of aggregate `agg` of one slot (the reference's O value, widened).
__device__ uint64_t b_emit(const BInst& I, const uint64_t* slot, int agg) {
    const Layout& L = I.L;
    const uint64_t cnt = (L.cnt >= 0) ? slot[L.cnt] : 0;
    if (agg == QDB_AGG_COUNT) return cnt;
    const bool isnull = cnt == 0;
    const bool mnq = agg == QDB_AGG_MIN;
    switch (I.vk) {
        case VK_I32: {
            int32_t v = 0;
            if (agg == QDB_AGG_MIN || agg == QDB_AGG_MAX) {
                if (isnull) v = mnq ? INT_MAX : INT_MIN;
                else {
                    const uint64_t w = slot[mnq ? L.mn : L.mx];
                    v = static_cast<int32_t>(mnq ? (w & 0xffffffffull) : (w >> 32));
                }
            } else if (agg == QDB_AGG_SUM) {
                v = isnull ? 0 : static_cast<int32_t>(static_cast<int64_t>(slot[L.sum]));
            } else {  // AVG truncates like GPUBinary<div, O, V*, int64_t*>
                const int32_t s = static_cast<int32_t>(static_cast<int64_t>(slot[L.sum]));
                v = isnull ? INT_MIN : static_cast<int32_t>(static_cast<int64_t>(s) / static_cast<int64_t>(cnt));
            }
            return static_cast<uint64_t>(static_cast<int64_t>(v));
        }
        case VK_I64: {
            int64_t v = 0;
            if (agg == QDB_AGG_MIN || agg == QDB_AGG_MAX) {
                if (isnull) v = mnq ? LLONG_MAX : LLONG_MIN;
                else v = static_cast<int64_t>(slot[mnq ? L.mn : L.mx]);
            } else if (agg == QDB_AGG_SUM) {
                v = isnull ? 0 : static_cast<int64_t>(slot[L.sum]);
            } else {
                v = isnull ? LLONG_MIN : static_cast<int64_t>(slot[L.sum]) / static_cast<int64_t>(cnt);
            }
            return static_cast<uint64_t>(v);
        }
        case VK_F32: {
            float v = 0.f;
            if (agg == QDB_AGG_MIN || agg == QDB_AGG_MAX) {
                if (isnull) v = mnq ? 3.402823466e+38f : -3.402823466e+38f;
                else {
                    const uint64_t w = slot[mnq ? L.mn : L.mx];
                    v = fdec(static_cast<int32_t>(mnq ? (w & 0xffffffffull) : (w >> 32)));
                }
            } else {
                double d;
                memcpy(&d, &slot[L.sum], 8);
                if (agg == QDB_AGG_SUM) v = isnull ? 0.f : static_cast<float>(d);
                else v = isnull ? __int_as_float(0x7fc00000) : static_cast<float>(d / static_cast<double>(cnt));
            }
            return dbits(static_cast<double>(v));
        }
        case VK_F64: {
            double v = 0.0;
            if (agg == QDB_AGG_MIN || agg == QDB_AGG_MAX) {
                if (isnull) v = mnq ? 1.7976931348623157e+308 : -1.7976931348623157e+308;
                else v = ddec(static_cast<int64_t>(slot[mnq ? L.mn : L.mx]));
            } else {
                double d;
                memcpy(&d, &slot[L.sum], 8);
                if (agg == QDB_AGG_SUM) v = isnull ? 0.0 : d;
                else v = isnull ? __longlong_as_double(0x7ff8000000000000ll) : d / static_cast<double>(cnt);
            }
            return dbits(v);
        }
        default: return 0;
    }
}

__global__ void __launch_bounds__(kBResThreads) gb_batch_results_kernel(const BatchArgs ba) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        for (int q = 0; q < kBQueues; ++q) ba.hdr->heads[q] = 0;
        ba.hdr->init_needed = 0;
    }
    const int i = blockIdx.x;
    if (i >= ba.hdr->n_inst) return;
    const BInst& I = ba.inst[i];
    const uint64_t total = I.main.mask + 3;
    const int W = I.L.W;
    const Layout L = I.L;
    uint64_t* res = ba.res + I.res_off;
    const int64_t cap = I.res_cap;
    __shared__ int tot_s;
    int64_t done = 0;
    // A chunk's slots are walked warp by warp (warp w: kWS consecutive slots, one per lane per step), so the key-word
    // loads are coalesced; a row's position is the chunk's base, its warp's offset and its rank in the ballot.
    constexpr int kWS = kBResChunk / (kBResThreads / 32);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    for (uint64_t c0 = 0; c0 < total; c0 += kBResChunk) {
        const uint64_t wb = c0 + static_cast<uint64_t>(warp) * kWS;
        int c = 0;
#pragma unroll 4
        for (int k = 0; k < kWS; k += 32) {
            const uint64_t v = wb + k + lane;
            c += __popc(__ballot_sync(0xffffffffu, v < total && I.main.slots[v * W] != kEmpty));
        }
        int64_t pos = done + b_block_scan(lane == 0 ? c : 0, &tot_s);
        pos = __shfl_sync(0xffffffffu, pos, 0);
        for (int k = 0; k < kWS; k += 32) {
            const uint64_t v = wb + k + lane;
            const bool pr = v < total && I.main.slots[v * W] != kEmpty;
            const unsigned bal = __ballot_sync(0xffffffffu, pr);
            if (pr) {
                const int64_t p = pos + __popc(bal & lt);
                uint64_t* slot = I.main.slots + v * W;
                if (p < cap) {
                    const uint64_t kw = slot[0];
                    int64_t key;
                    if (v == I.main.mask + 2) key = LLONG_MIN;  // the key equal to the empty marker
                    else if (I.kt == 4) key = static_cast<int32_t>(kw);
                    else key = static_cast<int64_t>(kw);
                    res[p] = static_cast<uint64_t>(key);
                    int col = 0;
                    for (int a = QDB_AGG_MIN; a <= QDB_AGG_COUNT; a <<= 1) {
                        if (!(I.aggs & a)) continue;
                        ++col;
                        res[static_cast<int64_t>(col) * cap + p] = b_emit(I, slot, a);
                    }
                }
                // Clean the slot for the next run.
                slot[0] = kEmpty;
                for (int w = 1; w < W; ++w) {
                    uint64_t x = 0;
                    if (w == L.mn && L.packed) x = kPackedMinMaxInit;
                    else if (w == L.mn) x = kMinInit64;
                    else if (w == L.mx) x = kMaxInit64;
                    slot[w] = x;
                }
            }
            pos += __popc(bal);
        }
        done += tot_s;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        int32_t st = static_cast<int32_t>(I.counters[1] & 0xffffffffull);
        if (ba.hdr->error != QDB_OK) st = ba.hdr->error;
        if (done > cap && st == QDB_OK) st = QDB_HASH_TABLE_FULL;
        ba.res_count[i] = done < cap ? done : cap;
        ba.status[i] = st;
        I.counters[0] = 0;
        I.counters[1] = 0;
    }
}

}  // namespace qdb
