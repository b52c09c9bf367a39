// Kernels of the batched GROUP BY: table initialisation, the persistent work-queue aggregation kernel and the
// result kernel.  The reference runs group_by_kernel once per query and block (GPUGroupBy.cuh:68-196,
// :395-410) and one GetResults per query (:478-587); here every query of a batch is a set of work items in
// one launch.
//
// Aggregation kernel: one CTA of 16 warps per SM.  The CTA drains three work queues in turn; in queue q the
// CTA is split into 2^q warp groups (16, 8 or 4 warps) that take work items independently, each with its
// own share of shared memory and its own named barrier, so small queries do not hold a whole SM.  A work
// item is a row range of one query.  The group streams the rows with 128-bit evict-first loads (each thread
// 4 or 8 consecutive rows per step), evaluates the WHERE interval, applies the key modulus and inserts the
// row
//   * shared placement: into one of R shared-memory tables of the group (warp w uses table w % R, so
//     low-cardinality queries spread their same-key atomics over R copies), then at the end of the item
//     every occupied shared slot is merged into the query's global table;
//   * global placement: straight into the query's global table, the probe loads of a thread's rows issued
//     together.
// Rows whose shared-memory probe fails (a cardinality estimate that was too low) go to the global table.
// Every item is timed with the global timer for the autotuner.
#include <climits>

#include "batch.cuh"

namespace qdb {

__device__ __forceinline__ void group_sync(int id, int nthreads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// ---------------------------------------------------------------------------------------------
// Table initialisation (only after a new plan: the result kernel cleans every slot it reads).
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) gb_batch_init_kernel(const BatchArgs ba) {
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
// Row loads.  base is a multiple of IPT and the columns are 16-byte aligned, so a full step is IPT * size / 16
// vector loads.
// ---------------------------------------------------------------------------------------------
template <int IPT>
__device__ __forceinline__ void load_i32(const void* col, int64_t base, bool full, int64_t r1, int32_t (&out)[IPT]) {
    const int32_t* p = static_cast<const int32_t*>(col) + base;
    if (full) {
#pragma unroll
        for (int j = 0; j < IPT / 4; ++j) {
            const int4 q = ld_stream16(p + 4 * j);
            out[4 * j + 0] = q.x;
            out[4 * j + 1] = q.y;
            out[4 * j + 2] = q.z;
            out[4 * j + 3] = q.w;
        }
    } else {
#pragma unroll
        for (int e = 0; e < IPT; ++e) out[e] = (base + e < r1) ? p[e] : 0;
    }
}

template <int IPT>
__device__ __forceinline__ void load_i64(const void* col, int64_t base, bool full, int64_t r1, int64_t (&out)[IPT]) {
    const int64_t* p = static_cast<const int64_t*>(col) + base;
    if (full) {
#pragma unroll
        for (int j = 0; j < IPT / 2; ++j) {
            const int4 q = ld_stream16(p + 2 * j);
            out[2 * j + 0] = (static_cast<int64_t>(static_cast<uint32_t>(q.y)) << 32) | static_cast<uint32_t>(q.x);
            out[2 * j + 1] = (static_cast<int64_t>(static_cast<uint32_t>(q.w)) << 32) | static_cast<uint32_t>(q.z);
        }
    } else {
#pragma unroll
        for (int e = 0; e < IPT; ++e) out[e] = (base + e < r1) ? p[e] : 0;
    }
}

template <typename VT, int IPT>
__device__ __forceinline__ void load_vals(const void* col, int64_t base, bool full, int64_t r1, VT (&out)[IPT]) {
    if constexpr (sizeof(VT) == 4) {
        int32_t t[IPT];
        load_i32<IPT>(col, base, full, r1, t);
#pragma unroll
        for (int e = 0; e < IPT; ++e) memcpy(&out[e], &t[e], 4);
    } else {
        int64_t t[IPT];
        load_i64<IPT>(col, base, full, r1, t);
#pragma unroll
        for (int e = 0; e < IPT; ++e) memcpy(&out[e], &t[e], 8);
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

template <typename VT>
__device__ __forceinline__ void b_s_acc(const BSmem& t, int s, VT v, bool has_vals, bool has_sum, bool has_min,
                                        bool has_max) {
    atomicAdd(t.cnt + s, 1u);
    if (!has_vals) return;
    if (has_sum) {
        if constexpr (std::is_floating_point<VT>::value)
            atomicAdd(reinterpret_cast<double*>(t.sum) + s, static_cast<double>(v));
        else
            atomicAdd(t.sum + s, static_cast<unsigned long long>(static_cast<long long>(v)));
    }
    if constexpr (sizeof(VT) == 4) {
        const int32_t e = enc32(v);
        if (has_min) atomicMin(reinterpret_cast<int*>(t.mn) + 2 * s, e);
        if (has_max) atomicMax(reinterpret_cast<int*>(t.mx) + 2 * s + 1, e);
    } else {
        const long long e = enc64(v);
        if (has_min) atomicMin(reinterpret_cast<long long*>(t.mn) + s, e);
        if (has_max) atomicMax(reinterpret_cast<long long*>(t.mx) + s, e);
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
// One work item: rows [r0, r1) of query I, processed by one warp group.
// ---------------------------------------------------------------------------------------------
template <typename VT, int IPT>
__device__ __forceinline__ void b_item(const BInst& I, int64_t r0, int64_t r1, unsigned char* gsm, int gtid,
                                    int gthreads, int bar, unsigned long long* claims) {
    constexpr bool V32 = sizeof(VT) == 4;
    const int S = I.S;
    const int RS = S * I.R;
    const bool has_vals = I.vk != VK_NONE;
    const bool has_sum = I.has_sum, has_min = I.has_min, has_max = I.has_max;
    const bool has_mm = has_min || has_max;
    const Layout L = I.L;
    const int W = L.W;
    const Region main = I.main;
    unsigned long long* counters = I.counters;

    BSmem t;
    t.key = reinterpret_cast<uint64_t*>(gsm);
    size_t off = static_cast<size_t>(RS) * 8;
    t.sum = reinterpret_cast<unsigned long long*>(gsm + off);
    if (has_sum) off += static_cast<size_t>(RS) * 8;
    t.mn = gsm + off;
    t.mx = gsm + off;
    if (has_mm) {
        off += static_cast<size_t>(RS) * 8;
        if (!V32) {
            t.mx = gsm + off;
            off += static_cast<size_t>(RS) * 8;
        }
    }
    t.cnt = reinterpret_cast<unsigned int*>(gsm + off);
    for (int i = gtid; i < RS; i += gthreads) {
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
    group_sync(bar, gthreads);

    // This warp's shared table (replica) as an offset into the arrays.
    const int tb = (I.R > 1) ? ((gtid >> 5) % I.R) * S : 0;
    BSmem mt = t;
    mt.key += tb;
    mt.sum += tb;
    mt.cnt += tb;
    mt.mn += static_cast<size_t>(tb) * 8;
    mt.mx += static_cast<size_t>(tb) * 8;
    const int shift = 32 - (31 - __clz(S > 0 ? S : 1));
    const int probe = I.probe;
    const bool k32 = I.kt == 4;
    const int64_t kmod = I.key_mod;
    const int pbytes = I.pbytes;
    const bool pfloat = I.pfloat != 0, pinv = I.pinv != 0;
    const int64_t plo = I.plo, phi = I.phi;

    for (int64_t base = r0 + static_cast<int64_t>(gtid) * IPT; base < r1;
         base += static_cast<int64_t>(gthreads) * IPT) {
        const bool full = base + IPT <= r1;
        uint64_t kw[IPT];
        bool ok[IPT];
        VT v[IPT];
        if (k32) {
            int32_t k[IPT];
            load_i32<IPT>(I.keys, base, full, r1, k);
            if (kmod > 0 && kmod <= INT_MAX) {
                const int32_t m = static_cast<int32_t>(kmod);
#pragma unroll
                for (int e = 0; e < IPT; ++e) k[e] = k[e] % m;
            } else if (kmod > 0) {  // |k| < kmod except INT32_MIN % 2^31
#pragma unroll
                for (int e = 0; e < IPT; ++e) k[e] = static_cast<int32_t>(static_cast<int64_t>(k[e]) % kmod);
            }
#pragma unroll
            for (int e = 0; e < IPT; ++e) kw[e] = key_word(k[e]);
        } else {
            int64_t k[IPT];
            load_i64<IPT>(I.keys, base, full, r1, k);
            if (kmod > 0) {
#pragma unroll
                for (int e = 0; e < IPT; ++e) k[e] = k[e] % kmod;
            }
#pragma unroll
            for (int e = 0; e < IPT; ++e) kw[e] = key_word(k[e]);
        }
        if (has_vals) load_vals<VT, IPT>(I.vals, base, full, r1, v);
        else {
#pragma unroll
            for (int e = 0; e < IPT; ++e) v[e] = VT{};
        }
#pragma unroll
        for (int e = 0; e < IPT; ++e) ok[e] = full || base + e < r1;
        if (pbytes == 4) {
            int32_t p[IPT];
            load_i32<IPT>(I.pcol, base, full, r1, p);
#pragma unroll
            for (int e = 0; e < IPT; ++e) {
                const int64_t o = pred_ord32(p[e], pfloat);
                ok[e] = ok[e] && (((o >= plo) && (o <= phi)) != pinv);
            }
        } else if (pbytes == 8) {
            int64_t p[IPT];
            load_i64<IPT>(I.pcol, base, full, r1, p);
#pragma unroll
            for (int e = 0; e < IPT; ++e) {
                const int64_t o = pred_ord64(p[e], pfloat);
                ok[e] = ok[e] && (((o >= plo) && (o <= phi)) != pinv);
            }
        }
        if (S > 0) {
#pragma unroll
            for (int e = 0; e < IPT; ++e) {
                if (!ok[e]) continue;
                int s = -1;
                if (kw[e] != kEmpty) {
                    bool found = false;
                    s = s_find(mt.key, S, probe, kw[e], smem_hash(kw[e], shift), &found);
                }
                if (s >= 0) {
                    b_s_acc<VT>(mt, s, v[e], has_vals, has_sum, has_min, has_max);
                } else {
                    uint64_t* slot = (kw[e] == kEmpty) ? g_special(main, W, 1, claims)
                                                       : g_find(main, W, kw[e], mix64(kw[e]), counters, claims);
                    if (slot) b_g_acc<VT>(slot, L, v[e], has_vals, has_sum, has_min, has_max);
                }
            }
        } else {
            uint64_t sl[IPT], cur[IPT];
#pragma unroll
            for (int e = 0; e < IPT; ++e) {
                sl[e] = mix64(kw[e]) & main.mask;
                cur[e] = (ok[e] && kw[e] != kEmpty) ? ld_volatile_u64(main.slots + sl[e] * W) : 0ull;
            }
#pragma unroll
            for (int e = 0; e < IPT; ++e) {
                if (!ok[e]) continue;
                uint64_t* slot = (kw[e] == kEmpty) ? g_special(main, W, 1, claims)
                                                   : g_find_from(main, W, kw[e], sl[e], cur[e], counters, claims);
                if (slot) b_g_acc<VT>(slot, L, v[e], has_vals, has_sum, has_min, has_max);
            }
        }
    }
    group_sync(bar, gthreads);

    // Merge the shared tables into the global table.
    if (S > 0) {
        const bool vfloat = std::is_floating_point<VT>::value;
        for (int i = gtid; i < RS; i += gthreads) {
            const uint64_t key = t.key[i];
            if (key == kEmpty) continue;
            uint64_t* slot = g_find(main, W, key, mix64(key), counters, claims);
            if (!slot) continue;
            const unsigned long long c = t.cnt[i];
            const uint64_t sumbits = has_sum ? t.sum[i] : 0ull;
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
            if (has_vals) {
                g_merge(slot, L, has_sum, has_min, has_max, V32, vfloat, c, sumbits, mn, mx);
            } else if (L.cnt >= 0) {
                atomicAdd(reinterpret_cast<unsigned long long*>(slot + L.cnt), c);
            }
        }
    }
    group_sync(bar, gthreads);
    if (gtid == 0) {
        publish_claims(counters, static_cast<unsigned long long>(I.capacity), *claims);
        *claims = 0;
    }
}

__global__ void __launch_bounds__(kBThreads, 1) gb_batch_agg_kernel(const BatchArgs ba) {
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ __align__(16) BInst s_inst[4];
    __shared__ int s_idx[4];
    __shared__ unsigned long long s_claims[4];
    const int warp = threadIdx.x >> 5;
    for (int q = 0; q < kBQueues; ++q) {
        const int qb = ba.hdr->q_begin[q];
        const int qe = ba.hdr->q_begin[q + 1];
        if (qb >= qe) continue;
        const int gw = kBWarps >> q;
        const int g = warp / gw;
        const int gthreads = gw * 32;
        const int gtid = threadIdx.x - g * gthreads;
        const int bar = 1 + g;
        const size_t gbytes = (static_cast<size_t>(ba.dyn_bytes) >> q) & ~static_cast<size_t>(127);
        unsigned char* gsm = sm + g * gbytes;
        if (gtid == 0) s_claims[g] = 0;
        for (;;) {
            if (gtid == 0) s_idx[g] = qb + static_cast<int>(atomicAdd(&ba.hdr->heads[q], 1ull));
            group_sync(bar, gthreads);
            const int idx = s_idx[g];
            if (idx >= qe) break;
            const BItem it = ba.items[idx];
            constexpr int kWords = static_cast<int>(sizeof(BInst) / 8);
            if (gtid < kWords)
                reinterpret_cast<uint64_t*>(&s_inst[g])[gtid] = reinterpret_cast<const uint64_t*>(ba.inst + it.inst)[gtid];
            group_sync(bar, gthreads);
            const unsigned long long t0 = global_ns();
            const BInst& I = s_inst[g];
            const bool wide = I.ipt == 8;
            switch (I.vk) {
                case VK_I64:
                    if (wide) b_item<int64_t, 8>(I, it.r0, it.r1, gsm, gtid, gthreads, bar, &s_claims[g]);
                    else b_item<int64_t, 4>(I, it.r0, it.r1, gsm, gtid, gthreads, bar, &s_claims[g]);
                    break;
                case VK_F32:
                    if (wide) b_item<float, 8>(I, it.r0, it.r1, gsm, gtid, gthreads, bar, &s_claims[g]);
                    else b_item<float, 4>(I, it.r0, it.r1, gsm, gtid, gthreads, bar, &s_claims[g]);
                    break;
                case VK_F64:
                    if (wide) b_item<double, 8>(I, it.r0, it.r1, gsm, gtid, gthreads, bar, &s_claims[g]);
                    else b_item<double, 4>(I, it.r0, it.r1, gsm, gtid, gthreads, bar, &s_claims[g]);
                    break;
                default:  // VK_I32 and tables without a value column
                    if (wide) b_item<int32_t, 8>(I, it.r0, it.r1, gsm, gtid, gthreads, bar, &s_claims[g]);
                    else b_item<int32_t, 4>(I, it.r0, it.r1, gsm, gtid, gthreads, bar, &s_claims[g]);
                    break;
            }
            if (gtid == 0) ba.item_ns[idx] = static_cast<long long>(global_ns() - t0);
            group_sync(bar, gthreads);
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
    for (uint64_t c0 = 0; c0 < total; c0 += kBResChunk) {
        const uint64_t b = c0 + static_cast<uint64_t>(threadIdx.x) * kBResPer;
        uint32_t pres = 0;
        int c = 0;
#pragma unroll 4
        for (int k = 0; k < kBResPer; ++k) {
            const uint64_t v = b + k;
            if (v < total && I.main.slots[v * W] != kEmpty) {
                pres |= 1u << k;
                ++c;
            }
        }
        int64_t pos = done + b_block_scan(c, &tot_s);
        for (int k = 0; k < kBResPer; ++k) {
            if (!((pres >> k) & 1u)) continue;
            const uint64_t v = b + k;
            uint64_t* slot = I.main.slots + v * W;
            if (pos < cap) {
                const uint64_t kw = slot[0];
                int64_t key;
                if (v == I.main.mask + 2) key = LLONG_MIN;  // the key equal to the empty marker
                else if (I.kt == 4) key = static_cast<int32_t>(kw);
                else key = static_cast<int64_t>(kw);
                res[pos] = static_cast<uint64_t>(key);
                int col = 0;
                for (int a = QDB_AGG_MIN; a <= QDB_AGG_COUNT; a <<= 1) {
                    if (!(I.aggs & a)) continue;
                    ++col;
                    res[static_cast<int64_t>(col) * cap + pos] = b_emit(I, slot, a);
                }
            }
            ++pos;
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
        done += tot_s;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        int32_t st = static_cast<int32_t>(I.counters[1] & 0xffffffffull);
        if (done > cap && st == QDB_OK) st = QDB_HASH_TABLE_FULL;
        ba.res_count[i] = done < cap ? done : cap;
        ba.status[i] = st;
        I.counters[0] = 0;
        I.counters[1] = 0;
    }
}

}  // namespace qdb
