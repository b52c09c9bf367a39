// GROUP BY table management, result extraction and partial-state exchange: the GPUGroupBy<AGG,O,K,V>
// operator surface (qikkDB/QueryEngine/GPUCore/GPUGroupBy.cuh:285-790) and its multi-key
// specialisation (qikkDB/QueryEngine/GPUCore/GPUGroupByMultiKey.cuh:262-1325) behind the C ABI.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <mutex>
#include <vector>

#include "aafl.cuh"
#include "groupby_fast.cuh"

namespace qdb {

// ---------------------------------------------------------------------------------------------
// Layout and sizing.
// ---------------------------------------------------------------------------------------------
Layout make_layout(int32_t aggs, ValKind vk) {
    Layout L;
    const bool has_vals = vk != VK_NONE;
    int w = 1;
    if (has_vals || (aggs & QDB_AGG_COUNT)) L.cnt = w++;
    if (has_vals && (aggs & (QDB_AGG_SUM | QDB_AGG_AVG))) L.sum = w++;
    if (has_vals && (aggs & (QDB_AGG_MIN | QDB_AGG_MAX))) {
        if (vk_is_32(vk)) {
            L.packed = 1;
            L.mn = L.mx = w++;
        } else {
            if (aggs & QDB_AGG_MIN) L.mn = w++;
            if (aggs & QDB_AGG_MAX) L.mx = w++;
        }
    }
    int W = 1;
    while (W < w) W <<= 1;
    L.W = W;
    return L;
}

static uint64_t next_pow2(uint64_t x) {
    uint64_t p = 1;
    while (p < x) p <<= 1;
    return p;
}

__global__ void init_region_kernel(uint64_t* slots, uint64_t nslots, Layout L, int32_t vk32) {
    const uint64_t total = nslots * static_cast<uint64_t>(L.W);
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const int w = static_cast<int>(i % L.W);
        uint64_t v = 0;
        if (w == 0) v = kEmpty;
        else if (w == L.mn && L.packed) v = kPackedMinMaxInit;
        else if (w == L.mn) v = kMinInit64;
        else if (w == L.mx) v = kMaxInit64;
        slots[i] = v;
    }
}

int32_t gb_init_region(qdb_gb* gb, Region& r, cudaStream_t s) {
    const uint64_t nslots = gb->cap + 2;
    if (!r.slots) {
        int32_t rc = dev_alloc(reinterpret_cast<void**>(&r.slots), nslots * gb->L.W * sizeof(uint64_t), s);
        if (rc != QDB_OK) return rc;
        r.mask = gb->cap - 1;
    }
    const DeviceInfo& di = device_info();
    uint64_t blocks = (nslots * gb->L.W + 255) / 256;
    if (blocks > static_cast<uint64_t>(di.sm_count) * 16) blocks = static_cast<uint64_t>(di.sm_count) * 16;
    init_region_kernel<<<static_cast<unsigned>(blocks), 256, 0, s>>>(r.slots, nslots, gb->L,
                                                                      vk_is_32(val_kind(gb->val_type)));
    note_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "init_region_kernel");
    return QDB_OK;
}

static int32_t launch_agg(const qdb_gb* gb, const AggArgs& a, int32_t ptype, bool nulls, size_t smem,
                          cudaStream_t st) {
    const ValKind vk = val_kind(gb->val_type);
    if (gb->n_key_cols == 2) return launch_agg_comp(a, vk, ptype, nulls, smem, st);
    switch (gb->key_type) {
        case QDB_INT32: return launch_agg_i32(a, vk, ptype, nulls, smem, st);
        case QDB_INT64: return launch_agg_i64(a, vk, ptype, nulls, smem, st);
        case QDB_FLOAT: return launch_agg_f32(a, vk, ptype, nulls, smem, st);
        case QDB_DOUBLE: return launch_agg_f64(a, vk, ptype, nulls, smem, st);
        default: return fail(QDB_ERR_INVALID, "unsupported key type");
    }
}

static int32_t launch_spill(const qdb_gb* gb, const AggArgs& a, size_t smem, int64_t grid, cudaStream_t st) {
    switch (val_kind(gb->val_type)) {
        case VK_NONE:
        case VK_I32: return launch_spill_t<int32_t>(a, smem, grid, st);
        case VK_I64: return launch_spill_t<int64_t>(a, smem, grid, st);
        case VK_F32: return launch_spill_t<float>(a, smem, grid, st);
        case VK_F64: return launch_spill_t<double>(a, smem, grid, st);
        default: return fail(QDB_ERR_INVALID, "unsupported value type");
    }
}

static int32_t launch_fast(const qdb_gb* gb, const AggArgs& a, int32_t ptype, size_t smem, cudaStream_t st) {
    const ValKind vk = val_kind(gb->val_type);
    if (a.kmod) {
        if (gb->n_key_cols == 1 && gb->key_type == QDB_INT32) return launch_fast_i32_mod(a, vk, ptype, smem, st);
        if (gb->n_key_cols == 1 && gb->key_type == QDB_INT64) return launch_fast_i64_mod(a, vk, ptype, smem, st);
        return fail(QDB_ERR_INVALID, "gb_fast_kernel: key % m needs a single INT32 or INT64 key");
    }
    if (gb->n_key_cols == 2) return launch_fast_comp(a, vk, ptype, smem, st);
    switch (gb->key_type) {
        case QDB_INT32: return launch_fast_i32(a, vk, ptype, smem, st);
        case QDB_INT64: return launch_fast_i64(a, vk, ptype, smem, st);
        case QDB_FLOAT: return launch_fast_f32(a, vk, ptype, smem, st);
        case QDB_DOUBLE: return launch_fast_f64(a, vk, ptype, smem, st);
        default: return fail(QDB_ERR_INVALID, "unsupported key type");
    }
}

static int32_t launch_fspill(const qdb_gb* gb, const AggArgs& a, size_t smem, int64_t grid, int32_t slices,
                             cudaStream_t st) {
    if (fast_mode(a) == 0) return launch_fspill_t<int32_t, 0>(a, smem, grid, slices, st);
    switch (val_kind(gb->val_type)) {
        case VK_I32: return launch_fspill_m<int32_t>(a, smem, grid, slices, st);
        case VK_I64: return launch_fspill_m<int64_t>(a, smem, grid, slices, st);
        case VK_F32: return launch_fspill_m<float>(a, smem, grid, slices, st);
        case VK_F64: return launch_fspill_m<double>(a, smem, grid, slices, st);
        default: return fail(QDB_ERR_INVALID, "unsupported value type");
    }
}

// The spill area of the aggregation pass: one per device, shared by every table and kept for the life of the
// process (grown on demand), because the reference's dispatcher creates a table per query and a multi-GB area
// allocated per table would grow the memory pool on every query.  A call borrows the area only while it enqueues
// its two launches; an event recorded after them on the call's stream orders the next borrower (on any stream)
// after them on the GPU.
namespace {
struct SpillArea {
    std::mutex mu;
    uint64_t* keys = nullptr;
    void* vals = nullptr;
    uint32_t* fill = nullptr;
    uint64_t rows = 0;
    int64_t cells = 0;
    int32_t vbytes = 0;
    cudaEvent_t done = nullptr;  // recorded after the last call that used the area
};
SpillArea g_spill[64];
}  // namespace

// Locks the device's spill area and makes it at least rows x (8 + vbytes) bytes with `cells` fill counters,
// ordered on stream s after every earlier use.  The caller fills *area and must call spill_release.
static int32_t spill_acquire(int dev, uint64_t rows, int vbytes, int64_t cells, cudaStream_t s, SpillArea** out) {
    if (dev < 0 || dev >= 64) return fail(QDB_ERR_INVALID, "spill area: device index out of range");
    SpillArea& A = g_spill[dev];
    A.mu.lock();
    if (!A.done && cudaEventCreateWithFlags(&A.done, cudaEventDisableTiming) != cudaSuccess) {
        A.mu.unlock();
        return cuda_fail(cudaGetLastError(), "cudaEventCreate(spill area)");
    }
    if (A.rows > 0) {
        const cudaError_t e = cudaStreamWaitEvent(s, A.done, 0);
        if (e != cudaSuccess) {
            A.mu.unlock();
            return cuda_fail(e, "cudaStreamWaitEvent(spill area)");
        }
    }
    if (A.rows < rows || A.vbytes < vbytes || A.cells < cells) {
        // grow every dimension to the largest seen, so that calls of different shapes do not reallocate in turn
        const uint64_t r = std::max<uint64_t>(rows, A.rows);
        const int64_t nc = std::max<int64_t>(cells, A.cells);
        const int32_t vb = std::max<int32_t>(vbytes, A.vbytes);
        dev_free(A.keys, s);
        dev_free(A.vals, s);
        dev_free(A.fill, s);
        A.keys = nullptr;
        A.vals = nullptr;
        A.fill = nullptr;
        A.rows = 0;
        A.cells = 0;
        A.vbytes = 0;
        int32_t rc = dev_alloc(reinterpret_cast<void**>(&A.fill), static_cast<size_t>(nc) * sizeof(uint32_t), s);
        if (rc == QDB_OK) rc = dev_alloc(reinterpret_cast<void**>(&A.keys), r * 8, s);
        if (rc == QDB_OK && vb) rc = dev_alloc(&A.vals, r * static_cast<uint64_t>(vb), s);
        if (rc != QDB_OK) {
            dev_free(A.keys, s);
            dev_free(A.vals, s);
            dev_free(A.fill, s);
            A.keys = nullptr;
            A.vals = nullptr;
            A.fill = nullptr;
            A.mu.unlock();
            return rc;
        }
        A.rows = r;
        A.cells = nc;
        A.vbytes = vb;
    }
    *out = &A;
    return QDB_OK;
}

// Records the end of this call's use of the area on stream s and unlocks it.
static void spill_release(SpillArea* A, cudaStream_t s) {
    cudaEventRecord(A->done, s);
    A->mu.unlock();
}

static bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

static int64_t env_int(const char* name, int64_t dflt) {
    const char* v = getenv(name);
    return (v && *v) ? strtoll(v, nullptr, 10) : dflt;
}

// ---------------------------------------------------------------------------------------------
// Predicate `col OP constant` -> interval of the column type.  The comparison the reference's
// kernel_filter makes (OP{}(a, b) on typed operands, in the C++ common type, GPUFilterConditions.cuh:9-120)
// is monotone in the column value for <, <=, >, >=, so the set of passing values is an interval of the
// column type (for == as well, and != is its complement).  The bounds are found by binary search over a
// monotone ordinal of the column type, evaluating the exact typed comparison on the host; the kernel then
// tests `(lo <= x && x <= hi) != invert`.  NaN columns values fail both bounds, so NaN passes only `!=`,
// matching IEEE comparisons.
// ---------------------------------------------------------------------------------------------
template <typename T>
struct Ordinal;
template <>
struct Ordinal<int32_t> {
    static uint64_t first() { return 0; }
    static uint64_t last() { return 0xffffffffull; }
    static int32_t at(uint64_t o) { return static_cast<int32_t>(static_cast<uint32_t>(o) ^ 0x80000000u); }
};
template <>
struct Ordinal<int64_t> {
    static uint64_t first() { return 0; }
    static uint64_t last() { return ~0ull; }
    static int64_t at(uint64_t o) { return static_cast<int64_t>(o ^ 0x8000000000000000ull); }
};
template <>
struct Ordinal<float> {
    static uint64_t of(float x) { return static_cast<uint32_t>(fenc(x)) ^ 0x80000000u; }
    static uint64_t first() { return of(-INFINITY); }
    static uint64_t last() { return of(INFINITY); }
    static float at(uint64_t o) { return fdec(static_cast<int32_t>(static_cast<uint32_t>(o) ^ 0x80000000u)); }
};
template <>
struct Ordinal<double> {
    static uint64_t of(double x) { return static_cast<uint64_t>(denc(x)) ^ 0x8000000000000000ull; }
    static uint64_t first() { return of(-INFINITY); }
    static uint64_t last() { return of(INFINITY); }
    static double at(uint64_t o) { return ddec(static_cast<int64_t>(o ^ 0x8000000000000000ull)); }
};

template <typename T>
static int64_t to_bits(T v) {
    if constexpr (sizeof(T) == 4) {
        int32_t w;
        memcpy(&w, &v, 4);
        return w;
    } else {
        int64_t w;
        memcpy(&w, &v, 8);
        return w;
    }
}

template <typename T, typename C>
static PredInterval interval_tc(int32_t op, C c) {
    using O = Ordinal<T>;
    const uint64_t L = O::first(), H = O::last();
    auto p = [&](uint64_t o, int32_t opx) { return cmp_op(opx, O::at(o), c); };
    auto last_true = [&](int32_t opx, uint64_t& out) {  // predicate non-increasing in the ordinal
        if (!p(L, opx)) return false;
        uint64_t lo = L, hi = H;
        while (lo < hi) {
            const uint64_t mid = lo + (hi - lo) / 2 + 1;
            if (p(mid, opx)) lo = mid;
            else hi = mid - 1;
        }
        out = lo;
        return true;
    };
    auto first_true = [&](int32_t opx, uint64_t& out) {  // predicate non-decreasing in the ordinal
        if (!p(H, opx)) return false;
        uint64_t lo = L, hi = H;
        while (lo < hi) {
            const uint64_t mid = lo + (hi - lo) / 2;
            if (p(mid, opx)) hi = mid;
            else lo = mid + 1;
        }
        out = lo;
        return true;
    };
    uint64_t a = L, b = H;
    bool ok = false;
    switch (op) {
        case QDB_LESS:
        case QDB_LESS_EQUAL: ok = last_true(op, b); break;
        case QDB_GREATER:
        case QDB_GREATER_EQUAL: ok = first_true(op, a); break;
        default: ok = first_true(QDB_GREATER_EQUAL, a) && last_true(QDB_LESS_EQUAL, b) && a <= b; break;
    }
    PredInterval pi;
    pi.invert = (op == QDB_NOT_EQUAL) ? 1 : 0;
    if (ok) {
        pi.lo = to_bits<T>(O::at(a));
        pi.hi = to_bits<T>(O::at(b));
    } else {  // empty: lo above hi
        pi.lo = to_bits<T>(O::at(H));
        pi.hi = to_bits<T>(O::at(L));
    }
    return pi;
}

template <typename T>
static PredInterval interval_t(const qdb_pred& p) {
    switch (p.const_type) {
        case QDB_INT32: return interval_tc<T>(p.op, static_cast<int32_t>(p.const_i));
        case QDB_INT64: return interval_tc<T>(p.op, static_cast<int64_t>(p.const_i));
        case QDB_FLOAT: return interval_tc<T>(p.op, static_cast<float>(p.const_f));
        default: return interval_tc<T>(p.op, p.const_f);
    }
}

PredInterval pred_interval(const qdb_pred& p) {
    switch (p.type) {
        case QDB_INT32: return interval_t<int32_t>(p);
        case QDB_INT64: return interval_t<int64_t>(p);
        case QDB_FLOAT: return interval_t<float>(p);
        default: return interval_t<double>(p);
    }
}

// ---------------------------------------------------------------------------------------------
// Plan and launch of the fast pass (groupby_fast.cuh) for a call without NULL masks or a precomputed mask whose
// columns are 16-byte aligned and hold at least one whole tile.  *used is false when the plan does not fit shared
// memory (the caller then takes the general pass).
// ---------------------------------------------------------------------------------------------
static int32_t process_fast(qdb_gb* gb, AggArgs a, const qdb_pred* pred, int32_t ptype, cudaStream_t s, bool* used) {
    *used = false;
    const DeviceInfo& di = device_info();
    const ValKind vk = val_kind(gb->val_type);
    // A table whose aggregates never read the values (COUNT only, no NULL masks here) streams the keys alone.
    if (fast_mode(a) == 0) a.vals = nullptr;
    const int ks = (gb->n_key_cols == 2) ? 4 : type_size(gb->key_type);
    const int vs = a.vals ? type_size(gb->val_type) : 0;
    const int ps = a.pcol ? type_size(pred->type) : 0;
    const int row_bytes = ks * gb->n_key_cols + vs + ps;
    // Stages: enough bytes in flight to cover the HBM latency at an SM's share of the bandwidth (about 48 KB), and at
    // least three when they fit (a warp may hold two stages while it carries rows over).
    const int stage_bytes = kFastT * row_bytes;
    int NS = static_cast<int>(env_int("QDB_FAST_STAGES", stage_bytes <= 16 * 1024 ? 4 : (stage_bytes <= 40 * 1024 ? 3 : 2)));
    NS = std::min(6, std::max(2, NS));
    // Compressed keys take each stage's key slots plus 64 bytes: a group is copied from the 16-byte boundary below
    // its first word (kzStage in groupby_fast.cuh).
    const size_t kz_extra = a.kz ? 64 : 0;
    const size_t ring = static_cast<size_t>(NS) * (stage_bytes + kz_extra);
    if (ring > 128 * 1024) return QDB_OK;
    // Ring columns: stage s, row i of column c at off_c + (s T + i) * size_c.
    StageLayout sl;
    int32_t off = 0;
    sl.key0 = off;
    off += NS * (kFastT * ks + static_cast<int32_t>(kz_extra));
    if (gb->n_key_cols == 2) {
        sl.key1 = off;
        off += NS * kFastT * ks;
    }
    if (vs) {
        sl.val = off;
        off += NS * kFastT * vs;
    }
    if (ps) {
        sl.pred = off;
        off += NS * kFastT * ps;
    }
    sl.bytes = stage_bytes;

    const bool has_mm = a.has_min || a.has_max;
    const size_t slot_bytes = 8 + 4 + (a.has_sum ? 8 : 0) + (has_mm ? (vk_is_32(vk) ? 8 : 16) : 0);
    const size_t bucket_bytes = 2 * slot_bytes;
    auto layout_table = [&](AggArgs& x, int NB) {  // offsets of the table arrays; returns the bytes used
        const size_t S = static_cast<size_t>(NB) * 2;
        size_t o = 0;
        x.NB = NB;
        x.so_keys = static_cast<int32_t>(o); o += S * 8;
        x.so_mn = static_cast<int32_t>(o); o += has_mm ? S * (vk_is_32(vk) ? 8 : 16) : 0;
        x.so_cnt = static_cast<int32_t>(o); o += S * 4;
        x.so_l0 = static_cast<int32_t>(o); o += a.has_sum ? S * 4 : 0;
        x.so_l1 = static_cast<int32_t>(o); o += a.has_sum ? S * 4 : 0;
        return (o + 127) & ~size_t(127);
    };

    // Spill plan: partitions small enough for the spill pass's table (one CTA per SM, the largest table shared
    // memory holds after the cell-fill prefix and the second-level counters) at half load.  The aggregation pass
    // writes at most 2^kMaxSpillBits partitions; a table needing more has two levels: the spill pass over the first
    // level aggregates what its table takes and sends the other rows to 2^spill_bits2 sub-partitions per partition,
    // which a third pass aggregates.  (Measured on 2^27 rows over 16.8M groups: one level of 8192 partitions, whose
    // 1.2M (partition, CTA) cells overflow L2 with partly written lines, still beats 1024 + 8 x 1024 partitions, whose
    // extra pass over many small items costs more than the better-combined writes save.)
    int spill_bits = -1;
    int spill_bits2 = 0;
    int NB2 = 0;
    const int64_t ctas_plan = std::min<int64_t>(di.sm_count, (a.n + kFastT - 1) / kFastT);
    const size_t prefix2 = ((static_cast<size_t>(ctas_plan) + 1) * 4 + 127) / 128 * 128;
    const size_t fill2_bytes = (size_t(4) << kMaxSpill2Bits);
    {
        const int64_t kb = env_int("QDB_SPILL_SMEM_KB", 0);
        const size_t budget2 = (kb > 0 ? static_cast<size_t>(kb) * 1024 : static_cast<size_t>(di.max_smem_optin) - 1024) -
                               prefix2 - fill2_bytes;
        NB2 = static_cast<int>(budget2 / bucket_bytes);
        if (NB2 >= 64 && env_int("QDB_AGG_NO_SPILL", 0) == 0) {
            const uint64_t per = static_cast<uint64_t>(NB2);  // distinct keys per partition at half load
            // At least two partitions per SM (512 on 148 SMs), so the spill pass's items balance over the SMs (the
            // last wave of a pass with 1.7 items per SM leaves a quarter of them idle); more partitions measured
            // slower (2^28-row filtered workload, aggregation + spill: 2.27 / 2.31 / 2.58 / 3.02 ms at 2 / 4 / 8 / 16
            // per SM, and 2.32 ms at one) ...
            const uint64_t min_parts =
                next_pow2(static_cast<uint64_t>(std::max<int64_t>(1, env_int("QDB_SPILL_PARTS_PER_SM", 2))) *
                          static_cast<uint64_t>(di.sm_count));
            const uint64_t parts = std::max(min_parts, next_pow2((static_cast<uint64_t>(gb->capacity) + per - 1) / per));
            int bits = 0;
            while ((1ull << bits) < parts) ++bits;
            // ... and a table sized for its partition's share of the groups at half load (the spill pass clears and
            // scans every slot of it per item).
            const uint64_t want = std::max<uint64_t>(64, next_pow2((static_cast<uint64_t>(gb->capacity) + parts - 1) / parts));
            if (want < static_cast<uint64_t>(NB2)) NB2 = static_cast<int>(want);
            const int max1 = static_cast<int>(env_int("QDB_SPILL_BITS_MAX", kMaxSpillBits));
            if (bits <= max1) {
                spill_bits = bits;
            } else if (bits <= max1 + kMaxSpill2Bits && int64_t(1) << max1 >= di.sm_count) {
                spill_bits = max1;
                spill_bits2 = bits - max1;
            }
        }
    }
    const size_t bar_bytes = 128;
    const size_t list_bytes = static_cast<size_t>(kFastWarps) * kListCap * 2;
    const size_t spill_words_bytes =
        spill_bits >= 0 ? ((size_t(4) << spill_bits) + kSeenWords * 4 + 127) & ~size_t(127) : 0;
    const size_t budget = static_cast<size_t>(di.max_smem_optin) - 1024 - ring - bar_bytes - list_bytes -
                          spill_words_bytes;
    int NBmax = static_cast<int>(budget / bucket_bytes);
    const int64_t forced = env_int("QDB_FAST_BUCKETS", 0);
    if (forced > 0 && forced < NBmax) NBmax = static_cast<int>(forced);
    if (NBmax < 64) return QDB_OK;
    // A table that holds every group at half load or less takes them all (sized for a quarter load when it can);
    // otherwise the largest table that fits, with the misses spilled by key hash.
    const uint64_t groups = static_cast<uint64_t>(gb->capacity) + 1;
    const bool fits = groups <= static_cast<uint64_t>(NBmax);
    const int NB = fits ? static_cast<int>(std::max<uint64_t>(64, std::min<uint64_t>(NBmax, 2 * groups))) : NBmax;
    if (fits) spill_bits = -1;
    const size_t tab_bytes = layout_table(a, NB);
    a.fits = fits ? 1 : 0;
    a.probe_b = fits ? 8 : 1;
    a.dedup = static_cast<int32_t>(env_int("QDB_DEDUP", 2));
    a.flush_rounds = static_cast<int32_t>(env_int("QDB_FLUSH_ROUNDS", 16));
    a.T = kFastT;
    a.NS = NS;
    a.sl = sl;
    a.tiles = (a.n + kFastT - 1) / kFastT;
    a.full_tiles = a.n / kFastT;
    a.staged = 1;

    SpillArea* spill = nullptr;
    if (spill_bits >= 0) {
        // One cell per (partition, CTA), each holding 5/4 of its share of this call's rows (at most 2^29 rows in all)
        // plus 64; rows of a full cell go to the global table.
        const int64_t parts = int64_t(1) << spill_bits;
        const int64_t ctas = std::min<int64_t>(di.sm_count, a.tiles);
        const int64_t rows = std::min<int64_t>(a.n + a.n / 4, int64_t(1) << 29);
        const int64_t cell = rows / (parts * ctas) + 64;
        // Records of 16 bytes (key word, value bits), or 8 (the key word) for a count-only table; one more fill word
        // is the spill pass's work counter.
        const uint64_t words = static_cast<uint64_t>(parts * ctas * cell) * (vs ? 2 : 1);
        // A second level takes as many records again, in 2^spill_bits2 cells per first-level partition, and its own
        // fill words (plus the third pass's work counter).
        const int64_t cells2 = spill_bits2 ? (parts << spill_bits2) : 0;
        int32_t rc = spill_acquire(gb->device, spill_bits2 ? 2 * words : words, 0,
                                   parts * ctas + 1 + (spill_bits2 ? cells2 + 1 : 0), s, &spill);
        if (rc != QDB_OK) return rc;
        a.spill_keys = spill->keys;
        a.spill_vals = nullptr;
        a.spill_fill = spill->fill;
        a.spill_cell = cell;
        a.spill_bits = spill_bits;
        a.spill_ctas = static_cast<int32_t>(ctas);
        if (spill_bits2) {
            a.spill2_keys = spill->keys + words;
            a.spill2_fill = spill->fill + parts * ctas + 1;
            a.spill2_cell = ctas * cell >> spill_bits2;
            a.spill2_bits = spill_bits2;
        }
    }
    a.so_bar = static_cast<int32_t>(tab_bytes);
    a.so_list = static_cast<int32_t>(tab_bytes + bar_bytes);
    a.so_spill = static_cast<int32_t>(a.so_list + list_bytes);
    a.so_stage = static_cast<int32_t>(a.so_spill + spill_words_bytes);
    const size_t smem = a.so_stage + ring;
    *used = true;
    int32_t rc = launch_fast(gb, a, ptype, smem, s);
    if (rc != QDB_OK || spill_bits < 0) {
        if (spill) spill_release(spill, s);
        return rc;
    }
    // Spill pass: one persistent CTA per SM, each with a table of NB2 buckets, taking (partition, slice) items; a
    // partition is cut into slices only when there are fewer partitions than CTAs.  Over the first of two levels the
    // table takes a key only into its home bucket and sends the rest on; the last level's table takes every key.
    AggArgs b = a;
    const size_t tab2 = layout_table(b, NB2);
    b.so_spill = static_cast<int32_t>(tab2);  // the prefix of the cell fills
    b.so_spill2 = static_cast<int32_t>(tab2 + prefix2);
    const size_t smem2 = tab2 + prefix2 + fill2_bytes;
    b.fits = spill_bits2 ? 0 : 1;
    b.probe_b = spill_bits2 ? 1 : 8;
    const int64_t parts = int64_t(1) << spill_bits;
    const int64_t ctas2 = static_cast<int64_t>(di.sm_count);
    const int64_t slices = std::max<int64_t>(1, std::min<int64_t>(a.spill_ctas, ctas2 / parts));
    rc = launch_fspill(gb, b, smem2, std::min<int64_t>(ctas2, parts * slices), static_cast<int32_t>(slices), s);
    if (rc == QDB_OK && spill_bits2) {
        // Third pass: every second-level cell is one partition of 2^(spill_bits + spill_bits2).
        AggArgs c = b;
        c.spill_keys = a.spill2_keys;
        c.spill_fill = a.spill2_fill;
        c.spill_cell = a.spill2_cell;
        c.spill_bits = spill_bits + spill_bits2;
        c.spill_ctas = 1;
        c.spill2_keys = nullptr;
        c.spill2_fill = nullptr;
        c.spill2_bits = 0;
        c.fits = 1;
        c.probe_b = 8;
        const int64_t items3 = int64_t(1) << c.spill_bits;
        rc = launch_fspill(gb, c, smem2, std::min<int64_t>(ctas2, items3), 1, s);
    }
    spill_release(spill, s);
    return rc;
}

}  // namespace qdb

using namespace qdb;

extern "C" {

int32_t qdb_gb_create(qdb_gb** out, int32_t agg_mask, int32_t key_type, int32_t n_key_cols, int32_t val_type,
                      int64_t max_groups, int32_t placement, void* stream) {
    if (!out) return fail(QDB_ERR_INVALID, "qdb_gb_create: null out");
    *out = nullptr;
    if (agg_mask & ~(QDB_AGG_MIN | QDB_AGG_MAX | QDB_AGG_SUM | QDB_AGG_AVG | QDB_AGG_COUNT))
        return fail(QDB_UNKNOWN_AGG_FUN, "qdb_gb_create: unknown aggregate bits");
    if (n_key_cols != 1 && n_key_cols != 2) return fail(QDB_ERR_INVALID, "qdb_gb_create: n_key_cols must be 1 or 2");
    if (n_key_cols == 2 && key_type != QDB_INT32)
        return fail(QDB_ERR_INVALID, "qdb_gb_create: composite keys are (int32, int32)");
    if (key_type != QDB_INT32 && key_type != QDB_INT64 && key_type != QDB_FLOAT && key_type != QDB_DOUBLE)
        return fail(QDB_ERR_INVALID, "qdb_gb_create: unsupported key type");
    if (val_type != 0 && val_kind(val_type) == VK_NONE)
        return fail(QDB_ERR_INVALID, "qdb_gb_create: unsupported value type");
    if (val_type == 0 && (agg_mask & (QDB_AGG_MIN | QDB_AGG_MAX | QDB_AGG_SUM | QDB_AGG_AVG)))
        return fail(QDB_ERR_INVALID, "qdb_gb_create: MIN/MAX/SUM/AVG need a value column");
    if (max_groups < 1) return fail(QDB_ERR_INVALID, "qdb_gb_create: max_groups must be >= 1");
    if (max_groups > (int64_t(1) << 30)) max_groups = int64_t(1) << 30;  // GB_BUFFER_SIZE_MAX
    int dev = 0;
    QDB_CUDA_TRY(cudaGetDevice(&dev));
    cudaStream_t s = as_stream(stream);

    qdb_gb* gb = new qdb_gb();
    gb->aggs = agg_mask;
    gb->key_type = key_type;
    gb->n_key_cols = n_key_cols;
    gb->val_type = val_type;
    gb->placement = placement;
    gb->device = dev;
    gb->capacity = max_groups;
    gb->cap = next_pow2(std::max<uint64_t>(16, static_cast<uint64_t>(max_groups) * 3 / 2 + 1));
    gb->L = make_layout(agg_mask, val_kind(val_type));
    int32_t rc = dev_alloc(reinterpret_cast<void**>(&gb->counters), 2 * sizeof(unsigned long long), s);
    if (rc == QDB_OK) rc = gb_init_region(gb, gb->main, s);
    if (rc == QDB_OK && cudaMemsetAsync(gb->counters, 0, 2 * sizeof(unsigned long long), s) != cudaSuccess)
        rc = cuda_fail(cudaGetLastError(), "cudaMemsetAsync(counters)");
    if (rc != QDB_OK) {
        qdb_gb_destroy(gb);
        return rc;
    }
    *out = gb;
    return QDB_OK;
}

int32_t qdb_gb_destroy(qdb_gb* gb) {
    if (!gb) return QDB_OK;
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != gb->device) cudaSetDevice(gb->device);
    // The table may still be in use by work queued on another stream: free in stream order on the
    // legacy stream, which orders after all blocking streams.
    dev_free(gb->main.slots, 0);
    dev_free(gb->aux.slots, 0);
    dev_free(gb->counters, 0);
    if (prev != gb->device) cudaSetDevice(prev);
    delete gb;
    return QDB_OK;
}

int32_t qdb_gb_max_hash_count(qdb_gb* gb, int64_t* out) {
    if (!gb || !out) return fail(QDB_ERR_INVALID, "qdb_gb_max_hash_count: null argument");
    *out = gb->capacity + 1;  // + 1 for the NULL key, as keyBufferSize_ (GPUGroupBy.cuh:315)
    return QDB_OK;
}

int32_t qdb_gb_group_count(qdb_gb* gb, int64_t* out, void* stream) {
    if (!gb || !out) return fail(QDB_ERR_INVALID, "qdb_gb_group_count: null argument");
    unsigned long long h = 0;
    QDB_CUDA_TRY(cudaMemcpyAsync(&h, gb->counters, sizeof(h), cudaMemcpyDeviceToHost, as_stream(stream)));
    QDB_CUDA_TRY(cudaStreamSynchronize(as_stream(stream)));
    *out = static_cast<int64_t>(h);
    return QDB_OK;
}

int32_t qdb_gb_reset(qdb_gb* gb, void* stream) {
    if (!gb) return fail(QDB_ERR_INVALID, "qdb_gb_reset: null table");
    cudaStream_t s = as_stream(stream);
    int32_t rc = gb_init_region(gb, gb->main, s);
    if (rc == QDB_OK && gb->aux.slots) rc = gb_init_region(gb, gb->aux, s);
    if (rc != QDB_OK) return rc;
    QDB_CUDA_TRY(cudaMemsetAsync(gb->counters, 0, 2 * sizeof(unsigned long long), s));
    return QDB_OK;
}

// A compressed-key call (kz) or a fused key % m call (km) that the fast pass cannot take: the caller decompresses the
// keys, or materialises the remainder column, instead.
constexpr int32_t kNotFused = -1;

static int32_t process_impl(qdb_gb* gb, const void* const* key_cols, const uint64_t* const* key_nulls, const void* vals,
                            const uint64_t* val_nulls, int64_t n, const qdb_pred* pred, const int8_t* mask,
                            void* stream, const AaflView* kz, const ModMagic* km = nullptr) {
    if (!gb) return fail(QDB_ERR_INVALID, "qdb_gb_process: null table");
    if (n < 0) return fail(QDB_ERR_INVALID, "qdb_gb_process: negative row count");
    if (n == 0) return QDB_OK;
    if (!kz && (!key_cols || !key_cols[0] || (gb->n_key_cols == 2 && !key_cols[1])))
        return fail(QDB_ERR_INVALID, "qdb_gb_process: missing key column");
    if (gb->val_type != 0 && !vals) return fail(QDB_ERR_INVALID, "qdb_gb_process: missing value column");
    int32_t ptype = 0;
    if (pred) {
        if (!pred->col) return fail(QDB_ERR_INVALID, "qdb_gb_process: predicate without column");
        if (pred->op < QDB_GREATER || pred->op > QDB_NOT_EQUAL)
            return fail(QDB_ERR_INVALID, "qdb_gb_process: predicate op must be a comparison");
        if (pred->type != QDB_INT32 && pred->type != QDB_INT64 && pred->type != QDB_FLOAT && pred->type != QDB_DOUBLE)
            return fail(QDB_ERR_INVALID, "qdb_gb_process: unsupported predicate column type");
        if (pred->const_type != QDB_INT32 && pred->const_type != QDB_INT64 && pred->const_type != QDB_FLOAT &&
            pred->const_type != QDB_DOUBLE)
            return fail(QDB_ERR_INVALID, "qdb_gb_process: unsupported predicate constant type");
        ptype = pred->type;
    }
    cudaStream_t s = as_stream(stream);
    const uint64_t* kn0 = key_nulls ? key_nulls[0] : nullptr;
    const uint64_t* kn1 = (key_nulls && gb->n_key_cols == 2) ? key_nulls[1] : nullptr;
    if (gb->n_key_cols == 2 && (kn0 || kn1) && !gb->aux.slots) {
        int32_t rc = gb_init_region(gb, gb->aux, s);
        if (rc != QDB_OK) return rc;
    }

    AggArgs a;
    a.key0 = kz ? nullptr : key_cols[0];
    a.key1 = (!kz && gb->n_key_cols == 2) ? key_cols[1] : nullptr;
    if (kz) {
        a.kz = 1;
        a.kz_words = kz->words;
        a.kz_pos = kz->pos;
        a.kz_bits = kz->bits;
        a.kz_off = kz->off;
        a.kz_len = kz->words_len;
    }
    if (km) {
        a.kmod = 1;
        a.km_d = km->d;
        a.km_m = km->m;
        a.km_s1 = km->s1;
        a.km_s2 = km->s2;
    }
    a.knull0 = kn0;
    a.knull1 = kn1;
    a.vals = gb->val_type ? vals : nullptr;
    a.vnull = gb->val_type ? val_nulls : nullptr;
    if (pred) {
        a.pcol = pred->col;
        a.pnull = pred->nulls;
        a.pi = pred_interval(*pred);
    }
    a.mask = mask;
    a.n = n;
    a.main = gb->main;
    a.aux = gb->aux;
    a.L = gb->L;
    const ValKind vk = val_kind(gb->val_type);
    a.has_sum = gb->L.sum >= 0;
    a.has_min = (gb->aggs & QDB_AGG_MIN) && gb->L.mn >= 0;
    a.has_max = (gb->aggs & QDB_AGG_MAX) && gb->L.mx >= 0;
    a.counters = gb->counters;
    a.capacity = static_cast<unsigned long long>(gb->capacity);
    const bool nulls = a.knull0 || a.knull1 || a.vnull || a.pnull;
    if (!nulls && !mask && gb->placement != QDB_PLACE_GLOBAL && n >= kFastT && env_int("QDB_AGG_FAST", 1) != 0 &&
        (kz || aligned16(a.key0)) && (!a.key1 || aligned16(a.key1)) && (!a.vals || aligned16(a.vals)) &&
        (!a.pcol || aligned16(a.pcol))) {
        bool used = false;
        const int32_t rc = process_fast(gb, a, pred, ptype, s, &used);
        if (rc != QDB_OK || used) return rc;
    }
    if (kz || km) return kNotFused;

    // Tile and stage plan: stages of about 32 KB (a stage costs a fixed hand-off between the producer and
    // the consumers, so small stages cannot reach the HBM bandwidth), three of them in the ring.
    const DeviceInfo& di = device_info();
    const int ks = (gb->n_key_cols == 2) ? 4 : type_size(gb->key_type);
    int row_bytes = ks * gb->n_key_cols + (a.vals ? type_size(gb->val_type) : 0) + (a.pcol ? type_size(pred->type) : 0) +
                    (a.mask ? 1 : 0);
    if (row_bytes < 1) row_bytes = 1;
    int Rw = static_cast<int>(env_int("QDB_AGG_ROWS_PER_WARP",
                                      (32 * 1024) / (row_bytes * kConsumerWarps)));
    Rw = std::min(512, std::max(kRowsPerWarpUnit, (Rw / kRowsPerWarpUnit) * kRowsPerWarpUnit));
    int T = kConsumerWarps * Rw;
    auto col_bytes = [&](int rows, int elem) { return static_cast<int32_t>(((size_t)rows * elem + 127) & ~size_t(127)); };
    auto plan_stage = [&](int rows) {
        StageLayout sl;
        int32_t off = 0;
        sl.key0 = off; off += col_bytes(rows, ks);
        if (gb->n_key_cols == 2) { sl.key1 = off; off += col_bytes(rows, ks); }
        if (a.vals) { sl.val = off; off += col_bytes(rows, type_size(gb->val_type)); }
        if (a.pcol) { sl.pred = off; off += col_bytes(rows, type_size(pred->type)); }
        if (a.mask) { sl.mask = off; off += col_bytes(rows, 1); }
        if (a.knull0) { sl.knull0 = off; off += col_bytes(rows / 64, 8); }
        if (a.knull1) { sl.knull1 = off; off += col_bytes(rows / 64, 8); }
        if (a.vnull) { sl.vnull = off; off += col_bytes(rows / 64, 8); }
        if (a.pnull) { sl.pnull = off; off += col_bytes(rows / 64, 8); }
        sl.bytes = off;
        return sl;
    };
    StageLayout sl = plan_stage(T);
    while (Rw > kRowsPerWarpUnit && sl.bytes > 48 * 1024) {
        Rw -= kRowsPerWarpUnit;
        T = kConsumerWarps * Rw;
        sl = plan_stage(T);
    }
    int NS = static_cast<int>(env_int("QDB_AGG_STAGES", sl.bytes * 3 <= 112 * 1024 ? 3 : 2));
    NS = std::min(8, std::max(2, NS));
    const bool aligned = aligned16(a.key0) && (!a.key1 || aligned16(a.key1)) && (!a.vals || aligned16(a.vals)) &&
                         (!a.pcol || aligned16(a.pcol)) && (!mask || aligned16(mask)) &&
                         (!a.knull0 || aligned16(a.knull0)) && (!a.knull1 || aligned16(a.knull1)) &&
                         (!a.vnull || aligned16(a.vnull)) && (!a.pnull || aligned16(a.pnull));
    a.T = T;
    a.NS = NS;
    a.sl = sl;
    a.tiles = (n + T - 1) / T;
    a.full_tiles = n / T;
    a.staged = aligned && a.full_tiles > 0 && env_int("QDB_AGG_DIRECT", 0) == 0;
    const size_t stage_area = a.staged ? static_cast<size_t>(NS) * sl.bytes : 0;
    const size_t bar_bytes = 128;
    const size_t list_bytes = (static_cast<size_t>(T) * 2 + 127) & ~size_t(127);
    const size_t queue_bytes = static_cast<size_t>(kConsumerWarps) * kQueueCap * (8 + 8 + 4);

    // Shared-memory table: bytes per slot (key, count, sum limbs, min/max).
    const bool has_mm = a.has_min || a.has_max;
    const bool vfloat = vk == VK_F32 || vk == VK_F64;
    const size_t limb_bytes = a.has_sum ? (vfloat ? 12 : 8) : 0;
    const size_t mm_bytes = has_mm ? (vk_is_32(vk) ? 8 : 16) : 0;
    const size_t bps = 8 + 4 + limb_bytes + mm_bytes;
    auto layout_table = [&](AggArgs& x, int S) {  // offsets of the table arrays; returns the bytes used
        const size_t S2 = static_cast<size_t>(S) + 2;
        size_t off = S2 * 8;
        x.so_mn = static_cast<int32_t>(off); off += S2 * mm_bytes;
        x.so_cnt = static_cast<int32_t>(off); off += S2 * 4;
        x.so_l0 = static_cast<int32_t>(off); off += a.has_sum ? S2 * 4 : 0;
        x.so_l1 = static_cast<int32_t>(off); off += a.has_sum ? S2 * 4 : 0;
        x.so_l2 = static_cast<int32_t>(off); off += (a.has_sum && vfloat) ? S2 * 4 : 0;
        return (off + 127) & ~size_t(127);
    };

    // Spill plan: when the table's group bound does not fit the shared table, misses are partitioned by key
    // hash into 2^bits partitions, each small enough for the spill pass's shared table.
    const bool smem_place = gb->placement != QDB_PLACE_GLOBAL;
    int spill_bits = -1;
    int S2spill = 0;
    if (smem_place && env_int("QDB_AGG_NO_SPILL", 0) == 0) {
        const size_t budget2 = static_cast<size_t>(env_int("QDB_SPILL_SMEM_KB", 50)) * 1024 - 1024;  // - the fill prefix  // 50 KB: four spill-pass CTAs per SM
        int S2 = 1 << 15;
        while (S2 >= 256 && static_cast<size_t>(S2 + 2) * bps + 256 > budget2) S2 >>= 1;
        if (S2 >= 256) {
            const uint64_t per = static_cast<uint64_t>(S2) / 2;  // distinct keys per partition at load factor 1/2
            const uint64_t parts = next_pow2((static_cast<uint64_t>(gb->capacity) + per - 1) / per);
            int bits = 0;
            while ((1ull << bits) < parts) ++bits;
            if (bits <= 10) {
                spill_bits = bits;
                S2spill = S2;
            }
        }
    }
    // spill cell fill counters, then a 32768-bit filter of keys seen once (admission to the shared table)
    const size_t spill_words_bytes = spill_bits >= 0 ? ((size_t(4) << spill_bits) + kSeenWords * 4 + 127) & ~size_t(127) : 0;
    const size_t budget = static_cast<size_t>(di.max_smem_optin) - 1024 - stage_area - bar_bytes - list_bytes -
                          queue_bytes - spill_words_bytes;

    size_t hash_bytes = 0;
    if (smem_place) {
        int S = 1 << 16;
        while (S >= 256 && static_cast<size_t>(S + 2) * bps + 128 > budget) S >>= 1;
        // A table much larger than the group count only costs initialisation and merge time.
        const uint64_t want = next_pow2(static_cast<uint64_t>(gb->capacity) * 2 + 2);
        if (static_cast<uint64_t>(S) > want) S = static_cast<int>(std::max<uint64_t>(want, 256));
        const int64_t forced = env_int("QDB_AGG_SMEM_SLOTS", 0);
        if (forced > 0 && forced < S) S = static_cast<int>(next_pow2(static_cast<uint64_t>(forced)));
        if (S >= 256) {
            a.S = S;
            const bool fits = static_cast<uint64_t>(gb->capacity) + 2 <= static_cast<uint64_t>(S) / 2;
            a.probe = fits ? S : static_cast<int>(env_int("QDB_AGG_PROBE", 4));
            hash_bytes = layout_table(a, S);
            if (fits) spill_bits = -1;  // every group fits the shared table: no misses to spill
        } else {
            spill_bits = -1;
        }
    }
    SpillArea* spill = nullptr;
    if (spill_bits >= 0) {
        // Spill area: one cell per (partition, CTA).  A cell holds 5/4 of its share of half this call's rows (at
        // most 2^28 rows in all) plus 64: warps whose shared-table hit rate is below 1/2 stop spilling, so hashed
        // misses overflow a cell only in the first tiles of such warps (and rows of a full cell go to the global
        // table).
        const int64_t parts = int64_t(1) << spill_bits;
        const int64_t ctas = std::min<int64_t>(di.sm_count, a.tiles);
        const int64_t rows = std::min<int64_t>((n + 1) / 2, int64_t(1) << 28);
        const int64_t cell = (rows + rows / 4) / (parts * ctas) + 64;
        const int vbytes = a.vals ? type_size(gb->val_type) : 0;
        int32_t rc = spill_acquire(gb->device, static_cast<uint64_t>(parts * ctas * cell), vbytes, parts * ctas, s, &spill);
        if (rc != QDB_OK) return rc;
        a.spill_keys = spill->keys;
        a.spill_vals = vbytes ? spill->vals : nullptr;
        a.spill_fill = spill->fill;
        a.spill_cell = cell;
        a.spill_bits = spill_bits;
        a.spill_ctas = static_cast<int32_t>(ctas);
    }
    a.so_bar = static_cast<int32_t>(hash_bytes);
    a.so_list = static_cast<int32_t>(hash_bytes + bar_bytes);
    a.so_queue = static_cast<int32_t>(hash_bytes + bar_bytes + list_bytes);
    a.so_spill = static_cast<int32_t>(a.so_queue + ((queue_bytes + 127) & ~size_t(127)));
    a.so_stage = static_cast<int32_t>(a.so_spill + spill_words_bytes);
    const size_t smem = a.so_stage + stage_area;
    int32_t rc = launch_agg(gb, a, ptype, nulls, smem, s);
    if (rc != QDB_OK || spill_bits < 0) {
        if (spill) spill_release(spill, s);
        return rc;
    }

    // Spill pass: partitions x slices CTAs, each with a shared table of S2spill slots.
    AggArgs b = a;
    b.S = S2spill;
    b.probe = 64;
    const size_t smem2 = layout_table(b, S2spill);
    const int64_t parts = int64_t(1) << spill_bits;
    const int64_t slices = std::max<int64_t>(1, std::min<int64_t>(a.spill_ctas, (4 * di.sm_count + parts - 1) / parts));
    rc = launch_spill(gb, b, smem2, parts * slices, s);
    spill_release(spill, s);
    return rc;
}


int32_t qdb_gb_process(qdb_gb* gb, const void* const* key_cols, const uint64_t* const* key_nulls, const void* vals,
                       const uint64_t* val_nulls, int64_t n, const qdb_pred* pred, const int8_t* mask,
                       void* stream) {
    return process_impl(gb, key_cols, key_nulls, vals, val_nulls, n, pred, mask, stream, nullptr);
}

int32_t qdb_gb_process_aafl(qdb_gb* gb, const qdb_aafl_col* keys, const void* vals, const qdb_pred* pred,
                            void* stream) {
    if (!gb || !keys) return fail(QDB_ERR_INVALID, "qdb_gb_process_aafl: null argument");
    if (gb->n_key_cols != 1 || keys->type != gb->key_type)
        return fail(QDB_ERR_INVALID, "qdb_gb_process_aafl: the block's type must be the single key type of the table");
    cudaStream_t s = as_stream(stream);
    AaflView v;
    int32_t rc = aafl_view(keys, &v, s);
    if (rc != QDB_OK || v.rows == 0) return rc;
    rc = process_impl(gb, nullptr, nullptr, vals, nullptr, v.rows, pred, nullptr, stream, &v);
    if (rc == kNotFused) {
        void* col = nullptr;
        rc = dev_alloc(&col, static_cast<size_t>(v.rows) * v.word_bytes, s);
        if (rc == QDB_OK) rc = qdb_aafl_decompress(keys, col, stream);
        const void* kc[1] = {col};
        if (rc == QDB_OK) rc = process_impl(gb, kc, nullptr, vals, nullptr, v.rows, pred, nullptr, stream, nullptr);
        dev_free(col, s);
    }
    dev_free(v.scratch, s);  // stream-ordered: after the pass that reads it
    return rc;
}

int32_t qdb_gb_process_mod(qdb_gb* gb, const void* keys, int64_t key_mod, const void* vals, const qdb_pred* pred,
                           int64_t n, void* stream) {
    if (!gb || (n > 0 && !keys)) return fail(QDB_ERR_INVALID, "qdb_gb_process_mod: null argument");
    if (gb->n_key_cols != 1 || (gb->key_type != QDB_INT32 && gb->key_type != QDB_INT64))
        return fail(QDB_ERR_INVALID, "qdb_gb_process_mod: the table must have a single INT32 or INT64 key");
    if (key_mod == 0) return fail(QDB_DIVISION_BY_ZERO, "qdb_gb_process_mod: modulo by zero");
    if (key_mod == INT64_MIN || (gb->key_type == QDB_INT32 && (key_mod > INT32_MAX || key_mod < INT32_MIN)))
        return fail(QDB_ERR_INVALID, "qdb_gb_process_mod: modulus out of the key type's range");
    if (n == 0) return QDB_OK;
    const ModMagic mm = mod_magic(static_cast<uint64_t>(key_mod < 0 ? -key_mod : key_mod));
    const void* kc[1] = {keys};
    int32_t rc = process_impl(gb, kc, nullptr, vals, nullptr, n, pred, nullptr, stream, nullptr, &mm);
    if (rc != kNotFused) return rc;
    // the fast pass does not apply: the remainder column first, as the dispatcher computes it
    cudaStream_t s = as_stream(stream);
    void* col = nullptr;
    rc = dev_alloc(&col, static_cast<size_t>(n) * type_size(gb->key_type), s);
    if (rc == QDB_OK) rc = qdb_arith_mod(gb->key_type, keys, key_mod, col, n, stream);
    const void* mc[1] = {col};
    if (rc == QDB_OK) rc = process_impl(gb, mc, nullptr, vals, nullptr, n, pred, nullptr, stream, nullptr);
    dev_free(col, s);
    return rc;
}

int32_t qdb_gb_check(qdb_gb* gb, void* stream) {
    if (!gb) return fail(QDB_ERR_INVALID, "qdb_gb_check: null table");
    cudaStream_t s = as_stream(stream);
    int32_t status = 0;
    QDB_CUDA_TRY(cudaMemcpyAsync(&status, &gb->counters[1], sizeof(status), cudaMemcpyDeviceToHost, s));
    QDB_CUDA_TRY(cudaStreamSynchronize(s));
    if (status != QDB_OK) {
        QDB_CUDA_TRY(cudaMemsetAsync(&gb->counters[1], 0, sizeof(unsigned long long), s));
        if (status == QDB_HASH_TABLE_FULL)
            return fail(QDB_HASH_TABLE_FULL, "GROUP BY hash table is full (more distinct keys than max_groups)");
        return fail(status, "GROUP BY kernel reported an error");
    }
    return QDB_OK;
}

int32_t qdb_gb_process_sync(qdb_gb* gb, const void* const* key_cols, const uint64_t* const* key_nulls,
                            const void* vals, const uint64_t* val_nulls, int64_t n, const qdb_pred* pred,
                            const int8_t* mask, void* stream) {
    int32_t rc = qdb_gb_process(gb, key_cols, key_nulls, vals, val_nulls, n, pred, mask, stream);
    if (rc != QDB_OK) return rc;
    return qdb_gb_check(gb, stream);
}

}  // extern "C"
