// GROUP BY over string keys: the replacement of GPUGroupBy<AGG, O, std::string, V>
// (qikkDB/QueryEngine/GPUCore/GPUGroupByString.cuh:39-169 and the class after it), whose kernel claims a slot by
// the row index of the string's first occurrence, compares keys byte by byte against the input blocks, and
// aggregates with global atomics into 256x replicated value buffers.
//
// Here a call is two passes.  The first dictionary-encodes the keys: a table that owns its keys maps every string
// to a slot, and each row's slot number is written to a scratch column.  The second is the numeric GROUP BY pass over
// (slot number, value) with the same NULL masks and row mask, so the aggregation of string keys runs on the same
// shared-memory tables, spill partitions and accumulators as integer keys.
//
// Keys come in the reference's GPUString layout: all characters concatenated, and int64 end offsets (string i is
// chars[i ? ends[i - 1] : 0, ends[i])).  The dictionary pass reads a string as little-endian 8-byte words: aligned
// loads of the character buffer, two of them funnel-shifted for an unaligned start; a load is issued only for an
// aligned word that holds one of the string's bytes (the buffer's own words, so no access leaves the pages the
// buffer lies in).  It hashes the words (length-seeded multiply-xorshift rounds, then the 64-bit finaliser) and
// probes linearly from the hash's home slot.  A slot is a header word (the key's hash; 0 = empty) and a 32-byte
// record: a meta word (0 until published, then (arena offset << 20) | (length + 1)) and the key's first 24 bytes;
// a longer key's remaining words go to a device arena (bump-allocated 8-byte words).
//   * An empty slot is claimed with a CAS of the hash into its header; the claimer writes the record's words and the
//     arena words, fences, and publishes the meta word.
//   * A row whose hash matches the header reads the meta word (waiting, bounded, while it is 0: a claimer that never
//     publishes ends the wait with QDB_ERR_TIMEOUT) and compares the key.  Records and arena words are read through
//     L1, so the hot keys of a skewed column are served by every SM's own L1 instead of one L2 slice.  An L1 sector
//     filled before the key was published still holds meta 0 (the reset cleared it, the publication writes it last),
//     so a nonzero meta read there comes with the key's words; a comparison that fails is repeated from L2
//     (ld.global.cg) before the probe moves on, so a stale word can never make one key two groups.
// More distinct keys than max_groups, or a full key arena, raise QDB_HASH_TABLE_FULL, as ProcessBlock does.
// GetResults takes the numeric table's groups (slot number, NULL flag, aggregates) and rebuilds each key's string from
// the records and the arena into a GPUString.
#include "groupby_agg.cuh"
#include "scan.cuh"

namespace qdb {

constexpr int kGbsThreads = 256;
constexpr uint64_t kMetaPoison = ~0ull;                 // a claimer that could not store its key
constexpr uint32_t kGbsWaitIters = 1u << 20;            // bounded wait for a claimer to publish its key
constexpr int kGbsInline = 3;                           // key words kept in the slot record
constexpr int64_t kGbsMaxLen = (int64_t(1) << 20) - 2;  // longest key the meta word encodes

struct GbsRec {
    uint64_t meta;
    uint64_t w[kGbsInline];
};

struct GbsDict {
    uint64_t* header = nullptr;  // [cap] 0: empty; else the key's hash (never 0)
    GbsRec* rec = nullptr;       // [cap] 32-byte aligned records
    uint64_t* arena = nullptr;   // words 3.. of long keys
    uint64_t arena_words = 0;
    unsigned long long* counters = nullptr;  // [0] arena words used, [1] status, [2] distinct keys
    uint64_t cap = 0;                        // slots (power of two)
    unsigned long long capacity = 0;         // max_groups
};

__host__ __device__ __forceinline__ int64_t gbs_meta_len(uint64_t m) { return static_cast<int64_t>(m & 0xfffffull) - 1; }
__host__ __device__ __forceinline__ uint64_t gbs_meta_off(uint64_t m) { return m >> 20; }

// Bytes [b, b + min(8, rem)) of the character buffer, zero-padded, as a little-endian word.  W is the buffer's
// aligned word view; W[k + 1] is loaded only when it holds one of those bytes.
__device__ __forceinline__ uint64_t gbs_word(const uint64_t* __restrict__ W, int64_t b, int64_t rem) {
    const int64_t k = b >> 3;
    const int sh = static_cast<int>(b & 7);
    uint64_t v = __ldg(W + k) >> (8 * sh);
    const int64_t take = rem < 8 ? rem : 8;
    if (sh && take > 8 - sh) v |= __ldg(W + k + 1) << (64 - 8 * sh);
    if (take < 8) v &= (1ull << (8 * take)) - 1ull;
    return v;
}

__device__ __forceinline__ uint64_t gbs_round(uint64_t h, uint64_t w) {
    h = (h ^ w) * 0x9E3779B97F4A7C15ull;
    return h ^ (h >> 29);
}

// Word j of the published key of record r (meta m): through L1, or from L2 when `l2`.
__device__ __forceinline__ uint64_t gbs_key_word(const GbsDict& t, const GbsRec* r, uint64_t m, int64_t j, bool l2) {
    if (j < kGbsInline) return l2 ? __ldcg(&r->w[j]) : r->w[j];
    const uint64_t* a = t.arena + gbs_meta_off(m) + (j - kGbsInline);
    return l2 ? __ldcg(a) : *a;
}

// Claims record r (slot pos) for the key (n bytes at byte offset b of W; w0..w2 its first three words, zero-padded)
// and publishes it.  Kept out of line: the probe loop stays small, and claims are rare after a table fills.
__device__ __noinline__ int64_t gbs_claim(GbsRec* r, uint64_t pos, uint64_t* arena, uint64_t arena_words,
                                          unsigned long long* counters, const uint64_t* __restrict__ W, int64_t b,
                                          int64_t n, uint64_t w0, uint64_t w1, uint64_t w2, unsigned* claims) {
    atomicAdd(claims, 1u);
    const int64_t words = (n + 7) >> 3;
    const uint64_t extra = words > kGbsInline ? static_cast<uint64_t>(words - kGbsInline) : 0ull;
    const unsigned long long o = extra ? atomicAdd(&counters[0], static_cast<unsigned long long>(extra)) : 0ull;
    if (o + extra > arena_words) {
        atomicExch(reinterpret_cast<int*>(&counters[1]), static_cast<int>(QDB_HASH_TABLE_FULL));
        atomicExch(reinterpret_cast<unsigned long long*>(&r->meta), kMetaPoison);
        return -1;
    }
    r->w[0] = w0;
    r->w[1] = w1;
    r->w[2] = w2;
    for (int64_t j = kGbsInline; j < words; ++j) arena[o + (j - kGbsInline)] = gbs_word(W, b + 8 * j, n - 8 * j);
    __threadfence();
    atomicExch(reinterpret_cast<unsigned long long*>(&r->meta),
               (static_cast<unsigned long long>(o) << 20) | static_cast<unsigned long long>(n + 1));
    return static_cast<int64_t>(pos);
}

// Finds or claims the string at byte offset b (n bytes) of the buffer W; returns its slot, or -1 (table or arena
// full, key too long, or a wait that gave up: the status word says which).  A key of at most 24 bytes lives in its
// record: its three words (zero-padded) are hashed and compared without loops, the record read as two 16-byte loads.
__device__ int64_t gbs_find(const GbsDict& t, const uint64_t* __restrict__ W, int64_t b, int64_t n, unsigned* claims) {
    if (n > kGbsMaxLen) {
        atomicExch(reinterpret_cast<int*>(&t.counters[1]), static_cast<int>(QDB_ERR_TOO_LARGE));
        return -1;
    }
    const bool shortk = n <= 8 * kGbsInline;
    uint64_t w[kGbsInline];
#pragma unroll
    for (int j = 0; j < kGbsInline; ++j) w[j] = 8 * j < n ? gbs_word(W, b + 8 * j, n - 8 * j) : 0ull;
    uint64_t h = 0x243F6A8885A308D3ull ^ (static_cast<uint64_t>(n) * 0xBF58476D1CE4E5B9ull);
#pragma unroll
    for (int j = 0; j < kGbsInline; ++j)
        if (8 * j < n) h = gbs_round(h, w[j]);
    for (int64_t j = 8 * kGbsInline; j < n; j += 8) h = gbs_round(h, gbs_word(W, b + j, n - j));
    h = mix64(h);
    if (h == 0) h = 1;
    const int64_t words = (n + 7) >> 3;
    const uint64_t mask = t.cap - 1;
    uint64_t pos = __umul64hi(h, t.cap);
    for (uint64_t probe = 0; probe < t.cap; ++probe, pos = (pos + 1) & mask) {
        uint64_t cur = t.header[pos];  // a stale 0 only sends the row to the CAS, which reads the live value
        GbsRec* r = t.rec + pos;
        if (cur == 0) {
            cur = atomicCAS(reinterpret_cast<unsigned long long*>(t.header + pos), 0ull, h);
            if (cur == 0) return gbs_claim(r, pos, t.arena, t.arena_words, t.counters, W, b, n, w[0], w[1], w[2], claims);
        }
        if (cur != h) continue;
        // Same hash: the published meta word, then the key.
        const ulonglong2* rq = reinterpret_cast<const ulonglong2*>(r);
        ulonglong2 q0 = rq[0], q1 = rq[1];  // (meta, w0), (w1, w2)
        bool l2 = false;
        for (uint32_t it = 0; q0.x == 0 && it < kGbsWaitIters; ++it) {
            __nanosleep(64);
            q0.x = ld_volatile_u64(&r->meta);
            l2 = true;  // the record's L1 copy predates the publication: read the key from L2
        }
        const uint64_t m = q0.x;
        if (m == 0) {
            atomicExch(reinterpret_cast<int*>(&t.counters[1]), static_cast<int>(QDB_ERR_TIMEOUT));
            return -1;
        }
        if (m == kMetaPoison || gbs_meta_len(m) != n) continue;
        if (l2) {
            q0 = __ldcg(rq);
            q1 = __ldcg(rq + 1);
        }
        bool eq = (q0.y == w[0]) & (q1.x == w[1]) & (q1.y == w[2]);
        if (!shortk)
            for (int64_t j = kGbsInline; j < words && eq; ++j)
                eq = gbs_key_word(t, r, m, j, l2) == gbs_word(W, b + 8 * j, n - 8 * j);
        if (!eq && !l2) {
            // a stale L1 copy cannot make a key miss its own slot: compare once more from L2
            const ulonglong2 c0 = __ldcg(rq), c1 = __ldcg(rq + 1);
            eq = (c0.y == w[0]) & (c1.x == w[1]) & (c1.y == w[2]);
            if (!shortk)
                for (int64_t j = kGbsInline; j < words && eq; ++j)
                    eq = gbs_key_word(t, r, m, j, true) == gbs_word(W, b + 8 * j, n - 8 * j);
        }
        if (eq) return static_cast<int64_t>(pos);
    }
    atomicExch(reinterpret_cast<int*>(&t.counters[1]), static_cast<int>(QDB_HASH_TABLE_FULL));
    return -1;
}

// Dictionary pass: ids[i] = the slot of row i's key (0 for rows the mask drops, NULL keys and failed rows).  Bounded
// to six blocks per SM (40 registers): the pass is latency-bound, and 48 resident warps beat 40 with fewer spills.
// `boff` is the offset of the characters' first byte within the aligned word view W.
__global__ void __launch_bounds__(kGbsThreads, 6) gbs_map_kernel(GbsDict t, const uint64_t* __restrict__ W, int64_t boff,
                                                              const int64_t* __restrict__ ends,
                                                              const uint64_t* __restrict__ knull,
                                                              const int8_t* __restrict__ mask, int64_t n,
                                                              int32_t* __restrict__ ids) {
    __shared__ unsigned s_claims;
    if (threadIdx.x == 0) s_claims = 0;
    __syncthreads();
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        int64_t slot = 0;
        const bool skip = (mask && mask[i] == 0) || (knull && ((knull[i >> 6] >> (i & 63)) & 1ull));
        if (!skip) {
            const int64_t b = i ? ends[i - 1] : 0;
            slot = gbs_find(t, W, boff + b, ends[i] - b, &s_claims);
            if (slot < 0) slot = 0;
        }
        ids[i] = static_cast<int32_t>(slot);
    }
    __syncthreads();
    if (threadIdx.x == 0 && s_claims) {
        if (atomicAdd(&t.counters[2], static_cast<unsigned long long>(s_claims)) + s_claims > t.capacity)
            atomicExch(reinterpret_cast<int*>(&t.counters[1]), static_cast<int>(QDB_HASH_TABLE_FULL));
    }
}

// Key lengths of the result groups: clen[r] = length of group r's key (0 for the NULL key).
__global__ void gbs_len_kernel(GbsDict t, const int32_t* __restrict__ slots, const uint64_t* __restrict__ knull,
                               int64_t g, long long* __restrict__ clen) {
    for (int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; r < g;
         r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const bool isnull = knull && ((knull[r >> 6] >> (r & 63)) & 1ull);
        clen[r] = isnull ? 0 : static_cast<long long>(gbs_meta_len(t.rec[slots[r]].meta));
    }
}

// Result keys: group r's characters at cpos[r], its end offset cpos[r] + length.
__global__ void gbs_emit_kernel(GbsDict t, const int32_t* __restrict__ slots, const uint64_t* __restrict__ knull,
                                int64_t g, const long long* __restrict__ cpos, char* __restrict__ out_chars,
                                int64_t* __restrict__ out_ends) {
    for (int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; r < g;
         r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const bool isnull = knull && ((knull[r >> 6] >> (r & 63)) & 1ull);
        const long long c0 = cpos[r];
        long long n = 0;
        if (!isnull) {
            const GbsRec* rc = t.rec + slots[r];
            const uint64_t m = rc->meta;
            n = gbs_meta_len(m);
            for (long long j = 0; j < n; j += 8) {
                const uint64_t w = (j >> 3) < kGbsInline ? rc->w[j >> 3] : t.arena[gbs_meta_off(m) + (j >> 3) - kGbsInline];
                for (long long c = j; c < n && c < j + 8; ++c)
                    out_chars[c0 + c] = static_cast<char>((w >> (8 * (c - j))) & 0xffu);
            }
        }
        out_ends[r] = c0 + n;
    }
}

// The keys of `groups` slots (knull bit set: the NULL key, an empty string) as a newly allocated GPUString.
static int32_t gbs_build_keys(const GbsDict& t, const int32_t* slots, const uint64_t* knull, int64_t groups,
                              char** out_chars, int64_t** out_ends, cudaStream_t s);

// Export records: slot numbers from the numeric table's key words, and the NULL-key flag as a bitmask.
__global__ void gbs_export_prep_kernel(const uint64_t* __restrict__ keys, const uint8_t* __restrict__ flags, int64_t n,
                                       int32_t* __restrict__ slots, unsigned long long* __restrict__ knull) {
    for (int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; r < n;
         r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const bool isnull = (flags[r] & 1u) != 0;  // bit 0 of the export flags: the NULL-key slot
        slots[r] = isnull ? 0 : static_cast<int32_t>(keys[r]);
        if (isnull) atomicOr(knull + (r >> 6), 1ull << (r & 63));
    }
}

// Merge of exported records: rows whose record is the NULL key are left out of the dictionary pass (mask 0); the
// slot numbers the pass returns become the numeric table's key words.
__global__ void gbs_merge_prep_kernel(const uint8_t* __restrict__ flags, int64_t n, int8_t* __restrict__ mask) {
    for (int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; r < n;
         r += static_cast<int64_t>(gridDim.x) * blockDim.x)
        mask[r] = (flags[r] & 1u) ? 0 : 1;
}

__global__ void gbs_keywords_kernel(const int32_t* __restrict__ ids, int64_t n, uint64_t* __restrict__ keys) {
    for (int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; r < n;
         r += static_cast<int64_t>(gridDim.x) * blockDim.x)
        keys[r] = static_cast<uint64_t>(static_cast<int64_t>(ids[r]));  // the int32 key word
}

static uint64_t gbs_pow2(uint64_t x) {
    uint64_t p = 16;
    while (p < x) p <<= 1;
    return p;
}

static unsigned gbs_grid(uint64_t n) {
    const DeviceInfo& di = device_info();
    return static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, uint64_t(di.sm_count) * 8)));
}

static int32_t gbs_build_keys(const GbsDict& t, const int32_t* slots, const uint64_t* knull, int64_t groups,
                              char** out_chars, int64_t** out_ends, cudaStream_t s) {
    *out_chars = nullptr;
    *out_ends = nullptr;
    long long *clen = nullptr, *tot = nullptr;
    int32_t rc = dev_alloc(reinterpret_cast<void**>(&clen), static_cast<size_t>(groups) * 8, s);
    if (rc == QDB_OK) rc = dev_alloc(reinterpret_cast<void**>(&tot), 8, s);
    long long nchars = 0;
    if (rc == QDB_OK) {
        gbs_len_kernel<<<gbs_grid(static_cast<uint64_t>(groups)), 256, 0, s>>>(t, slots, knull, groups, clen);
        note_launch();
        rc = exclusive_scan<long long>(clen, groups, tot, s);
        cudaError_t e = rc == QDB_OK ? cudaMemcpyAsync(&nchars, tot, 8, cudaMemcpyDeviceToHost, s) : cudaSuccess;
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (rc == QDB_OK && e != cudaSuccess) rc = cuda_fail(e, "string keys: lengths");
    }
    if (rc == QDB_OK)
        rc = dev_alloc(reinterpret_cast<void**>(out_chars), static_cast<size_t>(std::max<long long>(nchars, 1)), s);
    if (rc == QDB_OK) rc = dev_alloc(reinterpret_cast<void**>(out_ends), static_cast<size_t>(groups) * 8, s);
    if (rc == QDB_OK) {
        gbs_emit_kernel<<<gbs_grid(static_cast<uint64_t>(groups)), 256, 0, s>>>(t, slots, knull, groups, clen,
                                                                                *out_chars, *out_ends);
        note_launch();
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) rc = cuda_fail(e, "gbs_emit_kernel");
    }
    dev_free(clen, s);
    dev_free(tot, s);
    if (rc != QDB_OK) {
        dev_free(*out_chars, s);
        dev_free(*out_ends, s);
        *out_chars = nullptr;
        *out_ends = nullptr;
    }
    return rc;
}

}  // namespace qdb

struct qdb_gbs {
    int32_t aggs = 0;
    int32_t val_type = 0;
    int64_t max_groups = 0;
    qdb::GbsDict t;
    qdb_gb* num = nullptr;  // the numeric GROUP BY table over slot numbers
};

using namespace qdb;

extern "C" {

int32_t qdb_gbs_create(qdb_gbs** out, int32_t agg_mask, int32_t val_type, int64_t max_groups, int64_t max_key_bytes,
                       void* stream) {
    if (!out) return fail(QDB_ERR_INVALID, "qdb_gbs_create: null out");
    *out = nullptr;
    if (agg_mask & ~(QDB_AGG_MIN | QDB_AGG_MAX | QDB_AGG_SUM | QDB_AGG_AVG | QDB_AGG_COUNT))
        return fail(QDB_UNKNOWN_AGG_FUN, "qdb_gbs_create: unknown aggregate bits");
    const bool vt_ok = val_type == QDB_INT32 || val_type == QDB_INT64 || val_type == QDB_FLOAT || val_type == QDB_DOUBLE;
    if ((val_type != 0 && !vt_ok) || ((agg_mask & ~QDB_AGG_COUNT) && !vt_ok))
        return fail(QDB_ERR_INVALID, "qdb_gbs_create: value type must be INT32, INT64, FLOAT or DOUBLE (0: COUNT of rows)");
    if (max_groups < 1) return fail(QDB_ERR_INVALID, "qdb_gbs_create: max_groups must be positive");
    max_groups = std::min<int64_t>(max_groups, int64_t(1) << 30);
    qdb_gbs* g = new qdb_gbs();
    g->aggs = agg_mask;
    g->val_type = val_type;
    g->max_groups = max_groups;
    GbsDict& t = g->t;
    t.cap = gbs_pow2(static_cast<uint64_t>(max_groups) + static_cast<uint64_t>(max_groups) / 2);
    t.capacity = static_cast<unsigned long long>(max_groups);
    const uint64_t bytes = max_key_bytes > 0 ? static_cast<uint64_t>(max_key_bytes) : static_cast<uint64_t>(max_groups) * 32;
    t.arena_words = (bytes + 7) / 8;
    cudaStream_t s = as_stream(stream);
    int32_t rc = dev_alloc(reinterpret_cast<void**>(&t.header), t.cap * 8, s);
    if (rc == QDB_OK) rc = dev_alloc(reinterpret_cast<void**>(&t.rec), t.cap * sizeof(GbsRec), s);
    if (rc == QDB_OK) rc = dev_alloc(reinterpret_cast<void**>(&t.arena), std::max<uint64_t>(t.arena_words, 1) * 8, s);
    if (rc == QDB_OK) rc = dev_alloc(reinterpret_cast<void**>(&t.counters), 32, s);
    if (rc == QDB_OK) rc = qdb_gb_create(&g->num, agg_mask, QDB_INT32, 1, val_type, max_groups, QDB_PLACE_AUTO, stream);
    if (rc == QDB_OK) rc = qdb_gbs_reset(g, stream);
    if (rc != QDB_OK) {
        qdb_gbs_destroy(g);
        return rc;
    }
    *out = g;
    return QDB_OK;
}

int32_t qdb_gbs_destroy(qdb_gbs* g) {
    if (!g) return QDB_OK;
    GbsDict& t = g->t;
    for (void* p : {static_cast<void*>(t.header), static_cast<void*>(t.rec), static_cast<void*>(t.arena),
                    static_cast<void*>(t.counters)})
        if (p) dev_free(p, nullptr);
    if (g->num) qdb_gb_destroy(g->num);
    cudaStreamSynchronize(nullptr);
    delete g;
    return QDB_OK;
}

int32_t qdb_gbs_reset(qdb_gbs* g, void* stream) {
    if (!g) return fail(QDB_ERR_INVALID, "qdb_gbs_reset: null table");
    cudaStream_t s = as_stream(stream);
    const GbsDict& t = g->t;
    QDB_CUDA_TRY(cudaMemsetAsync(t.header, 0, t.cap * 8, s));
    QDB_CUDA_TRY(cudaMemsetAsync(t.rec, 0, t.cap * sizeof(GbsRec), s));
    QDB_CUDA_TRY(cudaMemsetAsync(t.counters, 0, 32, s));
    return qdb_gb_reset(g->num, stream);
}

int32_t qdb_gbs_process(qdb_gbs* g, const char* chars, const int64_t* ends, const uint64_t* key_nulls, const void* vals,
                        const uint64_t* val_nulls, const int8_t* mask, int64_t n, void* stream) {
    if (!g || n < 0) return fail(QDB_ERR_INVALID, "qdb_gbs_process: bad arguments");
    if (n == 0) return QDB_OK;
    // Without a value column a COUNT-only table counts rows (COUNT of the key column).
    if (!ends || (g->val_type && !vals && g->aggs != QDB_AGG_COUNT))
        return fail(QDB_ERR_INVALID, "qdb_gbs_process: null keys or values");
    cudaStream_t s = as_stream(stream);
    // Slot numbers, one per row; a COUNT-only call without values also lends this buffer as its (unread) value column.
    const size_t row_bytes = std::max<size_t>(4, static_cast<size_t>(type_size(g->val_type)));
    int32_t* ids = nullptr;
    int32_t rc = dev_alloc(reinterpret_cast<void**>(&ids), static_cast<size_t>(n) * row_bytes, s);
    if (rc != QDB_OK) return rc;
    const uintptr_t base = reinterpret_cast<uintptr_t>(chars);
    const uint64_t* W = reinterpret_cast<const uint64_t*>(base & ~uintptr_t(7));
    static int per_sm = 0;  // one wave: the blocks resident on every SM at once
    if (per_sm == 0) {
        int b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, gbs_map_kernel, kGbsThreads, 0) != cudaSuccess || b < 1) b = 4;
        per_sm = b;
    }
    const unsigned grid = static_cast<unsigned>(std::max<int64_t>(
        1, std::min<int64_t>((n + kGbsThreads - 1) / kGbsThreads, int64_t(device_info().sm_count) * per_sm)));
    gbs_map_kernel<<<grid, kGbsThreads, 0, s>>>(g->t, W, static_cast<int64_t>(base & 7), ends, key_nulls, mask, n, ids);
    note_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        dev_free(ids, s);
        return cuda_fail(e, "gbs_map_kernel");
    }
    const void* kc[1] = {ids};
    const uint64_t* kn[1] = {key_nulls};
    const void* v = vals ? vals : (g->val_type ? static_cast<const void*>(ids) : nullptr);
    rc = qdb_gb_process(g->num, kc, key_nulls ? kn : nullptr, v, vals ? val_nulls : nullptr, n, nullptr, mask, stream);
    dev_free(ids, s);  // stream-ordered: after the aggregation pass has read it
    return rc;
}

int32_t qdb_gbs_check(qdb_gbs* g, void* stream) {
    if (!g) return fail(QDB_ERR_INVALID, "qdb_gbs_check: null table");
    unsigned long long st = 0;
    QDB_CUDA_TRY(cudaMemcpyAsync(&st, g->t.counters + 1, 8, cudaMemcpyDeviceToHost, as_stream(stream)));
    QDB_CUDA_TRY(cudaStreamSynchronize(as_stream(stream)));
    const int32_t status = static_cast<int32_t>(st & 0xffffffffu);
    if (status != QDB_OK) {
        QDB_CUDA_TRY(cudaMemsetAsync(g->t.counters + 1, 0, 8, as_stream(stream)));
        qdb_gb_check(g->num, stream);  // clear the aggregation pass's status too
        const char* why = status == QDB_HASH_TABLE_FULL ? "string GROUP BY: more distinct keys than the table (or its "
                                                          "key arena) holds"
                          : status == QDB_ERR_TOO_LARGE ? "string GROUP BY: a key is longer than 2^20 - 2 bytes"
                                                        : "string GROUP BY: a wait for a key gave up";
        return fail(status, why);
    }
    return qdb_gb_check(g->num, stream);
}

int32_t qdb_gbs_results(qdb_gbs* g, int32_t n_aggs, const int32_t* aggs, char** out_chars, int64_t** out_ends,
                        uint64_t** out_key_nulls, void** out_vals, uint64_t** out_val_nulls, int64_t* out_count,
                        void* stream) {
    if (!g || !out_chars || !out_ends || !out_count || n_aggs < 0 || n_aggs > 5 || (n_aggs && (!aggs || !out_vals)))
        return fail(QDB_ERR_INVALID, "qdb_gbs_results: bad arguments");
    *out_chars = nullptr;
    *out_ends = nullptr;
    *out_count = 0;
    if (out_key_nulls) *out_key_nulls = nullptr;
    cudaStream_t s = as_stream(stream);
    void* slots = nullptr;
    uint64_t* knull = nullptr;
    int64_t groups = 0;
    int32_t rc = qdb_gb_results_multi(g->num, n_aggs, aggs, &slots, &knull, out_vals, out_val_nulls, &groups, stream);
    if (rc != QDB_OK) return rc;
    if (groups == 0) {
        dev_free(slots, s);
        dev_free(knull, s);
        return QDB_OK;
    }
    rc = gbs_build_keys(g->t, static_cast<const int32_t*>(slots), knull, groups, out_chars, out_ends, s);
    dev_free(slots, s);
    if (rc != QDB_OK) {
        dev_free(knull, s);
        for (int j = 0; j < n_aggs; ++j) {
            dev_free(out_vals[j], s);
            out_vals[j] = nullptr;
            if (out_val_nulls) {
                dev_free(out_val_nulls[j], s);
                out_val_nulls[j] = nullptr;
            }
        }
        return rc;
    }
    *out_count = groups;
    if (out_key_nulls) *out_key_nulls = knull;
    else dev_free(knull, s);
    return QDB_OK;
}

int32_t qdb_gbs_export(qdb_gbs* g, char** out_chars, int64_t** out_ends, uint64_t** out_state, uint8_t** out_flags,
                       int64_t* out_count, void* stream) {
    if (!g || !out_chars || !out_ends || !out_state || !out_flags || !out_count)
        return fail(QDB_ERR_INVALID, "qdb_gbs_export: null argument");
    *out_chars = nullptr;
    *out_ends = nullptr;
    *out_count = 0;
    cudaStream_t s = as_stream(stream);
    uint64_t* keys = nullptr;
    int64_t n = 0;
    int32_t rc = qdb_gb_export_partitioned(g->num, 1, &keys, out_state, out_flags, &n, stream);
    if (rc != QDB_OK) return rc;
    int32_t* slots = nullptr;
    unsigned long long* knull = nullptr;
    const size_t words = static_cast<size_t>((n + 63) / 64);
    if (n > 0) {
        rc = dev_alloc(reinterpret_cast<void**>(&slots), static_cast<size_t>(n) * 4, s);
        if (rc == QDB_OK) rc = dev_alloc(reinterpret_cast<void**>(&knull), words * 8, s);
        if (rc == QDB_OK) {
            cudaError_t e = cudaMemsetAsync(knull, 0, words * 8, s);
            if (e == cudaSuccess) {
                gbs_export_prep_kernel<<<gbs_grid(static_cast<uint64_t>(n)), 256, 0, s>>>(keys, *out_flags, n, slots, knull);
                note_launch();
                e = cudaGetLastError();
            }
            if (e != cudaSuccess) rc = cuda_fail(e, "gbs_export_prep_kernel");
        }
        if (rc == QDB_OK) rc = gbs_build_keys(g->t, slots, reinterpret_cast<const uint64_t*>(knull), n, out_chars, out_ends, s);
    }
    dev_free(keys, s);
    dev_free(slots, s);
    dev_free(knull, s);
    if (rc != QDB_OK) {
        dev_free(*out_state, s);
        dev_free(*out_flags, s);
        *out_state = nullptr;
        *out_flags = nullptr;
        return rc;
    }
    *out_count = n;
    return QDB_OK;
}

int32_t qdb_gbs_state_words(qdb_gbs* g, int32_t* out_words) {
    if (!g || !out_words) return fail(QDB_ERR_INVALID, "qdb_gbs_state_words: null argument");
    return qdb_gb_state_words(g->num, out_words);
}

int32_t qdb_gbs_merge_exported(qdb_gbs* g, const char* chars, const int64_t* ends, const uint64_t* state,
                               const uint8_t* flags, int64_t n, void* stream) {
    if (!g || n < 0 || (n > 0 && (!ends || !flags))) return fail(QDB_ERR_INVALID, "qdb_gbs_merge_exported: bad arguments");
    if (n == 0) return QDB_OK;
    cudaStream_t s = as_stream(stream);
    int8_t* mask = nullptr;
    int32_t* ids = nullptr;
    uint64_t* keys = nullptr;
    int32_t rc = dev_alloc(reinterpret_cast<void**>(&mask), static_cast<size_t>(n), s);
    if (rc == QDB_OK) rc = dev_alloc(reinterpret_cast<void**>(&ids), static_cast<size_t>(n) * 4, s);
    if (rc == QDB_OK) rc = dev_alloc(reinterpret_cast<void**>(&keys), static_cast<size_t>(n) * 8, s);
    if (rc == QDB_OK) {
        const unsigned grid = gbs_grid(static_cast<uint64_t>(n));
        gbs_merge_prep_kernel<<<grid, 256, 0, s>>>(flags, n, mask);
        const uintptr_t base = reinterpret_cast<uintptr_t>(chars);
        gbs_map_kernel<<<grid, kGbsThreads, 0, s>>>(g->t, reinterpret_cast<const uint64_t*>(base & ~uintptr_t(7)),
                                                    static_cast<int64_t>(base & 7), ends, nullptr, mask, n, ids);
        gbs_keywords_kernel<<<grid, 256, 0, s>>>(ids, n, keys);
        note_launch(3);
        const cudaError_t e = cudaGetLastError();
        rc = e == cudaSuccess ? qdb_gb_merge_partial(g->num, keys, state, flags, n, stream) : cuda_fail(e, "string merge");
    }
    dev_free(mask, s);
    dev_free(ids, s);
    dev_free(keys, s);
    return rc;
}

}  // extern "C"
