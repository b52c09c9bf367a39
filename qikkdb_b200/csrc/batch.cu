// Host side of the batched GROUP BY: validation, table and result arenas, the per-query execution plan
// (placement, warp-group width, rows per thread, work items), the measured autotuner, CUDA-graph capture
// and the C ABI.  The kernels are in batch_kernels.cu.
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "batch.cuh"

namespace qdb {

__global__ void gb_batch_init_kernel(const BatchArgs ba);
__global__ void gb_batch_agg_kernel(const BatchArgs ba);
__global__ void gb_batch_results_kernel(const BatchArgs ba);

// A plan family the autotuner chooses between, independent of one query's sizes.
struct BKind {
    int32_t place = QDB_PLACE_SHARED;  // QDB_PLACE_SHARED or QDB_PLACE_GLOBAL
    int32_t rep = 0;                   // shared tables per group: 0 -> 1, 1 -> 4, 2 -> one per consumer warp
    int32_t warps = kBCons;            // consumer warps per group: kBCons, kBCons / 2 or kBCons / 4
    int32_t rpt = 2;                   // rows each consumer thread takes from a stage tile (1..kBMaxRowsPerLane)
};

static uint64_t next_pow2_u(uint64_t x) {
    uint64_t p = 1;
    while (p < x) p <<= 1;
    return p;
}

static int ceil_log2(uint64_t x) {
    int l = 0;
    while ((uint64_t(1) << l) < x && l < 62) ++l;
    return l;
}

static int queue_of(int warps) { return warps == kBCons ? 0 : (warps == kBCons / 2 ? 1 : 2); }

// Process-wide tuning table: query class -> best plan family.
static std::mutex g_tune_mu;
static std::map<uint64_t, BKind> g_tune;

static uint64_t class_key(const qdb_gb_query& q) {
    const uint64_t vk = static_cast<uint64_t>(val_kind(q.val_type));
    const uint64_t kt = q.key_type == QDB_INT64 ? 1 : 0;
    const uint64_t pr = q.pred.col ? 1 : 0;
    const uint64_t card = static_cast<uint64_t>(std::min<int64_t>(q.max_groups, q.n_rows > 0 ? q.n_rows : 1));
    const uint64_t cb = static_cast<uint64_t>(ceil_log2(std::max<uint64_t>(card, 1)));
    const uint64_t rb = static_cast<uint64_t>(ceil_log2(static_cast<uint64_t>(std::max<int64_t>(q.n_rows, 1))) / 2);
    return vk | (kt << 3) | (pr << 4) | (cb << 5) | (rb << 11);
}

// Hashed slots of a query's global table: load factor at most 0.4, so that most probe sequences end at their first
// slot (every further probe is a dependent L2 round trip).
static uint64_t batch_table_cap(int64_t max_groups) {
    return next_pow2_u(std::max<uint64_t>(16, static_cast<uint64_t>(max_groups) * 5 / 2 + 1));
}

static bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Bytes of one shared-memory slot for a query (key, count, sum, min/max).
static size_t smem_slot_bytes(const qdb_gb_query& q) {
    const ValKind vk = val_kind(q.val_type);
    const bool has_vals = vk != VK_NONE;
    const bool has_sum = has_vals && (q.agg_mask & (QDB_AGG_SUM | QDB_AGG_AVG));
    const bool has_mm = has_vals && (q.agg_mask & (QDB_AGG_MIN | QDB_AGG_MAX));
    return 8 + 4 + (has_sum ? 8 : 0) + (has_mm ? (vk_is_32(vk) ? 8 : 16) : 0);
}

}  // namespace qdb

struct qdb_gb_batch {
    int device = 0;
    int32_t max_inst = 0;
    int64_t table_bytes = 0;
    int64_t result_bytes = 0;
    int64_t max_items = 0;
    size_t dyn_bytes = 0;
    int grid = 0;
    // device
    qdb::BHeader* d_hdr = nullptr;
    qdb::BInst* d_inst = nullptr;
    qdb::BItem* d_items = nullptr;
    qdb::BGroup* d_groups = nullptr;
    uint64_t* d_tables = nullptr;
    uint64_t* d_res = nullptr;
    unsigned long long* d_counters = nullptr;
    int64_t* d_res_count = nullptr;
    int32_t* d_status = nullptr;
    long long* d_item_ns = nullptr;
    // pinned host staging
    qdb::BHeader* h_hdr = nullptr;
    qdb::BInst* h_inst = nullptr;
    qdb::BItem* h_items = nullptr;
    qdb::BGroup* h_groups = nullptr;
    cudaEvent_t upload_done = nullptr;
    bool upload_recorded = false;
    // plan
    std::vector<qdb_gb_query> q;
    std::vector<qdb_gb_batch_cfg> cfg;
    std::vector<qdb::BItem> items;
    std::vector<int32_t> inst_group;   // scan group of every query
    int32_t n_groups = 0;
    bool share = true;                 // queries over the same columns share one scan
    int32_t n = 0;
    bool dirty = false;
    bool needs_init = false;
    int64_t total_rows = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
};

namespace qdb {

static void drop_graph(qdb_gb_batch* b) {
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->gexec = nullptr;
    b->graph = nullptr;
}

static BatchArgs batch_args(const qdb_gb_batch* b) {
    BatchArgs a;
    a.hdr = b->d_hdr;
    a.inst = b->d_inst;
    a.items = b->d_items;
    a.groups = b->d_groups;
    a.res = b->d_res;
    a.res_count = b->d_res_count;
    a.status = b->d_status;
    a.item_ns = b->d_item_ns;
    a.dyn_bytes = static_cast<int64_t>(b->dyn_bytes);
    return a;
}

// Shared-memory bytes available for the tables of one warp group at a given width.
static size_t table_space(const qdb_gb_batch* b, int warps) {
    const int q = queue_of(warps);
    const size_t gbytes = (b->dyn_bytes >> q) & ~static_cast<size_t>(127);
    return gbytes - kBHeaderBytes - b_ring_bytes(q);
}

static size_t align128(size_t x) { return (x + 127) & ~static_cast<size_t>(127); }

// The plan of query i for a plan family: falls back to the global table when the shared tables do not fit.
static qdb_gb_batch_cfg apply_kind(const qdb_gb_batch* b, const qdb_gb_query& q, const BKind& k) {
    qdb_gb_batch_cfg c{};
    c.warps = k.warps;
    c.rows_per_thread = k.rpt;
    c.placement = QDB_PLACE_GLOBAL;
    c.smem_slots = 0;
    c.replicas = 1;
    const int64_t card = std::min<int64_t>(q.max_groups, std::max<int64_t>(q.n_rows, 1));
    if (k.place == QDB_PLACE_SHARED) {
        const size_t bps = smem_slot_bytes(q);
        const size_t gb = table_space(b, k.warps);
        // load factor at most 0.625: short linear-probe runs, and as many queries as possible in shared memory
        const int S = static_cast<int>(std::min<int64_t>((std::max<int64_t>(64, (card * 8 + 4) / 5) + 31) / 32 * 32,
                                                         int64_t(1) << 20));
        int R = (k.rep == 0) ? 1 : (k.rep == 1 ? std::min(4, k.warps) : k.warps);
        while (R > 1 && align128(static_cast<size_t>(R) * S * bps) > gb) --R;
        if (align128(static_cast<size_t>(S) * bps) <= gb && S <= (1 << 20)) {
            c.placement = QDB_PLACE_SHARED;
            c.smem_slots = S;
            c.replicas = R;
        }
    }
    // Work items: big queries are cut so that every SM gets several items; an item of a shared placement is
    // long enough to amortise clearing and merging its tables.
    const int64_t per_sm = std::max<int64_t>(b->total_rows / (static_cast<int64_t>(b->grid) * 8), 1);
    int64_t chunk = std::min<int64_t>(std::max<int64_t>(per_sm * k.warps / kBCons, 32768), int64_t(8) << 20);
    if (c.placement == QDB_PLACE_SHARED)
        chunk = std::max<int64_t>(chunk, int64_t(16) * c.replicas * c.smem_slots);
    chunk = (chunk + 63) / 64 * 64;
    c.chunk_rows = chunk;
    return c;
}

static BKind heuristic_kind(const qdb_gb_query& q) {
    BKind k;
    const int64_t card = std::min<int64_t>(q.max_groups, std::max<int64_t>(q.n_rows, 1));
    k.place = QDB_PLACE_SHARED;
    k.rep = card <= 64 ? 2 : (card <= 512 ? 1 : 0);
    k.warps = q.n_rows < 32768 ? kBCons / 4 : (q.n_rows < 262144 ? kBCons / 2 : kBCons);
    k.rpt = card <= 4096 ? 1 : 2;
    return k;
}

static BKind tuned_kind(const qdb_gb_query& q) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune.find(class_key(q));
    return it == g_tune.end() ? heuristic_kind(q) : it->second;
}

// Result words of one query: max_groups + 2 rows of the key and every aggregate column.
static int64_t result_words(const qdb_gb_query& q) {
    const int64_t rows = q.max_groups + 2;
    return rows * (1 + __builtin_popcount(static_cast<unsigned>(q.agg_mask)));
}

// Rows of one stage tile of a group: as many as fit one ring stage (a multiple of 128 rows, so every column's
// tile is a whole number of 16-byte units and the rows spread evenly over the group's lanes).
static int stage_rows(int warps, int kt, int vb, int pb) {
    const int q = queue_of(warps);
    auto bytes = [&](int t) { return align128(size_t(t) * kt) + align128(size_t(t) * vb) + align128(size_t(t) * pb); };
    // every consumer warp compacts at most kBListRows rows of a tile (its share rounded up to 32 rows)
    const int max_rows = (kBListRows - 32) * warps;
    int T = 128;
    while (T + 128 <= max_rows && bytes(T + 128) <= static_cast<size_t>(b_stage_bytes(q))) T += 128;
    return T;
}

// Bytes of one query's shared tables.
static size_t query_table_bytes(const qdb_gb_query& q, const qdb_gb_batch_cfg& c) {
    if (c.placement != QDB_PLACE_SHARED) return 0;
    return align128(static_cast<size_t>(c.replicas) * c.smem_slots * smem_slot_bytes(q));
}

// Forms the scan groups (queries over the same columns, with the same warp-group width and tile, whose shared
// tables fit one group together), cuts every group into work items and stages the descriptors for upload.
static int32_t build_items(qdb_gb_batch* b) {
    struct Key {
        const void* k;
        const void* v;
        const void* p;
        int64_t n;
        int32_t kt, vt, pt, warps, rpt;
        bool operator<(const Key& o) const {
            return std::tie(k, v, p, n, kt, vt, pt, warps, rpt) < std::tie(o.k, o.v, o.p, o.n, o.kt, o.vt, o.pt, o.warps, o.rpt);
        }
    };
    std::vector<std::vector<int>> members;
    std::vector<size_t> used;
    std::map<Key, std::vector<int>> open;  // key -> indices of groups that may take more members
    b->inst_group.assign(b->n, -1);
    for (int i = 0; i < b->n; ++i) {
        const qdb_gb_query& q = b->q[i];
        const qdb_gb_batch_cfg& c = b->cfg[i];
        const size_t tb = query_table_bytes(q, c);
        const Key key{q.keys, q.val_type ? q.vals : nullptr, q.pred.col, q.n_rows, q.key_type, q.val_type,
                      q.pred.col ? q.pred.type : 0, c.warps, c.rows_per_thread};
        int gi = -1;
        if (b->share && q.n_rows > 0) {
            for (int cand : open[key])
                if (members[cand].size() < static_cast<size_t>(kBMaxMembers) && used[cand] + tb <= table_space(b, c.warps)) {
                    gi = cand;
                    break;
                }
        }
        if (gi < 0) {
            gi = static_cast<int>(members.size());
            members.emplace_back();
            used.push_back(0);
            open[key].push_back(gi);
        }
        b->h_inst[i].so_table = static_cast<int32_t>(used[gi]);
        used[gi] += tb;
        members[gi].push_back(i);
        b->inst_group[i] = gi;
    }
    b->n_groups = static_cast<int32_t>(members.size());
    std::vector<BItem> its[kBQueues];
    for (int gi = 0; gi < b->n_groups; ++gi) {
        const int i0 = members[gi][0];
        const qdb_gb_query& q = b->q[i0];
        const qdb_gb_batch_cfg& c = b->cfg[i0];
        BGroup& G = b->h_groups[gi];
        memset(&G, 0, sizeof(G));
        G.keys = q.keys;
        G.vals = q.val_type ? q.vals : nullptr;
        G.pcol = q.pred.col;
        G.n = q.n_rows;
        G.kt = type_size(q.key_type);
        G.vbytes = q.val_type ? type_size(q.val_type) : 0;
        G.pbytes = q.pred.col ? type_size(q.pred.type) : 0;
        G.vk = val_kind(q.val_type);
        G.n_members = static_cast<int32_t>(members[gi].size());
        for (int k = 0; k < G.n_members; ++k) G.members[k] = members[gi][k];
        G.stage_rows = stage_rows(c.warps, G.kt, G.vbytes, G.pbytes);
        G.rpt = c.rows_per_thread;
        // a shared scan does the work of every member per row: shorter items keep the queue balanced
        int64_t chunk = c.chunk_rows;
        for (int m : members[gi]) chunk = std::min<int64_t>(chunk, b->cfg[m].chunk_rows);
        chunk = std::max<int64_t>(4096, (chunk / G.n_members + 63) / 64 * 64);
        const int qi = queue_of(c.warps);
        for (int64_t r = 0; r < q.n_rows; r += chunk) {
            BItem it{};
            it.group = gi;
            it.queue = qi;
            it.r0 = r;
            it.r1 = std::min<int64_t>(q.n_rows, r + chunk);
            its[qi].push_back(it);
        }
    }
    b->items.clear();
    for (int qi = 0; qi < kBQueues; ++qi) {
        // Longest items first, so the queue's tail is made of short items.
        auto work = [&](const BItem& x) { return (x.r1 - x.r0) * b->h_groups[x.group].n_members; };
        std::stable_sort(its[qi].begin(), its[qi].end(), [&](const BItem& x, const BItem& y) { return work(x) > work(y); });
        b->h_hdr->q_begin[qi] = static_cast<int32_t>(b->items.size());
        b->items.insert(b->items.end(), its[qi].begin(), its[qi].end());
    }
    b->h_hdr->q_begin[kBQueues] = static_cast<int32_t>(b->items.size());
    if (static_cast<int64_t>(b->items.size()) > b->max_items) {
        // Grow the item buffers (the captured graph holds the old pointers).
        const int64_t want = static_cast<int64_t>(b->items.size()) * 2;
        if (b->upload_recorded) cudaEventSynchronize(b->upload_done);
        cudaDeviceSynchronize();
        cudaFree(b->d_items);
        cudaFree(b->d_item_ns);
        cudaFreeHost(b->h_items);
        b->d_items = nullptr;
        b->d_item_ns = nullptr;
        b->h_items = nullptr;
        QDB_CUDA_TRY(cudaMalloc(&b->d_items, want * sizeof(BItem)));
        QDB_CUDA_TRY(cudaMalloc(&b->d_item_ns, want * sizeof(long long)));
        QDB_CUDA_TRY(cudaMallocHost(&b->h_items, want * sizeof(BItem)));
        b->max_items = want;
        drop_graph(b);
    }
    for (size_t k = 0; k < b->items.size(); ++k) b->h_items[k] = b->items[k];
    for (int i = 0; i < b->n; ++i) {
        const qdb_gb_batch_cfg& c = b->cfg[i];
        BInst& I = b->h_inst[i];
        I.S = c.placement == QDB_PLACE_SHARED ? c.smem_slots : 0;
        I.R = c.placement == QDB_PLACE_SHARED ? c.replicas : 1;
        I.probe = std::min(I.S, 32);
    }
    b->h_hdr->n_inst = b->n;
    for (int qi = 0; qi < kBQueues; ++qi) b->h_hdr->heads[qi] = 0;
    b->dirty = true;
    return QDB_OK;
}

static int32_t upload(qdb_gb_batch* b, cudaStream_t s) {
    b->h_hdr->init_needed = b->needs_init ? 1 : 0;
    QDB_CUDA_TRY(cudaMemcpyAsync(b->d_hdr, b->h_hdr, sizeof(BHeader), cudaMemcpyHostToDevice, s));
    if (b->n > 0)
        QDB_CUDA_TRY(cudaMemcpyAsync(b->d_inst, b->h_inst, b->n * sizeof(BInst), cudaMemcpyHostToDevice, s));
    if (b->n_groups > 0)
        QDB_CUDA_TRY(cudaMemcpyAsync(b->d_groups, b->h_groups, b->n_groups * sizeof(BGroup), cudaMemcpyHostToDevice, s));
    if (!b->items.empty())
        QDB_CUDA_TRY(cudaMemcpyAsync(b->d_items, b->h_items, b->items.size() * sizeof(BItem),
                                     cudaMemcpyHostToDevice, s));
    QDB_CUDA_TRY(cudaEventRecord(b->upload_done, s));
    b->upload_recorded = true;
    b->dirty = false;
    return QDB_OK;
}

// The host staging buffers may still be read by an upload in flight.
static int32_t wait_staging(qdb_gb_batch* b) {
    if (b->upload_recorded) QDB_CUDA_TRY(cudaEventSynchronize(b->upload_done));
    return QDB_OK;
}

static int32_t launch_all(qdb_gb_batch* b, cudaStream_t s) {
    const BatchArgs a = batch_args(b);
    gb_batch_init_kernel<<<static_cast<unsigned>(b->max_inst), 1024, 0, s>>>(a);
    gb_batch_agg_kernel<<<static_cast<unsigned>(b->grid), kBThreads, b->dyn_bytes, s>>>(a);
    gb_batch_results_kernel<<<static_cast<unsigned>(b->max_inst), kBResThreads, 0, s>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "batch kernels launch");
    return QDB_OK;
}

static int32_t check_query(const qdb_gb_query& q) {
    if (q.key_type != QDB_INT32 && q.key_type != QDB_INT64)
        return fail(QDB_ERR_INVALID, "batch query: key_type must be INT32 or INT64");
    if (q.agg_mask & ~(QDB_AGG_MIN | QDB_AGG_MAX | QDB_AGG_SUM | QDB_AGG_AVG | QDB_AGG_COUNT))
        return fail(QDB_UNKNOWN_AGG_FUN, "batch query: unknown aggregate bits");
    if (q.val_type != 0 && val_kind(q.val_type) == VK_NONE)
        return fail(QDB_ERR_INVALID, "batch query: unsupported value type");
    if (q.val_type == 0 && (q.agg_mask & ~QDB_AGG_COUNT))
        return fail(QDB_ERR_INVALID, "batch query: MIN/MAX/SUM/AVG need a value column");
    if (q.n_rows < 0) return fail(QDB_ERR_INVALID, "batch query: negative row count");
    if (q.max_groups < 1) return fail(QDB_ERR_INVALID, "batch query: max_groups must be >= 1");
    if (q.key_mod < 0) return fail(QDB_ERR_INVALID, "batch query: negative key_mod");
    if (q.n_rows > 0) {
        if (!q.keys || !aligned16(q.keys)) return fail(QDB_ERR_INVALID, "batch query: keys missing or not 16-byte aligned");
        if (q.val_type && (!q.vals || !aligned16(q.vals)))
            return fail(QDB_ERR_INVALID, "batch query: values missing or not 16-byte aligned");
        if (q.pred.col && !aligned16(q.pred.col))
            return fail(QDB_ERR_INVALID, "batch query: predicate column not 16-byte aligned");
    }
    if (q.pred.col) {
        const qdb_pred& p = q.pred;
        if (p.nulls) return fail(QDB_ERR_INVALID, "batch query: predicate null masks are not supported");
        if (p.op < QDB_GREATER || p.op > QDB_NOT_EQUAL)
            return fail(QDB_ERR_INVALID, "batch query: predicate op must be a comparison");
        if (p.type != QDB_INT32 && p.type != QDB_INT64 && p.type != QDB_FLOAT && p.type != QDB_DOUBLE)
            return fail(QDB_ERR_INVALID, "batch query: unsupported predicate column type");
        if (p.const_type != QDB_INT32 && p.const_type != QDB_INT64 && p.const_type != QDB_FLOAT &&
            p.const_type != QDB_DOUBLE)
            return fail(QDB_ERR_INVALID, "batch query: unsupported predicate constant type");
    }
    return QDB_OK;
}

static int32_t check_cfg(const qdb_gb_batch* b, const qdb_gb_query& q, const qdb_gb_batch_cfg& c) {
    if (c.warps != kBCons && c.warps != kBCons / 2 && c.warps != kBCons / 4)
        return fail(QDB_ERR_INVALID, "batch cfg: warps must be 12, 6 or 3");
    if (c.rows_per_thread != 1 && c.rows_per_thread != 2 && c.rows_per_thread != 4)
        return fail(QDB_ERR_INVALID, "batch cfg: rows_per_thread must be 1, 2 or 4");
    if (c.chunk_rows < 64 || c.chunk_rows % 64) return fail(QDB_ERR_INVALID, "batch cfg: chunk_rows must be a positive multiple of 64");
    // an item's shared float sums are 64-bit fixed-point words with addends below 2^39
    if (c.chunk_rows > (int64_t(1) << 24)) return fail(QDB_ERR_INVALID, "batch cfg: chunk_rows must be at most 2^24");
    if (c.placement == QDB_PLACE_SHARED) {
        const int S = c.smem_slots;
        if (S < 64 || (S % 32)) return fail(QDB_ERR_INVALID, "batch cfg: smem_slots must be a multiple of 32, >= 64");
        if (c.replicas < 1 || c.replicas > c.warps) return fail(QDB_ERR_INVALID, "batch cfg: replicas must be in [1, warps]");
        if (query_table_bytes(q, c) > table_space(b, c.warps))
            return fail(QDB_ERR_TOO_LARGE, "batch cfg: shared-memory tables do not fit the warp group");
    } else if (c.placement != QDB_PLACE_GLOBAL) {
        return fail(QDB_ERR_INVALID, "batch cfg: placement must be SHARED or GLOBAL");
    }
    return QDB_OK;
}

// Predicate bound bit pattern -> ordinal used by the kernel.
static int64_t pred_ord_host(int32_t type, int64_t bits) {
    if (type == QDB_FLOAT) {
        const int32_t b = static_cast<int32_t>(bits);
        return static_cast<int64_t>(b ^ ((b >> 31) & 0x7fffffff));
    }
    if (type == QDB_DOUBLE) return bits ^ ((bits >> 63) & 0x7fffffffffffffffll);
    if (type == QDB_INT32) return static_cast<int64_t>(static_cast<int32_t>(bits));
    return bits;
}

static int32_t run_once(qdb_gb_batch* b, bool use_graph, cudaStream_t s) {
    if (b->dirty) {
        int32_t rc = upload(b, s);
        if (rc != QDB_OK) return rc;
    }
    if (use_graph && s != nullptr) {
        if (!b->gexec) {
            QDB_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            const BatchArgs a = batch_args(b);
            gb_batch_init_kernel<<<static_cast<unsigned>(b->max_inst), 1024, 0, s>>>(a);
            gb_batch_agg_kernel<<<static_cast<unsigned>(b->grid), kBThreads, b->dyn_bytes, s>>>(a);
            gb_batch_results_kernel<<<static_cast<unsigned>(b->max_inst), kBResThreads, 0, s>>>(a);
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(s, &g);
            if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture(batch)");
            b->graph = g;
            e = cudaGraphInstantiate(&b->gexec, g, 0);
            if (e != cudaSuccess) {
                drop_graph(b);
                return cuda_fail(e, "cudaGraphInstantiate(batch)");
            }
        }
        QDB_CUDA_TRY(cudaGraphLaunch(b->gexec, s));
    } else {
        int32_t rc = launch_all(b, s);
        if (rc != QDB_OK) return rc;
    }
    note_launch(3);
    b->needs_init = false;
    return QDB_OK;
}

int32_t batch_check_query(const qdb_gb_query& q) { return check_query(q); }

// Readback of a run for callers inside the library (the serving loop): enqueues, without synchronising, the
// copies of every query's group count and status and of the whole result region to host buffers.
int32_t batch_enqueue_readback(qdb_gb_batch* b, int64_t* h_counts, int32_t* h_status, void* h_res, int64_t h_res_bytes,
                               cudaStream_t s) {
    if (b->n == 0) return QDB_OK;
    const int64_t bytes = (b->h_inst[b->n - 1].res_off + result_words(b->q[b->n - 1])) * 8;
    if (bytes > h_res_bytes) return fail(QDB_ERR_TOO_LARGE, "batch readback: host result buffer too small");
    QDB_CUDA_TRY(cudaMemcpyAsync(h_counts, b->d_res_count, b->n * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    QDB_CUDA_TRY(cudaMemcpyAsync(h_status, b->d_status, b->n * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    QDB_CUDA_TRY(cudaMemcpyAsync(h_res, b->d_res, bytes, cudaMemcpyDeviceToHost, s));
    return QDB_OK;
}

// Where query i's results sit in the result region: first word, rows reserved per column, aggregate columns.
void batch_result_place(const qdb_gb_batch* b, int i, int64_t* off_words, int64_t* cap_rows, int32_t* n_cols) {
    *off_words = b->h_inst[i].res_off;
    *cap_rows = b->h_inst[i].res_cap;
    *n_cols = __builtin_popcount(static_cast<unsigned>(b->h_inst[i].aggs));
}

}  // namespace qdb

using namespace qdb;

extern "C" {

int32_t qdb_gb_batch_create(qdb_gb_batch** out, int32_t max_instances, int64_t table_bytes, int64_t result_bytes,
                            void* stream) {
    if (!out) return fail(QDB_ERR_INVALID, "qdb_gb_batch_create: null out");
    *out = nullptr;
    if (max_instances < 1 || max_instances > (1 << 20) || table_bytes < 0 || result_bytes < 0)
        return fail(QDB_ERR_INVALID, "qdb_gb_batch_create: bad sizes");
    (void)stream;
    qdb_gb_batch* b = new qdb_gb_batch();
    cudaGetDevice(&b->device);
    const DeviceInfo& di = device_info();
    b->max_inst = max_instances;
    b->table_bytes = table_bytes;
    b->result_bytes = result_bytes;
    b->max_items = static_cast<int64_t>(max_instances) * 4 + 1024;
    b->grid = di.sm_count;
    int32_t rc = QDB_OK;
    auto try_cuda = [&](cudaError_t e, const char* what) {
        if (rc == QDB_OK && e != cudaSuccess) rc = cuda_fail(e, what);
    };
    cudaFuncAttributes fa;
    try_cuda(cudaFuncGetAttributes(&fa, gb_batch_agg_kernel), "cudaFuncGetAttributes(gb_batch_agg_kernel)");
    if (rc == QDB_OK) {
        const size_t cap = std::min<size_t>(static_cast<size_t>(di.max_smem_optin), kBSmemCap);
        b->dyn_bytes = (cap - fa.sharedSizeBytes - 256) & ~static_cast<size_t>(1023);
        try_cuda(cudaFuncSetAttribute(gb_batch_agg_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(b->dyn_bytes)),
                 "cudaFuncSetAttribute(gb_batch_agg_kernel)");
    }
    try_cuda(cudaMalloc(&b->d_hdr, sizeof(BHeader)), "cudaMalloc(batch header)");
    try_cuda(cudaMalloc(&b->d_inst, max_instances * sizeof(BInst)), "cudaMalloc(batch descriptors)");
    try_cuda(cudaMalloc(&b->d_items, b->max_items * sizeof(BItem)), "cudaMalloc(batch items)");
    try_cuda(cudaMalloc(&b->d_groups, max_instances * sizeof(BGroup)), "cudaMalloc(batch scan groups)");
    try_cuda(cudaMallocHost(&b->h_groups, max_instances * sizeof(BGroup)), "cudaMallocHost(batch scan groups)");
    try_cuda(cudaMalloc(&b->d_item_ns, b->max_items * sizeof(long long)), "cudaMalloc(batch item times)");
    if (table_bytes > 0) try_cuda(cudaMalloc(&b->d_tables, table_bytes), "cudaMalloc(batch tables)");
    if (result_bytes > 0) try_cuda(cudaMalloc(&b->d_res, result_bytes), "cudaMalloc(batch results)");
    try_cuda(cudaMalloc(&b->d_counters, 2 * max_instances * sizeof(unsigned long long)), "cudaMalloc(batch counters)");
    try_cuda(cudaMalloc(&b->d_res_count, max_instances * sizeof(int64_t)), "cudaMalloc(batch counts)");
    try_cuda(cudaMalloc(&b->d_status, max_instances * sizeof(int32_t)), "cudaMalloc(batch status)");
    try_cuda(cudaMallocHost(&b->h_hdr, sizeof(BHeader)), "cudaMallocHost(batch header)");
    try_cuda(cudaMallocHost(&b->h_inst, max_instances * sizeof(BInst)), "cudaMallocHost(batch descriptors)");
    try_cuda(cudaMallocHost(&b->h_items, b->max_items * sizeof(BItem)), "cudaMallocHost(batch items)");
    try_cuda(cudaEventCreateWithFlags(&b->upload_done, cudaEventDisableTiming), "cudaEventCreate(batch)");
    if (rc == QDB_OK) {
        memset(b->h_hdr, 0, sizeof(BHeader));
        try_cuda(cudaMemset(b->d_hdr, 0, sizeof(BHeader)), "cudaMemset(batch header)");
        try_cuda(cudaMemset(b->d_counters, 0, 2 * max_instances * sizeof(unsigned long long)),
                 "cudaMemset(batch counters)");
        try_cuda(cudaMemset(b->d_res_count, 0, max_instances * sizeof(int64_t)), "cudaMemset(batch counts)");
        try_cuda(cudaMemset(b->d_status, 0, max_instances * sizeof(int32_t)), "cudaMemset(batch status)");
        try_cuda(cudaDeviceSynchronize(), "cudaDeviceSynchronize(batch create)");
    }
    if (rc != QDB_OK) {
        qdb_gb_batch_destroy(b);
        return rc;
    }
    *out = b;
    return QDB_OK;
}

int32_t qdb_gb_batch_destroy(qdb_gb_batch* b) {
    if (!b) return QDB_OK;
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != b->device) cudaSetDevice(b->device);
    cudaDeviceSynchronize();
    drop_graph(b);
    cudaFree(b->d_hdr);
    cudaFree(b->d_inst);
    cudaFree(b->d_items);
    cudaFree(b->d_item_ns);
    cudaFree(b->d_groups);
    cudaFree(b->d_tables);
    cudaFree(b->d_res);
    cudaFree(b->d_counters);
    cudaFree(b->d_res_count);
    cudaFree(b->d_status);
    if (b->h_hdr) cudaFreeHost(b->h_hdr);
    if (b->h_inst) cudaFreeHost(b->h_inst);
    if (b->h_items) cudaFreeHost(b->h_items);
    if (b->h_groups) cudaFreeHost(b->h_groups);
    if (b->upload_done) cudaEventDestroy(b->upload_done);
    if (prev != b->device) cudaSetDevice(prev);
    delete b;
    return QDB_OK;
}

int32_t qdb_gb_batch_set(qdb_gb_batch* b, const qdb_gb_query* queries, int32_t n, void* stream) {
    if (!b) return fail(QDB_ERR_INVALID, "qdb_gb_batch_set: null batch");
    if (n < 0 || n > b->max_inst || (n > 0 && !queries)) return fail(QDB_ERR_INVALID, "qdb_gb_batch_set: bad query count");
    std::vector<qdb_gb_query> qs(queries, queries + n);
    int64_t table_off = 0, res_off = 0, total_rows = 0;
    std::vector<int64_t> toff(n), roff(n);
    for (int i = 0; i < n; ++i) {
        int32_t rc = check_query(qs[i]);
        if (rc != QDB_OK) return rc;
        if (qs[i].max_groups > (int64_t(1) << 30)) qs[i].max_groups = int64_t(1) << 30;
        const uint64_t cap = batch_table_cap(qs[i].max_groups);
        const Layout L = make_layout(qs[i].agg_mask, val_kind(qs[i].val_type));
        toff[i] = table_off;
        table_off += static_cast<int64_t>((cap + 2) * L.W * 8 + 255) / 256 * 256;
        roff[i] = res_off;
        res_off += result_words(qs[i]) * 8;
        total_rows += qs[i].n_rows;
    }
    if (table_off > b->table_bytes) return fail(QDB_ERR_TOO_LARGE, "qdb_gb_batch_set: tables exceed the batch's table_bytes");
    if (res_off > b->result_bytes) return fail(QDB_ERR_TOO_LARGE, "qdb_gb_batch_set: results exceed the batch's result_bytes");
    int32_t rc = wait_staging(b);
    if (rc != QDB_OK) return rc;
    b->q = qs;
    b->n = n;
    b->total_rows = total_rows;
    b->cfg.assign(n, qdb_gb_batch_cfg{});
    for (int i = 0; i < n; ++i) {
        const qdb_gb_query& q = qs[i];
        b->cfg[i] = apply_kind(b, q, tuned_kind(q));
        BInst& I = b->h_inst[i];
        memset(&I, 0, sizeof(I));
        const ValKind vk = val_kind(q.val_type);
        const uint64_t cap = batch_table_cap(q.max_groups);
        I.counters = b->d_counters + 2 * i;
        I.main.slots = reinterpret_cast<uint64_t*>(reinterpret_cast<unsigned char*>(b->d_tables) + toff[i]);
        I.main.mask = cap - 1;
        I.n = q.n_rows;
        I.key_mod = q.key_mod;
        if (q.key_mod > 0) {
            const ModMagic mm = mod_magic(static_cast<uint64_t>(q.key_mod));
            I.mod_m = mm.m;
            I.mod_s1 = mm.s1;
            I.mod_s2 = mm.s2;
        }
        I.capacity = q.max_groups;
        I.res_off = roff[i] / 8;
        I.res_cap = q.max_groups + 2;
        I.L = make_layout(q.agg_mask, vk);
        I.kt = q.key_type == QDB_INT64 ? 8 : 4;
        I.vk = vk;
        I.aggs = q.agg_mask;
        I.has_sum = I.L.sum >= 0;
        I.has_min = (q.agg_mask & QDB_AGG_MIN) && I.L.mn >= 0;
        I.has_max = (q.agg_mask & QDB_AGG_MAX) && I.L.mx >= 0;
        if (q.pred.col) {
            const PredInterval pi = pred_interval(q.pred);
            I.pbytes = type_size(q.pred.type);
            I.pfloat = (q.pred.type == QDB_FLOAT || q.pred.type == QDB_DOUBLE) ? 1 : 0;
            I.pinv = pi.invert;
            I.plo = pred_ord_host(q.pred.type, pi.lo);
            I.phi = pred_ord_host(q.pred.type, pi.hi);
        }
    }
    b->needs_init = true;
    rc = build_items(b);
    if (rc != QDB_OK) return rc;
    return upload(b, as_stream(stream));
}

int32_t qdb_gb_batch_run(qdb_gb_batch* b, int32_t use_graph, void* stream) {
    if (!b) return fail(QDB_ERR_INVALID, "qdb_gb_batch_run: null batch");
    if (b->n == 0) return QDB_OK;
    return run_once(b, use_graph != 0, as_stream(stream));
}

int32_t qdb_gb_batch_fetch(qdb_gb_batch* b, int64_t* counts, int32_t* status, void* stream) {
    if (!b) return fail(QDB_ERR_INVALID, "qdb_gb_batch_fetch: null batch");
    cudaStream_t s = as_stream(stream);
    if (b->n > 0 && counts)
        QDB_CUDA_TRY(cudaMemcpyAsync(counts, b->d_res_count, b->n * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    if (b->n > 0 && status)
        QDB_CUDA_TRY(cudaMemcpyAsync(status, b->d_status, b->n * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    QDB_CUDA_TRY(cudaStreamSynchronize(s));
    return QDB_OK;
}

int32_t qdb_gb_batch_result(qdb_gb_batch* b, int32_t inst, const int64_t** keys, const void** cols, int32_t* n_cols,
                            int64_t* col_stride) {
    if (!b || inst < 0 || inst >= b->n) return fail(QDB_ERR_INVALID, "qdb_gb_batch_result: bad instance");
    const BInst& I = b->h_inst[inst];
    const uint64_t* base = b->d_res + I.res_off;
    if (keys) *keys = reinterpret_cast<const int64_t*>(base);
    if (cols) *cols = base + I.res_cap;
    if (n_cols) *n_cols = __builtin_popcount(static_cast<unsigned>(I.aggs));
    if (col_stride) *col_stride = I.res_cap;
    return QDB_OK;
}

int32_t qdb_gb_batch_copy_results(qdb_gb_batch* b, int32_t first, int32_t n, void* host, int64_t host_bytes,
                                  int64_t* needed, void* stream) {
    if (!b || first < 0 || n < 0 || first + n > b->n) return fail(QDB_ERR_INVALID, "qdb_gb_batch_copy_results: bad range");
    if (n == 0) {
        if (needed) *needed = 0;
        return QDB_OK;
    }
    const int64_t w0 = b->h_inst[first].res_off;
    const int64_t w1 = b->h_inst[first + n - 1].res_off + result_words(b->q[first + n - 1]);
    const int64_t bytes = (w1 - w0) * 8;
    if (needed) *needed = bytes;
    if (!host) return QDB_OK;
    if (host_bytes < bytes) return fail(QDB_ERR_TOO_LARGE, "qdb_gb_batch_copy_results: host buffer too small");
    cudaStream_t s = as_stream(stream);
    QDB_CUDA_TRY(cudaMemcpyAsync(host, b->d_res + w0, bytes, cudaMemcpyDeviceToHost, s));
    QDB_CUDA_TRY(cudaStreamSynchronize(s));
    return QDB_OK;
}

int32_t qdb_gb_batch_get_cfg(qdb_gb_batch* b, int32_t inst, qdb_gb_batch_cfg* cfg) {
    if (!b || !cfg || inst < 0 || inst >= b->n) return fail(QDB_ERR_INVALID, "qdb_gb_batch_get_cfg: bad instance");
    *cfg = b->cfg[inst];
    return QDB_OK;
}

int32_t qdb_gb_batch_set_cfg(qdb_gb_batch* b, int32_t inst, const qdb_gb_batch_cfg* cfg) {
    if (!b || !cfg || inst < 0 || inst >= b->n) return fail(QDB_ERR_INVALID, "qdb_gb_batch_set_cfg: bad instance");
    int32_t rc = check_cfg(b, b->q[inst], *cfg);
    if (rc != QDB_OK) return rc;
    rc = wait_staging(b);
    if (rc != QDB_OK) return rc;
    b->cfg[inst] = *cfg;
    return build_items(b);
}

int32_t qdb_gb_batch_item_times(qdb_gb_batch* b, int64_t* ns, void* stream) {
    if (!b || !ns) return fail(QDB_ERR_INVALID, "qdb_gb_batch_item_times: null argument");
    std::vector<long long> t(b->items.size());
    cudaStream_t s = as_stream(stream);
    if (!t.empty())
        QDB_CUDA_TRY(cudaMemcpyAsync(t.data(), b->d_item_ns, t.size() * sizeof(long long), cudaMemcpyDeviceToHost, s));
    QDB_CUDA_TRY(cudaStreamSynchronize(s));
    for (int i = 0; i < b->n; ++i) ns[i] = 0;
    for (size_t k = 0; k < t.size(); ++k) {
        const BGroup& G = b->h_groups[b->items[k].group];
        for (int m = 0; m < G.n_members; ++m) ns[G.members[m]] += t[k] / G.n_members;
    }
    return QDB_OK;
}

int32_t qdb_gb_batch_autotune(qdb_gb_batch* b, void* stream) {
    if (!b) return fail(QDB_ERR_INVALID, "qdb_gb_batch_autotune: null batch");
    if (b->n == 0) return QDB_OK;
    cudaStream_t s = as_stream(stream);
    const int n = b->n;
    std::vector<int64_t> ns(n);
    // Class of every query; costs are compared per class (SM-time summed over the class's queries), and every
    // query of a class runs the same plan family in every trial.
    std::vector<uint64_t> cls(n);
    std::map<uint64_t, int> first;
    for (int i = 0; i < n; ++i) {
        cls[i] = class_key(b->q[i]);
        first.emplace(cls[i], i);
    }
    std::vector<BKind> best(n);
    for (int i = 0; i < n; ++i) best[i] = tuned_kind(b->q[first[cls[i]]]);
    auto trial = [&](const std::vector<BKind>& kinds, std::vector<double>& cost) -> int32_t {
        int32_t rc = wait_staging(b);
        if (rc != QDB_OK) return rc;
        for (int i = 0; i < n; ++i) b->cfg[i] = apply_kind(b, b->q[i], kinds[i]);
        rc = build_items(b);
        if (rc == QDB_OK) rc = run_once(b, false, s);
        if (rc == QDB_OK) rc = qdb_gb_batch_item_times(b, ns.data(), stream);
        if (rc != QDB_OK) return rc;
        cost.assign(n, 0.0);
        for (int i = 0; i < n; ++i) cost[i] = static_cast<double>(ns[i]) * b->cfg[i].warps / kBCons;
        return QDB_OK;
    };
    // Coordinate search: placement and replication, then warp-group width, then rows per thread.
    for (int stage = 0; stage < 3; ++stage) {
        std::vector<std::vector<BKind>> cands;
        if (stage == 0) {
            const BKind variants[4] = {{QDB_PLACE_SHARED, 0, 0, 0}, {QDB_PLACE_SHARED, 1, 0, 0},
                                       {QDB_PLACE_SHARED, 2, 0, 0}, {QDB_PLACE_GLOBAL, 0, 0, 0}};
            for (const BKind& v : variants) {
                std::vector<BKind> ks(best);
                for (BKind& k : ks) {
                    k.place = v.place;
                    k.rep = v.rep;
                }
                cands.push_back(ks);
            }
        } else if (stage == 1) {
            for (int w : {kBCons, kBCons / 2, kBCons / 4}) {
                std::vector<BKind> ks(best);
                for (BKind& k : ks) k.warps = w;
                cands.push_back(ks);
            }
        } else {
            for (int rpt : {1, 2, 4}) {
                std::vector<BKind> ks(best);
                for (BKind& k : ks) k.rpt = rpt;
                cands.push_back(ks);
            }
        }
        std::map<uint64_t, std::vector<double>> class_cost;
        for (size_t c = 0; c < cands.size(); ++c) {
            std::vector<double> cost;
            int32_t rc = trial(cands[c], cost);
            if (rc != QDB_OK) return rc;
            for (int i = 0; i < n; ++i) {
                auto& v = class_cost[cls[i]];
                if (v.size() < cands.size()) v.assign(cands.size(), 0.0);
                v[c] += cost[i];
            }
        }
        for (int i = 0; i < n; ++i) {
            const auto& v = class_cost[cls[i]];
            const size_t arg = static_cast<size_t>(std::min_element(v.begin(), v.end()) - v.begin());
            best[i] = cands[arg][i];
        }
    }
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        for (int i = 0; i < n; ++i) g_tune[cls[i]] = best[i];
    }
    int32_t rc = wait_staging(b);
    if (rc != QDB_OK) return rc;
    for (int i = 0; i < n; ++i) b->cfg[i] = apply_kind(b, b->q[i], best[i]);
    rc = build_items(b);
    if (rc != QDB_OK) return rc;
    return upload(b, s);
}

int32_t qdb_gb_batch_required(const qdb_gb_query* queries, int32_t n, int64_t* table_bytes, int64_t* result_bytes) {
    if (n < 0 || (n > 0 && !queries)) return fail(QDB_ERR_INVALID, "qdb_gb_batch_required: bad query list");
    int64_t t = 0, r = 0;
    for (int i = 0; i < n; ++i) {
        qdb_gb_query q = queries[i];
        if (q.max_groups < 1) return fail(QDB_ERR_INVALID, "qdb_gb_batch_required: max_groups must be >= 1");
        if (q.max_groups > (int64_t(1) << 30)) q.max_groups = int64_t(1) << 30;
        const Layout L = make_layout(q.agg_mask, val_kind(q.val_type));
        t += static_cast<int64_t>((batch_table_cap(q.max_groups) + 2) * L.W * 8 + 255) / 256 * 256;
        r += result_words(q) * 8;
    }
    if (table_bytes) *table_bytes = t;
    if (result_bytes) *result_bytes = r;
    return QDB_OK;
}

int32_t qdb_gb_batch_set_sharing(qdb_gb_batch* b, int32_t share) {
    if (!b) return fail(QDB_ERR_INVALID, "qdb_gb_batch_set_sharing: null batch");
    int32_t rc = wait_staging(b);
    if (rc != QDB_OK) return rc;
    b->share = share != 0;
    return build_items(b);
}

int32_t qdb_gb_batch_tuning_reset(void) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune.clear();
    return QDB_OK;
}

int32_t qdb_gb_plain_run(const qdb_gb_query* queries, int32_t n, int32_t results_to_host, int64_t* out_groups,
                         void* stream) {
    if (n < 0 || (n > 0 && !queries)) return fail(QDB_ERR_INVALID, "qdb_gb_plain_run: bad arguments");
    static const int32_t kAggOrder[5] = {QDB_AGG_MIN, QDB_AGG_MAX, QDB_AGG_SUM, QDB_AGG_AVG, QDB_AGG_COUNT};
    std::vector<int64_t> host;
    for (int32_t i = 0; i < n; ++i) {
        const qdb_gb_query& q = queries[i];
        if (out_groups) out_groups[i] = 0;
        const int32_t ks = type_size(q.key_type);
        if (ks == 0 || q.n_rows < 0) return fail(QDB_ERR_INVALID, "qdb_gb_plain_run: bad query");
        // GROUP BY key % m: the dispatcher materialises the modulo column first (GPUBinary<mod>).
        const void* key = q.keys;
        void* modcol = nullptr;
        int32_t rc = QDB_OK;
        if (q.key_mod > 0 && q.n_rows > 0) {
            rc = qdb_malloc(&modcol, q.n_rows * ks, stream);
            if (rc == QDB_OK) rc = qdb_arith_mod(q.key_type, q.keys, q.key_mod, modcol, q.n_rows, stream);
            key = modcol;
        }
        qdb_gb* gb = nullptr;
        if (rc == QDB_OK)
            rc = qdb_gb_create(&gb, q.agg_mask, q.key_type, 1, q.val_type, q.max_groups, QDB_PLACE_AUTO, stream);
        if (rc == QDB_OK) {
            const void* kc[1] = {key};
            rc = qdb_gb_process_sync(gb, kc, nullptr, q.vals, nullptr, q.n_rows, q.pred.col ? &q.pred : nullptr,
                                     nullptr, stream);
        }
        int32_t aggs[5];
        int32_t na = 0;
        for (int32_t b : kAggOrder)
            if (q.agg_mask & b) aggs[na++] = b;
        void* okeys[1] = {nullptr};
        void* ovals[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
        int64_t g = 0;
        if (rc == QDB_OK) rc = qdb_gb_results_multi(gb, na, aggs, okeys, nullptr, ovals, nullptr, &g, stream);
        if (rc == QDB_OK && results_to_host && g > 0) {
            // keys, then every aggregate column (COUNT int64, the others of the value type) to host memory
            host.resize(static_cast<size_t>(g) * (1 + na));
            rc = qdb_memcpy_d2h(host.data(), okeys[0], g * ks, stream);
            for (int32_t j = 0; j < na && rc == QDB_OK; ++j) {
                const int64_t w = aggs[j] == QDB_AGG_COUNT ? 8 : type_size(q.val_type);
                rc = qdb_memcpy_d2h(host.data() + static_cast<size_t>(g) * (1 + j), ovals[j], g * w, stream);
            }
        }
        qdb_free(okeys[0], stream);
        for (void* v : ovals) qdb_free(v, stream);
        if (gb) qdb_gb_destroy(gb);
        qdb_free(modcol, stream);
        if (rc != QDB_OK) return rc;
        if (out_groups) out_groups[i] = g;
    }
    return qdb_stream_sync(stream);
}

}  // extern "C"
