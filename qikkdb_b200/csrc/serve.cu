// Serving loop: continuous batching of GROUP BY queries over device-resident columns on top of the batch engine
// (batch.cu).  No counterpart in the reference, whose server runs each query through a dispatcher one at a time
// per GPU.  Queries are submitted from any thread; one scheduler thread keeps up to `in_flight` batches on the GPU
// (one CUDA stream each, so a new batch's kernels start as the previous batch's last CTAs drain), admits pending
// queries in arrival order against the table and result budgets, reads back results, and resubmits queries whose
// table overflowed with twice the capacity.  Large queries (2^22 rows and up by default) skip the batch engine and
// take a slot alone through the single-query operators, whose fast pass hashes their rows faster.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "batch.cuh"

namespace qdb {


static int64_t now_ns() {
    return std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

// Queries of at least this many rows run alone through the single-query fast pass instead of a batch: the batch
// engine removes per-query launch and synchronisation costs, which such a query amortises, and its kernel hashes a
// row more slowly than the fast pass (shared table plus hash-partitioned spill).  A table-capacity threshold can
// route queries by their groups as well; it is off by default.
constexpr int64_t kServerPlainRows = int64_t(1) << 22;
constexpr int64_t kServerPlainGroups = 0;

struct Ticket {
    qdb_gb_query q{};
    int64_t submit_ns = 0, start_ns = 0, done_ns = 0;
    int32_t status = QDB_OK;
    int32_t retries = 0;
    int32_t batch_size = 0;
    int32_t n_cols = 0;
    int64_t n_groups = 0;
    std::vector<int64_t> data;  // keys, then every aggregate column
    bool done = false;
};

struct Slot {
    qdb_gb_batch* b = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t ev = nullptr;
    bool busy = false;
    std::vector<uint64_t> ids;
    int64_t* h_counts = nullptr;
    int32_t* h_status = nullptr;
    int64_t* h_res = nullptr;
    int64_t h_res_bytes = 0;
    // a query routed through the single-query operators (one per slot): its table and key % m column
    bool plain = false;
    qdb_gb* gb = nullptr;
};

// Sample of a key column (strided rows) kept per column for the cardinality estimates.
struct KeySample {
    std::vector<int64_t> keys;
    int64_t n = 0;
};

}  // namespace qdb

struct qdb_server {
    int device = 0;
    int32_t max_batch = 0;
    int32_t in_flight = 0;
    int64_t slot_table_bytes = 0;
    int64_t slot_result_bytes = 0;
    int64_t plain_rows = qdb::kServerPlainRows;
    int64_t plain_groups = qdb::kServerPlainGroups;
    std::mutex mu;
    std::condition_variable cv_work;
    std::condition_variable cv_done;
    std::unordered_map<uint64_t, qdb::Ticket*> tickets;
    std::deque<uint64_t> pending;
    uint64_t next_id = 1;
    std::vector<qdb::Slot> slots;
    std::map<std::pair<const void*, int64_t>, qdb::KeySample> samples;
    std::thread th;
    bool stop = false;
    qdb_server_stats stats{};
};

namespace qdb {

// GEE distinct-value estimate (Charikar, Chaudhuri, Motwani, Narasayya, PODS 2000) from a uniform sample of n of the
// column's N rows: sqrt(N / n) * f1 + sum_{j >= 2} f_j, where f_j counts the values seen exactly j times.
static int64_t gee_estimate(const std::vector<int64_t>& sample, int64_t N) {
    if (sample.empty()) return 1;
    std::unordered_map<int64_t, int32_t> freq;
    freq.reserve(sample.size() * 2);
    for (int64_t k : sample) ++freq[k];
    int64_t f1 = 0, rest = 0;
    for (const auto& kv : freq) (kv.second == 1 ? f1 : rest) += 1;
    const double est = std::sqrt(static_cast<double>(N) / static_cast<double>(sample.size())) * f1 + rest;
    return std::max<int64_t>(1, static_cast<int64_t>(std::ceil(est)));
}

// Table capacity of a query submitted with max_groups <= 0: the estimate of its keys' distinct count (after the
// key modulus), with 25% headroom, capped by the modulus and the row count.
static int64_t estimate_groups(qdb_server* sv, const qdb_gb_query& q) {
    constexpr int64_t kSample = 16384;
    const int64_t n = q.n_rows;
    if (n <= 0) return 1;
    KeySample* ks;
    {
        std::lock_guard<std::mutex> lock(sv->mu);
        ks = &sv->samples[{q.keys, n}];
    }
    if (ks->keys.empty()) {
        const int64_t m = std::min(n, kSample);
        const int kt = type_size(q.key_type);
        std::vector<unsigned char> raw(static_cast<size_t>(m) * kt);
        // strided sample: rows i * n / m (one small copy per row would be slow; copy a strided view instead)
        const int64_t stride = n / m;
        cudaMemcpy2D(raw.data(), kt, q.keys, static_cast<size_t>(stride) * kt, kt, static_cast<size_t>(m),
                     cudaMemcpyDeviceToHost);
        std::vector<int64_t> keys(m);
        for (int64_t i = 0; i < m; ++i) {
            if (kt == 4) {
                int32_t v;
                memcpy(&v, raw.data() + i * 4, 4);
                keys[i] = v;
            } else {
                memcpy(&keys[i], raw.data() + i * 8, 8);
            }
        }
        ks->n = n;
        ks->keys.swap(keys);
    }
    std::vector<int64_t> s(ks->keys);
    if (q.key_mod > 0)
        for (int64_t& k : s) k = k % q.key_mod;
    int64_t est = gee_estimate(s, n);
    est = est + est / 4 + 16;
    if (q.key_mod > 0) est = std::min(est, q.key_mod);
    return std::max<int64_t>(1, std::min(est, n));
}

static void finish_ticket(qdb_server* sv, Ticket* t, int32_t status) {
    t->status = status;
    t->done_ns = now_ns();
    t->done = true;
    sv->stats.completed += 1;
}

static void fail_slot_queries(qdb_server* sv, Slot& sl, int32_t status) {
    std::lock_guard<std::mutex> lock(sv->mu);
    for (uint64_t id : sl.ids) {
        auto it = sv->tickets.find(id);
        if (it != sv->tickets.end()) finish_ticket(sv, it->second, status);
    }
    sl.ids.clear();
    sl.busy = false;
    sv->cv_done.notify_all();
}

// Launches one batch on a free slot: plan, run (CUDA graph), results read back, completion event.
static void launch_slot(qdb_server* sv, Slot& sl, const std::vector<uint64_t>& ids) {
    std::vector<qdb_gb_query> qs;
    qs.reserve(ids.size());
    const int64_t t = now_ns();
    {
        std::lock_guard<std::mutex> lock(sv->mu);
        for (uint64_t id : ids) {
            Ticket* tk = sv->tickets[id];
            tk->start_ns = t;
            tk->batch_size = static_cast<int32_t>(ids.size());
            qs.push_back(tk->q);
        }
        sv->stats.batches += 1;
        sv->stats.queries_in_batches += static_cast<int64_t>(ids.size());
    }
    sl.ids = ids;
    sl.busy = true;
    int32_t rc = qdb_gb_batch_set(sl.b, qs.data(), static_cast<int32_t>(qs.size()), sl.s);
    if (rc == QDB_OK) rc = qdb_gb_batch_run(sl.b, 1, sl.s);
    if (rc == QDB_OK) rc = batch_enqueue_readback(sl.b, sl.h_counts, sl.h_status, sl.h_res, sl.h_res_bytes, sl.s);
    if (rc == QDB_OK && cudaEventRecord(sl.ev, sl.s) != cudaSuccess) rc = QDB_ERR_CUDA;
    if (rc != QDB_OK) fail_slot_queries(sv, sl, rc);
}

// A batch finished: copy every query's results out of the slot, or resubmit a query whose table overflowed.
static void complete_slot(qdb_server* sv, Slot& sl) {
    std::vector<uint64_t> retry;
    for (size_t k = 0; k < sl.ids.size(); ++k) {
        Ticket* t;
        {
            std::lock_guard<std::mutex> lock(sv->mu);
            t = sv->tickets[sl.ids[k]];
        }
        const int32_t st = sl.h_status[k];
        if (st == QDB_HASH_TABLE_FULL && t->retries < 16 && t->q.max_groups < (int64_t(1) << 30)) {
            t->q.max_groups = std::min<int64_t>(t->q.max_groups * 2, int64_t(1) << 30);
            t->retries += 1;
            retry.push_back(sl.ids[k]);
            continue;
        }
        int64_t off = 0, cap = 0;
        int32_t nc = 0;
        batch_result_place(sl.b, static_cast<int>(k), &off, &cap, &nc);
        const int64_t g = (st == QDB_OK) ? sl.h_counts[k] : 0;
        t->n_groups = g;
        t->n_cols = nc;
        t->data.resize(static_cast<size_t>(g) * (1 + nc));
        for (int c = 0; c <= nc; ++c)
            memcpy(t->data.data() + static_cast<size_t>(c) * g, sl.h_res + off + static_cast<int64_t>(c) * cap,
                   static_cast<size_t>(g) * 8);
        std::lock_guard<std::mutex> lock(sv->mu);
        finish_ticket(sv, t, st);
    }
    std::lock_guard<std::mutex> lock(sv->mu);
    for (auto it = retry.rbegin(); it != retry.rend(); ++it) sv->pending.push_front(*it);
    sv->stats.retries += static_cast<int64_t>(retry.size());
    sl.ids.clear();
    sl.busy = false;
    sv->cv_done.notify_all();
}

// The aggregate columns of a query in result order (MIN, MAX, SUM, AVG, COUNT).
static int32_t result_aggs(int32_t mask, int32_t* aggs) {
    static const int32_t kOrder[5] = {QDB_AGG_MIN, QDB_AGG_MAX, QDB_AGG_SUM, QDB_AGG_AVG, QDB_AGG_COUNT};
    int32_t na = 0;
    for (int32_t b : kOrder)
        if (mask & b) aggs[na++] = b;
    return na;
}

static void release_plain(Slot& sl) {
    if (sl.gb) qdb_gb_destroy(sl.gb);
    sl.gb = nullptr;
    sl.plain = false;
}

// Launches one query on a free slot through the single-query operators: a table of the query's capacity, ProcessBlock
// of key % m (the dispatcher's GPUBinary modulo column fused into the pass) with the fused WHERE, completion event.
static void launch_plain(qdb_server* sv, Slot& sl, uint64_t id) {
    Ticket* tk;
    {
        std::lock_guard<std::mutex> lock(sv->mu);
        tk = sv->tickets[id];
        tk->start_ns = now_ns();
        tk->batch_size = 1;
        sv->stats.plain_queries += 1;
    }
    sl.ids.assign(1, id);
    sl.busy = true;
    sl.plain = true;
    const qdb_gb_query& q = tk->q;
    int32_t rc = qdb_gb_create(&sl.gb, q.agg_mask, q.key_type, 1, q.val_type, q.max_groups, QDB_PLACE_AUTO, sl.s);
    if (rc == QDB_OK && q.n_rows > 0) {
        const void* vals = q.val_type ? q.vals : nullptr;
        const qdb_pred* pred = q.pred.col ? &q.pred : nullptr;
        if (q.key_mod > 0) {
            rc = qdb_gb_process_mod(sl.gb, q.keys, q.key_mod, vals, pred, q.n_rows, sl.s);
        } else {
            const void* kc[1] = {q.keys};
            rc = qdb_gb_process(sl.gb, kc, nullptr, vals, nullptr, q.n_rows, pred, nullptr, sl.s);
        }
    }
    if (rc == QDB_OK && cudaEventRecord(sl.ev, sl.s) != cudaSuccess) rc = QDB_ERR_CUDA;
    if (rc != QDB_OK) {
        cudaStreamSynchronize(sl.s);
        release_plain(sl);
        fail_slot_queries(sv, sl, rc);
    }
}

// Reads a plain query's results (GetResults) into the server's result layout: keys as int64, integer aggregates
// sign-extended to int64, float aggregates widened to double, COUNT as int64 -- the words the batch engine emits.
static int32_t read_plain_results(Slot& sl, Ticket* t) {
    const qdb_gb_query& q = t->q;
    int32_t aggs[5];
    const int32_t na = result_aggs(q.agg_mask, aggs);
    void* okeys[1] = {nullptr};
    void* ovals[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    int64_t g = 0;
    int32_t rc = qdb_gb_results_multi(sl.gb, na, aggs, okeys, nullptr, ovals, nullptr, &g, sl.s);
    const int ks = type_size(q.key_type);
    const int vs = q.val_type ? type_size(q.val_type) : 8;
    // raw columns to the slot's pinned buffer (g <= max_groups, so they fit the result budget the query was admitted
    // against: at most 8 bytes per word of max_groups + 2 rows)
    int64_t off[6] = {0, 0, 0, 0, 0, 0};
    int64_t need = static_cast<int64_t>(g) * ks;
    for (int32_t j = 0; j < na; ++j) {
        off[j + 1] = (need + 15) / 16 * 16;
        need = off[j + 1] + g * (aggs[j] == QDB_AGG_COUNT ? 8 : vs);
    }
    if (rc == QDB_OK && need > sl.h_res_bytes) rc = fail(QDB_ERR_TOO_LARGE, "server: plain results exceed the slot's buffer");
    unsigned char* h = reinterpret_cast<unsigned char*>(sl.h_res);
    if (rc == QDB_OK && g > 0) {
        if (cudaMemcpyAsync(h, okeys[0], static_cast<size_t>(g) * ks, cudaMemcpyDeviceToHost, sl.s) != cudaSuccess)
            rc = cuda_fail(cudaGetLastError(), "server: plain keys to host");
        for (int32_t j = 0; j < na && rc == QDB_OK; ++j) {
            const int w = aggs[j] == QDB_AGG_COUNT ? 8 : vs;
            if (cudaMemcpyAsync(h + off[j + 1], ovals[j], static_cast<size_t>(g) * w, cudaMemcpyDeviceToHost,
                                sl.s) != cudaSuccess)
                rc = cuda_fail(cudaGetLastError(), "server: plain results to host");
        }
        if (rc == QDB_OK && cudaStreamSynchronize(sl.s) != cudaSuccess)
            rc = cuda_fail(cudaGetLastError(), "server: plain results");
    }
    qdb_free(okeys[0], sl.s);
    for (void* v : ovals) qdb_free(v, sl.s);
    if (rc != QDB_OK) return rc;
    t->n_groups = g;
    t->n_cols = na;
    t->data.resize(static_cast<size_t>(g) * (1 + na));
    int64_t* d = t->data.data();
    for (int64_t i = 0; i < g; ++i) {
        if (ks == 4) {
            int32_t k;
            memcpy(&k, h + i * 4, 4);
            d[i] = k;
        } else {
            memcpy(&d[i], h + i * 8, 8);
        }
    }
    for (int32_t j = 0; j < na; ++j) {
        const unsigned char* src = h + off[j + 1];
        int64_t* dst = d + static_cast<size_t>(g) * (j + 1);
        if (aggs[j] == QDB_AGG_COUNT || q.val_type == QDB_INT64 || q.val_type == QDB_DOUBLE) {
            memcpy(dst, src, static_cast<size_t>(g) * 8);
        } else if (q.val_type == QDB_INT32) {
            for (int64_t i = 0; i < g; ++i) {
                int32_t v;
                memcpy(&v, src + i * 4, 4);
                dst[i] = v;
            }
        } else {  // QDB_FLOAT
            for (int64_t i = 0; i < g; ++i) {
                float f;
                memcpy(&f, src + i * 4, 4);
                const double x = static_cast<double>(f);
                memcpy(&dst[i], &x, 8);
            }
        }
    }
    return QDB_OK;
}

// A plain query finished: its results to the ticket, or a resubmission with twice the table after HASH_TABLE_FULL.
static void complete_plain(qdb_server* sv, Slot& sl) {
    Ticket* t;
    {
        std::lock_guard<std::mutex> lock(sv->mu);
        t = sv->tickets[sl.ids[0]];
    }
    int32_t st = qdb_gb_check(sl.gb, sl.s);
    bool retry = false;
    if (st == QDB_HASH_TABLE_FULL && t->retries < 16 && t->q.max_groups < (int64_t(1) << 30)) {
        t->q.max_groups = std::min<int64_t>(t->q.max_groups * 2, int64_t(1) << 30);
        t->retries += 1;
        retry = true;
    } else if (st == QDB_OK) {
        st = read_plain_results(sl, t);
    }
    release_plain(sl);
    std::lock_guard<std::mutex> lock(sv->mu);
    if (retry) {
        sv->pending.push_front(sl.ids[0]);
        sv->stats.retries += 1;
    } else {
        if (st != QDB_OK) {
            t->n_groups = 0;
            t->data.clear();
        }
        finish_ticket(sv, t, st);
    }
    sl.ids.clear();
    sl.busy = false;
    sv->cv_done.notify_all();
}

static void scheduler(qdb_server* sv) {
    cudaSetDevice(sv->device);
    for (;;) {
        bool progressed = false;
        // completions
        for (Slot& sl : sv->slots) {
            if (!sl.busy) continue;
            const cudaError_t e = cudaEventQuery(sl.ev);
            if (e == cudaSuccess) {
                if (sl.plain) complete_plain(sv, sl);
                else complete_slot(sv, sl);
                progressed = true;
            } else if (e != cudaErrorNotReady) {
                cudaGetLastError();
                if (sl.plain) release_plain(sl);
                fail_slot_queries(sv, sl, QDB_ERR_CUDA);
                progressed = true;
            }
        }
        // admissions
        for (Slot& sl : sv->slots) {
            if (sl.busy) continue;
            std::vector<uint64_t> ids;
            std::vector<uint64_t> need_estimate;
            {
                std::lock_guard<std::mutex> lock(sv->mu);
                for (uint64_t id : sv->pending)
                    if (sv->tickets[id]->q.max_groups <= 0) need_estimate.push_back(id);
            }
            for (uint64_t id : need_estimate) {
                Ticket* t;
                {
                    std::lock_guard<std::mutex> lock(sv->mu);
                    t = sv->tickets[id];
                }
                const int64_t est = estimate_groups(sv, t->q);
                std::lock_guard<std::mutex> lock(sv->mu);
                t->q.max_groups = est;
            }
            uint64_t plain_id = 0;
            {
                std::lock_guard<std::mutex> lock(sv->mu);
                int64_t tb = 0, rb = 0;
                // Pending queries in arrival order: the oldest, if it is for the single-query path, takes this slot
                // alone; otherwise the batch takes batch-path queries in order and passes over single-query ones,
                // which stay pending for the next free slot (so they do not cut the batch's shared scans short).
                auto it = sv->pending.begin();
                while (it != sv->pending.end() && static_cast<int32_t>(ids.size()) < sv->max_batch) {
                    const uint64_t id = *it;
                    Ticket* t = sv->tickets[id];
                    if (t->q.max_groups <= 0) break;  // arrived after this round's estimates: next round
                    int64_t qt = 0, qr = 0;
                    if (qdb_gb_batch_required(&t->q, 1, &qt, &qr) != QDB_OK || qt > sv->slot_table_bytes ||
                        qr > sv->slot_result_bytes) {
                        it = sv->pending.erase(it);
                        sv->stats.rejected += 1;
                        finish_ticket(sv, t, QDB_ERR_TOO_LARGE);
                        sv->cv_done.notify_all();
                        continue;
                    }
                    if ((sv->plain_rows > 0 && t->q.n_rows >= sv->plain_rows) ||
                        (sv->plain_groups > 0 && t->q.max_groups >= sv->plain_groups)) {
                        if (ids.empty() && it == sv->pending.begin()) {
                            plain_id = id;
                            sv->pending.pop_front();
                            break;
                        }
                        ++it;
                        continue;
                    }
                    if (tb + qt > sv->slot_table_bytes || rb + qr > sv->slot_result_bytes) break;
                    tb += qt;
                    rb += qr;
                    ids.push_back(id);
                    it = sv->pending.erase(it);
                }
            }
            if (plain_id != 0) {
                launch_plain(sv, sl, plain_id);
                progressed = true;
            } else if (!ids.empty()) {
                launch_slot(sv, sl, ids);
                progressed = true;
            }
        }
        std::unique_lock<std::mutex> lock(sv->mu);
        bool any_busy = false;
        for (const Slot& sl : sv->slots) any_busy = any_busy || sl.busy;
        if (sv->stop && sv->pending.empty() && !any_busy) return;
        if (!progressed) {
            if (any_busy) sv->cv_work.wait_for(lock, std::chrono::microseconds(20));
            else sv->cv_work.wait_for(lock, std::chrono::milliseconds(5),
                                      [&] { return sv->stop || !sv->pending.empty(); });
        }
    }
}

static uint64_t submit_at(qdb_server* sv, const qdb_gb_query& q, int64_t submit_ns) {
    Ticket* t = new Ticket();
    t->q = q;
    if (t->q.max_groups > (int64_t(1) << 30)) t->q.max_groups = int64_t(1) << 30;
    t->submit_ns = submit_ns;
    std::lock_guard<std::mutex> lock(sv->mu);
    const uint64_t id = sv->next_id++;
    sv->tickets[id] = t;
    sv->pending.push_back(id);
    sv->stats.submitted += 1;
    sv->cv_work.notify_one();
    return id;
}

}  // namespace qdb

using namespace qdb;

extern "C" {

int32_t qdb_server_create(qdb_server** out, int32_t max_batch, int32_t in_flight, int64_t table_budget_bytes,
                          int64_t result_budget_bytes) {
    if (!out) return fail(QDB_ERR_INVALID, "qdb_server_create: null out");
    *out = nullptr;
    if (max_batch < 1 || in_flight < 1 || in_flight > 8 || result_budget_bytes < in_flight)
        return fail(QDB_ERR_INVALID, "qdb_server_create: bad sizes");
    // The tables are carved out of the HBM that is free when the server starts (the reference sizes its device
    // allocators from cudaMemGetInfo, qikkDB/QueryEngine/Context.cu:58, CudaMemAllocator.cu:116): a reserve of an
    // eighth of the free memory (at least 2 GiB) stays for the spill area, result copies and other allocations, and
    // a table budget beyond what is left (or a budget <= 0, "all of it") is cut down to it.
    size_t free_b = 0, total_b = 0;
    QDB_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
    const int64_t reserve = std::max<int64_t>(int64_t(2) << 30, static_cast<int64_t>(free_b / 8));
    const int64_t avail = static_cast<int64_t>(free_b) - reserve - result_budget_bytes;
    if (avail < in_flight) return fail(QDB_ERR_NOMEM, "qdb_server_create: not enough free device memory");
    if (table_budget_bytes <= 0 || table_budget_bytes > avail) table_budget_bytes = avail;
    qdb_server* sv = new qdb_server();
    cudaGetDevice(&sv->device);
    sv->max_batch = max_batch;
    sv->in_flight = in_flight;
    sv->slot_table_bytes = table_budget_bytes / in_flight;
    sv->slot_result_bytes = result_budget_bytes / in_flight;
    sv->stats.table_budget_bytes = table_budget_bytes;
    sv->stats.hbm_free_at_create = static_cast<int64_t>(free_b);
    sv->slots.resize(in_flight);
    int32_t rc = QDB_OK;
    for (Slot& sl : sv->slots) {
        if (rc == QDB_OK) rc = qdb_gb_batch_create(&sl.b, max_batch, sv->slot_table_bytes, sv->slot_result_bytes, nullptr);
        if (rc == QDB_OK && cudaStreamCreateWithFlags(&sl.s, cudaStreamNonBlocking) != cudaSuccess)
            rc = cuda_fail(cudaGetLastError(), "cudaStreamCreate(server)");
        if (rc == QDB_OK && cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming) != cudaSuccess)
            rc = cuda_fail(cudaGetLastError(), "cudaEventCreate(server)");
        sl.h_res_bytes = sv->slot_result_bytes;
        if (rc == QDB_OK && cudaMallocHost(&sl.h_counts, max_batch * sizeof(int64_t)) != cudaSuccess)
            rc = cuda_fail(cudaGetLastError(), "cudaMallocHost(server counts)");
        if (rc == QDB_OK && cudaMallocHost(&sl.h_status, max_batch * sizeof(int32_t)) != cudaSuccess)
            rc = cuda_fail(cudaGetLastError(), "cudaMallocHost(server status)");
        if (rc == QDB_OK && cudaMallocHost(&sl.h_res, sl.h_res_bytes) != cudaSuccess)
            rc = cuda_fail(cudaGetLastError(), "cudaMallocHost(server results)");
    }
    if (rc != QDB_OK) {
        qdb_server_destroy(sv);
        return rc;
    }
    sv->th = std::thread(scheduler, sv);
    *out = sv;
    return QDB_OK;
}

int32_t qdb_server_destroy(qdb_server* sv) {
    if (!sv) return QDB_OK;
    if (sv->th.joinable()) {
        {
            std::lock_guard<std::mutex> lock(sv->mu);
            sv->stop = true;
            sv->cv_work.notify_all();
        }
        sv->th.join();
    }
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != sv->device) cudaSetDevice(sv->device);
    for (Slot& sl : sv->slots) {
        if (sl.s) cudaStreamSynchronize(sl.s);
        qdb_gb_batch_destroy(sl.b);
        if (sl.gb) qdb_gb_destroy(sl.gb);
        if (sl.ev) cudaEventDestroy(sl.ev);
        if (sl.s) cudaStreamDestroy(sl.s);
        if (sl.h_counts) cudaFreeHost(sl.h_counts);
        if (sl.h_status) cudaFreeHost(sl.h_status);
        if (sl.h_res) cudaFreeHost(sl.h_res);
    }
    for (auto& kv : sv->tickets) delete kv.second;
    if (prev != sv->device) cudaSetDevice(prev);
    delete sv;
    return QDB_OK;
}

int32_t qdb_server_submit(qdb_server* sv, const qdb_gb_query* q, uint64_t* ticket) {
    if (!sv || !q || !ticket) return fail(QDB_ERR_INVALID, "qdb_server_submit: null argument");
    qdb_gb_query c = *q;
    if (c.max_groups < 0) c.max_groups = 0;
    // validate now (a table size of 0 means "estimate it"), so that the caller gets the error
    qdb_gb_query v = c;
    if (v.max_groups == 0) v.max_groups = 1;
    const int32_t rc = batch_check_query(v);
    if (rc != QDB_OK) return rc;
    *ticket = submit_at(sv, c, now_ns());
    return QDB_OK;
}

int32_t qdb_server_wait(qdb_server* sv, uint64_t ticket, int64_t timeout_ms, qdb_server_result* out) {
    if (!sv || !out) return fail(QDB_ERR_INVALID, "qdb_server_wait: null argument");
    std::unique_lock<std::mutex> lock(sv->mu);
    auto it = sv->tickets.find(ticket);
    if (it == sv->tickets.end()) return fail(QDB_ERR_INVALID, "qdb_server_wait: unknown ticket");
    Ticket* t = it->second;
    if (timeout_ms < 0) {
        sv->cv_done.wait(lock, [&] { return t->done; });
    } else if (!sv->cv_done.wait_for(lock, std::chrono::milliseconds(timeout_ms), [&] { return t->done; })) {
        return fail(QDB_ERR_TIMEOUT, "qdb_server_wait: query not done yet");
    }
    out->status = t->status;
    out->n_cols = t->n_cols;
    out->n_groups = t->n_groups;
    out->keys = t->data.data();
    out->cols = t->data.data() + t->n_groups;
    out->submit_ns = t->submit_ns;
    out->start_ns = t->start_ns;
    out->done_ns = t->done_ns;
    out->retries = t->retries;
    out->batch_size = t->batch_size;
    out->max_groups = t->q.max_groups;
    return QDB_OK;
}

int32_t qdb_server_release(qdb_server* sv, uint64_t ticket) {
    if (!sv) return fail(QDB_ERR_INVALID, "qdb_server_release: null server");
    std::lock_guard<std::mutex> lock(sv->mu);
    auto it = sv->tickets.find(ticket);
    if (it == sv->tickets.end()) return fail(QDB_ERR_INVALID, "qdb_server_release: unknown ticket");
    if (!it->second->done) return fail(QDB_ERR_INVALID, "qdb_server_release: query still running");
    delete it->second;
    sv->tickets.erase(it);
    return QDB_OK;
}

int32_t qdb_server_set_plain_route(qdb_server* sv, int64_t min_rows, int64_t min_groups) {
    if (!sv) return fail(QDB_ERR_INVALID, "qdb_server_set_plain_route: null server");
    std::lock_guard<std::mutex> lock(sv->mu);
    sv->plain_rows = min_rows;
    sv->plain_groups = min_groups;
    return QDB_OK;
}

int32_t qdb_server_stats_get(qdb_server* sv, qdb_server_stats* out) {
    if (!sv || !out) return fail(QDB_ERR_INVALID, "qdb_server_stats_get: null argument");
    std::lock_guard<std::mutex> lock(sv->mu);
    *out = sv->stats;
    return QDB_OK;
}

int32_t qdb_server_run_open_loop(qdb_server* sv, const qdb_gb_query* queries, int32_t n, const int64_t* arrival_ns,
                                 int64_t* latency_ns, int32_t* status, int64_t* wall_ns) {
    if (!sv || n < 0 || (n > 0 && (!queries || !arrival_ns || !latency_ns || !status)))
        return fail(QDB_ERR_INVALID, "qdb_server_run_open_loop: bad arguments");
    for (int i = 1; i < n; ++i)
        if (arrival_ns[i] < arrival_ns[i - 1]) return fail(QDB_ERR_INVALID, "qdb_server_run_open_loop: arrivals must not decrease");
    std::vector<uint64_t> ids(n);
    const int64_t t0 = now_ns() + 1000000;  // 1 ms to settle
    for (int i = 0; i < n; ++i) {
        const int64_t target = t0 + arrival_ns[i];
        for (;;) {
            const int64_t d = target - now_ns();
            if (d <= 0) break;
            if (d > 300000) std::this_thread::sleep_for(std::chrono::nanoseconds(d - 200000));
        }
        qdb_gb_query c = queries[i];
        if (c.max_groups < 0) c.max_groups = 0;
        qdb_gb_query v = c;
        if (v.max_groups == 0) v.max_groups = 1;
        const int32_t rc = batch_check_query(v);
        if (rc != QDB_OK) return rc;
        ids[i] = submit_at(sv, c, target);
    }
    int64_t last = t0;
    for (int i = 0; i < n; ++i) {
        qdb_server_result r;
        int32_t rc = qdb_server_wait(sv, ids[i], -1, &r);
        if (rc != QDB_OK) return rc;
        latency_ns[i] = r.done_ns - (t0 + arrival_ns[i]);
        status[i] = r.status;
        last = std::max(last, r.done_ns);
        qdb_server_release(sv, ids[i]);
    }
    if (wall_ns) *wall_ns = n > 0 ? last - (t0 + arrival_ns[0]) : 0;
    return QDB_OK;
}

}  // extern "C"
