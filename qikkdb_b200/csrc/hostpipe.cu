// GROUP BY over host-resident columns: the H2D upload of each block overlapped with the aggregation of the
// previous one.  The reference uploads every block synchronously through its column cache before the
// operators run (qikkDB/GpuSqlParser/Dispatcher/GpuSqlDispatcherVMFunctions.h:185-260, GPUMemoryCache.h:100-141);
// here the columns are streamed in chunks through two device staging buffers: a copy stream fills buffer
// b while the caller's stream aggregates buffer 1-b, ordered by events.  Host buffers should be pinned
// (page-locked) for the copies to run asynchronously.
#include <vector>

#include "groupby.cuh"

namespace qdb {

struct HostPipe {
    cudaStream_t copy = nullptr;
    cudaEvent_t copied[2] = {nullptr, nullptr};
    cudaEvent_t consumed[2] = {nullptr, nullptr};
    void* stage[2] = {nullptr, nullptr};
    size_t stage_bytes = 0;
    int device = -1;
};

static HostPipe* pipe_for(qdb_gb* gb) {
    static thread_local std::vector<HostPipe> pipes;
    int dev = 0;
    cudaGetDevice(&dev);
    if (static_cast<int>(pipes.size()) <= dev) pipes.resize(dev + 1);
    HostPipe& p = pipes[dev];
    if (!p.copy) {
        if (cudaStreamCreateWithFlags(&p.copy, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
        for (int i = 0; i < 2; ++i) {
            cudaEventCreateWithFlags(&p.copied[i], cudaEventDisableTiming);
            cudaEventCreateWithFlags(&p.consumed[i], cudaEventDisableTiming);
        }
        p.device = dev;
    }
    (void)gb;
    return &p;
}

}  // namespace qdb

using namespace qdb;

extern "C" int32_t qdb_gb_process_host(qdb_gb* gb, const void* const* key_cols, const uint64_t* const* key_nulls,
                                       const void* vals, const uint64_t* val_nulls, int64_t n, const qdb_pred* pred,
                                       const int8_t* mask, int64_t chunk_rows, void* stream) {
    if (!gb || !key_cols) return fail(QDB_ERR_INVALID, "qdb_gb_process_host: null argument");
    if (n <= 0) return QDB_OK;
    if (chunk_rows <= 0) chunk_rows = int64_t(1) << 24;
    chunk_rows = ((chunk_rows + 4095) / 4096) * 4096;  // whole tiles, whole null-mask words
    if (chunk_rows > n) chunk_rows = ((n + 4095) / 4096) * 4096;
    cudaStream_t s = as_stream(stream);
    HostPipe* hp = pipe_for(gb);
    if (!hp) return fail(QDB_ERR_CUDA, "qdb_gb_process_host: could not create the copy stream");

    const int nk = gb->n_key_cols;
    const size_t ks = (nk == 2) ? 4 : type_size(gb->key_type);
    const size_t vs = gb->val_type ? type_size(gb->val_type) : 0;
    const size_t ps = pred ? type_size(pred->type) : 0;
    const size_t nullw = static_cast<size_t>(chunk_rows / 64) * 8;
    // staging layout per buffer: keys[nk], key nulls[nk], values, value nulls, predicate, predicate nulls, mask
    struct Off {
        size_t key[2], knull[2], val, vnull, pcol, pnull, mask, total;
    } o{};
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t at = off;
        off += (bytes + 255) & ~size_t(255);
        return at;
    };
    for (int c = 0; c < nk; ++c) {
        o.key[c] = take(chunk_rows * ks);
        o.knull[c] = (key_nulls && key_nulls[c]) ? take(nullw) : SIZE_MAX;
    }
    o.val = vs ? take(chunk_rows * vs) : SIZE_MAX;
    o.vnull = (vs && val_nulls) ? take(nullw) : SIZE_MAX;
    o.pcol = pred ? take(chunk_rows * ps) : SIZE_MAX;
    o.pnull = (pred && pred->nulls) ? take(nullw) : SIZE_MAX;
    o.mask = mask ? take(chunk_rows) : SIZE_MAX;
    o.total = off;

    if (hp->stage_bytes < o.total) {
        // Earlier calls may have run on other streams: wait for their last use of each buffer and for the copies.
        for (int b = 0; b < 2; ++b) QDB_CUDA_TRY(cudaEventSynchronize(hp->consumed[b]));
        QDB_CUDA_TRY(cudaStreamSynchronize(hp->copy));
        for (int b = 0; b < 2; ++b) {
            if (hp->stage[b]) cudaFree(hp->stage[b]);
            hp->stage[b] = nullptr;
        }
        hp->stage_bytes = 0;
        for (int b = 0; b < 2; ++b) QDB_CUDA_TRY(cudaMalloc(&hp->stage[b], o.total));
        hp->stage_bytes = o.total;
    }
    // consumed[b] keeps the record of the last aggregation that read buffer b, on whichever stream the call that
    // queued it used, so the copy stream's wait below orders this call after earlier calls on other streams too
    // (an event never recorded makes the wait a no-op).  It is re-recorded only after this call's own use of b.

    const int64_t nchunks = (n + chunk_rows - 1) / chunk_rows;
    for (int64_t c = 0; c < nchunks; ++c) {
        const int b = static_cast<int>(c & 1);
        const int64_t r0 = c * chunk_rows;
        const int64_t rows = std::min<int64_t>(chunk_rows, n - r0);
        const size_t w0 = static_cast<size_t>(r0 / 64);
        const size_t nwb = static_cast<size_t>((rows + 63) / 64) * 8;
        char* st = static_cast<char*>(hp->stage[b]);
        QDB_CUDA_TRY(cudaStreamWaitEvent(hp->copy, hp->consumed[b], 0));
        auto up = [&](size_t at, const void* src, size_t bytes) -> cudaError_t {
            return cudaMemcpyAsync(st + at, src, bytes, cudaMemcpyHostToDevice, hp->copy);
        };
        const void* dk[2] = {nullptr, nullptr};
        const uint64_t* dkn[2] = {nullptr, nullptr};
        for (int k = 0; k < nk; ++k) {
            QDB_CUDA_TRY(up(o.key[k], static_cast<const char*>(key_cols[k]) + r0 * ks, rows * ks));
            dk[k] = st + o.key[k];
            if (o.knull[k] != SIZE_MAX) {
                QDB_CUDA_TRY(up(o.knull[k], key_nulls[k] + w0, nwb));
                dkn[k] = reinterpret_cast<const uint64_t*>(st + o.knull[k]);
            }
        }
        const void* dv = nullptr;
        const uint64_t* dvn = nullptr;
        if (o.val != SIZE_MAX) {
            QDB_CUDA_TRY(up(o.val, static_cast<const char*>(vals) + r0 * vs, rows * vs));
            dv = st + o.val;
        }
        if (o.vnull != SIZE_MAX) {
            QDB_CUDA_TRY(up(o.vnull, val_nulls + w0, nwb));
            dvn = reinterpret_cast<const uint64_t*>(st + o.vnull);
        }
        qdb_pred dp{};
        if (pred) {
            dp = *pred;
            QDB_CUDA_TRY(up(o.pcol, static_cast<const char*>(pred->col) + r0 * ps, rows * ps));
            dp.col = st + o.pcol;
            dp.nulls = nullptr;
            if (o.pnull != SIZE_MAX) {
                QDB_CUDA_TRY(up(o.pnull, pred->nulls + w0, nwb));
                dp.nulls = reinterpret_cast<const uint64_t*>(st + o.pnull);
            }
        }
        const int8_t* dm = nullptr;
        if (o.mask != SIZE_MAX) {
            QDB_CUDA_TRY(up(o.mask, mask + r0, rows));
            dm = reinterpret_cast<const int8_t*>(st + o.mask);
        }
        QDB_CUDA_TRY(cudaEventRecord(hp->copied[b], hp->copy));
        QDB_CUDA_TRY(cudaStreamWaitEvent(s, hp->copied[b], 0));
        int32_t rc = qdb_gb_process(gb, dk, (key_nulls ? dkn : nullptr), dv, dvn, rows, pred ? &dp : nullptr, dm,
                                    stream);
        if (rc != QDB_OK) return rc;
        QDB_CUDA_TRY(cudaEventRecord(hp->consumed[b], s));
    }
    return QDB_OK;
}
