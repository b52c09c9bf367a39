// Device-side structures of the batched GROUP BY (many independent queries in one persistent launch).
#pragma once

#include "groupby_agg.cuh"

namespace qdb {

constexpr int kBCons = 12;                          // consumer warps per CTA
constexpr int kBProd = 4;                           // producer warps per CTA (one per warp group)
constexpr int kBThreads = (kBCons + kBProd) * 32;   // 512 threads (128 registers each), one CTA per SM
constexpr int kBQueues = 3;                         // work queues for 1, 2 and 4 warp groups per CTA (12, 6, 3 warps)
constexpr int kBStages = 3;                         // shared-memory ring stages per warp group
constexpr int kBStageBytes = 24 * 1024;             // stage bytes at one group per CTA (halved per extra group level)
constexpr int kBHeaderBytes = 256;                  // mbarriers and stage metadata of one warp group
constexpr int kBMaxMembers = 8;                     // queries sharing one scan of their columns
constexpr int kBMaxRowsPerLane = 4;
constexpr int kBListRows = 256;                     // rows of a stage tile one consumer warp compacts (u16 list)
constexpr int kBSmemCap = 192 * 1024;              // shared memory per CTA: the rest stays L1 for the probe loads
constexpr int kBResThreads = 1024;
constexpr int kBResPer = 8;
constexpr int kBResChunk = kBResThreads * kBResPer;

// Shared memory of one warp group in queue q: [header | tables ... | stage ring].
__host__ __device__ constexpr int b_stage_bytes(int q) { return kBStageBytes >> q; }
__host__ __device__ constexpr int b_ring_bytes(int q) { return kBStages * (kBStageBytes >> q); }

// One query of the batch as the kernels see it.
struct BInst {
    unsigned long long* counters;  // [0] groups claimed, [1] status word
    Region main;                   // the query's global table (cap hashed slots + NULL slot + escape slot)
    int64_t n;
    int64_t key_mod;               // > 0: the key is key % key_mod
    int64_t capacity;              // distinct keys allowed before HASH_TABLE_FULL
    int64_t plo, phi;              // predicate interval in the ordinal space of the predicate column
    int64_t res_off;               // first result word of this query
    int64_t res_cap;               // result rows reserved (capacity + 2)
    Layout L;
    int32_t kt;                    // key bytes: 4 or 8
    int32_t vk;                    // ValKind of the value column
    int32_t pbytes;                // predicate column bytes: 0 (no predicate), 4 or 8
    int32_t pfloat;                // predicate column is IEEE floating point
    int32_t pinv;                  // keep = (lo <= x <= hi) != pinv
    int32_t has_sum, has_min, has_max;
    int32_t aggs;
    int32_t S;                     // slots of one shared-memory table (a multiple of 32), 0 = global placement
    int32_t R;                     // shared-memory tables of this query per warp group
    int32_t probe;                 // shared-memory probe limit
    int32_t so_table;              // byte offset of this query's shared tables in the group's table region
    int32_t mod_s1;                // key modulus as multiply-high constants (mod_magic of key_mod)
    uint64_t mod_m;
    int32_t mod_s2;
    int32_t pad;
};
static_assert(sizeof(BInst) % 8 == 0, "BInst is 64-bit aligned");

// Queries that read the same columns and are aggregated in one scan (one tile load serves every member).
struct BGroup {
    const void* keys;
    const void* vals;
    const void* pcol;
    int64_t n;
    int32_t kt, vbytes, pbytes, vk;
    int32_t n_members;
    int32_t stage_rows;            // rows per stage tile (as many as fit one ring stage, a multiple of 4)
    int32_t rpt;                   // rows each consumer thread handles per step of a tile (1, 2 or 4)
    int32_t pad;
    int32_t members[kBMaxMembers];
};

// A contiguous row range of one scan group.
struct BItem {
    int32_t group;
    int32_t queue;
    int64_t r0;
    int64_t r1;
    int64_t pad;
};

// Per-run control block in device memory.  The host writes it with every new plan; the result kernel resets
// the queue heads and init flag at the end of every run, so a captured graph can be replayed as is.
struct BHeader {
    unsigned long long heads[kBQueues];
    int32_t q_begin[kBQueues + 1];  // queue q holds items [q_begin[q], q_begin[q + 1])
    int32_t n_inst;
    int32_t init_needed;
    int32_t error;                  // QDB_ERR_TIMEOUT when a bounded wait gave up (reset by the init kernel)
    int32_t pad;
};

struct BatchArgs {
    BHeader* hdr;
    const BInst* inst;
    const BGroup* groups;
    const BItem* items;
    uint64_t* res;        // result words
    int64_t* res_count;   // per query: groups emitted
    int32_t* status;      // per query: QDB_OK or the latched error
    long long* item_ns;   // per item: device time of the item (globaltimer)
    int64_t dyn_bytes;    // dynamic shared memory of the aggregation kernel
};

// Host-side helpers of the batch for the serving loop (batch.cu).
int32_t batch_check_query(const qdb_gb_query& q);
int32_t batch_enqueue_readback(qdb_gb_batch* b, int64_t* h_counts, int32_t* h_status, void* h_res, int64_t h_res_bytes,
                               cudaStream_t s);
void batch_result_place(const qdb_gb_batch* b, int i, int64_t* off_words, int64_t* cap_rows, int32_t* n_cols);

}  // namespace qdb
