// Device-side structures of the batched GROUP BY (many independent queries in one persistent launch).
#pragma once

#include "groupby_agg.cuh"

namespace qdb {

constexpr int kBWarps = 16;                  // warps per CTA of the batch kernel
constexpr int kBThreads = kBWarps * 32;      // 512 threads: 128 registers per thread at one CTA per SM, no spills
constexpr int kBQueues = 3;                  // work queues for 1, 2 and 4 warp groups per CTA (16, 8, 4 warps)
constexpr int kBResThreads = 256;
constexpr int kBResPer = 16;
constexpr int kBResChunk = kBResThreads * kBResPer;

// One query of the batch as the kernels see it (copied into shared memory at the start of every work item).
struct BInst {
    const void* keys;
    const void* vals;
    const void* pcol;
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
    int32_t S;                     // slots of one shared-memory table (power of two), 0 = global placement
    int32_t R;                     // shared-memory tables per warp group
    int32_t probe;                 // shared-memory probe limit
    int32_t ipt;                   // rows per thread per step (4 or 8)
    int32_t pad;
};
static_assert(sizeof(BInst) % 8 == 0, "BInst is copied as 64-bit words");

// A contiguous row range of one query.
struct BItem {
    int32_t inst;
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
};

struct BatchArgs {
    BHeader* hdr;
    const BInst* inst;
    const BItem* items;
    uint64_t* res;        // result words
    int64_t* res_count;   // per query: groups emitted
    int32_t* status;      // per query: QDB_OK or the latched error
    long long* item_ns;   // per item: device time of the item (globaltimer)
    int64_t dyn_bytes;    // dynamic shared memory of the aggregation kernel
};

}  // namespace qdb
