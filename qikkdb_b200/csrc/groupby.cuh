// Internal definitions of the GROUP BY table shared by the aggregation, result and batch kernels.
#pragma once

#include "qdb_common.cuh"

namespace qdb {

// Word layout of one table slot.  Word 0 is the key word.  The remaining words hold the running state
// of every aggregate the table carries; a table carries several aggregates at once so that
// SUM/MIN/MAX/COUNT/AVG of one query come out of one pass (the reference needs one table per
// aggregate, qikkDB/QueryEngine/GPUCore/GPUGroupBy.cuh:285-362).
//   cnt : number of non-NULL values aggregated (uint64).  A group whose cnt is 0 has a NULL value
//         (the reference's valuesNullArray, GPUGroupBy.cuh:182-185), and AVG = sum / cnt.
//   sum : two's-complement uint64 for integer values (wraps exactly like the reference's integer
//         atomicAdd, AggregationFunctions.cuh:219-228) or an FP64 accumulator for float/double values.
//   mn/mx : for 32-bit values one word holds both (low half min, high half max, as int32 or as the
//         order-preserving encoding of a float); for 64-bit values one word each.
struct Layout {
    int32_t W = 1;       // words per slot, a power of two
    int32_t cnt = -1;
    int32_t sum = -1;
    int32_t mn = -1;
    int32_t mx = -1;
    int32_t packed = 0;  // 1: mn and mx share one word
};

// One open-addressing region: `cap` hashed slots (cap a power of two) followed by two special slots:
// slot cap holds the NULL key (the reference's slot 0, GPUGroupBy.cuh:163-167) and slot cap+1 holds
// the one key value that equals kEmpty.
struct Region {
    uint64_t* slots = nullptr;
    uint64_t mask = 0;  // cap - 1
};

enum ValKind : int32_t { VK_NONE = 0, VK_I32 = 1, VK_I64 = 2, VK_F32 = 3, VK_F64 = 4 };

inline ValKind val_kind(int32_t t) {
    switch (t) {
        case QDB_INT32: return VK_I32;
        case QDB_INT64: return VK_I64;
        case QDB_FLOAT: return VK_F32;
        case QDB_DOUBLE: return VK_F64;
        default: return VK_NONE;
    }
}

inline bool vk_is_32(ValKind vk) { return vk == VK_I32 || vk == VK_F32; }

// Row-level kinds of a key.
enum KeyKind : int32_t { KK_NORMAL = 0, KK_NULL = 1, KK_ESCAPE = 2, KK_AUX = 3 };

// Identity words of the min/max state (encoded space).
constexpr uint64_t kPackedMinMaxInit = (static_cast<uint64_t>(0x80000000u) << 32) | 0x7fffffffu;
constexpr uint64_t kMinInit64 = 0x7fffffffffffffffull;
constexpr uint64_t kMaxInit64 = 0x8000000000000000ull;

// The virtual slot space of a table for whole-table passes: the main region's cap + 2 slots,
// followed by the composite-NULL region's cap + 2 slots when that region exists.
struct SlotSpace {
    const uint64_t* main = nullptr;
    const uint64_t* aux = nullptr;
    uint64_t cap = 0;    // hashed slots per region
    int32_t W = 1;
    uint64_t total = 0;  // main (cap + 2) + aux (cap + 2, when present)
};

#ifdef __CUDACC__
__device__ __forceinline__ const uint64_t* slot_at(const SlotSpace& sp, uint64_t v) {
    const uint64_t per = sp.cap + 2;
    return (v < per) ? sp.main + v * sp.W : sp.aux + (v - per) * sp.W;
}

__device__ __forceinline__ bool present(const SlotSpace& sp, uint64_t v) {
    return v < sp.total && slot_at(sp, v)[0] != kEmpty;
}
#endif

}  // namespace qdb

// The opaque table handle of the C ABI.
struct qdb_gb {
    int32_t aggs = 0;
    int32_t key_type = 0;
    int32_t n_key_cols = 1;
    int32_t val_type = 0;
    int32_t placement = 0;
    int32_t device = 0;
    int64_t capacity = 0;  // distinct groups allowed before HASH_TABLE_FULL
    uint64_t cap = 0;      // hashed slots per region (power of two)
    qdb::Layout L;
    qdb::Region main;
    qdb::Region aux;       // composite keys with a NULL component (allocated on first use)
    unsigned long long* counters = nullptr;  // [0] groups claimed, [1] status word (int32 in low half)
    int64_t last_hint_rows = 0;
};

namespace qdb {
int32_t gb_init_region(qdb_gb* gb, Region& r, cudaStream_t s);

inline SlotSpace slot_space(const qdb_gb* gb) {
    SlotSpace sp;
    sp.main = gb->main.slots;
    sp.aux = gb->aux.slots;
    sp.cap = gb->cap;
    sp.W = gb->L.W;
    sp.total = (gb->cap + 2) * (gb->aux.slots ? 2 : 1);
    return sp;
}
}  // namespace qdb
