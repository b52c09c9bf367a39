/*
 * qdb_gb.h - C ABI of the B200 GROUP BY hot path (filter -> compaction -> hash aggregate).
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, and returns an int32
 * status whose values 0..8 are the reference's QueryEngineErrorType
 * (qikkDB/QueryEngine/GPUError.h:17-28); values >= 100 are this library's own.
 * Device pointers are CUDA device pointers on the current device.  `stream` is a
 * cudaStream_t passed as void* (NULL = the legacy default stream, which is what the
 * reference's operators use, qikkDB/QueryEngine/GPUCore/GPUMemory.cuh:89-189).
 *
 * Buffers that an entry point hands back (`out` pointers) are allocated by the library
 * on `stream` with the stream-ordered allocator and must be released with qdb_free(),
 * mirroring GPUMemory::alloc / GPUMemory::free ownership in the reference
 * (qikkDB/QueryEngine/GPUCore/GPUGroupBy.cuh:501, GPUReconstruct.cuh:296).
 *
 * Null masks are the reference's bit-packed `nullmask_t` (uint64_t, bit i%64 of word i/64,
 * qikkDB/QueryEngine/GPUCore/NullValues.cuh:6-12, NullValues.cu:3-57).
 */
#ifndef QDB_GB_H
#define QDB_GB_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes: 0..8 mirror QueryEngineErrorType (qikkDB/QueryEngine/GPUError.h:17-28) ---- */
enum qdb_status {
    QDB_OK = 0,                 /* GPU_EXTENSION_SUCCESS */
    QDB_ERROR = 1,              /* GPU_EXTENSION_ERROR (CUDA or argument error) */
    QDB_DIVISION_BY_ZERO = 2,   /* GPU_DIVISION_BY_ZERO_ERROR */
    QDB_INTEGER_OVERFLOW = 3,   /* GPU_INTEGER_OVERFLOW_ERROR */
    QDB_HASH_TABLE_FULL = 4,    /* GPU_HASH_TABLE_FULL: more distinct keys than the table holds */
    QDB_UNKNOWN_AGG_FUN = 5,    /* GPU_UNKNOWN_AGG_FUN */
    QDB_NOT_FOUND = 6,          /* GPU_NOT_FOUND_ERROR: no CUDA device */
    QDB_ERR_INVALID = 100,      /* bad argument (type code, size, null pointer) */
    QDB_ERR_NOMEM = 101,        /* device allocation failed */
    QDB_ERR_CUDA = 102,         /* a CUDA runtime call failed; see qdb_last_error() */
    QDB_ERR_TIMEOUT = 103,      /* a bounded device-side wait gave up */
    QDB_ERR_TOO_LARGE = 104     /* size beyond a stated maximum */
};

/* ---- element types (codes follow the reference's COLUMN_* DataType values, qikkDB/DataType.h:7-27) ---- */
enum qdb_type {
    QDB_INT32 = 8,   /* COLUMN_INT */
    QDB_INT64 = 9,   /* COLUMN_LONG */
    QDB_FLOAT = 10,  /* COLUMN_FLOAT */
    QDB_DOUBLE = 11, /* COLUMN_DOUBLE */
    QDB_INT8 = 15    /* COLUMN_INT8_T (filter operands / masks only) */
};

/* ---- aggregate bits (AggregationFunctions::{min,max,sum,avg,count,none},
 *      qikkDB/QueryEngine/GPUCore/AggregationFunctions.cuh:17-366). A table may carry several
 *      aggregates at once (one fused pass); AGG none is agg_mask == 0. ---- */
enum qdb_agg {
    QDB_AGG_MIN = 1,
    QDB_AGG_MAX = 2,
    QDB_AGG_SUM = 4,
    QDB_AGG_AVG = 8,
    QDB_AGG_COUNT = 16
};

/* ---- filter operators (FilterConditions::*, qikkDB/QueryEngine/GPUCore/GPUFilterConditions.cuh:9-180) ---- */
enum qdb_cmp {
    QDB_GREATER = 0,
    QDB_GREATER_EQUAL = 1,
    QDB_LESS = 2,
    QDB_LESS_EQUAL = 3,
    QDB_EQUAL = 4,
    QDB_NOT_EQUAL = 5,
    QDB_LOGICAL_AND = 6,
    QDB_LOGICAL_OR = 7
};

/* ---- table placement hints for the aggregation pass ---- */
enum qdb_placement {
    QDB_PLACE_AUTO = 0,   /* choose from the capacity hint */
    QDB_PLACE_SHARED = 1, /* per-CTA shared-memory table with global spill (low cardinality / skew) */
    QDB_PLACE_GLOBAL = 2  /* global open-addressing table only (high cardinality) */
};

/* A predicate `col OP constant` evaluated inside the aggregation pass (the fused form of
 * GPUBinary<OP,int8_t,T*,U>::Binary + GPUReconstruct::reconstructColKeep, which the reference
 * runs as separate kernels, qikkDB/QueryEngine/GPUCore/GPUBinary.cuh:555-579,
 * GPUReconstruct.cuh:272-355).  Rows whose predicate column is NULL are filtered out, as
 * kernel_filter does (qikkDB/QueryEngine/GPUCore/GPUFilter.cuh:22-44). */
typedef struct qdb_pred {
    const void* col;         /* device column */
    int32_t type;            /* qdb_type of col (INT32, INT64, FLOAT, DOUBLE) */
    int32_t op;              /* qdb_cmp (comparison ops only) */
    int32_t const_type;      /* qdb_type of the constant; the comparison runs in the C++ common type
                                of (column type, constant type), as kernel_filter's `a < b` does */
    int32_t reserved;
    int64_t const_i;         /* the constant when const_type is INT32 or INT64 */
    double const_f;          /* the constant when const_type is FLOAT (exactly representable) or DOUBLE */
    const uint64_t* nulls;   /* optional null bitmask of col */
} qdb_pred;

typedef struct qdb_gb qdb_gb; /* opaque GROUP BY table */

/* Last error message of the calling thread (never NULL). */
const char* qdb_last_error(void);
/* Library version string. */
const char* qdb_version(void);
/* Number of kernels this library has launched in the process so far (for launch accounting). */
int64_t qdb_launch_count(void);
/* Number of CUDA devices visible (0 when none); returns QDB_OK. */
int32_t qdb_device_count(int32_t* out_count);

/* ---- memory helpers (GPUMemory::alloc/free/copy*, qikkDB/QueryEngine/GPUCore/GPUMemory.cuh:89-189) ---- */
int32_t qdb_malloc(void** out_ptr, int64_t bytes, void* stream);
int32_t qdb_free(void* ptr, void* stream);
int32_t qdb_memcpy_h2d(void* dst, const void* src, int64_t bytes, void* stream);
int32_t qdb_memcpy_d2h(void* dst, const void* src, int64_t bytes, void* stream);
int32_t qdb_memcpy_d2d(void* dst, const void* src, int64_t bytes, void* stream);
int32_t qdb_memset(void* dst, int32_t byte_value, int64_t bytes, void* stream);
int32_t qdb_stream_sync(void* stream);
/* Context::bindDeviceToContext / getBoundDeviceID (qikkDB/QueryEngine/Context.cu:134-139): the calling thread's
 * current device, on which every other entry point works. */
int32_t qdb_set_device(int32_t device);
int32_t qdb_get_device(int32_t* out_device);
/* Synchronous copy between two devices' memory, the transfer the reference's multi-GPU GetResults makes through
 * host buffers when it gathers every GPU's table (qikkDB/QueryEngine/GPUCore/GPUGroupBy.cuh:594-790). */
int32_t qdb_memcpy_peer(void* dst, int32_t dst_device, const void* src, int32_t src_device, int64_t bytes);

/* ---- GROUP BY table: GPUGroupBy<AGG,O,K,V> (qikkDB/QueryEngine/GPUCore/GPUGroupBy.cuh:285-790) and
 *      the multi-key specialisation (qikkDB/QueryEngine/GPUCore/GPUGroupByMultiKey.cuh:262-1325). ----
 *
 * qdb_gb_create replaces the constructor GPUGroupBy(maxHashCount, keySizeMultiplier)
 * (GPUGroupBy.cuh:313): `max_groups` = maxHashCount * keySizeMultiplier, capped at 2^30 like
 * GB_BUFFER_SIZE_MAX (IGroupBy.h:5).  key_type is a qdb_type; n_key_cols is 1, or 2 for a composite
 * (int32 x int32) key.  val_type is a qdb_type or 0 for a table without a value column.
 * agg_mask is an OR of qdb_agg bits.  placement is a qdb_placement hint. */
int32_t qdb_gb_create(qdb_gb** out, int32_t agg_mask, int32_t key_type, int32_t n_key_cols,
                      int32_t val_type, int64_t max_groups, int32_t placement, void* stream);
/* ~GPUGroupBy (GPUGroupBy.cuh:374-386). */
int32_t qdb_gb_destroy(qdb_gb* gb);
/* GetMaxHashCount (GPUGroupBy.cuh:414): the reference's keyBufferSize_ (max_groups + 1 NULL slot). */
int32_t qdb_gb_max_hash_count(qdb_gb* gb, int64_t* out);
/* Number of distinct non-NULL keys inserted so far (reads a device counter; synchronises stream). */
int32_t qdb_gb_group_count(qdb_gb* gb, int64_t* out, void* stream);

/* ProcessBlock (GPUGroupBy.cuh:395-410; multi-key GPUGroupByMultiKey.cuh:535-627), asynchronous:
 * key_cols[n_key_cols] device key columns, key_nulls[n_key_cols] optional null bitmasks (array may be
 * NULL), vals/val_nulls the value column (NULL when val_type == 0), n rows.  `pred` (optional) is a
 * fused filter; `mask` (optional) is a precomputed int8 filter mask (non-zero = keep).  Both may be
 * given; a row is aggregated when it passes both.  Errors raised by the kernel (HASH_TABLE_FULL) are
 * latched in the table and returned by qdb_gb_check (the ErrorFlagSwapper::Swap step,
 * qikkDB/QueryEngine/GPUCore/ErrorFlagSwapper.h:32-50).  A table whose max_groups exceeds one shared-memory
 * table (and placement is not QDB_PLACE_GLOBAL) uses the device's spill area, allocated by the first call that
 * needs it and kept, grown on demand, until the process exits. */
int32_t qdb_gb_process(qdb_gb* gb, const void* const* key_cols, const uint64_t* const* key_nulls,
                       const void* vals, const uint64_t* val_nulls, int64_t n, const qdb_pred* pred,
                       const int8_t* mask, void* stream);
/* ProcessBlock over HOST-resident columns (every pointer, including pred->col / pred->nulls and the masks, is a
 * host pointer): the columns are uploaded in chunks of `chunk_rows` rows (rounded up to 4096; <= 0 picks 16M)
 * through two device staging buffers, each chunk's upload overlapping the aggregation of the previous one.
 * Host buffers should be pinned for the overlap.  Asynchronous on `stream` like qdb_gb_process; the caller keeps
 * the host buffers alive until `stream` has passed this call.  Replaces the synchronous per-block LoadCol upload
 * (qikkDB/GpuSqlParser/Dispatcher/GpuSqlDispatcherVMFunctions.h:185-260) in front of ProcessBlock. */
int32_t qdb_gb_process_host(qdb_gb* gb, const void* const* key_cols, const uint64_t* const* key_nulls,
                            const void* vals, const uint64_t* val_nulls, int64_t n, const qdb_pred* pred,
                            const int8_t* mask, int64_t chunk_rows, void* stream);
/* ---- compressed column blocks: AAFL (qikkDB/Compression/GPUCompression.cu:25-148, :474-522; the block format
 *      of CompressionGPU::compressDataAAFL and the bit packing of feathergpu fl/aafl.cuh, fl/afl.cuh) ----
 * A block as the reference stores it, on the device: int64 rows, int64 elements (its length in elements of the
 * type), int64 blocks (= ceil(rows / 32)), uint64 position[blocks], uint8 bit_length[blocks], then the packed words.
 * Rows come in groups of 32 W (W = bits of the type): row d is lane d % 32, value (d % 32W) / 32 of its group, and
 * takes bit_length[g] bits of the lane's stream (words position[g] + lane + 32 k), to which the offset (the block's
 * min, or 0 when max - min does not fit the type) is added back.  FLOAT blocks are their int32 bit patterns (the
 * reference compresses only single-sign float blocks).  min_bits / max_bits carry the block's min and max (the
 * BlockBase statistics the dispatcher passes to Decompress) as the type's bit pattern in the low bytes. */
typedef struct qdb_aafl_col {
    const void* data;    /* device: the compressed block */
    int32_t type;        /* QDB_INT32, QDB_INT64 or QDB_FLOAT */
    int32_t reserved;
    int64_t rows;        /* the header's three counts */
    int64_t elements;
    int64_t blocks;
    int64_t min_bits;
    int64_t max_bits;
} qdb_aafl_col;
/* CompressionGPU::decompressDataAAFLOnDevice: writes the block's rows to `out` (device, rows elements of the
 * type).  A block whose words do not match its header latches nothing here: the call returns QDB_ERR_INVALID after
 * synchronising `stream` when a position or bit length points outside the packed words. */
int32_t qdb_aafl_decompress(const qdb_aafl_col* col, void* out, void* stream);
/* CompressionGPU::compressDataAAFL (GPUCompression.cu:25-148, on a device column): compresses `rows` values of
 * `type` at `in` with the block's min and max (bit patterns as in qdb_aafl_col) into a newly allocated block
 * (*out_block, *out_elements elements of the type; release with qdb_free), groups placed in row order.  A block that
 * would not be smaller than the column (or a FLOAT column whose values mix signs) stays plain: *out_block is NULL.
 * Synchronises `stream`. */
int32_t qdb_aafl_compress(int32_t type, const void* in, int64_t rows, int64_t min_bits, int64_t max_bits,
                          void** out_block, int64_t* out_elements, void* stream);
/* ProcessBlock of a single-key table whose key column is an AAFL block (the dispatcher's decompress-then-aggregate,
 * GpuSqlDispatcherVMFunctions.h:228-250, fused): in the fast pass the consumer warps unpack their rows' keys from the
 * packed words into shared memory, so the key column costs its compressed bytes of HBM traffic.  `vals` (plain,
 * val_type's column of rows values) and `pred` (plain columns) as in qdb_gb_process; no NULL masks.  When the fast
 * pass does not apply (a table placed QDB_PLACE_GLOBAL, fewer than 2048 rows, unaligned columns) the keys are
 * decompressed into a temporary column first.  The key type must be the table's.  Asynchronous like qdb_gb_process;
 * a malformed block latches QDB_ERR_INVALID for qdb_gb_check. */
int32_t qdb_gb_process_aafl(qdb_gb* gb, const qdb_aafl_col* keys, const void* vals, const qdb_pred* pred,
                            void* stream);
/* ProcessBlock of the expression key % key_mod (C++ remainder) of a single INT32 or INT64 key column: the
 * dispatcher's GPUBinary<ArithmeticOperations::mod> column (GPUBinary.cuh:145-166) followed by ProcessBlock
 * (GPUGroupBy.cuh:395-410), fused -- the fast pass takes each key's remainder (multiply-high by the invariant |m|) as
 * it reads the key, so no remainder column is written or read.  Where the fast pass does not apply (fewer than 2048
 * rows, unaligned columns, a table placed QDB_PLACE_GLOBAL) the remainder column is materialised first.  `vals` and
 * `pred` as in qdb_gb_process, no NULL masks; key_mod must fit the key type (QDB_DIVISION_BY_ZERO for 0).
 * Asynchronous like qdb_gb_process. */
int32_t qdb_gb_process_mod(qdb_gb* gb, const void* keys, int64_t key_mod, const void* vals, const qdb_pred* pred,
                           int64_t n, void* stream);
/* Synchronises `stream`, returns and clears the latched kernel status (QDB_OK or QDB_HASH_TABLE_FULL). */
int32_t qdb_gb_check(qdb_gb* gb, void* stream);
/* ProcessBlock followed by the Swap check: the synchronous form the reference exposes. */
int32_t qdb_gb_process_sync(qdb_gb* gb, const void* const* key_cols, const uint64_t* const* key_nulls,
                            const void* vals, const uint64_t* val_nulls, int64_t n, const qdb_pred* pred,
                            const int8_t* mask, void* stream);

/* GetResults (GPUGroupBy.cuh:478-587; multi-key GPUGroupByMultiKey.cuh:742-912).
 * For one aggregate `agg` (a single qdb_agg bit, or 0 for GROUP BY without aggregation):
 * out_keys[n_key_cols] receive newly allocated device key columns, out_key_nulls[n_key_cols] (optional)
 * their null bitmasks, *out_vals the values (type: V for MIN/MAX/SUM/AVG, int64 for COUNT),
 * *out_val_nulls (optional) the value null bitmask, *out_count the group count.  An empty result yields
 * NULL pointers and count 0 (GPUReconstruct.cuh:311-318).  Synchronises `stream` (the count is read back). */
int32_t qdb_gb_results(qdb_gb* gb, int32_t agg, void** out_keys, uint64_t** out_key_nulls, void** out_vals,
                       uint64_t** out_val_nulls, int64_t* out_count, void* stream);
/* Several aggregates from one fused table in one pass: aggs[n_aggs] are qdb_agg bits, out_vals[i] and
 * out_val_nulls[i] (optional array) receive aggregate i. */
int32_t qdb_gb_results_multi(qdb_gb* gb, int32_t n_aggs, const int32_t* aggs, void** out_keys,
                             uint64_t** out_key_nulls, void** out_vals, uint64_t** out_val_nulls,
                             int64_t* out_count, void* stream);
/* Clears the table to its freshly created state (asynchronous). */
int32_t qdb_gb_reset(qdb_gb* gb, void* stream);

/* ---- raw partial state, for merging tables across GPUs (GetResults over `tables`,
 *      GPUGroupBy.cuh:594-790, and ReconstructRawNumbers, :433-471) ----
 * A partial record is (key word, state words).  qdb_gb_export_partitioned writes every occupied slot,
 * bucketed by owner = hash(key) mod n_parts, into newly allocated device buffers: *out_keys (uint64 key
 * words, int64 for composite packing), *out_state (state words, qdb_gb_state_words() per record),
 * *out_flags (uint8: bit0 NULL key slot, bit1 escaped key slot, bit2 composite-with-null key),
 * and host array part_counts[n_parts]. Synchronises `stream`. */
int32_t qdb_gb_state_words(qdb_gb* gb, int32_t* out_words);
int32_t qdb_gb_export_partitioned(qdb_gb* gb, int32_t n_parts, uint64_t** out_keys, uint64_t** out_state,
                                  uint8_t** out_flags, int64_t* part_counts, void* stream);
/* Merges `n` exported records (device buffers in the export layout) into `gb` (asynchronous). */
int32_t qdb_gb_merge_partial(qdb_gb* gb, const uint64_t* keys, const uint64_t* state, const uint8_t* flags,
                             int64_t n, void* stream);

/* ---- filter: GPUBinary<FilterConditions::OP,int8_t,L,R>::Binary
 *      (qikkDB/QueryEngine/GPUCore/GPUBinary.cuh:555-579, kernel_filter GPUFilter.cuh:22-44) ----
 * out_mask[i] = OP(a[i] or a, b[i] or b) && !null(i).  When a side is a constant (`*_is_col` == 0) its
 * pointer is a HOST pointer to one value of its type.  const-const fills the mask (GPUBinary.cuh:573). */
int32_t qdb_filter(int32_t op, int32_t a_type, int32_t a_is_col, const void* a, int32_t b_type, int32_t b_is_col,
                   const void* b, const uint64_t* null_mask, int8_t* out_mask, int64_t n, void* stream);

/* GPUBinary<ArithmeticOperations::mod, T, T*, T>::Binary (qikkDB/QueryEngine/GPUCore/GPUBinary.cuh:145-166) for a
 * column and a constant: out[i] = in[i] % modulus (C++ remainder) for INT32 / INT64 columns; the `key % m` column
 * the dispatcher materialises before a GROUP BY over that expression.  modulus 0 returns QDB_DIVISION_BY_ZERO. */
int32_t qdb_arith_mod(int32_t type, const void* in, int64_t modulus, void* out, int64_t n, void* stream);

/* ---- compaction: GPUReconstruct (qikkDB/QueryEngine/GPUCore/GPUReconstruct.cuh:204-355, :487-640) ----
 * qdb_reconstruct_keep: reconstructColKeep<T> with elem_bytes = sizeof(T) (1, 2, 4 or 8).  A NULL mask
 * returns `in` itself and n (no copy), as the reference does (GPUReconstruct.cuh:320-327).
 * null_in/out_null_mask: optional null bitmask to compact alongside. Synchronises `stream`. */
int32_t qdb_reconstruct_keep(int32_t elem_bytes, const void* in, const int8_t* mask, int64_t n, void** out,
                             int64_t* out_count, const uint64_t* null_in, uint64_t** out_null_mask,
                             void* stream);
/* Compaction that allocates nothing.  No counterpart in the reference: it exists for callers that own all
 * device memory themselves (a buffer pool that accounts every byte of HBM, a serving loop admitting queries
 * against a fixed HBM budget) and so cannot let a library call cudaMalloc or cudaFree during a query: such an
 * allocation can fail mid-query under their memory pressure, escapes their accounting, and cudaFree
 * synchronises the device.  Same selection as qdb_reconstruct_keep (mask required), but the caller passes
 * the output buffer `out` (room for out_capacity elements of elem_bytes) and, when null_in is given, an
 * output null mask with room for ceil(out_capacity / 64) words; *out_count receives the number of selected
 * rows (the call synchronises `stream` to read it).  Selecting more than out_capacity rows returns
 * QDB_ERR_TOO_LARGE and writes nothing.  Limit: n <= 268435456 (2^28) rows, else QDB_ERR_TOO_LARGE.
 * Scratch is a fixed 512 KiB array that the library holds on every GPU that loads it until the process
 * exits; the first call on a device looks up that array's device address, so make the first call before
 * any stream capture.  All calls on a device share the array: calls that overlap on the GPU (other streams,
 * other host threads) race and must be serialised by the caller. */
int32_t qdb_reconstruct_keep_noalloc(int32_t elem_bytes, const void* in, const int8_t* mask, int64_t n, void* out,
                                     int64_t out_capacity, int64_t* out_count, const uint64_t* null_in,
                                     uint64_t* out_null_mask, void* stream);
/* GenerateIndexesKeep<int32_t,int8_t> (GPUReconstruct.cuh:518-566): int32 row indices where mask != 0. */
int32_t qdb_generate_indexes(const int8_t* mask, int64_t n, int32_t** out, int64_t* out_count, void* stream);
/* PrefixSum<int32_t,int8_t> (GPUReconstruct.cuh:573-583): inclusive sum of mask into out[n] (caller-owned). */
int32_t qdb_prefix_sum(const int8_t* mask, int64_t n, int32_t* out, void* stream);
/* CompressNullMask (GPUReconstruct.cu:756-764): uint8 array (bit0 of each byte) -> bit-packed mask
 * (newly allocated, ceil(n/64) words). */
int32_t qdb_compress_null_mask(const uint8_t* in, int64_t n, uint64_t** out, void* stream);

/* ---- ORDER BY over result columns: GPUOrderBy (qikkDB/QueryEngine/GPUCore/GPUOrderBy.cuh:88-195) ----
 * qdb_order_by_column is one GPUOrderBy::OrderByColumn step: it re-sorts the permutation `indices` (n int32
 * row numbers, device, caller-owned; first != 0 starts from the identity 0..n-1 instead of reading it) stably by
 * the column `col` (qdb_type INT32, INT64, FLOAT or DOUBLE), ascending, or descending when descending != 0.  NULL
 * rows (bits of the optional null mask) order as lowest(T), as the reference's TransformNullValsToSmallestVal makes
 * them; floats order by their IEEE bits (-0.0 before +0.0), as a radix sort does.  Calling it for the ORDER BY
 * columns from the last to the first, as the dispatcher does, leaves the lexicographic order with the first column
 * most significant and ties in input order.  qdb_order_by does that for n_cols columns at once.
 * qdb_reorder is ReOrderByIdx with OFFSET / LIMIT: out[i] = in[indices[offset + i]] for i < count;
 * qdb_reorder_nulls is ReOrderNullValuesByIdx the same way (out holds ceil(count / 64) words).  Asynchronous. */
int32_t qdb_order_by_column(int32_t type, const void* col, const uint64_t* nulls, int32_t descending, int64_t n,
                            int32_t first, int32_t* indices, void* stream);
int32_t qdb_order_by(int32_t n_cols, const int32_t* types, const void* const* cols, const uint64_t* const* nulls,
                     const int32_t* descending, int64_t n, int32_t* out_indices, void* stream);
int32_t qdb_reorder(int32_t elem_bytes, const void* in, const int32_t* indices, int64_t offset, int64_t count,
                    void* out, void* stream);
int32_t qdb_reorder_nulls(const uint64_t* in, const int32_t* indices, int64_t offset, int64_t count, uint64_t* out,
                          void* stream);

/* ---- scalar aggregation: GPUAggregation::col<AGG, OUT, IN> (qikkDB/QueryEngine/GPUCore/GPUAggregation.cuh:15-37)
 * over a WHERE-filtered column, fused, accumulated over a query's blocks ----
 * A qdb_scalar accumulates COUNT, SUM, MIN and MAX of one value column (val_type INT32, INT64, FLOAT or DOUBLE) over
 * every qdb_scalar_process call: rows that pass `pred` (optional, `col OP constant` as in qdb_gb_process) and `mask`
 * (optional int8, non-zero = keep) and whose value is not NULL (val_nulls optional).  qdb_scalar_result reads one
 * aggregate (one qdb_agg bit) into *out_value, typed as the GROUP BY results are: V for MIN/MAX/SUM/AVG (an integer
 * SUM wraps in V, an integer AVG is the wrapped sum over the count, truncated; float sums are accumulated in FP64),
 * int64 for COUNT; *out_is_null is 1 for MIN/MAX/SUM/AVG over no row.  qdb_scalar_result synchronises `stream`. */
typedef struct qdb_scalar qdb_scalar; /* opaque scalar accumulator */
int32_t qdb_scalar_create(qdb_scalar** out, int32_t val_type, void* stream);
int32_t qdb_scalar_destroy(qdb_scalar* q);
int32_t qdb_scalar_reset(qdb_scalar* q, void* stream);
int32_t qdb_scalar_process(qdb_scalar* q, const void* vals, const uint64_t* val_nulls, int64_t n, const qdb_pred* pred,
                           const int8_t* mask, void* stream);
int32_t qdb_scalar_result(qdb_scalar* q, int32_t agg, void* out_value, int32_t* out_is_null, void* stream);
/* Block skipping (GpuSqlDispatcher::WhereEvaluation, qikkDB/GpuSqlParser/GpuSqlDispatcher.cpp:1116-1125): whether a
 * block whose predicate column has non-NULL values in [*block_min, *block_max] (host values of pred->type) can hold a
 * row passing `pred`; *may_pass = 0 lets the caller skip loading and processing the block.  Host only. */
int32_t qdb_pred_block_may_pass(const qdb_pred* pred, const void* block_min, const void* block_max, int32_t* may_pass);

/* ---- GROUP BY over string keys: GPUGroupBy<AGG, O, std::string, V>
 *      (qikkDB/QueryEngine/GPUCore/GPUGroupByString.cuh:171-785, kernel :39-169) ----
 * Keys come in the reference's GPUString layout (GPUMemory.cuh GPUString): `chars` all characters concatenated,
 * `ends[i]` the int64 end offset of string i (string i is chars[i ? ends[i-1] : 0, ends[i])).  qdb_gbs_create sizes
 * the table for max_groups distinct non-NULL keys (the NULL key has its own slot, as keyBufferSize_ adds one) and a
 * key arena of max_key_bytes for the bytes of keys beyond their first 24 (<= 0: 32 per group); a key is at most
 * 2^20 - 2 bytes long.  agg_mask as qdb_gb_create; val_type 0 is allowed with QDB_AGG_COUNT only and counts rows.
 * qdb_gbs_process (asynchronous) aggregates the rows whose `mask` (optional int8, non-zero = keep) is set (a
 * COUNT-only table given no `vals` counts rows); NULL keys (key_nulls, optional) form one group; NULL values
 * (val_nulls, optional) are skipped, a group whose values are all NULL has a NULL aggregate and COUNT 0.  More
 * distinct keys than max_groups, or more key bytes than the arena holds, latch QDB_HASH_TABLE_FULL (a longer key
 * QDB_ERR_TOO_LARGE), which qdb_gbs_check (it synchronises `stream`) returns and clears.  qdb_gbs_results (GetResults, GPUGroupByString.cuh:446-563) allocates
 * the result keys as a GPUString (*out_chars, *out_ends), their NULL bitmask (optional), and per requested aggregate
 * (aggs[n_aggs], n_aggs <= 5) a column typed as qdb_gb_results types it plus its NULL bitmask (optional array);
 * an empty result yields NULL pointers and count 0.  It synchronises `stream`. */
typedef struct qdb_gbs qdb_gbs; /* opaque string-key GROUP BY table */
int32_t qdb_gbs_create(qdb_gbs** out, int32_t agg_mask, int32_t val_type, int64_t max_groups, int64_t max_key_bytes,
                       void* stream);
int32_t qdb_gbs_destroy(qdb_gbs* g);
int32_t qdb_gbs_reset(qdb_gbs* g, void* stream);
int32_t qdb_gbs_process(qdb_gbs* g, const char* chars, const int64_t* ends, const uint64_t* key_nulls, const void* vals,
                        const uint64_t* val_nulls, const int8_t* mask, int64_t n, void* stream);
int32_t qdb_gbs_check(qdb_gbs* g, void* stream);
/* The partial state of a string table, for GetResults over several GPUs' tables (GPUGroupByString.cuh:565-785, which
 * gathers every table's keys and values on the host): qdb_gbs_export writes every group as a record (its key string
 * into a newly allocated GPUString *out_chars / *out_ends, the NULL key as an empty string, and the numeric table's
 * state words and flags as qdb_gb_export_partitioned lays them out) and synchronises `stream`;
 * qdb_gbs_merge_exported adds `n` such records, copied to this table's device, into `g` (asynchronous; overflow
 * latches QDB_HASH_TABLE_FULL for qdb_gbs_check). */
int32_t qdb_gbs_export(qdb_gbs* g, char** out_chars, int64_t** out_ends, uint64_t** out_state, uint8_t** out_flags,
                       int64_t* out_count, void* stream);
int32_t qdb_gbs_merge_exported(qdb_gbs* g, const char* chars, const int64_t* ends, const uint64_t* state,
                               const uint8_t* flags, int64_t n, void* stream);
/* State words per exported record of `g` (the size of *out_state is count times this). */
int32_t qdb_gbs_state_words(qdb_gbs* g, int32_t* out_words);
int32_t qdb_gbs_results(qdb_gbs* g, int32_t n_aggs, const int32_t* aggs, char** out_chars, int64_t** out_ends,
                        uint64_t** out_key_nulls, void** out_vals, uint64_t** out_val_nulls, int64_t* out_count,
                        void* stream);

/* ---- batched GROUP BY: many independent queries in one persistent launch ----
 * The reference runs one GPUGroupBy per query, each with its own kernel launches and host synchronisations
 * (GpuSqlDispatcherAggregationFunctions.h:377-507 via GroupByHelper, :99-318).  A batch holds up to
 * max_instances such queries over device-resident columns and executes all of them with one work-queue-driven
 * persistent kernel (plus a table-initialisation and a result kernel), optionally replayed as one CUDA graph.
 * Per query it picks the table placement (shared-memory replicas or the global table), the number of warps that
 * cooperate on one work item (the effective CTA size) and the rows each thread loads per step, from a tuning
 * table that qdb_gb_batch_autotune fills by timing candidate plans on the batch's own queries.
 * Batch instances carry no NULL masks; queries with NULLs use qdb_gb_process. */
typedef struct qdb_gb_query {
    int32_t agg_mask;        /* qdb_agg bits; without a value column only QDB_AGG_COUNT */
    int32_t key_type;        /* QDB_INT32 or QDB_INT64 */
    int32_t val_type;        /* 0 (no value column) or QDB_INT32 / QDB_INT64 / QDB_FLOAT / QDB_DOUBLE */
    int32_t reserved;
    const void* keys;        /* device column of n_rows keys, 16-byte aligned */
    const void* vals;        /* device column of n_rows values, 16-byte aligned, or NULL when val_type == 0 */
    int64_t n_rows;
    int64_t max_groups;      /* distinct-key bound (a cardinality estimate): sizes the table; a query that
                                exceeds it reports QDB_HASH_TABLE_FULL, as ProcessBlock does */
    int64_t key_mod;         /* > 0: GROUP BY key % key_mod (C++ remainder, the GPUBinary modulo the dispatcher
                                would materialise first); 0: GROUP BY key */
    qdb_pred pred;           /* WHERE col OP constant; pred.col == NULL for none (pred.nulls must be NULL) */
} qdb_gb_query;

/* Execution plan of one batch instance (what the autotuner chooses). */
typedef struct qdb_gb_batch_cfg {
    int32_t placement;       /* QDB_PLACE_SHARED: shared-memory tables merged into the global table at the end of
                                every work item; QDB_PLACE_GLOBAL: every row goes to the global table */
    int32_t smem_slots;      /* slots of one shared-memory table (a multiple of 32, >= 64), shared placement */
    int32_t replicas;        /* shared-memory tables per warp group (warp w uses table w % replicas) */
    int32_t warps;           /* consumer warps cooperating on one work item: 12, 6 or 3 (1, 2 or 4 warp groups per
                                CTA, each with its own producer warp and share of shared memory) */
    int32_t rows_per_thread; /* rows each consumer thread takes per step through a staged column tile: 1, 2 or 4
                                (the probe loads of one step's rows are in flight together) */
    int32_t reserved;
    int64_t chunk_rows;      /* rows per work item (a multiple of 64) */
} qdb_gb_batch_cfg;

typedef struct qdb_gb_batch qdb_gb_batch; /* opaque batch */

/* Allocates a batch for up to max_instances queries whose hash tables take at most table_bytes of device memory
 * and whose results take at most result_bytes (per query (max_groups + 2) * (1 + aggregates) * 8 bytes). */
int32_t qdb_gb_batch_create(qdb_gb_batch** out, int32_t max_instances, int64_t table_bytes, int64_t result_bytes,
                            void* stream);
int32_t qdb_gb_batch_destroy(qdb_gb_batch* b);
/* Replaces the batch's queries and plans them (placement, warps, rows per thread, work items) from the tuning
 * table; uploads the plan asynchronously.  QDB_ERR_TOO_LARGE when the tables or results do not fit. */
int32_t qdb_gb_batch_set(qdb_gb_batch* b, const qdb_gb_query* queries, int32_t n, void* stream);
/* Executes every query of the batch: table initialisation (after a new plan), the persistent aggregation
 * kernel, and the result kernel (which leaves the tables clean for the next run).  use_graph != 0 replays
 * one CUDA graph holding the three kernels (captured on first use).  Asynchronous. */
int32_t qdb_gb_batch_run(qdb_gb_batch* b, int32_t use_graph, void* stream);
/* Synchronises `stream` and copies every query's group count and status (QDB_OK / QDB_HASH_TABLE_FULL) of the
 * last run to host arrays of n entries (either may be NULL). */
int32_t qdb_gb_batch_fetch(qdb_gb_batch* b, int64_t* counts, int32_t* status, void* stream);
/* Device pointers of query `inst`'s results of the last run, valid until the next run or set: keys[count] as
 * int64, and one column of count 8-byte words per aggregate of agg_mask in bit order (MIN, MAX, SUM, AVG,
 * COUNT), column j starting col_stride words after column j - 1: integer results as int64 (the output-type
 * value sign-extended), float results as double (the output-type value widened exactly).  *n_cols receives
 * the number of aggregate columns.  The output types are the reference's O: V for MIN/MAX/SUM/AVG, int64 for
 * COUNT (GpuSqlDispatcherAggregationFunctions.cu:49-168). */
int32_t qdb_gb_batch_result(qdb_gb_batch* b, int32_t inst, const int64_t** keys, const void** cols,
                            int32_t* n_cols, int64_t* col_stride);
/* Copies the result region of queries [first, first + n) to host memory: for each query, max_groups + 2 rows of
 * (1 + n_cols) int64-sized words in the layout of qdb_gb_batch_result (keys first, then each column).
 * host_bytes is the size of `host`; the needed size is returned in *needed (call with host == NULL to ask). */
int32_t qdb_gb_batch_copy_results(qdb_gb_batch* b, int32_t first, int32_t n, void* host, int64_t host_bytes,
                                  int64_t* needed, void* stream);
/* Reads and overrides the plan of query `inst` (the override lasts until the next qdb_gb_batch_set). */
int32_t qdb_gb_batch_get_cfg(qdb_gb_batch* b, int32_t inst, qdb_gb_batch_cfg* cfg);
int32_t qdb_gb_batch_set_cfg(qdb_gb_batch* b, int32_t inst, const qdb_gb_batch_cfg* cfg);
/* Times candidate plans on the batch's own queries (one run per candidate, every work item timed on the device)
 * and records, per query class (value type, cardinality, rows), the plan with the lowest SM-time per row in the
 * process-wide tuning table; then re-plans the batch from it.  Synchronises `stream`. */
int32_t qdb_gb_batch_autotune(qdb_gb_batch* b, void* stream);
/* Device time of the last run's aggregation kernel per work item, summed per query, in nanoseconds
 * (host array of n entries; requires a run after qdb_gb_batch_autotune or with timing enabled). */
int32_t qdb_gb_batch_item_times(qdb_gb_batch* b, int64_t* ns, void* stream);
/* Device bytes that qdb_gb_batch_set needs for the tables and the results of these queries (for sizing a batch
 * or admitting queries against a memory budget). */
int32_t qdb_gb_batch_required(const qdb_gb_query* queries, int32_t n, int64_t* table_bytes, int64_t* result_bytes);
/* share != 0 (the default): queries of the batch that read the same columns (same key, value and predicate
 * columns and row count) and run with the same warp-group width are aggregated in one scan, up to 8 per scan,
 * as long as their shared-memory tables fit one warp group together; each column tile is then loaded once for
 * all of them.  share == 0: every query scans its columns on its own.  Re-plans the batch. */
int32_t qdb_gb_batch_set_sharing(qdb_gb_batch* b, int32_t share);
/* Clears the process-wide tuning table (plans fall back to the built-in heuristic). */
int32_t qdb_gb_batch_tuning_reset(void);
/* The one-query-at-a-time path the batch replaces, looped in C: for each query in turn, as the dispatcher runs a
 * GROUP BY (GpuSqlDispatcherAggregationFunctions.h:377-507): the `key % key_mod` column when key_mod > 0
 * (GPUBinary<mod>), a table of max_groups (qdb_gb_create), ProcessBlock with the fused WHERE and the Swap check
 * (qdb_gb_process_sync), GetResults of every aggregate (qdb_gb_results_multi), with results_to_host != 0 the keys
 * and aggregate columns copied to host memory, then every buffer freed and the table destroyed.  out_groups[i]
 * (optional) receives query i's group count.  Returns at the first failing query; synchronises `stream`. */
int32_t qdb_gb_plain_run(const qdb_gb_query* queries, int32_t n, int32_t results_to_host, int64_t* out_groups,
                         void* stream);

/* ---- serving loop: continuous batching of GROUP BY queries over device-resident columns ----
 * No counterpart in the reference: its server hands every query to a dispatcher that runs the operators one
 * query at a time per GPU (qikkDB/QueryEngine/GpuSqlDispatcher.cpp, TCPClientHandler).  Here queries are
 * submitted from any thread and return at once with a ticket; one scheduler thread keeps up to `in_flight`
 * batches on the GPU (each on its own stream, executed by the batch engine above, so their work overlaps on the
 * device), admits pending queries in arrival order into the next free batch while their hash tables fit the
 * table budget (table_budget_bytes over all batches in flight, split evenly between them) and their results
 * fit the result budget, and on completion copies every query's results to host memory.  Large queries (see
 * qdb_server_set_plain_route) take a slot alone through the single-query operators instead.  A query whose
 * max_groups is 0 gets its table sized from a cardinality estimate (a sample of its key column, GEE estimator of
 * Charikar, Chaudhuri, Motwani and Narasayya, PODS 2000, capped by key_mod); a query that reports
 * QDB_HASH_TABLE_FULL is resubmitted with twice the table, like the dispatcher's restart on GPU_HASH_TABLE_FULL
 * (GpuSqlDispatcherAggregationFunctions.h:452-470).  The columns must stay allocated until the query is done. */
typedef struct qdb_server qdb_server; /* opaque serving loop */

typedef struct qdb_server_result {
    int32_t status;          /* QDB_OK, or the query's error */
    int32_t n_cols;          /* aggregate columns (agg_mask bits in the order MIN, MAX, SUM, AVG, COUNT) */
    int64_t n_groups;
    const int64_t* keys;     /* host: n_groups keys as int64 (owned by the server until qdb_server_release) */
    const int64_t* cols;     /* host: column j at cols + j * n_groups, 8-byte words as in qdb_gb_batch_result */
    int64_t submit_ns;       /* steady-clock timestamps (ns) */
    int64_t start_ns;        /* when its (last) batch was launched */
    int64_t done_ns;         /* when its results were on the host */
    int32_t retries;         /* resubmissions after HASH_TABLE_FULL */
    int32_t batch_size;      /* queries in the batch that completed it */
    int64_t max_groups;      /* table capacity it finally ran with */
} qdb_server_result;

typedef struct qdb_server_stats {
    int64_t submitted, completed, batches, retries, rejected;
    int64_t queries_in_batches; /* sum of batch sizes (mean batch size = queries_in_batches / batches) */
    int64_t table_budget_bytes; /* the table budget the server admits against (after the free-HBM cut) */
    int64_t hbm_free_at_create; /* free device memory when the server was created (cudaMemGetInfo) */
    int64_t plain_queries;      /* queries run alone through the single-query operators (qdb_server_set_plain_route) */
} qdb_server_stats;

/* table_budget_bytes is cut down to the device memory free at creation less a reserve (an eighth of the free
 * memory, at least 2 GiB) and the result budget; <= 0 takes all of that.  QDB_ERR_NOMEM when nothing is left. */
int32_t qdb_server_create(qdb_server** out, int32_t max_batch, int32_t in_flight, int64_t table_budget_bytes,
                          int64_t result_budget_bytes);
/* Waits for the queries in flight, stops the scheduler and frees everything (tickets included). */
int32_t qdb_server_destroy(qdb_server* s);
/* Thread-safe; copies the query.  *ticket identifies it in qdb_server_wait / qdb_server_release. */
int32_t qdb_server_submit(qdb_server* s, const qdb_gb_query* q, uint64_t* ticket);
/* Blocks until the query is done or timeout_ms passes (QDB_ERR_TIMEOUT; timeout_ms < 0 waits for ever). */
int32_t qdb_server_wait(qdb_server* s, uint64_t ticket, int64_t timeout_ms, qdb_server_result* out);
/* Frees a finished ticket and its host results. */
int32_t qdb_server_release(qdb_server* s, uint64_t ticket);
int32_t qdb_server_stats_get(qdb_server* s, qdb_server_stats* out);
/* Queries of at least min_rows rows, or whose table capacity (given, or the cardinality estimate) is at least
 * min_groups, skip the batch engine and run alone on a slot through the single-query operators: qdb_gb_create,
 * qdb_gb_process_mod (key % key_mod fused into the pass) or qdb_gb_process, with the fused WHERE, then
 * qdb_gb_results_multi, their results converted to the words of qdb_gb_batch_result.  Batching pays for small
 * queries, whose launch and synchronisation costs it removes; a large query amortises those, and the single-query
 * fast pass (shared table plus hash-partitioned spill) hashes its rows faster than the batch kernel.  A threshold
 * <= 0 is off.  The batch engine still takes single-query-path queries' places in arrival order: the oldest pending
 * query, if it is for the single-query path, takes the next free slot alone.  Defaults: min_rows 2^22, min_groups
 * off. */
int32_t qdb_server_set_plain_route(qdb_server* s, int64_t min_rows, int64_t min_groups);
/* Open-loop driver: submits queries[i] when arrival_ns[i] (ns after the call, non-decreasing) has come, whatever
 * is still in flight, waits for all of them and writes latency_ns[i] = results on host - arrival time (so queueing
 * delay counts) and status[i]; tickets are released.  *wall_ns = first arrival to last completion. */
int32_t qdb_server_run_open_loop(qdb_server* s, const qdb_gb_query* queries, int32_t n, const int64_t* arrival_ns,
                                 int64_t* latency_ns, int32_t* status, int64_t* wall_ns);

#ifdef __cplusplus
}
#endif

#endif /* QDB_GB_H */
