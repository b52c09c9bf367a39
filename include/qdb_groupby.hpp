/*
 * qdb_groupby.hpp - C++ drop-in for qikkDB's GROUP BY operator templates, implemented on the C ABI of qdb_gb.h.
 *
 * A caller written against the reference's operators keeps its code: the class and function names, template
 * parameters, argument order and meaning, output ownership (outputs allocated on the device, released with
 * GPUMemory::free) and error behaviour (a query_engine_error carrying the QueryEngineErrorType) are those of
 *   GPUGroupBy<AGG,O,K,V>                 qikkDB/QueryEngine/GPUCore/GPUGroupBy.cuh:285-790
 *   GPUGroupBy<AGG,O,std::vector<void*>,V> qikkDB/QueryEngine/GPUCore/GPUGroupByMultiKey.cuh:262-912
 *   GPUGroupBy<AGG,O,std::string,V>       qikkDB/QueryEngine/GPUCore/GPUGroupByString.cuh:171-785
 *   GPUBinary<FilterConditions::OP,int8_t,L,R>::Binary   GPUBinary.cuh:555-579
 *   GPUReconstruct::{reconstructColKeep, reconstructCol, GenerateIndexesKeep, GenerateIndexes, PrefixSum,
 *                    CompressNullMask}   GPUReconstruct.cuh:204-640
 *   GPUOrderBy::{OrderByColumn, ReOrderByIdx, ReOrderNullValuesByIdx}   GPUOrderBy.cuh:88-195
 *   GPUAggregation::col<AGG, OUT, IN>      GPUAggregation.cuh:15-37
 *   CompressionGPU::{compressDataAAFL, decompressDataAAFL, decompressDataAAFLOnDevice}
 *                                          qikkDB/Compression/GPUCompression.h:10-80
 *   GPUMemory::{alloc, allocAndSet, free, copyHostToDevice, copyDeviceToHost, copyDeviceToDevice, memset}
 *                                          GPUMemory.cuh:18-236
 *   query_engine_error / gpu_error / QueryEngineErrorType   qikkDB/QueryEngine/GPUError.h:17-75
 * Everything runs on the legacy default stream and every operator returns after its work is done, as the
 * reference's operators do; the library behind it is qikkdb_b200/libqdbgb.so (link with -lqdbgb).
 *
 * Differences a caller can see: a table may be created for K, V in {int32_t, int64_t, float, double}; the
 * multi-key form takes two COLUMN_INT key columns (other key type lists raise GPU_EXTENSION_ERROR); AGG avg
 * and min/max/sum require O == V and count requires O == int64_t (checked at compile time, as the reference's
 * dispatch tables pair them); float SUM/AVG are accumulated to FP64 accuracy.
 */
#ifndef QDB_GROUPBY_HPP
#define QDB_GROUPBY_HPP

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "qdb_gb.h"

typedef uint64_t nullmask_t;  /* bit-packed NULL flags: bit i%64 of word i/64 (NullValues.cuh:6-12) */
typedef uint8_t nullarray_t;  /* one byte per row (NullValues.cuh) */

/* Status values of the reference's error enum; the library's qdb_status 0..8 carry the same numbers. */
enum QueryEngineErrorType {
    GPU_EXTENSION_SUCCESS = 0,
    GPU_EXTENSION_ERROR,
    GPU_DIVISION_BY_ZERO_ERROR,
    GPU_INTEGER_OVERFLOW_ERROR,
    GPU_HASH_TABLE_FULL,
    GPU_UNKNOWN_AGG_FUN,
    GPU_NOT_FOUND_ERROR,
    GPU_MEMORY_MAPPING_NOT_SUPPORTED_ERROR,
    GPU_DRIVER_NOT_FOUND_EXCEPTION
};

/* Column type codes (qikkDB/DataType.h:7-27); the library's qdb_type uses the COLUMN_* numbers. */
enum DataType {
    CONST_ERROR = -1,
    CONST_INT = 0,
    CONST_LONG = 1,
    CONST_FLOAT = 2,
    CONST_DOUBLE = 3,
    CONST_POINT = 4,
    CONST_POLYGON = 5,
    CONST_STRING = 6,
    CONST_INT8_T = 7,
    COLUMN_INT = 8,
    COLUMN_LONG = 9,
    COLUMN_FLOAT = 10,
    COLUMN_DOUBLE = 11,
    COLUMN_POINT = 12,
    COLUMN_POLYGON = 13,
    COLUMN_STRING = 14,
    COLUMN_INT8_T = 15,
    DATA_TYPE_SIZE = 16
};

/* A failed CUDA call or library-side argument check (codes >= 100 of qdb_status). */
class gpu_error : public std::runtime_error {
public:
    explicit gpu_error(const std::string& what_arg) : std::runtime_error(what_arg) {}
};

/* A query-engine condition such as GPU_HASH_TABLE_FULL, which the caller may handle (grow and restart). */
class query_engine_error : public gpu_error {
public:
    query_engine_error(QueryEngineErrorType type, const std::string& message)
        : gpu_error("query engine error " + std::to_string(static_cast<int>(type)) +
                    (message.empty() ? std::string() : ": " + message)),
          type_(type) {}
    QueryEngineErrorType GetQueryEngineError() const { return type_; }

private:
    QueryEngineErrorType type_;
};

/* Throws unless type is GPU_EXTENSION_SUCCESS (GPUError.cpp:42-60). */
inline void CheckQueryEngineError(QueryEngineErrorType type, const std::string& message = std::string()) {
    if (type != GPU_EXTENSION_SUCCESS) throw query_engine_error(type, message);
}

namespace qdb_cpp {

/* Turns a qdb_status into the reference's exception: 1..8 query_engine_error, library codes gpu_error. */
inline void check(int32_t status) {
    if (status == QDB_OK) return;
    const std::string msg = qdb_last_error();
    if (status > 0 && status <= GPU_DRIVER_NOT_FOUND_EXCEPTION)
        throw query_engine_error(static_cast<QueryEngineErrorType>(status), msg);
    throw gpu_error("qikkdb_b200 status " + std::to_string(status) + ": " + msg);
}

template <typename T>
struct type_of;
template <> struct type_of<int32_t> { static constexpr int32_t code = QDB_INT32; };
template <> struct type_of<int64_t> { static constexpr int32_t code = QDB_INT64; };
template <> struct type_of<float> { static constexpr int32_t code = QDB_FLOAT; };
template <> struct type_of<double> { static constexpr int32_t code = QDB_DOUBLE; };
template <> struct type_of<int8_t> { static constexpr int32_t code = QDB_INT8; };

inline void sync() { check(qdb_stream_sync(nullptr)); }

inline int32_t current_device() {
    int32_t d = 0;
    check(qdb_get_device(&d));
    return d;
}

/* Makes `device` current for the lifetime of the guard (tables of other GPUs are exported on their own). */
class device_guard {
public:
    explicit device_guard(int32_t device) : prev_(current_device()) {
        if (device != prev_) check(qdb_set_device(device));
    }
    ~device_guard() { qdb_set_device(prev_); }
    device_guard(const device_guard&) = delete;
    device_guard& operator=(const device_guard&) = delete;

private:
    int32_t prev_;
};

}  // namespace qdb_cpp

/* ---- GPUMemory (GPUMemory.cuh:18-236): device buffers of the library's stream-ordered pool ---- */
namespace GPUMemory {
template <typename T>
inline void alloc(T** p, size_t dataElementCount) {
    void* v = nullptr;
    qdb_cpp::check(qdb_malloc(&v, static_cast<int64_t>(dataElementCount * sizeof(T)), nullptr));
    *p = static_cast<T*>(v);
}
template <typename T>
inline void allocAndSet(T** p, int32_t value, size_t dataElementCount) {
    alloc(p, dataElementCount);
    qdb_cpp::check(qdb_memset(*p, value, static_cast<int64_t>(dataElementCount * sizeof(T)), nullptr));
}
template <typename T>
inline void free(T* p) {
    if (p) qdb_cpp::check(qdb_free(const_cast<void*>(static_cast<const void*>(p)), nullptr));
}
template <typename T>
inline void memset(T* p, int32_t value, size_t dataElementCount) {
    qdb_cpp::check(qdb_memset(p, value, static_cast<int64_t>(dataElementCount * sizeof(T)), nullptr));
}
template <typename T>
inline void copyHostToDevice(T* dst, const T* src, size_t dataElementCount) {
    qdb_cpp::check(qdb_memcpy_h2d(dst, src, static_cast<int64_t>(dataElementCount * sizeof(T)), nullptr));
    qdb_cpp::sync();
}
template <typename T>
inline void copyDeviceToHost(T* dst, const T* src, size_t dataElementCount) {
    qdb_cpp::check(qdb_memcpy_d2h(dst, src, static_cast<int64_t>(dataElementCount * sizeof(T)), nullptr));
    qdb_cpp::sync();
}
template <typename T>
inline void copyDeviceToDevice(T* dst, const T* src, size_t dataElementCount) {
    qdb_cpp::check(qdb_memcpy_d2d(dst, src, static_cast<int64_t>(dataElementCount * sizeof(T)), nullptr));
}
/* Words of a null bitmask for dataElementCount rows (NullValues.cu:13-16). */
inline size_t CalculateNullMaskSize(size_t dataElementCount) { return (dataElementCount + 63) / 64; }
/* A device string column (GPUMemory.cuh GPUString): every string's characters concatenated, and the int64 end
 * offset of each string (string i is allChars[i ? stringIndices[i-1] : 0, stringIndices[i])). */
struct GPUString {
    char* allChars;
    int64_t* stringIndices;
};
inline void free(GPUString s) {
    free(s.allChars);
    free(s.stringIndices);
}
}  // namespace GPUMemory

/* Owning device pointer (cuda_ptr.h): freed with GPUMemory::free. */
template <typename T>
class cuda_ptr {
public:
    cuda_ptr() = default;
    explicit cuda_ptr(size_t dataElementCount) { GPUMemory::alloc(&p_, dataElementCount); }
    cuda_ptr(size_t dataElementCount, int32_t value) { GPUMemory::allocAndSet(&p_, value, dataElementCount); }
    explicit cuda_ptr(T* adopt) : p_(adopt) {}
    ~cuda_ptr() { reset(); }
    cuda_ptr(cuda_ptr&& o) noexcept : p_(o.p_) { o.p_ = nullptr; }
    cuda_ptr& operator=(cuda_ptr&& o) noexcept {
        if (this != &o) {
            reset();
            p_ = o.p_;
            o.p_ = nullptr;
        }
        return *this;
    }
    cuda_ptr(const cuda_ptr&) = delete;
    cuda_ptr& operator=(const cuda_ptr&) = delete;
    T* get() const { return p_; }
    T* release() {
        T* p = p_;
        p_ = nullptr;
        return p;
    }
    void reset() {
        if (p_) qdb_free(p_, nullptr);
        p_ = nullptr;
    }

private:
    T* p_ = nullptr;
};

/* ---- AggregationFunctions (AggregationFunctions.cuh:17-366): tags selecting the aggregate ---- */
namespace AggregationFunctions {
struct min { static constexpr int32_t bit = QDB_AGG_MIN; };
struct max { static constexpr int32_t bit = QDB_AGG_MAX; };
struct sum { static constexpr int32_t bit = QDB_AGG_SUM; };
struct avg { static constexpr int32_t bit = QDB_AGG_AVG; };
struct count { static constexpr int32_t bit = QDB_AGG_COUNT; };
struct none { static constexpr int32_t bit = 0; };
}  // namespace AggregationFunctions

/* ---- FilterConditions (GPUFilterConditions.cuh:9-180): comparison and logical functors ---- */
namespace FilterConditions {
struct greater {
    static constexpr int32_t code = QDB_GREATER;
    template <typename T, typename U> bool operator()(T a, U b) const { return a > b; }
};
struct greaterEqual {
    static constexpr int32_t code = QDB_GREATER_EQUAL;
    template <typename T, typename U> bool operator()(T a, U b) const { return a >= b; }
};
struct less {
    static constexpr int32_t code = QDB_LESS;
    template <typename T, typename U> bool operator()(T a, U b) const { return a < b; }
};
struct lessEqual {
    static constexpr int32_t code = QDB_LESS_EQUAL;
    template <typename T, typename U> bool operator()(T a, U b) const { return a <= b; }
};
struct equal {
    static constexpr int32_t code = QDB_EQUAL;
    template <typename T, typename U> bool operator()(T a, U b) const { return a == b; }
};
struct notEqual {
    static constexpr int32_t code = QDB_NOT_EQUAL;
    template <typename T, typename U> bool operator()(T a, U b) const { return a != b; }
};
struct logicalAnd {
    static constexpr int32_t code = QDB_LOGICAL_AND;
    template <typename T, typename U> bool operator()(T a, U b) const { return a && b; }
};
struct logicalOr {
    static constexpr int32_t code = QDB_LOGICAL_OR;
    template <typename T, typename U> bool operator()(T a, U b) const { return a || b; }
};
}  // namespace FilterConditions

/* Base of every table (IGroupBy.h): lets a dispatcher keep one table per GPU in one vector. */
class IGroupBy {
protected:
    IGroupBy() = default;

public:
    virtual ~IGroupBy() = default;
};

constexpr int32_t GB_VALUE_BUFFER_DEFAULT_MULTIPLIER = 256;
constexpr size_t GB_BUFFER_SIZE_MAX = size_t(1) << 30;

namespace qdb_cpp {

/* The table handle shared by the single- and multi-key forms: creation, one fused ProcessBlock, results of one
 * aggregate, and the cross-GPU merge of GetResults(..., tables). */
class table {
public:
    table(int32_t agg_bit, int32_t key_type, int32_t n_key_cols, int32_t val_type, int64_t max_groups)
        : agg_(agg_bit), n_key_cols_(n_key_cols), device_(current_device()) {
        check(qdb_gb_create(&gb_, agg_bit, key_type, n_key_cols, agg_bit ? val_type : 0, max_groups, QDB_PLACE_AUTO,
                            nullptr));
        key_type_ = key_type;
        val_type_ = agg_bit ? val_type : 0;
        max_groups_ = max_groups;
    }
    ~table() {
        if (gb_) qdb_gb_destroy(gb_);
    }
    table(const table&) = delete;
    table& operator=(const table&) = delete;

    /* ProcessBlock + ErrorFlagSwapper::Swap: throws GPU_HASH_TABLE_FULL when the keys overflow the table. */
    void process(const void* const* keys, const nullmask_t* const* key_nulls, const void* vals,
                 const nullmask_t* val_nulls, int32_t n) {
        if (n <= 0) return;
        check(qdb_gb_process_sync(gb_, keys, reinterpret_cast<const uint64_t* const*>(key_nulls),
                                  val_type_ ? vals : nullptr, val_type_ ? val_nulls : nullptr, n, nullptr, nullptr,
                                  nullptr));
    }

    /* GetResults for this table's aggregate: newly allocated device columns (NULL when there are no groups). */
    void results(void** out_keys, nullmask_t** out_key_nulls, void** out_vals, nullmask_t** out_val_nulls,
                 int32_t* out_count) {
        int64_t count = 0;
        check(qdb_gb_results(gb_, agg_, out_keys, reinterpret_cast<uint64_t**>(out_key_nulls), agg_ ? out_vals : nullptr,
                             agg_ ? reinterpret_cast<uint64_t**>(out_val_nulls) : nullptr, &count, nullptr));
        *out_count = static_cast<int32_t>(count);
    }

    /* Merges every occupied slot of `src` (a table of the same shape, on any GPU) into this table. */
    void merge_from(table& src) {
        uint64_t *keys = nullptr, *state = nullptr;
        uint8_t* flags = nullptr;
        int64_t count = 0;
        {
            device_guard g(src.device_);
            check(qdb_gb_export_partitioned(src.gb_, 1, &keys, &state, &flags, &count, nullptr));
        }
        if (count == 0) return;
        int32_t words = 0;
        check(qdb_gb_state_words(gb_, &words));
        cuda_ptr<uint64_t> k, s;
        cuda_ptr<uint8_t> f;
        if (src.device_ == device_) {
            k = cuda_ptr<uint64_t>(keys);
            s = cuda_ptr<uint64_t>(state);
            f = cuda_ptr<uint8_t>(flags);
        } else {
            /* records of another GPU are copied into this GPU's memory first, then released on their own GPU */
            k = cuda_ptr<uint64_t>(static_cast<size_t>(count));
            f = cuda_ptr<uint8_t>(static_cast<size_t>(count));
            check(qdb_memcpy_peer(k.get(), device_, keys, src.device_, count * 8));
            check(qdb_memcpy_peer(f.get(), device_, flags, src.device_, count));
            if (words > 0) {
                s = cuda_ptr<uint64_t>(static_cast<size_t>(count) * words);
                check(qdb_memcpy_peer(s.get(), device_, state, src.device_, count * words * 8));
            }
            device_guard g(src.device_);
            qdb_free(keys, nullptr);
            qdb_free(state, nullptr);
            qdb_free(flags, nullptr);
            sync();
        }
        check(qdb_gb_merge_partial(gb_, k.get(), s.get(), f.get(), count, nullptr));
        check(qdb_gb_check(gb_, nullptr));
    }

    int64_t max_hash_count() const {
        int64_t v = 0;
        check(qdb_gb_max_hash_count(gb_, &v));
        return v;
    }
    int64_t max_groups() const { return max_groups_; }
    int32_t agg() const { return agg_; }
    int32_t key_type() const { return key_type_; }
    int32_t val_type() const { return val_type_; }
    int32_t n_key_cols() const { return n_key_cols_; }

private:
    qdb_gb* gb_ = nullptr;
    int32_t agg_;
    int32_t n_key_cols_;
    int32_t device_;
    int32_t key_type_ = 0;
    int32_t val_type_ = 0;
    int64_t max_groups_ = 0;
};

inline int64_t table_size(int32_t maxHashCount, int32_t keySizeMultiplier) {
    const int64_t want = static_cast<int64_t>(maxHashCount) * keySizeMultiplier;
    return want < static_cast<int64_t>(GB_BUFFER_SIZE_MAX) ? want : static_cast<int64_t>(GB_BUFFER_SIZE_MAX);
}

template <typename AGG, typename O, typename V>
constexpr bool output_type_ok() {
    return std::is_same<AGG, AggregationFunctions::count>::value ? std::is_same<O, int64_t>::value
                                                                 : (std::is_same<AGG, AggregationFunctions::none>::value ||
                                                                    std::is_same<O, V>::value);
}

}  // namespace qdb_cpp

/* ---- GPUGroupBy<AGG, O, K, V>: single-key GROUP BY table (GPUGroupBy.cuh:285-790) ---- */
template <typename AGG, typename O, typename K, typename V>
class GPUGroupBy : public IGroupBy {
    static_assert(qdb_cpp::output_type_ok<AGG, O, V>(),
                  "GROUP BY output type: O must be int64_t for COUNT and V for MIN, MAX, SUM and AVG");

public:
    /* GPUGroupBy(maxHashCount, keySizeMultiplier) (GPUGroupBy.cuh:313): a table for up to
     * min(maxHashCount * keySizeMultiplier, 2^30) distinct non-NULL keys. */
    GPUGroupBy(const int32_t maxHashCount, const int32_t keySizeMultiplier)
        : t_(AGG::bit, qdb_cpp::type_of<K>::code, 1, qdb_cpp::type_of<V>::code,
             qdb_cpp::table_size(maxHashCount, keySizeMultiplier)) {}

    /* GPUGroupBy(maxHashCount, keys, firstKeyIsNull) (GPUGroupBy.cuh:367): a table that already holds the
     * maxHashCount device keys `keys` (keys[0] stands for the NULL key when firstKeyIsNull), each with no value
     * yet; used to gather the key set of several tables before their values are merged. */
    GPUGroupBy(const int32_t maxHashCount, K* keys, bool firstKeyIsNull)
        : t_(AGG::bit, qdb_cpp::type_of<K>::code, 1, qdb_cpp::type_of<V>::code,
             static_cast<int64_t>(maxHashCount) - (firstKeyIsNull ? 1 : 0)) {
        if (maxHashCount <= 0) return;
        /* The keys enter as a block whose rows all have NULL values: every key becomes a group, no aggregate
         * changes, and a NULL first key becomes the NULL-key group. */
        const size_t words = GPUMemory::CalculateNullMaskSize(static_cast<size_t>(maxHashCount));
        std::vector<nullmask_t> kn(words, 0), vn(words, ~nullmask_t(0));
        if (firstKeyIsNull) kn[0] = 1;
        cuda_ptr<nullmask_t> dkn(words), dvn(words);
        cuda_ptr<V> vals(static_cast<size_t>(maxHashCount), 0);
        GPUMemory::copyHostToDevice(dkn.get(), kn.data(), words);
        GPUMemory::copyHostToDevice(dvn.get(), vn.data(), words);
        const void* kc[1] = {keys};
        const nullmask_t* knc[1] = {dkn.get()};
        t_.process(kc, knc, vals.get(), dvn.get(), maxHashCount);
    }

    GPUGroupBy(const GPUGroupBy&) = delete;
    GPUGroupBy& operator=(const GPUGroupBy&) = delete;

    /* ProcessBlock (GPUGroupBy.cuh:395): aggregates one block; throws query_engine_error(GPU_HASH_TABLE_FULL)
     * when the block brings more distinct keys than the table holds. */
    void ProcessBlock(K* inKeys, V* inValues, int32_t dataElementCount, nullmask_t* inKeysNullMask = nullptr,
                      nullmask_t* inValuesNullMask = nullptr) {
        const void* kc[1] = {inKeys};
        const nullmask_t* knc[1] = {inKeysNullMask};
        t_.process(kc, inKeysNullMask ? knc : nullptr, inValues, inValuesNullMask, dataElementCount);
    }

    /* GetMaxHashCount (GPUGroupBy.cuh:414). */
    int32_t GetMaxHashCount() { return static_cast<int32_t>(t_.max_hash_count()); }

    /* GetResults (GPUGroupBy.cuh:478): newly allocated device keys and values (free with GPUMemory::free); an
     * empty result leaves NULL pointers and a count of 0.  outValues stays NULL for AGG none. */
    void GetResults(K** outKeys, O** outValues, int32_t* outDataElementCount, nullmask_t** outKeysNullMask = nullptr,
                    nullmask_t** outValuesNullMask = nullptr) {
        void* k[1] = {nullptr};
        nullmask_t* kn[1] = {nullptr};
        void* v = nullptr;
        t_.results(k, outKeysNullMask ? kn : nullptr, outValues ? &v : nullptr, outValuesNullMask, outDataElementCount);
        *outKeys = static_cast<K*>(k[0]);
        if (outKeysNullMask) *outKeysNullMask = kn[0];
        if (outValues) *outValues = static_cast<O*>(v);
    }

    /* GetResults over the tables of every GPU (GPUGroupBy.cuh:594): the partial states of all tables are merged
     * into a new table on the current GPU, whose results are returned. */
    void GetResults(K** outKeys, O** outValues, int32_t* outDataElementCount,
                    std::vector<std::unique_ptr<IGroupBy>>& tables, nullmask_t** outKeysNullMask = nullptr,
                    nullmask_t** outValuesNullMask = nullptr) {
        if (tables.size() <= 1) {
            GetResults(outKeys, outValues, outDataElementCount, outKeysNullMask, outValuesNullMask);
            return;
        }
        int64_t groups = 0;
        for (auto& tb : tables) groups += static_cast<GPUGroupBy*>(tb.get())->t_.max_groups();
        GPUGroupBy merged(static_cast<int32_t>(groups < INT32_MAX ? groups : INT32_MAX), 1);
        for (auto& tb : tables) merged.t_.merge_from(static_cast<GPUGroupBy*>(tb.get())->t_);
        merged.GetResults(outKeys, outValues, outDataElementCount, outKeysNullMask, outValuesNullMask);
    }

private:
    qdb_cpp::table t_;
};

/* ---- GPUGroupBy<AGG, O, std::vector<void*>, V>: composite-key GROUP BY (GPUGroupByMultiKey.cuh:262-912) ---- */
template <typename AGG, typename O, typename V>
class GPUGroupBy<AGG, O, std::vector<void*>, V> : public IGroupBy {
    static_assert(qdb_cpp::output_type_ok<AGG, O, V>(),
                  "GROUP BY output type: O must be int64_t for COUNT and V for MIN, MAX, SUM and AVG");

public:
    /* GPUGroupBy(maxHashCount, keySizeMultiplier, keyTypes) (GPUGroupByMultiKey.cuh:330); keyTypes must be
     * {COLUMN_INT, COLUMN_INT}. */
    GPUGroupBy(const int32_t maxHashCount, const int32_t keySizeMultiplier, const std::vector<DataType>& keyTypes)
        : keyTypes_(checked(keyTypes)),
          t_(AGG::bit, QDB_INT32, 2, qdb_cpp::type_of<V>::code, qdb_cpp::table_size(maxHashCount, keySizeMultiplier)) {}

    GPUGroupBy(const GPUGroupBy&) = delete;
    GPUGroupBy& operator=(const GPUGroupBy&) = delete;

    /* ProcessBlock (GPUGroupByMultiKey.cuh:535). */
    void ProcessBlock(std::vector<void*> inKeysVector, std::vector<nullmask_t*> inKeysNullMaskVector, V* inValues,
                      int32_t dataElementCount, nullmask_t* inValuesNullMask = nullptr) {
        if (dataElementCount <= 0) return;
        if (inKeysVector.size() != keyTypes_.size())
            CheckQueryEngineError(GPU_EXTENSION_ERROR, "Incorrect number of key columns in ProcessBlock");
        const void* kc[2] = {inKeysVector[0], inKeysVector[1]};
        const nullmask_t* knc[2] = {nullptr, nullptr};
        bool any_null = false;
        for (size_t c = 0; c < 2 && c < inKeysNullMaskVector.size(); ++c) {
            knc[c] = inKeysNullMaskVector[c];
            any_null = any_null || knc[c];
        }
        t_.process(kc, any_null ? knc : nullptr, inValues, inValuesNullMask, dataElementCount);
    }

    int32_t GetMaxHashCount() { return static_cast<int32_t>(t_.max_hash_count()); }

    /* GetResults (GPUGroupByMultiKey.cuh:742): one newly allocated device column per key (release them with
     * FreeKeysVector), the values, and optional null masks. */
    void GetResults(std::vector<void*>* outKeysVector, O** outValues, int32_t* outDataElementCount,
                    std::vector<nullmask_t*>* outKeysNullMasksVector = nullptr, nullmask_t** outValuesNullMask = nullptr) {
        void* k[2] = {nullptr, nullptr};
        nullmask_t* kn[2] = {nullptr, nullptr};
        void* v = nullptr;
        t_.results(k, outKeysNullMasksVector ? kn : nullptr, outValues ? &v : nullptr, outValuesNullMask,
                   outDataElementCount);
        outKeysVector->assign(k, k + 2);
        if (outKeysNullMasksVector) outKeysNullMasksVector->assign(kn, kn + 2);
        if (outValues) *outValues = static_cast<O*>(v);
    }

private:
    static const std::vector<DataType>& checked(const std::vector<DataType>& kt) {
        if (kt.size() != 2 || kt[0] != COLUMN_INT || kt[1] != COLUMN_INT)
            CheckQueryEngineError(GPU_EXTENSION_ERROR, "multi-key GROUP BY supports (COLUMN_INT, COLUMN_INT) keys");
        return kt;
    }
    std::vector<DataType> keyTypes_;
    qdb_cpp::table t_;
};

/* ---- GPUGroupBy<AGG, O, std::string, V>: GROUP BY over string keys (GPUGroupByString.cuh:171-785) ----
 * The keys arrive as a GPUString block.  The table keeps its own copy of every distinct key (a device arena of
 * 32 characters per group on average); GetResults returns the keys as a newly allocated GPUString (release it
 * with GPUMemory::free).  COUNT given no values (inValues NULL) counts rows. */
template <typename AGG, typename O, typename V>
class GPUGroupBy<AGG, O, std::string, V> : public IGroupBy {
    static_assert(qdb_cpp::output_type_ok<AGG, O, V>(),
                  "GROUP BY output type: O must be int64_t for COUNT and V for MIN, MAX, SUM and AVG");

public:
    /* GPUGroupBy(maxHashCount, keySizeMultiplier) (GPUGroupByString.cuh:210): up to
     * min(maxHashCount * keySizeMultiplier, 2^30) distinct non-NULL keys, plus the NULL key. */
    GPUGroupBy(const int32_t maxHashCount, const int32_t keySizeMultiplier)
        : max_groups_(qdb_cpp::table_size(maxHashCount, keySizeMultiplier)), device_(qdb_cpp::current_device()) {
        qdb_cpp::check(qdb_gbs_create(&g_, AGG::bit, AGG::bit ? qdb_cpp::type_of<V>::code : 0, max_groups_, 0, nullptr));
    }
    ~GPUGroupBy() {
        if (g_) qdb_gbs_destroy(g_);
    }
    GPUGroupBy(const GPUGroupBy&) = delete;
    GPUGroupBy& operator=(const GPUGroupBy&) = delete;

    /* ProcessBlock (GPUGroupByString.cuh:333): throws query_engine_error(GPU_HASH_TABLE_FULL) when the block
     * brings more distinct keys than the table holds. */
    void ProcessBlock(GPUMemory::GPUString inKeys, V* inValues, int32_t dataElementCount,
                      nullmask_t* inKeysNullMask = nullptr, nullmask_t* inValuesNullMask = nullptr) {
        if (dataElementCount <= 0) return;
        qdb_cpp::check(qdb_gbs_process(g_, inKeys.allChars, inKeys.stringIndices, inKeysNullMask,
                                       AGG::bit ? inValues : nullptr, AGG::bit ? inValuesNullMask : nullptr, nullptr,
                                       dataElementCount, nullptr));
        qdb_cpp::check(qdb_gbs_check(g_, nullptr));
    }

    /* GetMaxHashCount: the key buffer size, max_groups plus the NULL slot. */
    int32_t GetMaxHashCount() { return static_cast<int32_t>(max_groups_ + 1); }

    /* GetResults (GPUGroupByString.cuh:446): newly allocated keys and values (NULL pointers and a count of 0 for
     * an empty result).  outValues stays NULL for AGG none. */
    void GetResults(GPUMemory::GPUString* outKeys, O** outValues, int32_t* outDataElementCount,
                    nullmask_t** outKeysNullMask = nullptr, nullmask_t** outValuesNullMask = nullptr) {
        const int32_t agg = AGG::bit;
        void* v = nullptr;
        uint64_t* vn = nullptr;
        int64_t count = 0;
        qdb_cpp::check(qdb_gbs_results(g_, agg ? 1 : 0, &agg, &outKeys->allChars, &outKeys->stringIndices,
                                       reinterpret_cast<uint64_t**>(outKeysNullMask), agg ? &v : nullptr,
                                       agg && outValuesNullMask ? &vn : nullptr, &count, nullptr));
        *outDataElementCount = static_cast<int32_t>(count);
        if (outValues) *outValues = static_cast<O*>(v);
        else GPUMemory::free(v);
        if (outValuesNullMask) *outValuesNullMask = reinterpret_cast<nullmask_t*>(vn);
    }

    /* GetResults over the tables of every GPU (GPUGroupByString.cuh:565): every table's groups (key strings and
     * partial states) are merged into a new table on the current GPU, whose results are returned. */
    void GetResults(GPUMemory::GPUString* outKeys, O** outValues, int32_t* outDataElementCount,
                    std::vector<std::unique_ptr<IGroupBy>>& tables, nullmask_t** outKeysNullMask = nullptr,
                    nullmask_t** outValuesNullMask = nullptr) {
        if (tables.size() <= 1) {
            GetResults(outKeys, outValues, outDataElementCount, outKeysNullMask, outValuesNullMask);
            return;
        }
        int64_t groups = 0;
        for (auto& tb : tables) groups += static_cast<GPUGroupBy*>(tb.get())->max_groups_;
        GPUGroupBy merged(static_cast<int32_t>(groups < INT32_MAX ? groups : INT32_MAX), 1);
        for (auto& tb : tables) merged.merge_from(*static_cast<GPUGroupBy*>(tb.get()));
        merged.GetResults(outKeys, outValues, outDataElementCount, outKeysNullMask, outValuesNullMask);
    }

private:
    /* Adds every group of `src` (on any GPU) to this table. */
    void merge_from(GPUGroupBy& src) {
        char* chars = nullptr;
        int64_t* ends = nullptr;
        uint64_t* state = nullptr;
        uint8_t* flags = nullptr;
        int64_t n = 0;
        int32_t words = 0;
        {
            qdb_cpp::device_guard g(src.device_);
            qdb_cpp::check(qdb_gbs_export(src.g_, &chars, &ends, &state, &flags, &n, nullptr));
            qdb_cpp::check(qdb_gbs_state_words(src.g_, &words));
        }
        if (n == 0) return;
        if (src.device_ == device_) {
            qdb_cpp::check(qdb_gbs_merge_exported(g_, chars, ends, state, flags, n, nullptr));
            qdb_cpp::check(qdb_gbs_check(g_, nullptr));
            GPUMemory::free(chars);
            GPUMemory::free(ends);
            GPUMemory::free(state);
            GPUMemory::free(flags);
            return;
        }
        /* records of another GPU are copied into this GPU's memory first, then released on their own GPU */
        int64_t nchars = 0;
        {
            qdb_cpp::device_guard g(src.device_);
            GPUMemory::copyDeviceToHost(&nchars, ends + (n - 1), 1);
        }
        cuda_ptr<char> c(static_cast<size_t>(nchars > 0 ? nchars : 1));
        cuda_ptr<int64_t> e(static_cast<size_t>(n));
        cuda_ptr<uint64_t> st(static_cast<size_t>(n) * static_cast<size_t>(words > 0 ? words : 1));
        cuda_ptr<uint8_t> f(static_cast<size_t>(n));
        if (nchars > 0) qdb_cpp::check(qdb_memcpy_peer(c.get(), device_, chars, src.device_, nchars));
        qdb_cpp::check(qdb_memcpy_peer(e.get(), device_, ends, src.device_, n * 8));
        if (words > 0) qdb_cpp::check(qdb_memcpy_peer(st.get(), device_, state, src.device_, n * words * 8));
        qdb_cpp::check(qdb_memcpy_peer(f.get(), device_, flags, src.device_, n));
        {
            qdb_cpp::device_guard g(src.device_);
            GPUMemory::free(chars);
            GPUMemory::free(ends);
            GPUMemory::free(state);
            GPUMemory::free(flags);
            qdb_cpp::sync();
        }
        qdb_cpp::check(qdb_gbs_merge_exported(g_, c.get(), e.get(), st.get(), f.get(), n, nullptr));
        qdb_cpp::check(qdb_gbs_check(g_, nullptr));
    }

    qdb_gbs* g_ = nullptr;
    int64_t max_groups_;
    int32_t device_;
};

/* Releases the key columns returned by the multi-key GetResults (GPUGroupByMultiKey.cu:403-418). */
inline void FreeKeysVector(std::vector<void*> keysVector, std::vector<DataType> keyTypes) {
    for (size_t i = 0; i < keysVector.size() && i < keyTypes.size(); ++i) GPUMemory::free(keysVector[i]);
}

/* ---- GPUBinary<OP, int8_t, L, R>::Binary: filter mask (GPUBinary.cuh:555-579) ----
 * L and R are each a device column pointer (T*) or a constant (T); OP is a FilterConditions functor.
 * outMask[i] = OP(A[i], B[i]) && !null(i).  Constant-constant fills the mask. */
template <typename OP, typename OUT, typename L, typename R>
class GPUBinary {
    static_assert(std::is_same<OUT, int8_t>::value, "GPUBinary here implements the filter form (OUT = int8_t)");

    template <typename X>
    static void side(const X& x, int32_t& type, int32_t& is_col, const void*& ptr) {
        using T = typename std::remove_cv<typename std::remove_pointer<X>::type>::type;
        type = qdb_cpp::type_of<T>::code;
        if constexpr (std::is_pointer<X>::value) {
            is_col = 1;
            ptr = x;
        } else {
            is_col = 0;
            ptr = &x;  // a host pointer to the constant
        }
    }

public:
    static void Binary(int8_t* outMask, L ACol, R BCol, int32_t dataElementCount, nullmask_t* nullBitMask = nullptr) {
        int32_t at, ac, bt, bc;
        const void *ap, *bp;
        side(ACol, at, ac, ap);
        side(BCol, bt, bc, bp);
        qdb_cpp::check(qdb_filter(OP::code, at, ac, ap, bt, bc, bp, nullBitMask, outMask, dataElementCount, nullptr));
        qdb_cpp::sync();
    }
};

/* ---- GPUReconstruct: stream compaction by an int8 mask (GPUReconstruct.cuh:204-640) ---- */
class GPUReconstruct {
public:
    /* reconstructColKeep (GPUReconstruct.cuh:272): the rows of ACol whose mask byte is non-zero, in a newly
     * allocated device column (NULL when none is selected).  A NULL mask hands back ACol itself and
     * dataElementCount, as the reference does. */
    template <typename T>
    static void reconstructColKeep(T** outCol, int32_t* outDataElementCount, T* ACol, int8_t* inMask,
                                   int32_t dataElementCount, nullmask_t** outNullMask = nullptr,
                                   nullmask_t* nullMask = nullptr) {
        void* out = nullptr;
        uint64_t* onm = nullptr;
        int64_t count = 0;
        qdb_cpp::check(qdb_reconstruct_keep(static_cast<int32_t>(sizeof(T)), ACol, inMask, dataElementCount, &out,
                                            &count, nullMask, (outNullMask && nullMask) ? &onm : nullptr, nullptr));
        *outCol = static_cast<T*>(out);
        *outDataElementCount = static_cast<int32_t>(count);
        if (outNullMask) *outNullMask = nullMask ? reinterpret_cast<nullmask_t*>(onm) : nullptr;
    }

    /* reconstructCol (GPUReconstruct.cuh:204): as reconstructColKeep, into the HOST buffer outData (room for
     * dataElementCount rows) and, when both masks are given, the host null mask outNullMask. */
    template <typename T>
    static void reconstructCol(T* outData, int32_t* outDataElementCount, T* ACol, int8_t* inMask,
                               int32_t dataElementCount, nullmask_t* outNullMask = nullptr,
                               nullmask_t* nullMask = nullptr) {
        T* dev = nullptr;
        nullmask_t* dnm = nullptr;
        reconstructColKeep(&dev, outDataElementCount, ACol, inMask, dataElementCount,
                           (outNullMask && nullMask) ? &dnm : nullptr, nullMask);
        const int32_t n = *outDataElementCount;
        if (n > 0) GPUMemory::copyDeviceToHost(outData, dev, static_cast<size_t>(n));
        if (dnm && n > 0) GPUMemory::copyDeviceToHost(outNullMask, dnm, GPUMemory::CalculateNullMaskSize(n));
        if (inMask) {
            GPUMemory::free(dev);
            GPUMemory::free(dnm);
        }
    }

    /* GenerateIndexesKeep<int32_t, int8_t> (GPUReconstruct.cuh:518): row indices where the mask is non-zero, in a
     * newly allocated device array. */
    template <typename T, typename M>
    static void GenerateIndexesKeep(T** outData, int32_t* outDataElementCount, M* inMask, int32_t dataElementCount) {
        static_assert(std::is_same<T, int32_t>::value && sizeof(M) == 1, "indexes are int32_t over an int8_t mask");
        int32_t* out = nullptr;
        int64_t count = 0;
        qdb_cpp::check(qdb_generate_indexes(reinterpret_cast<const int8_t*>(inMask), dataElementCount, &out, &count,
                                            nullptr));
        *outData = out;
        *outDataElementCount = static_cast<int32_t>(count);
    }

    /* GenerateIndexes (GPUReconstruct.cuh:487): as GenerateIndexesKeep, into the HOST buffer outData. */
    template <typename T, typename M>
    static void GenerateIndexes(T* outData, int32_t* outDataElementCount, M* inMask, int32_t dataElementCount) {
        T* dev = nullptr;
        GenerateIndexesKeep(&dev, outDataElementCount, inMask, dataElementCount);
        if (*outDataElementCount > 0) GPUMemory::copyDeviceToHost(outData, dev, static_cast<size_t>(*outDataElementCount));
        GPUMemory::free(dev);
    }

    /* PrefixSum<int32_t, int8_t> (GPUReconstruct.cuh:573): inclusive running count of the mask into the device
     * array prefixSumPointer (dataElementCount entries). */
    template <typename T, typename M>
    static void PrefixSum(T* prefixSumPointer, M* inMask, int32_t dataElementCount) {
        static_assert(std::is_same<T, int32_t>::value && sizeof(M) == 1, "prefix sums are int32_t over an int8_t mask");
        qdb_cpp::check(qdb_prefix_sum(reinterpret_cast<const int8_t*>(inMask), dataElementCount, prefixSumPointer, nullptr));
        qdb_cpp::sync();
    }

    /* CompressNullMask (GPUReconstruct.cu:756-764): one NULL byte per row to a bit-packed device mask. */
    static cuda_ptr<nullmask_t> CompressNullMask(nullarray_t* inputNullArray, int32_t dataElementCount) {
        uint64_t* out = nullptr;
        qdb_cpp::check(qdb_compress_null_mask(inputNullArray, dataElementCount, &out, nullptr));
        qdb_cpp::sync();
        return cuda_ptr<nullmask_t>(reinterpret_cast<nullmask_t*>(out));
    }
};

/* ---- GPUAggregation::col<AGG, OUT, IN> (GPUAggregation.cuh:15-37): one aggregate of a whole device column into
 * the device value *outValue.  OUT is IN for MIN/MAX/SUM/AVG (an integer SUM wraps in IN, an integer AVG truncates)
 * and int64_t for COUNT; an empty column leaves 0. ---- */
class GPUAggregation {
public:
    template <typename AGG, typename OUT, typename IN>
    static void col(OUT* outValue, IN* ACol, int32_t dataElementCount) {
        static_assert(qdb_cpp::output_type_ok<AGG, OUT, IN>(), "aggregate output type: OUT = IN, or int64_t for COUNT");
        static_assert(!std::is_same<AGG, AggregationFunctions::none>::value, "GPUAggregation needs an aggregate");
        qdb_scalar* q = nullptr;
        qdb_cpp::check(qdb_scalar_create(&q, qdb_cpp::type_of<IN>::code, nullptr));
        OUT v{};
        int32_t is_null = 0;
        int32_t rc = qdb_scalar_process(q, ACol, nullptr, dataElementCount, nullptr, nullptr, nullptr);
        if (rc == QDB_OK) rc = qdb_scalar_result(q, AGG::bit, &v, &is_null, nullptr);
        qdb_scalar_destroy(q);
        qdb_cpp::check(rc);
        GPUMemory::copyHostToDevice(outValue, &v, 1);
    }
};

/* ---- ORDER BY over result columns: GPUOrderBy (GPUOrderBy.cuh:88-195, OrderByType.h, IOrderBy.h) ---- */
namespace OrderBy {
enum Order { ASC, DESC };
}  // namespace OrderBy

class IOrderBy {
protected:
    IOrderBy() = default;

public:
    virtual ~IOrderBy() = default;
};

/* The dispatcher creates one GPUOrderBy per result, calls OrderByColumn for the ORDER BY columns from the last to
 * the first (each call re-sorts the kept permutation stably by one column; NULL rows order as lowest(T)), and
 * reorders every result column and null mask by the indices. */
class GPUOrderBy : public IOrderBy {
public:
    explicit GPUOrderBy(int32_t dataElementCount) : n_(dataElementCount > 0 ? dataElementCount : 0) {
        GPUMemory::alloc(&indices_, n_ > 0 ? static_cast<size_t>(n_) : 1);
    }
    ~GPUOrderBy() override { qdb_free(indices_, nullptr); }
    GPUOrderBy(const GPUOrderBy&) = delete;
    GPUOrderBy& operator=(const GPUOrderBy&) = delete;

    template <typename T>
    void OrderByColumn(int32_t* outIndices, T* inCol, nullmask_t* nullBitMask, int32_t dataElementCount,
                       OrderBy::Order order) {
        qdb_cpp::check(qdb_order_by_column(qdb_cpp::type_of<T>::code, inCol, nullBitMask, order == OrderBy::DESC,
                                           dataElementCount, first_ ? 1 : 0, indices_, nullptr));
        first_ = false;
        if (outIndices && dataElementCount > 0) GPUMemory::copyDeviceToDevice(outIndices, indices_, dataElementCount);
        qdb_cpp::sync();
    }

    /* outCol[i] = inCol[inIndices[i]] (ReOrderByIdx, kernel_reorder_by_idx). */
    template <typename T>
    static void ReOrderByIdx(T* outCol, int32_t* inIndices, T* inCol, int32_t dataElementCount) {
        qdb_cpp::check(qdb_reorder(static_cast<int32_t>(sizeof(T)), inCol, inIndices, 0, dataElementCount, outCol,
                                   nullptr));
        qdb_cpp::sync();
    }

    /* The null bits reordered the same way (ReOrderNullValuesByIdx). */
    static void ReOrderNullValuesByIdx(nullmask_t* outNullBitMask, int32_t* indices, nullmask_t* inNullBitMask,
                                       int32_t rowCount) {
        qdb_cpp::check(qdb_reorder_nulls(inNullBitMask, indices, 0, rowCount, outNullBitMask, nullptr));
        qdb_cpp::sync();
    }

private:
    int32_t n_;
    int32_t* indices_ = nullptr;
    bool first_ = true;
};

/* ---- CompressionGPU (qikkDB/Compression/GPUCompression.h:10-80): AAFL column blocks ----
 * The same block format (header, position ids, bit lengths, packed words); compression and decompression run on the
 * GPU.  Supported element types: int32_t, int64_t and float (single-sign blocks); other types return false, as the
 * reference does for double.  A block that would not shrink is not compressed (false). */
class CompressionGPU {
    template <typename T>
    static int32_t code() {
        return std::is_same<T, int32_t>::value ? QDB_INT32
               : std::is_same<T, int64_t>::value ? QDB_INT64
               : std::is_same<T, float>::value   ? QDB_FLOAT
                                                 : 0;
    }
    template <typename T>
    static int64_t bits(T v) {
        if (sizeof(T) == 8) {
            int64_t b;
            std::memcpy(&b, &v, 8);
            return b;
        }
        int32_t b;
        std::memcpy(&b, &v, 4);
        return b;
    }

public:
    static const char CWARP_SIZE = 32;

    /* compressDataAAFL (GPUCompression.cu:150-225): host column in, host block out. */
    template <typename T>
    static bool compressDataAAFL(T* const hostUncompressed, int64_t uncompressedElementsCount,
                                 std::vector<T>& hostCompressed, int64_t& compressedElementsCount, T minValue,
                                 T maxValue) {
        if (code<T>() == 0 || uncompressedElementsCount <= 0) return false;
        cuda_ptr<T> d(static_cast<size_t>(uncompressedElementsCount));
        GPUMemory::copyHostToDevice(d.get(), hostUncompressed, static_cast<size_t>(uncompressedElementsCount));
        void* blk = nullptr;
        int64_t elems = 0;
        qdb_cpp::check(qdb_aafl_compress(code<T>(), d.get(), uncompressedElementsCount, bits(minValue), bits(maxValue),
                                         &blk, &elems, nullptr));
        if (!blk) return false;
        hostCompressed.resize(static_cast<size_t>(elems));
        GPUMemory::copyDeviceToHost(hostCompressed.data(), static_cast<const T*>(blk), static_cast<size_t>(elems));
        GPUMemory::free(blk);
        compressedElementsCount = elems;
        return true;
    }

    /* decompressDataAAFLOnDevice (GPUCompression.cu:474-522): a device block into a device column. */
    template <typename T>
    static bool decompressDataAAFLOnDevice(T* const deviceCompressed, int64_t uncompressedElementsCount,
                                           int64_t compressedElementsCount, int64_t compressionBlocksCount,
                                           T* const deviceUncompressed, T minValue, T maxValue) {
        if (code<T>() == 0) return false;
        qdb_aafl_col c{deviceCompressed, code<T>(), 0, uncompressedElementsCount, compressedElementsCount,
                       compressionBlocksCount, bits(minValue), bits(maxValue)};
        qdb_cpp::check(qdb_aafl_decompress(&c, deviceUncompressed, nullptr));
        return true;
    }

    /* decompressDataAAFL (GPUCompression.cu:366-440): host block in (its header gives the counts), host column out. */
    template <typename T>
    static bool decompressDataAAFL(T* const hostCompressed, int64_t compressedElementsCount,
                                   std::vector<T>& hostUncompressed, int64_t& uncompressedElementsCount, T minValue,
                                   T maxValue) {
        if (code<T>() == 0 || compressedElementsCount * static_cast<int64_t>(sizeof(T)) < 24) return false;
        int64_t hdr[3];
        std::memcpy(hdr, hostCompressed, 24);
        cuda_ptr<T> blk(static_cast<size_t>(compressedElementsCount));
        GPUMemory::copyHostToDevice(blk.get(), hostCompressed, static_cast<size_t>(compressedElementsCount));
        cuda_ptr<T> out(static_cast<size_t>(hdr[0] > 0 ? hdr[0] : 1));
        decompressDataAAFLOnDevice(blk.get(), hdr[0], hdr[1], hdr[2], out.get(), minValue, maxValue);
        hostUncompressed.resize(static_cast<size_t>(hdr[0]));
        GPUMemory::copyDeviceToHost(hostUncompressed.data(), out.get(), static_cast<size_t>(hdr[0]));
        uncompressedElementsCount = hdr[0];
        return true;
    }
};

#endif /* QDB_GROUPBY_HPP */
