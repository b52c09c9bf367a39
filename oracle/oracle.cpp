// ORACLE - test infrastructure only.  Nothing in the product imports, links or calls this file; only
// tests/, __graft_entry__.smoke() and bench.py's CPU baseline leg use it, as the checker.
//
// A CPU restatement of the GROUP BY path's semantics, pinned by the reference's own known-answer tests
// (tests/golden/reference_kats.json, transcribed from qikkDB_test/DispatcherGroupByTests.cpp,
// DispatcherNullTests.cpp, GPUGroupByTests.cu, GPUFilterTests.cu and GPUReconstructTests.cu).
//
// The aggregation follows the std::unordered_map accumulate pattern the reference's tests use as ground
// truth (qikkDB_test/DispatcherNullTests.cpp:931-960, :1101-1140; DispatcherGroupByTests.cpp:34-71) with
// the operator semantics of GPUGroupBy (qikkDB/QueryEngine/GPUCore/GPUGroupBy.cuh:68-196, :478-587):
//   * all NULL keys form one group (GPUGroupBy.cuh:163-167); for composite keys a NULL component matches
//     only NULL, whatever the stored value (GPUGroupByMultiKey.cu:70-226);
//   * NULL values are skipped; a group with no non-NULL value has a NULL aggregate
//     (valuesNullArray, GPUGroupBy.cuh:182-185); COUNT counts non-NULL values and is never NULL;
//   * integer SUM wraps in the value type (atomicAdd on int32 / uint64, AggregationFunctions.cuh:219-228);
//   * integer AVG is the wrapped sum divided by the count with truncation (GPUBinary<div, O, V*, int64_t*>,
//     ArithmeticOperations.h div; pinned by DispatcherGroupByTests.cpp:1349-1353);
//   * float SUM/AVG are accumulated in FP64 (the north-star tolerance is stated against FP64);
//   * NULL-aggregate placeholders: MIN -> max(V), MAX -> lowest(V), SUM -> 0, AVG -> GetNullConstant<V>()
//     (qikkDB/QueryEngine/NullConstants.cuh:9-25).
// The filter follows kernel_filter (qikkDB/QueryEngine/GPUCore/GPUFilter.cuh:22-44): OP(a, b) evaluated in
// the C++ common type of the operands, && !null(i).  Compaction follows reconstructColKeep /
// GenerateIndexes (qikkDB/QueryEngine/GPUCore/GPUReconstruct.cuh:29-71, :272-355, :518-566).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <random>
#include <string_view>
#include <thread>
#include <type_traits>
#include <unordered_map>
#include <vector>

namespace {

enum { T_INT32 = 8, T_INT64 = 9, T_FLOAT = 10, T_DOUBLE = 11, T_INT8 = 15 };
enum { OP_GT = 0, OP_GE = 1, OP_LT = 2, OP_LE = 3, OP_EQ = 4, OP_NE = 5, OP_AND = 6, OP_OR = 7 };

inline bool bit(const uint64_t* m, int64_t i) { return m && ((m[i >> 6] >> (i & 63)) & 1ull); }

template <typename A, typename B>
inline bool cmp(int op, A a, B b) {
    switch (op) {
        case OP_GT: return a > b;
        case OP_GE: return a >= b;
        case OP_LT: return a < b;
        case OP_LE: return a <= b;
        case OP_EQ: return a == b;
        case OP_NE: return a != b;
        case OP_AND: return a && b;
        case OP_OR: return a || b;
        default: return false;
    }
}

template <typename T>
inline T load(const void* p, int64_t i) {
    T v;
    memcpy(&v, static_cast<const char*>(p) + i * sizeof(T), sizeof(T));
    return v;
}

template <typename A>
inline bool cmp_const(int op, A a, int ctype, int64_t ci, double cf) {
    switch (ctype) {
        case T_INT32: return cmp(op, a, static_cast<int32_t>(ci));
        case T_INT64: return cmp(op, a, static_cast<int64_t>(ci));
        case T_FLOAT: return cmp(op, a, static_cast<float>(cf));
        case T_DOUBLE: return cmp(op, a, cf);
        case T_INT8: return cmp(op, a, static_cast<int8_t>(ci));
        default: return false;
    }
}

inline bool pred_row(int ptype, const void* col, int64_t i, int op, int ctype, int64_t ci, double cf) {
    switch (ptype) {
        case T_INT32: return cmp_const(op, load<int32_t>(col, i), ctype, ci, cf);
        case T_INT64: return cmp_const(op, load<int64_t>(col, i), ctype, ci, cf);
        case T_FLOAT: return cmp_const(op, load<float>(col, i), ctype, ci, cf);
        case T_DOUBLE: return cmp_const(op, load<double>(col, i), ctype, ci, cf);
        case T_INT8: return cmp_const(op, load<int8_t>(col, i), ctype, ci, cf);
        default: return false;
    }
}

// Group key: per component a NULL flag and a value held as int64 (integers) or as the double value
// (floats, compared with ==, so -0.0 and +0.0 are one key).
struct Key {
    uint8_t n0 = 0, n1 = 0;
    int64_t i0 = 0, i1 = 0;
    double f0 = 0.0;
    bool operator==(const Key& o) const {
        return n0 == o.n0 && n1 == o.n1 && (n0 || (i0 == o.i0 && f0 == o.f0)) && (n1 || i1 == o.i1);
    }
};

struct KeyHash {
    size_t operator()(const Key& k) const {
        size_t h = std::hash<int>()(k.n0 * 2 + k.n1);
        if (!k.n0) {
            h ^= std::hash<int64_t>()(k.i0) * 31;
            h ^= std::hash<double>()(k.f0 == 0.0 ? 0.0 : k.f0) * 131;
        }
        if (!k.n1) h ^= std::hash<int64_t>()(k.i1) * 1009;
        return h;
    }
};

struct State {
    int64_t cnt = 0;        // non-NULL values
    uint64_t isum = 0;      // wrapping integer sum
    double fsum = 0.0;      // FP64 sum of float values
    int64_t imin = 0, imax = 0;
    double fmin = 0.0, fmax = 0.0;
};

struct Input {
    int key_type, n_key_cols;
    const void *k0, *k1;
    const uint64_t *kn0, *kn1;
    int val_type;
    const void* vals;
    const uint64_t* vn;
    int64_t n;
    int ptype;
    const void* pcol;
    const uint64_t* pn;
    int pop, ctype;
    int64_t ci;
    double cf;
    const int8_t* mask;
};

inline bool is_float(int t) { return t == T_FLOAT || t == T_DOUBLE; }

void accumulate(const Input& in, int64_t b, int64_t e, std::unordered_map<Key, State, KeyHash>& m) {
    const bool vfloat = is_float(in.val_type);
    for (int64_t i = b; i < e; ++i) {
        if (in.ptype && !(pred_row(in.ptype, in.pcol, i, in.pop, in.ctype, in.ci, in.cf) && !bit(in.pn, i))) continue;
        if (in.mask && in.mask[i] == 0) continue;
        Key k;
        k.n0 = bit(in.kn0, i);
        if (!k.n0) {
            switch (in.key_type) {
                case T_INT32: k.i0 = load<int32_t>(in.k0, i); break;
                case T_INT64: k.i0 = load<int64_t>(in.k0, i); break;
                case T_FLOAT: k.f0 = load<float>(in.k0, i); break;
                case T_DOUBLE: k.f0 = load<double>(in.k0, i); break;
            }
        }
        if (in.n_key_cols == 2) {
            k.n1 = bit(in.kn1, i);
            if (!k.n1) k.i1 = load<int32_t>(in.k1, i);
        }
        State& s = m[k];
        if (!in.vals) {
            ++s.cnt;
            continue;
        }
        if (bit(in.vn, i)) continue;
        if (vfloat) {
            const double v = in.val_type == T_FLOAT ? static_cast<double>(load<float>(in.vals, i)) : load<double>(in.vals, i);
            if (s.cnt == 0) s.fmin = s.fmax = v;
            else {
                if (v < s.fmin) s.fmin = v;
                if (v > s.fmax) s.fmax = v;
            }
            s.fsum += v;
        } else {
            const int64_t v = in.val_type == T_INT32 ? load<int32_t>(in.vals, i) : load<int64_t>(in.vals, i);
            if (s.cnt == 0) s.imin = s.imax = v;
            else {
                s.imin = std::min(s.imin, v);
                s.imax = std::max(s.imax, v);
            }
            s.isum += static_cast<uint64_t>(v);
        }
        ++s.cnt;
    }
}

void merge_into(std::unordered_map<Key, State, KeyHash>& dst, const std::unordered_map<Key, State, KeyHash>& src,
                bool vfloat) {
    for (const auto& kv : src) {
        auto it = dst.find(kv.first);
        if (it == dst.end()) {
            dst.emplace(kv.first, kv.second);
            continue;
        }
        State& d = it->second;
        const State& s = kv.second;
        if (s.cnt) {
            if (d.cnt == 0) {
                d.imin = s.imin; d.imax = s.imax; d.fmin = s.fmin; d.fmax = s.fmax;
            } else if (vfloat) {
                d.fmin = std::min(d.fmin, s.fmin);
                d.fmax = std::max(d.fmax, s.fmax);
            } else {
                d.imin = std::min(d.imin, s.imin);
                d.imax = std::max(d.imax, s.imax);
            }
        }
        d.cnt += s.cnt;
        d.isum += s.isum;
        d.fsum += s.fsum;
    }
}

}  // namespace

struct oracle_result {
    int key_type = 0, n_key_cols = 1, val_type = 0;
    std::vector<std::pair<Key, State>> rows;
    double agg_seconds = 0.0;
    int threads = 1;
};

extern "C" {

// GROUP BY oracle. Null masks are bit-packed (uint64 words).  pred_type 0 = no predicate.  threads <= 0 uses
// every hardware thread.  The result rows are sorted by key (NULL first per component).
oracle_result* oracle_groupby(int32_t key_type, int32_t n_key_cols, const void* key0, const void* key1,
                              const uint64_t* knull0, const uint64_t* knull1, int32_t val_type, const void* vals,
                              const uint64_t* vnull, int64_t n, int32_t pred_type, const void* pred_col,
                              const uint64_t* pred_nulls, int32_t pred_op, int32_t const_type, int64_t const_i,
                              double const_f, const int8_t* mask, int32_t threads, int32_t sort_rows) {
    Input in{key_type, n_key_cols, key0, key1, knull0, knull1, val_type, val_type ? vals : nullptr, vnull, n,
             pred_type, pred_col, pred_nulls, pred_op, const_type, const_i, const_f, mask};
    int t = threads > 0 ? threads : static_cast<int>(std::thread::hardware_concurrency());
    if (t < 1) t = 1;
    if (n < 4096) t = 1;
    auto* res = new oracle_result();
    res->key_type = key_type;
    res->n_key_cols = n_key_cols;
    res->val_type = val_type;
    res->threads = t;
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<std::unordered_map<Key, State, KeyHash>> maps(t);
    if (t == 1) {
        accumulate(in, 0, n, maps[0]);
    } else {
        std::vector<std::thread> pool;
        const int64_t chunk = (n + t - 1) / t;
        for (int k = 0; k < t; ++k) {
            const int64_t b = std::min<int64_t>(n, k * chunk), e = std::min<int64_t>(n, b + chunk);
            pool.emplace_back([&, k, b, e] { accumulate(in, b, e, maps[k]); });
        }
        for (auto& th : pool) th.join();
        // Pairwise tree merge keeps the merge parallel as well.
        for (int step = 1; step < t; step *= 2) {
            std::vector<std::thread> mp;
            for (int k = 0; k + step < t; k += 2 * step)
                mp.emplace_back([&, k, step] {
                    merge_into(maps[k], maps[k + step], is_float(val_type));
                    maps[k + step].clear();
                });
            for (auto& th : mp) th.join();
        }
    }
    const auto t1 = std::chrono::steady_clock::now();
    res->agg_seconds = std::chrono::duration<double>(t1 - t0).count();
    res->rows.assign(maps[0].begin(), maps[0].end());
    if (sort_rows) {
        const bool kf = is_float(key_type);
        std::sort(res->rows.begin(), res->rows.end(), [kf](const auto& a, const auto& b) {
            const Key &x = a.first, &y = b.first;
            if (x.n0 != y.n0) return x.n0 > y.n0;
            if (!x.n0) {
                if (kf) {
                    if (x.f0 != y.f0) return x.f0 < y.f0;
                } else if (x.i0 != y.i0) {
                    return x.i0 < y.i0;
                }
            }
            if (x.n1 != y.n1) return x.n1 > y.n1;
            if (!x.n1 && x.i1 != y.i1) return x.i1 < y.i1;
            return false;
        });
    }
    return res;
}

int64_t oracle_result_count(const oracle_result* r) { return static_cast<int64_t>(r->rows.size()); }
double oracle_result_seconds(const oracle_result* r) { return r->agg_seconds; }
int32_t oracle_result_threads(const oracle_result* r) { return r->threads; }

// Fetches the result rows.  Keys: int64 for integer key types, double for float key types (8 bytes/row);
// key nulls as bytes.  Aggregates (each optional): int64 for integer values, double for float values;
// cnt is int64.  Values at NULL-aggregate rows follow the reference placeholders.
void oracle_result_fetch(const oracle_result* r, void* key0, void* key1, uint8_t* knull0, uint8_t* knull1,
                         int64_t* cnt, void* sum, void* mn, void* mx, void* avg, uint8_t* vnull) {
    const bool kf = is_float(r->key_type);
    const bool vf = is_float(r->val_type);
    const bool v32 = r->val_type == T_INT32 || r->val_type == T_FLOAT;
    for (size_t i = 0; i < r->rows.size(); ++i) {
        const Key& k = r->rows[i].first;
        const State& s = r->rows[i].second;
        if (key0) {
            if (kf) static_cast<double*>(key0)[i] = k.n0 ? 0.0 : k.f0;
            else static_cast<int64_t*>(key0)[i] = k.n0 ? 0 : k.i0;
        }
        if (key1) static_cast<int64_t*>(key1)[i] = k.n1 ? 0 : k.i1;
        if (knull0) knull0[i] = k.n0;
        if (knull1) knull1[i] = k.n1;
        if (cnt) cnt[i] = s.cnt;
        if (vnull) vnull[i] = s.cnt == 0;
        if (vf) {
            const double fmax = v32 ? std::numeric_limits<float>::max() : std::numeric_limits<double>::max();
            if (sum) static_cast<double*>(sum)[i] = s.cnt ? s.fsum : 0.0;
            if (mn) static_cast<double*>(mn)[i] = s.cnt ? s.fmin : fmax;
            if (mx) static_cast<double*>(mx)[i] = s.cnt ? s.fmax : -fmax;
            if (avg) static_cast<double*>(avg)[i] = s.cnt ? s.fsum / static_cast<double>(s.cnt) : std::nan("");
        } else {
            const int64_t vmax = v32 ? std::numeric_limits<int32_t>::max() : std::numeric_limits<int64_t>::max();
            const int64_t vmin = v32 ? std::numeric_limits<int32_t>::min() : std::numeric_limits<int64_t>::min();
            // wrap the sum into the value type
            const int64_t wsum = v32 ? static_cast<int64_t>(static_cast<int32_t>(static_cast<uint32_t>(s.isum)))
                                     : static_cast<int64_t>(s.isum);
            if (sum) static_cast<int64_t*>(sum)[i] = s.cnt ? wsum : 0;
            if (mn) static_cast<int64_t*>(mn)[i] = s.cnt ? s.imin : vmax;
            if (mx) static_cast<int64_t*>(mx)[i] = s.cnt ? s.imax : vmin;
            if (avg) static_cast<int64_t*>(avg)[i] = s.cnt ? wsum / s.cnt : vmin;
        }
    }
}

void oracle_result_free(oracle_result* r) { delete r; }

// Filter oracle: out[i] = OP(a, b) && !null(i); a side with *_is_col == 0 is a pointer to one value.
void oracle_filter(int32_t op, int32_t a_type, int32_t a_is_col, const void* a, int32_t b_type, int32_t b_is_col,
                   const void* b, const uint64_t* nulls, int8_t* out, int64_t n) {
    for (int64_t i = 0; i < n; ++i) {
        const int64_t ia = a_is_col ? i : 0, ib = b_is_col ? i : 0;
        bool r = false;
        // dispatch on both types
        auto with_b = [&](auto av) {
            switch (b_type) {
                case T_INT8: r = cmp(op, av, load<int8_t>(b, ib)); break;
                case T_INT32: r = cmp(op, av, load<int32_t>(b, ib)); break;
                case T_INT64: r = cmp(op, av, load<int64_t>(b, ib)); break;
                case T_FLOAT: r = cmp(op, av, load<float>(b, ib)); break;
                case T_DOUBLE: r = cmp(op, av, load<double>(b, ib)); break;
            }
        };
        switch (a_type) {
            case T_INT8: with_b(load<int8_t>(a, ia)); break;
            case T_INT32: with_b(load<int32_t>(a, ia)); break;
            case T_INT64: with_b(load<int64_t>(a, ia)); break;
            case T_FLOAT: with_b(load<float>(a, ia)); break;
            case T_DOUBLE: with_b(load<double>(a, ia)); break;
        }
        // const-const fills the mask without looking at nulls (GPUBinary.cuh:573-575)
        if (a_is_col || b_is_col) r = r && !bit(nulls, i);
        out[i] = r ? 1 : 0;
    }
}

// Compaction oracle: selected elements in order; returns the count.  null_out (optional, zeroed by the
// caller, ceil(count/64) words) receives the compacted null bits.
int64_t oracle_compact(int32_t elem_bytes, const void* in, const int8_t* mask, int64_t n, void* out,
                       const uint64_t* null_in, uint64_t* null_out) {
    int64_t c = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (!mask[i]) continue;
        memcpy(static_cast<char*>(out) + c * elem_bytes, static_cast<const char*>(in) + i * elem_bytes, elem_bytes);
        if (null_out && bit(null_in, i)) null_out[c >> 6] |= 1ull << (c & 63);
        ++c;
    }
    return c;
}

// ORDER BY oracle (qikkDB/QueryEngine/GPUCore/GPUOrderBy.cuh:88-195 as the dispatcher drives it): the row
// permutation that sorts by the columns, column 0 most significant, each ascending or descending, ties in input
// order.  As the reference does, a NULL row takes the value lowest(T) before the comparison
// (TransformNullValsToSmallestVal), and values compare the way its CUB radix sort orders them: integers by value,
// IEEE values by their bits mapped to an unsigned order (negative: all bits flipped; else the sign bit set), so
// -0.0 precedes +0.0.  Descending reverses the comparison only (the radix sort stays stable).
namespace {
uint64_t ob_key(int32_t type, const void* col, const uint64_t* nulls, int64_t r) {
    const bool null = nulls && bit(nulls, r);
    switch (type) {
        case T_INT32: {
            const int32_t v = null ? std::numeric_limits<int32_t>::lowest() : static_cast<const int32_t*>(col)[r];
            return static_cast<uint32_t>(v) ^ 0x80000000u;
        }
        case T_INT64: {
            const int64_t v = null ? std::numeric_limits<int64_t>::lowest() : static_cast<const int64_t*>(col)[r];
            return static_cast<uint64_t>(v) ^ 0x8000000000000000ull;
        }
        case T_FLOAT: {
            const float v = null ? std::numeric_limits<float>::lowest() : static_cast<const float*>(col)[r];
            uint32_t b;
            memcpy(&b, &v, 4);
            return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
        }
        default: {
            const double v = null ? std::numeric_limits<double>::lowest() : static_cast<const double*>(col)[r];
            uint64_t b;
            memcpy(&b, &v, 8);
            return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
        }
    }
}
}  // namespace

void oracle_order_by(int32_t n_cols, const int32_t* types, const void* const* cols, const uint64_t* const* nulls,
                     const int32_t* descending, int64_t n, int32_t* out) {
    std::vector<std::vector<uint64_t>> keys(n_cols, std::vector<uint64_t>(static_cast<size_t>(n)));
    for (int c = 0; c < n_cols; ++c)
        for (int64_t r = 0; r < n; ++r) keys[c][r] = ob_key(types[c], cols[c], nulls ? nulls[c] : nullptr, r);
    std::vector<int32_t> idx(static_cast<size_t>(n));
    for (int64_t r = 0; r < n; ++r) idx[r] = static_cast<int32_t>(r);
    std::stable_sort(idx.begin(), idx.end(), [&](int32_t x, int32_t y) {
        for (int c = 0; c < n_cols; ++c) {
            const uint64_t a = keys[c][x], b = keys[c][y];
            if (a != b) return (descending && descending[c]) ? a > b : a < b;
        }
        return false;
    });
    std::copy(idx.begin(), idx.end(), out);
}

// String keys (GPUString layout: concatenated chars, int64 end offsets).  The reference's string GROUP BY
// identifies a group by the row of the key's first occurrence (sourceIndices, GPUGroupByString.cuh:39-169);
// this writes that row for every non-NULL row (rows with a NULL key get -1), so that GROUP BY over strings is
// the integer GROUP BY above over these ids.  Returns the number of distinct non-NULL strings.
int64_t oracle_string_ids(const char* chars, const int64_t* ends, const uint64_t* knull, int64_t n, int64_t* out) {
    std::unordered_map<std::string_view, int64_t> first;
    first.reserve(static_cast<size_t>(n < 1024 ? 1024 : n / 4));
    for (int64_t i = 0; i < n; ++i) {
        if (bit(knull, i)) {
            out[i] = -1;
            continue;
        }
        const int64_t b = i ? ends[i - 1] : 0;
        const std::string_view s(chars + b, static_cast<size_t>(ends[i] - b));
        out[i] = first.emplace(s, i).first->second;
    }
    return static_cast<int64_t>(first.size());
}

// ---- AAFL compressed blocks (the block format of qikkDB/Compression/GPUCompression.cu:25-148 with the bit
// packing of feathergpu fl/aafl.cuh:5-58 and fl/afl.cuh:6-77), restated for 32- and 64-bit integers and for
// floats of one sign (compressed as their int32 bit patterns, GPUCompression.cu:197-225).
// A block of T elements: int64 rows, int64 elements (the block's length in T), int64 blocks (= ceil(rows / 32));
// uint64 position[blocks]; uint8 bit_length[blocks]; then the packed words (T).  Rows are packed in groups of
// 32 W (W = bits of T): row d of group g is lane d % 32, index i = (d % 32W) / 32; lane l's values i = 0, 1, ...
// occupy bits [i b, (i + 1) b) of the lane's bit stream, word k of which is words[position[g] + l + 32 k]
// (least significant bit first), b = bit_length[g] = significant bits of the group's largest (value - offset).
// The compressor here places the groups' words in group order (the reference takes them in the order its warps
// finish); any placement decodes the same.
}  // extern "C"

namespace {

template <typename T>
T aafl_offset(T mn, T mx) {
    // offset = min, or 0 when max - min does not fit T; -min wraps as two's complement does for lowest(T)
    using U = typename std::make_unsigned<T>::type;
    T off = mn;
    if (mn < 0 && mx > 0) {
        const T neg = static_cast<T>(U(0) - static_cast<U>(mn));
        if (std::numeric_limits<T>::max() - mx < neg) off = 0;
    }
    return off;
}

template <typename T>
int64_t aafl_compress_t(const T* v, int64_t n, T mn, T mx, T* out, int64_t cap) {
    using U = typename std::make_unsigned<T>::type;
    constexpr int W = sizeof(T) * 8;
    const T off = aafl_offset(mn, mx);
    const int64_t blocks = (n + 31) / 32;
    const int64_t groups = (n + 32 * W - 1) / (32 * W);
    std::vector<uint64_t> pos(static_cast<size_t>(blocks), 0);
    std::vector<uint8_t> bl(static_cast<size_t>(blocks), 0);
    std::vector<U> words;
    for (int64_t g = 0; g < groups; ++g) {
        const int64_t d0 = g * 32 * W;
        U mxv = 0;
        for (int64_t d = d0; d < std::min<int64_t>(n, d0 + 32 * W); ++d) mxv = std::max<U>(mxv, static_cast<U>(static_cast<U>(v[d]) - static_cast<U>(off)));
        int b = 0;
        while (b < W && (mxv >> b) != 0) ++b;
        const int64_t rem = n - d0;
        int64_t space = static_cast<int64_t>(b) * 32;
        if (rem < 32 * W) space = ((((rem + W - 1) / W) * b + 31) / 32) * 32;  // GPUCompression's last-group size
        pos[static_cast<size_t>(g)] = words.size();
        bl[static_cast<size_t>(g)] = static_cast<uint8_t>(b);
        const size_t base = words.size();
        words.resize(base + static_cast<size_t>(space), 0);
        if (b == 0) continue;
        for (int l = 0; l < 32; ++l) {
            for (int i = 0; i < W; ++i) {
                const int64_t d = d0 + l + 32 * i;
                if (d >= n) break;
                const U x = static_cast<U>(static_cast<U>(v[d]) - static_cast<U>(off));
                const int64_t o = static_cast<int64_t>(i) * b;
                const int64_t k = o / W;
                const int p = static_cast<int>(o % W);
                words[base + static_cast<size_t>(l + 32 * k)] |= static_cast<U>(x << p);
                if (p + b > W) words[base + static_cast<size_t>(l + 32 * (k + 1))] |= static_cast<U>(x >> (W - p));
            }
        }
    }
    const int64_t data_bytes = static_cast<int64_t>(words.size()) * static_cast<int64_t>(sizeof(T));
    const int64_t total = data_bytes + std::max<int64_t>(8 * blocks, sizeof(T)) + std::max<int64_t>(blocks, sizeof(T)) + 24;
    const int64_t elems = (total + static_cast<int64_t>(sizeof(T)) - 1) / static_cast<int64_t>(sizeof(T));
    if (elems >= n) return 0;  // compression does not pay: the block stays plain
    if (elems > cap) return -elems;
    char* o = reinterpret_cast<char*>(out);
    std::memset(o, 0, static_cast<size_t>(elems) * sizeof(T));
    const int64_t hdr[3] = {n, elems, blocks};
    std::memcpy(o, hdr, 24);
    std::memcpy(o + 24, pos.data(), static_cast<size_t>(blocks) * 8);
    std::memcpy(o + 24 + 8 * blocks, bl.data(), static_cast<size_t>(blocks));
    std::memcpy(o + 24 + 9 * blocks, words.data(), static_cast<size_t>(data_bytes));
    return elems;
}

template <typename T>
void aafl_decompress_t(const T* c, T mn, T mx, T* out) {
    using U = typename std::make_unsigned<T>::type;
    constexpr int W = sizeof(T) * 8;
    const char* b = reinterpret_cast<const char*>(c);
    int64_t hdr[3];
    std::memcpy(hdr, b, 24);
    const int64_t n = hdr[0], blocks = hdr[2];
    const T off = aafl_offset(mn, mx);
    const int64_t groups = (n + 32 * W - 1) / (32 * W);
    for (int64_t g = 0; g < groups; ++g) {
        uint64_t base;
        std::memcpy(&base, b + 24 + 8 * g, 8);
        const int bits = static_cast<uint8_t>(b[24 + 8 * blocks + g]);
        const char* words = b + 24 + 9 * blocks;
        auto word = [&](int64_t idx) {
            U w;
            std::memcpy(&w, words + idx * static_cast<int64_t>(sizeof(T)), sizeof(T));
            return w;
        };
        for (int l = 0; l < 32; ++l) {
            for (int i = 0; i < W; ++i) {
                const int64_t d = g * 32 * W + l + 32 * i;
                if (d >= n) break;
                U x = 0;
                if (bits) {
                    const int64_t o = static_cast<int64_t>(i) * bits;
                    const int64_t k = o / W;
                    const int p = static_cast<int>(o % W);
                    x = static_cast<U>(word(static_cast<int64_t>(base) + l + 32 * k) >> p);
                    if (p + bits > W) x |= static_cast<U>(word(static_cast<int64_t>(base) + l + 32 * (k + 1)) << (W - p));
                    if (bits < W) x &= static_cast<U>((U(1) << bits) - 1);
                }
                out[d] = static_cast<T>(static_cast<U>(x + static_cast<U>(off)));
            }
        }
    }
}

}  // namespace

extern "C" {

// Compresses n values of type (T_INT32, T_INT64, T_FLOAT) with the block's min and max (host values of the type).
// Returns the block's length in elements (written to out), 0 when the block stays plain (compression would not
// shrink it, or a float block mixes signs), or -needed when cap elements are too few.
int64_t oracle_aafl_compress(int32_t type, const void* in, int64_t n, const void* mn, const void* mx, void* out,
                             int64_t cap) {
    switch (type) {
        case T_INT32: return aafl_compress_t(static_cast<const int32_t*>(in), n, *static_cast<const int32_t*>(mn),
                                             *static_cast<const int32_t*>(mx), static_cast<int32_t*>(out), cap);
        case T_INT64: return aafl_compress_t(static_cast<const int64_t*>(in), n, *static_cast<const int64_t*>(mn),
                                             *static_cast<const int64_t*>(mx), static_cast<int64_t*>(out), cap);
        case T_FLOAT: {
            const float fmn = *static_cast<const float*>(mn), fmx = *static_cast<const float*>(mx);
            if (!((fmn >= 0 && fmx >= 0) || (fmn <= 0 && fmx <= 0))) return 0;
            int32_t a, b;
            std::memcpy(&a, &fmn, 4);
            std::memcpy(&b, &fmx, 4);
            if (a > b) std::swap(a, b);
            return aafl_compress_t(static_cast<const int32_t*>(in), n, a, b, static_cast<int32_t*>(out), cap);
        }
        default: return 0;
    }
}

// Decompresses a block (its header gives the row count) into out.
void oracle_aafl_decompress(int32_t type, const void* in, const void* mn, const void* mx, void* out) {
    switch (type) {
        case T_INT32:
            aafl_decompress_t(static_cast<const int32_t*>(in), *static_cast<const int32_t*>(mn),
                              *static_cast<const int32_t*>(mx), static_cast<int32_t*>(out));
            break;
        case T_INT64:
            aafl_decompress_t(static_cast<const int64_t*>(in), *static_cast<const int64_t*>(mn),
                              *static_cast<const int64_t*>(mx), static_cast<int64_t*>(out));
            break;
        case T_FLOAT: {
            int32_t a, b;
            std::memcpy(&a, mn, 4);
            std::memcpy(&b, mx, 4);
            if (a > b) std::swap(a, b);
            aafl_decompress_t(static_cast<const int32_t*>(in), a, b, static_cast<int32_t*>(out));
            break;
        }
        default: break;
    }
}

int64_t oracle_indexes(const int8_t* mask, int64_t n, int32_t* out) {
    int64_t c = 0;
    for (int64_t i = 0; i < n; ++i)
        if (mask[i]) out[c++] = static_cast<int32_t>(i);
    return c;
}

void oracle_prefix_sum(const int8_t* mask, int64_t n, int32_t* out) {
    int32_t run = 0;
    for (int64_t i = 0; i < n; ++i) out[i] = (run += mask[i]);
}

// Inputs of the reference's filter tests, generated as those tests do: a default-seeded
// std::default_random_engine with uniform_int_distribution<int32_t>(INT32_MIN, INT32_MAX) for integer types and
// uniform_real_distribution<float>(-32000, 32000) for float (qikkDB_test/GPUFilterTests.cu:13-45, :190-215).
// mode 0: column-column (A[i], B[i] drawn alternately); mode 1: column then one constant (b[0]).
void oracle_reference_filter_inputs(int32_t type, int32_t mode, int64_t n, void* a, void* b) {
    std::default_random_engine gen;
    std::uniform_int_distribution<int32_t> di(std::numeric_limits<int32_t>::lowest(), std::numeric_limits<int32_t>::max());
    std::uniform_real_distribution<float> df(-32000.0f, 32000.0f);
    auto put = [&](void* dst, int64_t i) {
        switch (type) {
            case T_INT32: static_cast<int32_t*>(dst)[i] = di(gen); break;
            case T_INT64: static_cast<int64_t*>(dst)[i] = di(gen); break;
            case T_FLOAT: static_cast<float*>(dst)[i] = df(gen); break;
        }
    };
    if (mode == 0) {
        for (int64_t i = 0; i < n; ++i) {
            put(a, i);
            put(b, i);
        }
    } else {
        for (int64_t i = 0; i < n; ++i) put(a, i);
        put(b, 0);
    }
}

}  // extern "C"
