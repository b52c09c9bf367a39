// A reference-shaped caller of the C++ drop-in header (include/qdb_groupby.hpp), compiled with g++ against
// libqdbgb.so.  It reads known-answer GROUP BY cases from stdin and runs each one the way qikkDB's dispatcher
// drives the operators (GpuSqlDispatcherAggregationFunctions.h:377-553): block by block, the WHERE mask from
// GPUBinary<FilterConditions::OP, int8_t, int32_t*, int32_t>::Binary, keys and values compacted with
// GPUReconstruct::reconstructColKeep, GPUGroupBy<AGG, O, K, V>::ProcessBlock (the multi-key form for two key
// columns), a restart with a doubled key-size multiplier on GPU_HASH_TABLE_FULL (GpuSqlDispatcher.cpp:378-394),
// then GetResults.  It prints every group, which the test compares with the reference's expected results.
//
// Input, per case (whitespace separated):
//   case <name> <agg> <key columns> <rows> <block> <table size> <grow on full> <has values> <has key nulls>
//        <has value nulls> <predicate op or -1> <predicate constant>
//   then the key columns, the key null flags (when given), the values, the value null flags and the predicate
//   column (when given), <rows> numbers each.
// Output, per case:  "result <name> <groups> <multiplier>", then per group "<key...> <key null...> <value null> <value>".
// With the single argument "version" it prints the library version and exits (no GPU needed); "order", "scalar",
// "string" and "compress" run the ORDER BY, scalar-aggregation, string-key GROUP BY and compressed-block operators
// (described at their functions).
#include <cstdint>
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "qdb_groupby.hpp"

namespace {

struct Case {
    std::string name, agg;
    int nk = 1;
    int32_t n = 0, block = 0;
    int64_t table = 0;
    int grow = 0, has_vals = 0, has_kn = 0, has_vn = 0, pred_op = -1;
    int32_t pred_const = 0;
    std::vector<int32_t> keys[2];
    std::vector<int> kn[2];
    std::vector<int32_t> vals, pred;
    std::vector<int> vn;
};

bool read_case(Case& c) {
    std::string tag;
    if (!(std::cin >> tag)) return false;
    if (tag != "case") throw std::runtime_error("bad input: expected 'case', got " + tag);
    std::cin >> c.name >> c.agg >> c.nk >> c.n >> c.block >> c.table >> c.grow >> c.has_vals >> c.has_kn >> c.has_vn >>
        c.pred_op >> c.pred_const;
    auto rd = [&](auto& v) {
        v.resize(c.n);
        for (auto& x : v) std::cin >> x;
    };
    for (int k = 0; k < c.nk; ++k) rd(c.keys[k]);
    if (c.has_kn)
        for (int k = 0; k < c.nk; ++k) rd(c.kn[k]);
    if (c.has_vals) rd(c.vals);
    if (c.has_vn) rd(c.vn);
    if (c.pred_op >= 0) rd(c.pred);
    return true;
}

// Bit-packed null mask of rows [r0, r0 + rows) of `flags`, on the device (NULL when the case has no flags).
cuda_ptr<nullmask_t> device_mask(const std::vector<int>& flags, int32_t r0, int32_t rows) {
    if (flags.empty()) return cuda_ptr<nullmask_t>();
    std::vector<nullmask_t> w(GPUMemory::CalculateNullMaskSize(rows), 0);
    for (int32_t i = 0; i < rows; ++i)
        if (flags[r0 + i]) w[i / 64] |= nullmask_t(1) << (i % 64);
    cuda_ptr<nullmask_t> d(w.size());
    GPUMemory::copyHostToDevice(d.get(), w.data(), w.size());
    return d;
}

template <typename T>
cuda_ptr<T> device_col(const std::vector<T>& v, int32_t r0, int32_t rows) {
    cuda_ptr<T> d(static_cast<size_t>(rows));
    GPUMemory::copyHostToDevice(d.get(), v.data() + r0, static_cast<size_t>(rows));
    return d;
}

template <typename OP>
void where(int8_t* mask, int32_t* col, int32_t constant, int32_t n) {
    GPUBinary<OP, int8_t, int32_t*, int32_t>::Binary(mask, col, constant, n, nullptr);
}

void filter(int op, int8_t* mask, int32_t* col, int32_t constant, int32_t n) {
    switch (op) {
        case QDB_GREATER: where<FilterConditions::greater>(mask, col, constant, n); break;
        case QDB_GREATER_EQUAL: where<FilterConditions::greaterEqual>(mask, col, constant, n); break;
        case QDB_LESS: where<FilterConditions::less>(mask, col, constant, n); break;
        case QDB_LESS_EQUAL: where<FilterConditions::lessEqual>(mask, col, constant, n); break;
        case QDB_EQUAL: where<FilterConditions::equal>(mask, col, constant, n); break;
        case QDB_NOT_EQUAL: where<FilterConditions::notEqual>(mask, col, constant, n); break;
        default: throw std::runtime_error("unsupported predicate op");
    }
}

// One block of a case, compacted by its WHERE mask when it has one.  The compacted columns are owned here (a
// block without a predicate hands the uploaded columns through unchanged).
struct Block {
    int32_t rows = 0;
    cuda_ptr<int32_t> up_keys[2], up_vals, up_pred;
    cuda_ptr<nullmask_t> up_kn[2], up_vn;
    cuda_ptr<int32_t> keys[2], vals;
    cuda_ptr<nullmask_t> kn[2], vn;
    int32_t* k[2] = {nullptr, nullptr};
    nullmask_t* knp[2] = {nullptr, nullptr};
    int32_t* v = nullptr;
    nullmask_t* vnp = nullptr;
};

void prepare(const Case& c, int32_t r0, int32_t rows, Block& b) {
    for (int k = 0; k < c.nk; ++k) {
        b.up_keys[k] = device_col(c.keys[k], r0, rows);
        if (c.has_kn) b.up_kn[k] = device_mask(c.kn[k], r0, rows);
    }
    if (c.has_vals) b.up_vals = device_col(c.vals, r0, rows);
    if (c.has_vn) b.up_vn = device_mask(c.vn, r0, rows);
    if (c.pred_op < 0) {
        b.rows = rows;
        for (int k = 0; k < c.nk; ++k) {
            b.k[k] = b.up_keys[k].get();
            b.knp[k] = b.up_kn[k].get();
        }
        b.v = b.up_vals.get();
        b.vnp = b.up_vn.get();
        return;
    }
    b.up_pred = device_col(c.pred, r0, rows);
    cuda_ptr<int8_t> mask(static_cast<size_t>(rows));
    filter(c.pred_op, mask.get(), b.up_pred.get(), c.pred_const, rows);
    for (int k = 0; k < c.nk; ++k) {
        int32_t* out = nullptr;
        nullmask_t* onm = nullptr;
        GPUReconstruct::reconstructColKeep(&out, &b.rows, b.up_keys[k].get(), mask.get(), rows,
                                           c.has_kn ? &onm : nullptr, b.up_kn[k].get());
        b.keys[k] = cuda_ptr<int32_t>(out);
        b.kn[k] = cuda_ptr<nullmask_t>(onm);
        b.k[k] = out;
        b.knp[k] = onm;
    }
    if (c.has_vals) {
        int32_t* out = nullptr;
        nullmask_t* onm = nullptr;
        int32_t cnt = 0;
        GPUReconstruct::reconstructColKeep(&out, &cnt, b.up_vals.get(), mask.get(), rows, c.has_vn ? &onm : nullptr,
                                           b.up_vn.get());
        b.vals = cuda_ptr<int32_t>(out);
        b.vn = cuda_ptr<nullmask_t>(onm);
        b.v = out;
        b.vnp = onm;
    }
}

template <typename T>
std::vector<T> to_host(const T* d, int32_t n) {
    std::vector<T> h(n);
    if (n > 0) GPUMemory::copyDeviceToHost(h.data(), d, static_cast<size_t>(n));
    return h;
}

std::vector<int> unpack(const nullmask_t* d, int32_t n) {
    std::vector<int> flags(n, 0);
    if (!d || n == 0) return flags;
    std::vector<nullmask_t> w = to_host(d, static_cast<int32_t>(GPUMemory::CalculateNullMaskSize(n)));
    for (int32_t i = 0; i < n; ++i) flags[i] = static_cast<int>((w[i / 64] >> (i % 64)) & 1);
    return flags;
}

template <typename AGG, typename O>
void print_groups(const Case& c, int multiplier, int32_t count, const std::vector<void*>& keys,
                  const std::vector<nullmask_t*>& knulls, O* vals, nullmask_t* vnulls) {
    std::printf("result %s %d %d\n", c.name.c_str(), count, multiplier);
    std::vector<std::vector<int32_t>> hk;
    std::vector<std::vector<int>> hkn;
    for (int k = 0; k < c.nk; ++k) {
        hk.push_back(to_host(static_cast<int32_t*>(keys[k]), count));
        hkn.push_back(unpack(knulls[k], count));
    }
    std::vector<O> hv = vals ? to_host(vals, count) : std::vector<O>(count, O{});
    std::vector<int> hvn = unpack(vnulls, count);
    for (int32_t i = 0; i < count; ++i) {
        for (int k = 0; k < c.nk; ++k) std::printf("%d ", hk[k][i]);
        for (int k = 0; k < c.nk; ++k) std::printf("%d ", hkn[k][i]);
        const bool none = std::is_same<AGG, AggregationFunctions::none>::value;
        std::printf("%d %lld\n", none ? 1 : hvn[i], static_cast<long long>(hv[i]));
    }
}

// Runs every block into a fresh table of `multiplier` times the case's size; throws GPU_HASH_TABLE_FULL through.
template <typename AGG, typename O>
void run_single(const Case& c, int multiplier) {
    const int32_t size = static_cast<int32_t>(c.table ? c.table : 262144);  // GroupByBuckets default
    GPUGroupBy<AGG, O, int32_t, int32_t> gb(size, multiplier);
    const int32_t block = c.block > 0 ? c.block : c.n;
    for (int32_t r0 = 0; r0 < c.n; r0 += block) {
        Block b;
        prepare(c, r0, std::min(block, c.n - r0), b);
        if (b.rows > 0) gb.ProcessBlock(b.k[0], b.v, b.rows, b.knp[0], b.vnp);
    }
    int32_t* keys = nullptr;
    O* vals = nullptr;
    nullmask_t *kn = nullptr, *vn = nullptr;
    int32_t count = 0;
    gb.GetResults(&keys, std::is_same<AGG, AggregationFunctions::none>::value ? nullptr : &vals, &count, &kn, &vn);
    print_groups<AGG, O>(c, multiplier, count, {keys}, {kn}, vals, vn);
    GPUMemory::free(keys);
    GPUMemory::free(vals);
    GPUMemory::free(kn);
    GPUMemory::free(vn);
}

template <typename AGG, typename O>
void run_multi(const Case& c, int multiplier) {
    const int32_t size = static_cast<int32_t>(c.table ? c.table : 262144);
    std::vector<DataType> types = {COLUMN_INT, COLUMN_INT};
    GPUGroupBy<AGG, O, std::vector<void*>, int32_t> gb(size, multiplier, types);
    const int32_t block = c.block > 0 ? c.block : c.n;
    for (int32_t r0 = 0; r0 < c.n; r0 += block) {
        Block b;
        prepare(c, r0, std::min(block, c.n - r0), b);
        if (b.rows > 0) gb.ProcessBlock({b.k[0], b.k[1]}, {b.knp[0], b.knp[1]}, b.v, b.rows, b.vnp);
    }
    std::vector<void*> keys;
    std::vector<nullmask_t*> kn;
    O* vals = nullptr;
    nullmask_t* vn = nullptr;
    int32_t count = 0;
    gb.GetResults(&keys, std::is_same<AGG, AggregationFunctions::none>::value ? nullptr : &vals, &count, &kn, &vn);
    print_groups<AGG, O>(c, multiplier, count, keys, kn, vals, vn);
    FreeKeysVector(keys, types);
    for (nullmask_t* m : kn) GPUMemory::free(m);
    GPUMemory::free(vals);
    GPUMemory::free(vn);
}

template <typename AGG, typename O>
void run(const Case& c) {
    for (int multiplier = 1;; multiplier *= 2) {
        try {
            if (c.nk == 2) run_multi<AGG, O>(c, multiplier);
            else run_single<AGG, O>(c, multiplier);
            return;
        } catch (const query_engine_error& e) {
            if (!c.grow || e.GetQueryEngineError() != GPU_HASH_TABLE_FULL || multiplier >= 64) throw;
        }
    }
}

}  // namespace

// "order" mode: GROUP BY SUM then ORDER BY key or value (DispatcherGroupByTests.cpp:1551-1588) through
// GPUGroupBy + GPUOrderBy::OrderByColumn + GPUOrderBy::ReOrderByIdx.  Input per case: "ocase <name> <by_value> <desc>
// <rows>", the keys, the values.  Output: "oresult <name> <groups>" and one "<key> <sum>" line per group, in order.
int run_order() {
    std::string tag, name;
    while (std::cin >> tag) {
        int by_value = 0, desc = 0;
        int32_t n = 0;
        std::cin >> name >> by_value >> desc >> n;
        std::vector<int32_t> k(n), v(n);
        for (auto& x : k) std::cin >> x;
        for (auto& x : v) std::cin >> x;
        cuda_ptr<int32_t> dk = device_col(k, 0, n), dv = device_col(v, 0, n);
        GPUGroupBy<AggregationFunctions::sum, int32_t, int32_t, int32_t> gb(1024, 1);
        gb.ProcessBlock(dk.get(), dv.get(), n);
        int32_t *keys = nullptr, *sums = nullptr, g = 0;
        gb.GetResults(&keys, &sums, &g);
        GPUOrderBy ob(g);
        cuda_ptr<int32_t> idx(static_cast<size_t>(g > 0 ? g : 1));
        ob.OrderByColumn(idx.get(), by_value ? sums : keys, nullptr, g, desc ? OrderBy::DESC : OrderBy::ASC);
        cuda_ptr<int32_t> ok(static_cast<size_t>(g > 0 ? g : 1)), os(static_cast<size_t>(g > 0 ? g : 1));
        GPUOrderBy::ReOrderByIdx(ok.get(), idx.get(), keys, g);
        GPUOrderBy::ReOrderByIdx(os.get(), idx.get(), sums, g);
        std::vector<int32_t> hk = to_host(ok.get(), g), hs = to_host(os.get(), g);
        std::printf("oresult %s %d\n", name.c_str(), g);
        for (int32_t i = 0; i < g; ++i) std::printf("%d %d\n", hk[i], hs[i]);
        GPUMemory::free(keys);
        GPUMemory::free(sums);
    }
    return 0;
}

// "scalar" mode: the aggregates of GPUAggregationTests.cu (min, max, sum, avg, count of one column) through
// GPUAggregation::col.  Input: "<type code> <rows>" then the values.  Output: "<min> <max> <sum> <avg> <count>".
template <typename T>
void scalar_case(int32_t n) {
    std::vector<T> v(n);
    for (auto& x : v) std::cin >> x;
    cuda_ptr<T> d = device_col(v, 0, n);
    cuda_ptr<T> out(4);
    cuda_ptr<int64_t> cnt(1);
    GPUAggregation::col<AggregationFunctions::min>(out.get(), d.get(), n);
    GPUAggregation::col<AggregationFunctions::max>(out.get() + 1, d.get(), n);
    GPUAggregation::col<AggregationFunctions::sum>(out.get() + 2, d.get(), n);
    GPUAggregation::col<AggregationFunctions::avg>(out.get() + 3, d.get(), n);
    GPUAggregation::col<AggregationFunctions::count>(cnt.get(), d.get(), n);
    std::vector<T> h = to_host(out.get(), 4);
    std::vector<int64_t> c = to_host(cnt.get(), 1);
    std::cout.precision(17);
    std::cout << h[0] << " " << h[1] << " " << h[2] << " " << h[3] << " " << c[0] << "\n";
}

int run_scalar() {
    int32_t type = 0, n = 0;
    while (std::cin >> type >> n) {
        if (type == COLUMN_INT) scalar_case<int32_t>(n);
        else if (type == COLUMN_LONG) scalar_case<int64_t>(n);
        else if (type == COLUMN_FLOAT) scalar_case<float>(n);
        else scalar_case<double>(n);
    }
    return 0;
}

// "string" mode: GROUP BY over string keys (GPUGroupByTests.cu:474-516, DispatcherGroupByTests.cpp:1422-1467,
// DispatcherNullTests.cpp:1372-1750) through GPUGroupBy<AGG, O, std::string, int32_t>, block by block.  Input per
// case: "scase <name> <agg> <blocks>", then per block "<rows>" and per row "<key> <value> <keep>": key N (NULL),
// - (empty) or the bytes in hex; value N (NULL), X (no value column) or an integer; keep 0 drops the row before
// the block is built, as the dispatcher's WHERE compaction does.  Output: "sresult <name> <groups>" and one
// "<key> <value>" line per group (value N for a NULL aggregate).
template <typename AGG, typename O>
void string_case(const std::string& name, int32_t blocks) {
    GPUGroupBy<AGG, O, std::string, int32_t> gb(8, 1);
    for (int32_t b = 0; b < blocks; ++b) {
        int32_t rows = 0;
        std::cin >> rows;
        std::string chars;
        std::vector<int64_t> ends;
        std::vector<int32_t> vals;
        std::vector<nullmask_t> kn(GPUMemory::CalculateNullMaskSize(rows) + 1, 0), vn(kn.size(), 0);
        bool any_kn = false, any_vn = false, have_vals = true;
        for (int32_t r = 0; r < rows; ++r) {
            std::string k, v;
            int keep = 1;
            std::cin >> k >> v >> keep;
            if (!keep) continue;
            const size_t i = ends.size();
            if (k == "N") {
                kn[i / 64] |= nullmask_t(1) << (i % 64);
                any_kn = true;
            } else if (k != "-") {
                for (size_t c = 0; c + 1 < k.size(); c += 2) chars.push_back(static_cast<char>(std::stoi(k.substr(c, 2), nullptr, 16)));
            }
            ends.push_back(static_cast<int64_t>(chars.size()));
            if (v == "X") have_vals = false;
            else if (v == "N") {
                vn[i / 64] |= nullmask_t(1) << (i % 64);
                any_vn = true;
                vals.push_back(0);
            } else {
                vals.push_back(std::stoi(v));
            }
        }
        const int32_t n = static_cast<int32_t>(ends.size());
        if (n == 0) continue;
        cuda_ptr<char> dc(chars.size() + 1);
        if (!chars.empty()) GPUMemory::copyHostToDevice(dc.get(), chars.data(), chars.size());
        cuda_ptr<int64_t> de = device_col(ends, 0, n);
        cuda_ptr<nullmask_t> dkn = device_col(kn, 0, static_cast<int32_t>(kn.size()));
        cuda_ptr<nullmask_t> dvn = device_col(vn, 0, static_cast<int32_t>(vn.size()));
        cuda_ptr<int32_t> dv(have_vals ? static_cast<size_t>(n) : 1);
        if (have_vals) GPUMemory::copyHostToDevice(dv.get(), vals.data(), static_cast<size_t>(n));
        gb.ProcessBlock(GPUMemory::GPUString{dc.get(), de.get()}, have_vals ? dv.get() : nullptr, n,
                        any_kn ? dkn.get() : nullptr, any_vn ? dvn.get() : nullptr);
    }
    GPUMemory::GPUString keys{nullptr, nullptr};
    O* vals = nullptr;
    nullmask_t *kn = nullptr, *vn = nullptr;
    int32_t g = 0;
    gb.GetResults(&keys, &vals, &g, &kn, &vn);
    std::printf("sresult %s %d\n", name.c_str(), g);
    if (g > 0) {
        std::vector<int64_t> ends = to_host(keys.stringIndices, g);
        std::string chars(static_cast<size_t>(ends[g - 1]), '\0');
        if (!chars.empty()) GPUMemory::copyDeviceToHost(&chars[0], keys.allChars, chars.size());
        std::vector<O> hv = to_host(vals, g);
        std::vector<nullmask_t> hkn = to_host(kn, static_cast<int32_t>(GPUMemory::CalculateNullMaskSize(g)));
        std::vector<nullmask_t> hvn = to_host(vn, static_cast<int32_t>(GPUMemory::CalculateNullMaskSize(g)));
        for (int32_t i = 0; i < g; ++i) {
            const int64_t b0 = i ? ends[i - 1] : 0;
            std::string key;
            if ((hkn[i / 64] >> (i % 64)) & 1) key = "N";
            else if (ends[i] == b0) key = "-";
            else
                for (int64_t c = b0; c < ends[i]; ++c) {
                    char hx[3];
                    std::snprintf(hx, sizeof(hx), "%02x", static_cast<unsigned char>(chars[static_cast<size_t>(c)]));
                    key += hx;
                }
            if ((hvn[i / 64] >> (i % 64)) & 1) std::printf("%s N\n", key.c_str());
            else std::printf("%s %lld\n", key.c_str(), static_cast<long long>(hv[i]));
        }
    }
    GPUMemory::free(keys);
    GPUMemory::free(vals);
    GPUMemory::free(kn);
    GPUMemory::free(vn);
}

// "smerge" mode: as "string", with the blocks dealt alternately to two tables that GetResults(..., tables) merges
// (the multi-GPU GetResults, GPUGroupByString.cuh:565).
template <typename AGG, typename O>
void string_merge_case(const std::string& name, int32_t blocks) {
    std::vector<std::unique_ptr<IGroupBy>> tables;
    tables.emplace_back(new GPUGroupBy<AGG, O, std::string, int32_t>(8, 1));
    tables.emplace_back(new GPUGroupBy<AGG, O, std::string, int32_t>(8, 1));
    for (int32_t b = 0; b < blocks; ++b) {
        auto& gb = *static_cast<GPUGroupBy<AGG, O, std::string, int32_t>*>(tables[b % 2].get());
        int32_t rows = 0;
        std::cin >> rows;
        std::string chars;
        std::vector<int64_t> ends;
        std::vector<int32_t> vals;
        std::vector<nullmask_t> kn(GPUMemory::CalculateNullMaskSize(rows) + 1, 0), vn(kn.size(), 0);
        bool any_kn = false, any_vn = false, have_vals = true;
        for (int32_t r = 0; r < rows; ++r) {
            std::string k, v;
            int keep = 1;
            std::cin >> k >> v >> keep;
            if (!keep) continue;
            const size_t i = ends.size();
            if (k == "N") {
                kn[i / 64] |= nullmask_t(1) << (i % 64);
                any_kn = true;
            } else if (k != "-") {
                for (size_t c = 0; c + 1 < k.size(); c += 2) chars.push_back(static_cast<char>(std::stoi(k.substr(c, 2), nullptr, 16)));
            }
            ends.push_back(static_cast<int64_t>(chars.size()));
            if (v == "X") have_vals = false;
            else if (v == "N") {
                vn[i / 64] |= nullmask_t(1) << (i % 64);
                any_vn = true;
                vals.push_back(0);
            } else {
                vals.push_back(std::stoi(v));
            }
        }
        const int32_t n = static_cast<int32_t>(ends.size());
        if (n == 0) continue;
        cuda_ptr<char> dc(chars.size() + 1);
        if (!chars.empty()) GPUMemory::copyHostToDevice(dc.get(), chars.data(), chars.size());
        cuda_ptr<int64_t> de = device_col(ends, 0, n);
        cuda_ptr<nullmask_t> dkn = device_col(kn, 0, static_cast<int32_t>(kn.size()));
        cuda_ptr<nullmask_t> dvn = device_col(vn, 0, static_cast<int32_t>(vn.size()));
        cuda_ptr<int32_t> dv(have_vals ? static_cast<size_t>(n) : 1);
        if (have_vals) GPUMemory::copyHostToDevice(dv.get(), vals.data(), static_cast<size_t>(n));
        gb.ProcessBlock(GPUMemory::GPUString{dc.get(), de.get()}, have_vals ? dv.get() : nullptr, n,
                        any_kn ? dkn.get() : nullptr, any_vn ? dvn.get() : nullptr);
    }
    GPUMemory::GPUString keys{nullptr, nullptr};
    O* vals = nullptr;
    nullmask_t *kn = nullptr, *vn = nullptr;
    int32_t g = 0;
    static_cast<GPUGroupBy<AGG, O, std::string, int32_t>*>(tables[0].get())->GetResults(&keys, &vals, &g, tables, &kn, &vn);
    std::printf("sresult %s %d\n", name.c_str(), g);
    if (g > 0) {
        std::vector<int64_t> ends = to_host(keys.stringIndices, g);
        std::string chars(static_cast<size_t>(ends[g - 1]), '\0');
        if (!chars.empty()) GPUMemory::copyDeviceToHost(&chars[0], keys.allChars, chars.size());
        std::vector<O> hv = to_host(vals, g);
        std::vector<nullmask_t> hkn = to_host(kn, static_cast<int32_t>(GPUMemory::CalculateNullMaskSize(g)));
        std::vector<nullmask_t> hvn = to_host(vn, static_cast<int32_t>(GPUMemory::CalculateNullMaskSize(g)));
        for (int32_t i = 0; i < g; ++i) {
            const int64_t b0 = i ? ends[i - 1] : 0;
            std::string key;
            if ((hkn[i / 64] >> (i % 64)) & 1) key = "N";
            else if (ends[i] == b0) key = "-";
            else
                for (int64_t c = b0; c < ends[i]; ++c) {
                    char hx[3];
                    std::snprintf(hx, sizeof(hx), "%02x", static_cast<unsigned char>(chars[static_cast<size_t>(c)]));
                    key += hx;
                }
            if ((hvn[i / 64] >> (i % 64)) & 1) std::printf("%s N\n", key.c_str());
            else std::printf("%s %lld\n", key.c_str(), static_cast<long long>(hv[i]));
        }
    }
    GPUMemory::free(keys);
    GPUMemory::free(vals);
    GPUMemory::free(kn);
    GPUMemory::free(vn);
}

int run_string_merge() {
    std::string tag, name, agg;
    int32_t blocks = 0;
    while (std::cin >> tag >> name >> agg >> blocks) {
        if (agg == "sum") string_merge_case<AggregationFunctions::sum, int32_t>(name, blocks);
        else if (agg == "min") string_merge_case<AggregationFunctions::min, int32_t>(name, blocks);
        else if (agg == "max") string_merge_case<AggregationFunctions::max, int32_t>(name, blocks);
        else if (agg == "avg") string_merge_case<AggregationFunctions::avg, int32_t>(name, blocks);
        else string_merge_case<AggregationFunctions::count, int64_t>(name, blocks);
    }
    return 0;
}

int run_string() {
    std::string tag, name, agg;
    int32_t blocks = 0;
    while (std::cin >> tag >> name >> agg >> blocks) {
        if (agg == "sum") string_case<AggregationFunctions::sum, int32_t>(name, blocks);
        else if (agg == "min") string_case<AggregationFunctions::min, int32_t>(name, blocks);
        else if (agg == "max") string_case<AggregationFunctions::max, int32_t>(name, blocks);
        else if (agg == "avg") string_case<AggregationFunctions::avg, int32_t>(name, blocks);
        else string_case<AggregationFunctions::count, int64_t>(name, blocks);
    }
    return 0;
}

// "compress" mode: CompressionGPU on the columns of GPUCompressionTests.cpp.  Input per case: "<type code> <rows>" and
// the values.  Output: "plain", or "block" and the block's first eight words (int32 words for 4-byte types, int64
// for 8-byte ones), then "roundtrip <1|0>" from decompressDataAAFL (host) and decompressDataAAFLOnDevice.
template <typename T, typename Word>
void compress_case(int32_t n) {
    std::vector<T> v(n);
    for (auto& x : v) std::cin >> x;
    const T mn = *std::min_element(v.begin(), v.end()), mx = *std::max_element(v.begin(), v.end());
    std::vector<T> blk;
    int64_t elems = 0;
    if (!CompressionGPU::compressDataAAFL(v.data(), n, blk, elems, mn, mx)) {
        std::printf("plain\n");
        return;
    }
    std::printf("block");
    const Word* w = reinterpret_cast<const Word*>(blk.data());
    for (int i = 0; i < 8; ++i) std::printf(" %lld", static_cast<long long>(w[i]));
    std::printf("\n");
    std::vector<T> back;
    int64_t rows = 0;
    bool ok = CompressionGPU::decompressDataAAFL(blk.data(), elems, back, rows, mn, mx) && rows == n &&
              std::memcmp(back.data(), v.data(), sizeof(T) * static_cast<size_t>(n)) == 0;
    int64_t hdr[3];
    std::memcpy(hdr, blk.data(), 24);
    cuda_ptr<T> db(static_cast<size_t>(elems)), out(static_cast<size_t>(n));
    GPUMemory::copyHostToDevice(db.get(), blk.data(), static_cast<size_t>(elems));
    ok = ok && CompressionGPU::decompressDataAAFLOnDevice(db.get(), hdr[0], hdr[1], hdr[2], out.get(), mn, mx);
    std::vector<T> dev = to_host(out.get(), n);
    ok = ok && std::memcmp(dev.data(), v.data(), sizeof(T) * static_cast<size_t>(n)) == 0;
    std::printf("roundtrip %d\n", ok ? 1 : 0);
}

int run_compress() {
    int32_t type = 0, n = 0;
    while (std::cin >> type >> n) {
        if (type == COLUMN_INT) compress_case<int32_t, int32_t>(n);
        else if (type == COLUMN_LONG) compress_case<int64_t, int64_t>(n);
        else compress_case<float, int32_t>(n);
    }
    return 0;
}

int main(int argc, char** argv) {
    if (argc > 1 && std::string(argv[1]) == "version") {
        std::printf("%s\n", qdb_version());
        return 0;
    }
    try {
        if (argc > 1 && std::string(argv[1]) == "order") return run_order();
        if (argc > 1 && std::string(argv[1]) == "scalar") return run_scalar();
        if (argc > 1 && std::string(argv[1]) == "string") return run_string();
        if (argc > 1 && std::string(argv[1]) == "compress") return run_compress();
        if (argc > 1 && std::string(argv[1]) == "smerge") return run_string_merge();
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 2;
    }
    try {
        Case c;
        while (read_case(c)) {
            if (c.agg == "sum") run<AggregationFunctions::sum, int32_t>(c);
            else if (c.agg == "min") run<AggregationFunctions::min, int32_t>(c);
            else if (c.agg == "max") run<AggregationFunctions::max, int32_t>(c);
            else if (c.agg == "avg") run<AggregationFunctions::avg, int32_t>(c);
            else if (c.agg == "count") run<AggregationFunctions::count, int64_t>(c);
            else if (c.agg == "none") run<AggregationFunctions::none, int32_t>(c);
            else throw query_engine_error(GPU_UNKNOWN_AGG_FUN, c.agg);
            c = Case();
        }
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 2;
    }
    return 0;
}
