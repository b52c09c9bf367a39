// Seeded synthetic column generators for the GROUP BY workloads (host C++, multithreaded).
//
// Every value is a pure function of (seed, stream, row index): row i draws from the SplitMix64 sequence
// (Steele, Lea and Flood, "Fast splittable pseudorandom number generators", OOPSLA 2014) started at a
// state derived from (seed, stream).  Output is therefore identical for any thread count, and a column
// can be regenerated in pieces.  Transcendental functions (log, cos, exp) run only here, on the host, so
// the CPU oracle and the GPU see the same bytes.
//
// Distributions: uniform integers and floats; lognormal via the Box-Muller transform; Zipf(s) over ranks
// 1..N via Vose's alias method ("A linear algorithm for generating random numbers with a given
// distribution", IEEE TSE 1991), with ranks optionally mapped to 64-bit keys through a fixed bijection.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

inline uint64_t sm_mix(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

constexpr uint64_t kGolden = 0x9e3779b97f4a7c15ull;

struct Stream {
    uint64_t base;
    Stream(uint64_t seed, uint64_t stream) : base(sm_mix(seed ^ sm_mix(stream + kGolden))) {}
    // k-th 64-bit draw of row i (k < 4)
    inline uint64_t draw(int64_t i, int k = 0) const {
        return sm_mix(base + (static_cast<uint64_t>(i) * 4 + static_cast<uint64_t>(k) + 1) * kGolden);
    }
};

inline uint64_t bounded(uint64_t u, uint64_t range) {  // floor(u * range / 2^64)
    return static_cast<uint64_t>((static_cast<unsigned __int128>(u) * range) >> 64);
}

inline double unit_open(uint64_t u) {  // (0, 1), 53-bit
    return (static_cast<double>(u >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

int resolve_threads(int threads, int64_t n) {
    int t = threads > 0 ? threads : static_cast<int>(std::thread::hardware_concurrency());
    if (t < 1) t = 1;
    const int64_t min_rows = 1 << 16;
    if (n / min_rows < t) t = static_cast<int>(std::max<int64_t>(1, n / min_rows));
    return t;
}

template <typename F>
void parallel_rows(int64_t n, int threads, F f) {
    const int t = resolve_threads(threads, n);
    if (t == 1) {
        f(int64_t(0), n);
        return;
    }
    std::vector<std::thread> pool;
    const int64_t chunk = (n + t - 1) / t;
    for (int k = 0; k < t; ++k) {
        const int64_t b = k * chunk, e = std::min(n, b + chunk);
        if (b >= e) break;
        pool.emplace_back([=] { f(b, e); });
    }
    for (auto& th : pool) th.join();
}

}  // namespace

extern "C" {

// Version tag of the generator definitions; fixtures record it.
int32_t qdbgen_version(void) { return 1; }

// The key bijection applied to Zipf ranks (never yields INT64_MIN for ranks < 2^40).
int64_t qdbgen_rank_key(int64_t rank) {
    uint64_t k = sm_mix(static_cast<uint64_t>(rank) ^ 0x5bd1e9955bd1e995ull);
    if (k == 0x8000000000000000ull) k ^= 1ull;  // keep the value space free of INT64_MIN
    return static_cast<int64_t>(k);
}

int32_t qdbgen_uniform_i32(uint64_t seed, uint64_t stream, int64_t n, int32_t lo, int32_t hi, int32_t* out,
                           int32_t threads) {
    if (n < 0 || !out || hi < lo) return 1;
    const Stream st(seed, stream);
    const uint64_t range = static_cast<uint64_t>(static_cast<int64_t>(hi) - lo) + 1;
    parallel_rows(n, threads, [&](int64_t b, int64_t e) {
        for (int64_t i = b; i < e; ++i) out[i] = static_cast<int32_t>(lo + static_cast<int64_t>(bounded(st.draw(i), range)));
    });
    return 0;
}

int32_t qdbgen_uniform_i64(uint64_t seed, uint64_t stream, int64_t n, int64_t lo, int64_t hi, int64_t* out,
                           int32_t threads) {
    if (n < 0 || !out || hi < lo) return 1;
    const Stream st(seed, stream);
    const uint64_t range = static_cast<uint64_t>(hi) - static_cast<uint64_t>(lo) + 1;  // 0 = full 64-bit range
    parallel_rows(n, threads, [&](int64_t b, int64_t e) {
        for (int64_t i = b; i < e; ++i) {
            const uint64_t u = st.draw(i);
            out[i] = static_cast<int64_t>(static_cast<uint64_t>(lo) + (range ? bounded(u, range) : u));
        }
    });
    return 0;
}

// Uniform float32 in [lo, hi) on a 2^-24 grid of the unit interval.
int32_t qdbgen_uniform_f32(uint64_t seed, uint64_t stream, int64_t n, float lo, float hi, float* out, int32_t threads) {
    if (n < 0 || !out) return 1;
    const Stream st(seed, stream);
    parallel_rows(n, threads, [&](int64_t b, int64_t e) {
        for (int64_t i = b; i < e; ++i) {
            const float u = static_cast<float>(st.draw(i) >> 40) * (1.0f / 16777216.0f);
            out[i] = lo + (hi - lo) * u;
        }
    });
    return 0;
}

// Lognormal float32: exp(mu + sigma * z), z standard normal by Box-Muller from two draws.
int32_t qdbgen_lognormal_f32(uint64_t seed, uint64_t stream, int64_t n, double mu, double sigma, float* out,
                             int32_t threads) {
    if (n < 0 || !out) return 1;
    const Stream st(seed, stream);
    parallel_rows(n, threads, [&](int64_t b, int64_t e) {
        for (int64_t i = b; i < e; ++i) {
            const double u1 = unit_open(st.draw(i, 0)), u2 = unit_open(st.draw(i, 1));
            const double z = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
            out[i] = static_cast<float>(std::exp(mu + sigma * z));
        }
    });
    return 0;
}

// Zipf(s) over ranks 1..N.  map_keys = 1 writes qdbgen_rank_key(rank), 0 writes the rank itself.
int32_t qdbgen_zipf_i64(uint64_t seed, uint64_t stream, int64_t n, int64_t N, double s, int32_t map_keys,
                        int64_t* out, int32_t threads) {
    if (n < 0 || !out || N < 1 || N > (int64_t(1) << 31)) return 1;
    // Vose's alias table over ranks.
    std::vector<double> p(N);
    double total = 0.0;
    for (int64_t r = 0; r < N; ++r) total += (p[r] = std::pow(static_cast<double>(r + 1), -s));
    std::vector<double> prob(N);
    std::vector<int32_t> alias(N, 0);
    std::vector<int32_t> small, large;
    small.reserve(N);
    large.reserve(N);
    for (int64_t r = 0; r < N; ++r) {
        p[r] = p[r] * static_cast<double>(N) / total;
        (p[r] < 1.0 ? small : large).push_back(static_cast<int32_t>(r));
    }
    while (!small.empty() && !large.empty()) {
        const int32_t l = small.back(), g = large.back();
        small.pop_back();
        prob[l] = p[l];
        alias[l] = g;
        p[g] = (p[g] + p[l]) - 1.0;
        if (p[g] < 1.0) {
            large.pop_back();
            small.push_back(g);
        }
    }
    for (int32_t g : large) prob[g] = 1.0;
    for (int32_t l : small) prob[l] = 1.0;
    std::vector<int64_t> keys;
    if (map_keys) {
        keys.resize(N);
        for (int64_t r = 0; r < N; ++r) keys[r] = qdbgen_rank_key(r + 1);
    }
    const Stream st(seed, stream);
    parallel_rows(n, threads, [&](int64_t b, int64_t e) {
        for (int64_t i = b; i < e; ++i) {
            const int64_t col = static_cast<int64_t>(bounded(st.draw(i, 0), static_cast<uint64_t>(N)));
            const double coin = unit_open(st.draw(i, 1));
            const int64_t idx = (coin < prob[col]) ? col : alias[col];
            out[i] = map_keys ? keys[idx] : idx + 1;
        }
    });
    return 0;
}

// Log-uniform integers in [lo, hi]: floor(exp(U(ln lo, ln(hi + 1)))) clamped to [lo, hi].
int32_t qdbgen_loguniform_i64(uint64_t seed, uint64_t stream, int64_t n, int64_t lo, int64_t hi, int64_t* out,
                              int32_t threads) {
    if (n < 0 || !out || lo < 1 || hi < lo) return 1;
    const Stream st(seed, stream);
    const double a = std::log(static_cast<double>(lo)), b = std::log(static_cast<double>(hi) + 1.0);
    parallel_rows(n, threads, [&](int64_t bb, int64_t e) {
        for (int64_t i = bb; i < e; ++i) {
            int64_t v = static_cast<int64_t>(std::floor(std::exp(a + (b - a) * unit_open(st.draw(i)))));
            out[i] = std::min(hi, std::max(lo, v));
        }
    });
    return 0;
}

}  // extern "C"
