// Seeded synthetic column generators (host C++), used by tests and the bench.
// vgen_splitmix64 is Steele, Lea and Flood's SplitMix64 (2014) in counter form:
// element i is the finaliser applied to seed + (i + 1) * golden gamma.
// The f64 uniform generator uses std::mt19937_64 + std::uniform_real_distribution
// so it reproduces the columns the reference's own validation programs build
// (examples/validate.cpp:22-25: seed 42, U[0,1000)).
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <random>
#include <thread>
#include <vector>

namespace {

uint64_t splitmix_at(uint64_t seed, uint64_t i) {
    uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

double unit_at(uint64_t seed, uint64_t i) { return static_cast<double>(splitmix_at(seed, i) >> 11) * 0x1.0p-53; }

}  // namespace

extern "C" {

void vgen_uniform_f64_mt(uint64_t seed, size_t n, double lo, double hi, double* out) {
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> dist(lo, hi);
    for (size_t i = 0; i < n; ++i) out[i] = dist(rng);
}

void vgen_splitmix64(uint64_t seed, size_t n, uint64_t* out) {
    for (size_t i = 0; i < n; ++i) {
        uint64_t z = seed + (static_cast<uint64_t>(i) + 1) * 0x9E3779B97F4A7C15ull;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        out[i] = z ^ (z >> 31);
    }
}

// Probe keys of the hash-join workload: with probability 1 - miss_frac a build
// key drawn Zipf(s) over the build rows (rank r has weight (r+1)^-s; ranks
// mapped to build rows by a seeded permutation), else an odd key (the build
// keys are even, so it never matches).  Sampling uses Vose's alias method
// (Vose 1991) with a counter-based SplitMix64 stream per row, so the output
// does not depend on the thread count.
void vgen_join_probe_i64(uint64_t seed, const int64_t* build, size_t nb, double s, double miss_frac, size_t n,
                         int64_t* out, unsigned threads) {
    if (nb == 0) return;
    std::vector<double> prob(nb);
    std::vector<uint32_t> alias(nb);
    {
        std::vector<double> w(nb);
        double tot = 0.0;
        for (size_t r = 0; r < nb; ++r) tot += (w[r] = std::pow(static_cast<double>(r + 1), -s));
        std::vector<uint32_t> small, large;
        for (size_t r = 0; r < nb; ++r) {
            w[r] = w[r] * static_cast<double>(nb) / tot;
            (w[r] < 1.0 ? small : large).push_back(static_cast<uint32_t>(r));
        }
        while (!small.empty() && !large.empty()) {
            const uint32_t a = small.back(), b = large.back();
            small.pop_back();
            prob[a] = w[a];
            alias[a] = b;
            w[b] = (w[b] + w[a]) - 1.0;
            if (w[b] < 1.0) {
                large.pop_back();
                small.push_back(b);
            }
        }
        for (uint32_t r : large) { prob[r] = 1.0; alias[r] = r; }
        for (uint32_t r : small) { prob[r] = 1.0; alias[r] = r; }
    }
    std::vector<uint32_t> perm(nb);
    for (size_t r = 0; r < nb; ++r) perm[r] = static_cast<uint32_t>(r);
    for (size_t r = nb - 1; r > 0; --r) {  // Fisher-Yates on a SplitMix64 stream
        const size_t j = static_cast<size_t>(splitmix_at(seed ^ 0x5EEDull, r) % (r + 1));
        std::swap(perm[r], perm[j]);
    }
    if (threads == 0) threads = 1;
    auto work = [&](size_t lo, size_t hi) {
        for (size_t i = lo; i < hi; ++i) {
            const uint64_t c = 3ull * i;
            if (unit_at(seed, c + 2) < miss_frac) {
                out[i] = static_cast<int64_t>((splitmix_at(seed, c + 1) >> 1) | 1ull);
                continue;
            }
            size_t j = static_cast<size_t>(unit_at(seed, c) * static_cast<double>(nb));
            if (j >= nb) j = nb - 1;
            const uint32_t r = unit_at(seed, c + 1) < prob[j] ? static_cast<uint32_t>(j) : alias[j];
            out[i] = build[perm[r]];
        }
    };
    std::vector<std::thread> th;
    const size_t per = (n + threads - 1) / threads;
    for (unsigned t = 0; t < threads; ++t) {
        const size_t lo = std::min(n, t * per), hi = std::min(n, lo + per);
        if (lo < hi) th.emplace_back(work, lo, hi);
    }
    for (auto& x : th) x.join();
}

}  // extern "C"
