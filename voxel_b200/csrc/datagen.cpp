// Seeded synthetic column generators (host C++), used by tests and the bench.
// vgen_splitmix64 is Steele, Lea and Flood's SplitMix64 (2014) in counter form:
// element i is the finaliser applied to seed + (i + 1) * golden gamma.
// The f64 uniform generator uses std::mt19937_64 + std::uniform_real_distribution
// so it reproduces the columns the reference's own validation programs build
// (examples/validate.cpp:22-25: seed 42, U[0,1000)).
#include <cstddef>
#include <cstdint>
#include <random>

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

}  // extern "C"
