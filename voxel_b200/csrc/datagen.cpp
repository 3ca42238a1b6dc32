// Seeded synthetic column generators (host C++), used by tests and the bench.
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

}  // extern "C"
