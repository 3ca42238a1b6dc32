// Device view of the hash-join build table (join.cu): one 16-byte slot per
// distinct build key {key, start, len} pointing at the key's run of build
// rows in the sorted build keys; open addressing with linear probing from
// the splitmix64 finaliser of the key (the mixer of the reference's
// HashValue<i64>, include/voxel/ops/hash.hpp:328-333).
#pragma once

#include <stdint.h>

namespace vx {

struct __align__(16) Slot {
    int64_t key;
    uint32_t start;
    uint32_t len;  // 0 = empty
};

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
    // splitmix64 finaliser, the mixer HashValue<i64> uses (ops/hash.hpp:328-333)
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

__device__ __forceinline__ Slot lookup(const Slot* __restrict__ table, uint64_t mask, int64_t k) {
    uint64_t h = mix64(static_cast<uint64_t>(k)) & mask;
    for (uint64_t probes = 0; probes <= mask; ++probes) {
        Slot s;
        const uint4 raw = __ldg(reinterpret_cast<const uint4*>(table + h));
        s.key = static_cast<int64_t>((static_cast<uint64_t>(raw.y) << 32) | raw.x);
        s.start = raw.z;
        s.len = raw.w;
        if (s.len == 0) break;
        if (s.key == k) return s;
        h = (h + 1) & mask;
    }
    Slot miss;
    miss.key = 0;
    miss.start = 0;
    miss.len = 0;
    return miss;
}

}  // namespace vx
