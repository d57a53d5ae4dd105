// Basic integer types and sentinels shared by the host-side code of the
// partitioner (METIS IO, generators, initial partitioner, drivers).
//
// Vertex ids and CSR offsets are u32, weights are s32, block ids are u32, as in
// the reference (src/utility/definitions.h:48-55). Objective sums (edge cut,
// communication cost J) are carried in s64.
#pragma once
#include <cstdint>
#include <cstddef>
#include <memory>
#include <type_traits>
#include <utility>
#include <vector>
#include <string>

namespace hp {

typedef int8_t s8;
typedef int16_t s16;
typedef int32_t s32;
typedef int64_t s64;
typedef uint8_t u8;
typedef uint16_t u16;
typedef uint32_t u32;
typedef uint64_t u64;

// Sentinels with the reference's values (src/utility/definitions.h:51-55,
// src/coarsening/two_hop_matching.h:48).
constexpr s32 GAIN_MIN = INT32_MIN;
constexpr u32 NULL_PART = 0xFFFFFFFFu - 1u;
constexpr u32 HASH_RECLAIM = 0xFFFFFFFFu - 2u;
constexpr u32 NO_MOVE = 0xFFFFFFFFu - 3u;
constexpr u32 NO_BLOCK_ID = 0xFFFFFFFFu;
constexpr u32 SENTINEL = 0xFFFFFFFFu;

// Allocator whose resize() leaves elements of trivially constructible types
// uninitialised, so that large host arrays are first touched (and their pages
// faulted in) by the threads that fill them rather than by one zero-fill.
// Every resize() of such a vector is followed by writes to all new elements.
template<typename T>
struct NoInitAlloc : std::allocator<T> {
    template<typename U>
    struct rebind {
        using other = NoInitAlloc<U>;
    };
    NoInitAlloc() = default;
    template<typename U>
    NoInitAlloc(const NoInitAlloc<U> &) noexcept {}
    template<typename U>
    void construct(U *p) noexcept(std::is_nothrow_default_constructible<U>::value) {
        ::new ((void *) p) U;
    }
    template<typename U, typename... Args>
    void construct(U *p, Args &&...args) {
        ::new ((void *) p) U(std::forward<Args>(args)...);
    }
};
template<typename T>
using hvec = std::vector<T, NoInitAlloc<T> >;

// A host CSR graph. `m` counts directed entries (2x the undirected edges), as
// the reference stores it (src/datastructures/host_graph.h:195). Empty `ew` /
// `vw` mean unit weights ("uniform" in the reference).
struct HostCSR {
    u32 n = 0;
    u32 m = 0;
    hvec<u32> xadj;  // n+1
    hvec<u32> adj;   // m
    hvec<s32> ew;    // m or empty
    hvec<s32> vw;    // n or empty
    s64 total_vw() const {
        if (vw.empty()) return (s64) n;
        s64 s = 0;
        for (s32 w: vw) s += w;
        return s;
    }
};

// Deterministic 64-bit generator (xorshift64*), used wherever the host code
// needs seeded randomness (generators, initial partitioner).
struct Rng64 {
    u64 s;
    explicit Rng64(u64 seed) : s(seed * 0x9E3779B97F4A7C15ull + 0xD1B54A32D192ED03ull) {
        if (s == 0) s = 0x106689D45497FDB5ull;
        for (int i = 0; i < 4; ++i) next();
    }
    u64 next() {
        s ^= s >> 12;
        s ^= s << 25;
        s ^= s >> 27;
        return s * 0x2545F4914F6CDD1Dull;
    }
    u32 next_u32() { return (u32) (next() >> 32); }
    // uniform in [0, bound) for bound > 0
    u32 below(u32 bound) { return (u32) (((u64) next_u32() * (u64) bound) >> 32); }
    double uniform() { return (double) (next() >> 11) * (1.0 / 9007199254740992.0); }
};

// splitmix64 finaliser: a stateless hash used for counter-based generation.
inline u64 splitmix64(u64 x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

} // namespace hp
