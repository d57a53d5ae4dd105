// Common device-side definitions for the sm_100a partitioner kernels.
#pragma once
#include <atomic>
#include <cstdint>
#include <cuda_runtime.h>

#include "../host/hp_types.h"

namespace hp {

// ---- tuning constants ------------------------------------------------------
constexpr int NUM_SMS_HINT = 148;           // B200: 148 SMs on two dies
constexpr int BLOCK = 256;                  // default block size
constexpr u32 THREAD_DEG_MAX = 16;          // thread-per-vertex rows up to this degree
constexpr u32 WARP_DEG_MAX = 2048;          // warp-per-vertex rows up to this degree
constexpr u32 JET_MAX_ITERATIONS = 12;      // jet_label_propagation.h:36
constexpr u32 JET_MAX_WEAK_ITERATIONS = 2;  // jet_label_propagation.h:37
constexpr u32 MAX_SECTIONS = 128;           // jet_label_propagation.h:41
constexpr u32 MAX_BUCKETS = 50;             // jet_label_propagation.h:42
constexpr u32 MATCH_SEED = 12345u;          // two_hop_matching.h:590
constexpr u32 MAX_K = 1u << 16;             // largest supported block count

// ---- error codes returned through the C ABI --------------------------------
enum Status : int {
    HP_OK = 0,
    HP_ERR_ARG = 1,
    HP_ERR_CUDA = 2,
    HP_ERR_OOM = 3,
    HP_ERR_IO = 4,
    HP_ERR_GRAPH = 5,
    HP_ERR_DEVICE = 6,  // a kernel reported an error through the status word
};

// Device-side error bits (written into the context's status word).
enum DevErr : u32 {
    DEV_ERR_NONE = 0,
    DEV_ERR_BAD_ID = 1u << 0,       // neighbour id out of range
    DEV_ERR_BAD_WEIGHT = 1u << 1,   // non-positive weight
    DEV_ERR_HASH_FULL = 1u << 2,    // a bounded probe sequence ran out
    DEV_ERR_SPIN = 1u << 3,         // a bounded wait gave up
    DEV_ERR_RANGE = 1u << 4,        // an index check failed
};

// ---- integer helpers -----------------------------------------------------------
__host__ __device__ __forceinline__ s32 wadd(s32 a, s32 b) { return (s32) ((u32) a + (u32) b); }
__host__ __device__ __forceinline__ s32 wsub(s32 a, s32 b) { return (s32) ((u32) a - (u32) b); }
__host__ __device__ __forceinline__ s32 wmul(s32 a, s32 b) { return (s32) ((u32) a * (u32) b); }

// xorshift32: two_hop_matching.h:93-100 (identical to mix32, graph.h:39-45)
__host__ __device__ __forceinline__ u32 xorshift32(u32 x) {
    x ^= x << 13;
    x ^= x >> 17;
    x ^= x << 5;
    return x;
}

__host__ __device__ __forceinline__ u32 rotl32(u32 x, int r) { return (x << r) | (x >> (32 - r)); }

// MurmurHash3_x86_32 of one 4-byte little-endian block, seed 0: the
// Kokkos::pod_hash<u32> used at two_hop_matching.h:317 and :458.
__host__ __device__ __forceinline__ u32 murmur3_u32(u32 key) {
    u32 k = key * 0xcc9e2d51u;
    k = rotl32(k, 15);
    k *= 0x1b873593u;
    u32 h = k;  // seed 0
    h = rotl32(h, 13);
    h = h * 5u + 0xe6546b64u;
    h ^= 4u;
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

// gain_bucket (jet_label_propagation.h:147-180) as an exact integer rule:
// with g = -gx / vwgt, g >= 1 -> 25 + min{k : 1.5^k >= g} (<= 49), and
// g < 1 -> 25 - min{k : 1.5^k >= 1/g} (>= 2). 128-bit products keep it exact.
__host__ __device__ __forceinline__ u32 gain_bucket(s32 gx, s32 vwgt) {
    if (gx > 0) return 0;
    if (gx == 0) return 1;
    unsigned __int128 a = (unsigned __int128) (u64) (-(s64) gx);
    unsigned __int128 b = (unsigned __int128) (u64) (vwgt < 1 ? 1 : vwgt);
    unsigned __int128 p2 = 1, p3 = 1;
    u32 k = 0;
    if (a >= b) {
        while (k < 24 && a * p2 > b * p3) {
            ++k;
            p2 *= 2;
            p3 *= 3;
        }
        return 25 + k;
    }
    while (k < 23 && b * p2 > a * p3) {
        ++k;
        p2 *= 2;
        p3 *= 3;
    }
    return 25 - k;
}

// ---- warp helpers ------------------------------------------------------------
constexpr unsigned FULL = 0xFFFFFFFFu;

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ int warp_in_block() { return threadIdx.x >> 5; }

template<typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

__device__ __forceinline__ s32 warp_max_s32(s32 v) { return __reduce_max_sync(FULL, v); }

// Appends `pred` items to a global list with one atomic per warp; returns the
// slot for this lane (valid when pred). All lanes of the warp must call it.
__device__ __forceinline__ u32 warp_append(u32 *counter, bool pred) {
    unsigned mask = __ballot_sync(FULL, pred);
    if (mask == 0) return 0;
    int leader = __ffs(mask) - 1;
    u32 base = 0;
    if (lane_id() == leader) base = atomicAdd(counter, (u32) __popc(mask));
    base = __shfl_sync(FULL, base, leader);
    return base + (u32) __popc(mask & ((1u << lane_id()) - 1u));
}

// Block-wide version of warp_append: one global atomic per block. All
// threads of the block must call it; `sm` holds 33 u32.
__device__ __forceinline__ u32 block_append(u32 *counter, bool pred, u32 *sm) {
    const unsigned mask = __ballot_sync(FULL, pred);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) sm[w] = (u32) __popc(mask);
    __syncthreads();
    if (threadIdx.x == 0) {
        u32 tot = 0;
        for (u32 i = 0; i < (blockDim.x >> 5); ++i) {
            const u32 c = sm[i];
            sm[i] = tot;
            tot += c;
        }
        sm[32] = tot ? atomicAdd(counter, tot) : 0u;
    }
    __syncthreads();
    const u32 r = sm[32] + sm[w] + (u32) __popc(mask & ((1u << lane) - 1u));
    __syncthreads();
    return r;
}

__device__ __forceinline__ void set_error(u32 *err, u32 bits) { atomicOr(err, bits); }

// Grid-wide barrier for kernels launched with cudaLaunchCooperativeKernel
// (all blocks resident), with a bounded wait. bar[0] counts arrivals and
// bar[1] is the generation; both are zero before the launch. Thread 0 of each
// block arrives and polls the generation at most GRID_BARRIER_SPINS times
// (about a second); when that runs out it sets DEV_ERR_SPIN in *err. Returns
// false in every thread of the block once *err carries DEV_ERR_SPIN, so the
// caller leaves its loops; every later wait of the other blocks is bounded
// too, so the kernel ends and the host reads the error.
constexpr unsigned long long GRID_BARRIER_SPINS = 1ull << 24;

__device__ __forceinline__ bool grid_barrier(u32 *bar, u32 *err) {
    __shared__ u32 s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile u32 *vgen = bar + 1;
        const u32 gen = *vgen;
        __threadfence();
        if (atomicAdd(&bar[0], 1u) == gridDim.x * gridDim.y * gridDim.z - 1) {
            atomicExch(&bar[0], 0u);
            __threadfence();
            atomicAdd(&bar[1], 1u);
        } else {
            unsigned long long spins = 0;
            while (*vgen == gen) {
                if (++spins > GRID_BARRIER_SPINS) {
                    set_error(err, DEV_ERR_SPIN);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        s_ok = (*(volatile u32 *) err & DEV_ERR_SPIN) == 0u;
    }
    __syncthreads();
    return s_ok != 0u;
}

// Number of kernels this process has launched (every launch site calls
// note_launch()).
extern std::atomic<unsigned long long> g_kernel_launches;
// Launches of the calling host thread (graph capture counts its own launches
// with it while other threads may launch concurrently).
extern thread_local unsigned long long t_kernel_launches;
inline void note_launch() {
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    ++t_kernel_launches;
}

// Grid sizing: a multiple of the SM count, capped by the work.
inline u32 grid_for(u64 items, u32 per_block, u32 max_blocks = NUM_SMS_HINT * 16) {
    u64 b = (items + per_block - 1) / per_block;
    if (b == 0) b = 1;
    if (b > max_blocks) b = max_blocks;
    return (u32) b;
}

} // namespace hp
