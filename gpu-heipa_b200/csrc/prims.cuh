// Device-wide primitives: block scan, reduce-then-scan over a functor, stable
// select (compaction) and a stable LSD radix sort of (key, u32 value) pairs.
// All are deterministic: results never depend on thread scheduling.
#pragma once
#include "context.h"

namespace hp {

// Exclusive scan of one value per thread across the block; `total` receives
// the block sum. `smem` must hold 32 elements. All threads must call it.
template<typename T>
__device__ __forceinline__ T block_exclusive_scan(T v, T &total, T *smem) {
    const int lane = lane_id(), w = warp_in_block(), nw = blockDim.x >> 5;
    T x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(FULL, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) smem[w] = x;
    __syncthreads();
    if (w == 0) {
        T s = lane < nw ? smem[lane] : T(0);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T y = __shfl_up_sync(FULL, s, o);
            if (lane >= o) s += y;
        }
        if (lane < nw) smem[lane] = s;
    }
    __syncthreads();
    T wp = w > 0 ? smem[w - 1] : T(0);
    total = smem[nw - 1];
    __syncthreads();
    return wp + x - v;
}

constexpr int SCAN_ITEMS = 16;
constexpr int SCAN_TILE = BLOCK * SCAN_ITEMS;

// Element count of a launch sized for n_max elements: min(n_max, *dn + add)
// when a device count is given (read by the kernel, so the launch needs no
// host synchronisation and can be captured in a CUDA graph).
__device__ __forceinline__ u64 count_of(u64 n_max, const u32 *dn, u32 add) {
    if (!dn) return n_max;
    const u64 c = (u64) *dn + add;
    return c < n_max ? c : n_max;
}

template<typename T, typename Load>
__global__ void __launch_bounds__(BLOCK) k_scan_reduce(u64 n, const u32 *dn, u32 dn_add, Load load, T *tile_sums) {
    __shared__ T sm[32];
    n = count_of(n, dn, dn_add);
    const u64 base = (u64) blockIdx.x * SCAN_TILE;
    T s = T(0);
#pragma unroll 4
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        u64 idx = base + (u64) i * BLOCK + threadIdx.x;
        if (idx < n) s += load(idx);
    }
    T total;
    block_exclusive_scan<T>(s, total, sm);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

template<typename T>
__global__ void __launch_bounds__(1024) k_scan_tiles(T *sums, u32 ntiles, T *total_out) {
    __shared__ T sm[32];
    T carry = T(0);
    for (u32 base = 0; base < ntiles; base += blockDim.x) {
        u32 i = base + threadIdx.x;
        T v = i < ntiles ? sums[i] : T(0);
        T tot;
        T p = block_exclusive_scan<T>(v, tot, sm);
        if (i < ntiles) sums[i] = carry + p;
        carry += tot;
    }
    if (threadIdx.x == 0 && total_out) *total_out = carry;
}

template<typename T, typename Load, typename Store>
__global__ void __launch_bounds__(BLOCK) k_scan_apply(u64 n, const u32 *dn, u32 dn_add, Load load, Store store,
                                                      const T *tile_offsets) {
    __shared__ T sm[32];
    n = count_of(n, dn, dn_add);
    if ((u64) blockIdx.x * SCAN_TILE >= n) return;
    const u64 base = (u64) blockIdx.x * SCAN_TILE + (u64) threadIdx.x * SCAN_ITEMS;
    T vals[SCAN_ITEMS];
    T s = T(0);
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        u64 idx = base + i;
        vals[i] = idx < n ? load(idx) : T(0);
        s += vals[i];
    }
    T total;
    T pre = block_exclusive_scan<T>(s, total, sm) + tile_offsets[blockIdx.x];
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        u64 idx = base + i;
        if (idx < n) store(idx, pre, vals[i]);
        pre += vals[i];
    }
}

// Exclusive scan over i in [0, n): prefix(i) = sum_{j<i} load(j); calls
// store(i, prefix(i), load(i)) for every i. Writes the total to *total_dev
// when given (device pointer). With dn, n is min(n, *dn + dn_add), read on
// the device. Deterministic for integer T.
template<typename T, typename Load, typename Store>
void device_scan(Ctx &ctx, u64 n, Load load, Store store, T *total_dev, const u32 *dn = nullptr, u32 dn_add = 0) {
    ScratchScope ss(ctx.arena);
    u64 nt = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (nt == 0) nt = 1;
    T *sums = ctx.balloc<T>(nt);
    k_scan_reduce<T><<<(u32) nt, BLOCK, 0, ctx.stream>>>(n, dn, dn_add, load, sums); note_launch();
    k_scan_tiles<T><<<1, 1024, 0, ctx.stream>>>(sums, (u32) nt, total_dev); note_launch();
    k_scan_apply<T><<<(u32) nt, BLOCK, 0, ctx.stream>>>(n, dn, dn_add, load, store, sums); note_launch();
    HP_LAUNCH_CHECK();
}

// Stable compaction: writes item(i) for every i with pred(i) to out, in
// ascending i; the count goes to *count_dev.
template<typename Pred, typename Item>
void device_select(Ctx &ctx, u64 n, Pred pred, Item item, u32 *out, u32 *count_dev) {
    device_scan<u32>(
        ctx, n, [=] __device__(u64 i) -> u32 { return pred(i) ? 1u : 0u; },
        [=] __device__(u64 i, u32 p, u32 v) {
            if (v) out[p] = item(i);
        },
        count_dev);
}

// ---- stable LSD radix sort of (key, value) pairs -----------------------------
constexpr int RS_ITEMS = 16;
constexpr int RS_TILE = BLOCK * RS_ITEMS;

template<typename K>
__global__ void __launch_bounds__(BLOCK) k_rs_hist(const K *keys, u64 n, const u32 *dn, int shift, u32 *hist,
                                                   u32 ntiles) {
    __shared__ u32 cnt[256];
    n = count_of(n, dn, 0);
    cnt[threadIdx.x] = 0;
    __syncthreads();
    const u64 base = (u64) blockIdx.x * RS_TILE;
    for (int i = 0; i < RS_ITEMS; ++i) {
        u64 idx = base + (u64) i * BLOCK + threadIdx.x;
        if (idx < n) atomicAdd(&cnt[(u32) (keys[idx] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[(u64) threadIdx.x * ntiles + blockIdx.x] = cnt[threadIdx.x];
}

template<typename K>
__global__ void __launch_bounds__(BLOCK) k_rs_scatter(const K *kin, const u32 *vin, K *kout, u32 *vout, u64 n,
                                                       const u32 *dn, int shift, const u32 *offs, u32 ntiles) {
    n = count_of(n, dn, 0);
    if ((u64) blockIdx.x * RS_TILE >= n) return;
    __shared__ u32 run[256];
    __shared__ u32 wc[BLOCK / 32][256];
    const int t = threadIdx.x, w = warp_in_block(), lane = lane_id();
    run[t] = offs[(u64) t * ntiles + blockIdx.x];
    const u64 base = (u64) blockIdx.x * RS_TILE;
    const unsigned lt_mask = (1u << lane) - 1u;
    for (int r = 0; r < RS_ITEMS; ++r) {
#pragma unroll
        for (int x = 0; x < BLOCK / 32; ++x) wc[x][t] = 0;
        __syncthreads();
        const u64 idx = base + (u64) r * BLOCK + t;
        const bool valid = idx < n;
        K k = valid ? kin[idx] : K(0);
        u32 d = valid ? ((u32) (k >> shift) & 255u) : 256u;
        unsigned mask = __match_any_sync(FULL, d);
        u32 rank = (u32) __popc(mask & lt_mask);
        bool leader = (__ffs(mask) - 1) == lane;
        if (valid && leader) wc[w][d] = (u32) __popc(mask);
        __syncthreads();
        if (valid) {
            u32 off = run[d] + rank;
            for (int x = 0; x < w; ++x) off += wc[x][d];
            kout[off] = k;
            vout[off] = vin[idx];
        }
        __syncthreads();
        u32 add = 0;
#pragma unroll
        for (int x = 0; x < BLOCK / 32; ++x) add += wc[x][t];
        run[t] += add;
        __syncthreads();
    }
}

// Sorts n pairs by key bits [begin_bit, end_bit), stably; keys/vals are
// updated in place (scratch double buffers come from the arena's back end).
// With dn, the pair count is min(n, *dn), read on the device (buffers are
// sized for n).
template<typename K>
void radix_sort_pairs(Ctx &ctx, K *keys, u32 *vals, u64 n, int begin_bit, int end_bit, const u32 *dn = nullptr) {
    if (n <= 1 || end_bit <= begin_bit) return;
    ScratchScope ss(ctx.arena);
    u32 ntiles = (u32) ((n + RS_TILE - 1) / RS_TILE);
    K *k_alt = ctx.balloc<K>(n);
    u32 *v_alt = ctx.balloc<u32>(n);
    u32 *hist = ctx.balloc<u32>((u64) 256 * ntiles);
    K *ks = keys, *kd = k_alt;
    u32 *vs = vals, *vd = v_alt;
    for (int shift = begin_bit; shift < end_bit; shift += 8) {
        k_rs_hist<K><<<ntiles, BLOCK, 0, ctx.stream>>>(ks, n, dn, shift, hist, ntiles); note_launch();
        u64 hn = (u64) 256 * ntiles;
        device_scan<u32>(
            ctx, hn, [=] __device__(u64 i) -> u32 { return hist[i]; },
            [=] __device__(u64 i, u32 p, u32) { hist[i] = p; }, (u32 *) nullptr);
        k_rs_scatter<K><<<ntiles, BLOCK, 0, ctx.stream>>>(ks, vs, kd, vd, n, dn, shift, hist, ntiles); note_launch();
        HP_LAUNCH_CHECK();
        std::swap(ks, kd);
        std::swap(vs, vd);
    }
    if (ks != keys) {
        HP_CUDA(cudaMemcpyAsync(keys, ks, sizeof(K) * n, cudaMemcpyDeviceToDevice, ctx.stream));
        HP_CUDA(cudaMemcpyAsync(vals, vs, sizeof(u32) * n, cudaMemcpyDeviceToDevice, ctx.stream));
    }
}

// Number of significant bits of x (0 for x == 0).
inline int bits_for(u64 x) {
    int b = 0;
    while (x) {
        ++b;
        x >>= 1;
    }
    return b;
}

template<typename T>
__global__ void k_fill(T *p, u64 n, T v) {
    for (u64 i = (u64) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64) gridDim.x * blockDim.x) p[i] = v;
}

template<typename T>
void device_fill(Ctx &ctx, T *p, u64 n, T v) {
    if (n == 0) return;
    k_fill<T><<<ctx.grid(n, BLOCK), BLOCK, 0, ctx.stream>>>(p, n, v); note_launch();
    HP_LAUNCH_CHECK();
}

__global__ void k_iota(u32 *p, u64 n);
void device_iota(Ctx &ctx, u32 *p, u64 n);

} // namespace hp
