// Edge cut of a caller-owned device CSR graph, computed without allocating
// any memory: hp_edge_cut_noalloc (declared in include/gpuheipa.h).
//
// Who needs it: a caller that holds its graph in device memory it does not
// want to hand over (a PyTorch tensor, a serving engine's pre-reserved pool)
// and that must not allocate device memory while it serves a request.
// cudaMalloc/cudaFree synchronise the whole device (stalling every other
// stream of the process), can fail when a caching allocator has reserved most
// of HBM, and would make the call's footprint depend on the request. The
// arena-backed hp_edge_cut needs an hp_ctx whose arena is sized for whole
// solves (gigabytes). This entry point instead uses one fixed scratch area in
// static device memory of this module, reserved by the driver when the module
// is loaded: 256 bytes of counters plus room for a partition of up to
// HP_EDGE_CUT_NOALLOC_MAX_N labels (16 MiB + 256 B in total).
//
// The objective is edge_cut (src/utility/edge_cut.h:71-90): the sum over CSR
// entries (u, v) with part[u] != part[v] of the entry's weight, halved because
// every undirected edge appears twice.
#include "../../include/gpuheipa.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

namespace {

constexpr uint32_t kMaxN = HP_EDGE_CUT_NOALLOC_MAX_N;
constexpr size_t kHeadBytes = 256;  // counters: [0] weighted cut entries, [1] rejected rows/entries
constexpr size_t kScratchBytes = kHeadBytes + sizeof(uint32_t) * (size_t) kMaxN;
constexpr int kMaxDevices = 64;
constexpr int kBlock = 256;
constexpr int kBlocksPerSm = 8;

}  // namespace

// One scratch area per device: the module's copy of this variable on each
// device. The counters must be zero when the kernel starts; every call clears
// them on its stream before the launch. The partition staging area needs no
// initial value: each call overwrites entries [0, n) and reads only those.
static __device__ __align__(256) unsigned char g_cut_scratch[kScratchBytes];

namespace {

struct DeviceScratch {
    unsigned char *base = nullptr;  // device address of g_cut_scratch on this device
    int sms = 0;
};

std::mutex g_setup_mu;
DeviceScratch g_scratch[kMaxDevices];

// First call per device: resolve the address of the static scratch with that
// device current (this also makes the driver load the module there) and read
// the SM count for the grid size. Later calls only read the table.
int scratch_for_device(int dev, DeviceScratch *out) {
    std::lock_guard<std::mutex> lock(g_setup_mu);
    DeviceScratch &s = g_scratch[dev];
    if (!s.base) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_cut_scratch) != cudaSuccess || !p) return HP_ERR_CUDA;
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
            return HP_ERR_CUDA;
        s.sms = sms;
        s.base = static_cast<unsigned char *>(p);
    }
    *out = s;
    return HP_OK;
}

// The pointer must be device (or managed) memory usable from device `dev`;
// host memory would fault in the kernel, so it is rejected here.
bool on_device(const void *p, int dev) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();  // clear the non-sticky error of the query
        return false;
    }
    if (a.type == cudaMemoryTypeManaged) return true;
    return a.type == cudaMemoryTypeDevice && a.device == dev;
}

// `part` is read on the host (copied into the scratch area), so device memory
// there is a caller error.
bool is_device_memory(const void *p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice;
}

// Every failing CUDA call leaves its error in the runtime's per-thread state;
// clear it so that it is not reported later against the caller's own work.
int cuda_failure() {
    cudaGetLastError();
    return HP_ERR_CUDA;
}

// One warp per vertex (grid-stride over warps). Every row and entry is bounds
// checked against n and m: a row with xadj[u+1] < xadj[u] or xadj[u+1] > m, an
// entry with adj[e] >= n, or an edge weight <= 0 (hp_graph_upload rejects the
// same graphs) is skipped and counted in counters[1], so bad input yields an
// error status and never an out-of-range access.
__global__ void __launch_bounds__(kBlock)
k_edge_cut_staged(uint32_t n, uint32_t m, const uint32_t *__restrict__ xadj, const uint32_t *__restrict__ adj,
                  const int32_t *__restrict__ ew, const uint32_t *__restrict__ part,
                  unsigned long long *__restrict__ counters) {
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    long long acc = 0;
    unsigned long long bad = 0;
    for (uint32_t u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < n; u += warps) {
        const uint32_t beg = xadj[u];
        const uint32_t end = xadj[u + 1];
        if (end < beg || end > m) {
            bad += lane == 0;
            continue;
        }
        const uint32_t pu = part[u];
        for (uint32_t e = beg + lane; e < end; e += 32) {
            const uint32_t v = adj[e];
            const int32_t w = ew ? ew[e] : 1;
            if (v >= n || w <= 0) {
                ++bad;
                continue;
            }
            if (part[v] != pu) acc += (long long) w;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        acc += __shfl_xor_sync(0xffffffffu, acc, o);
        bad += __shfl_xor_sync(0xffffffffu, bad, o);
    }
    if (lane == 0) {
        if (acc) atomicAdd(&counters[0], (unsigned long long) acc);
        if (bad) atomicAdd(&counters[1], bad);
    }
}

}  // namespace

extern "C" int hp_edge_cut_noalloc(uint32_t n, uint32_t m, const uint32_t *d_xadj, const uint32_t *d_adj,
                                   const int32_t *d_ew, const uint32_t *part, void *stream, int64_t *cut) {
    if (!cut || !d_xadj || !part || (m > 0 && !d_adj)) return HP_ERR_ARG;
    if (n > kMaxN) return HP_ERR_TOO_LARGE;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return HP_ERR_CUDA;
    if (dev < 0 || dev >= kMaxDevices) return HP_ERR_DEVICE;
    if (!on_device(d_xadj, dev) || (m > 0 && !on_device(d_adj, dev)) || (d_ew && !on_device(d_ew, dev)))
        return HP_ERR_ARG;
    if (is_device_memory(part)) return HP_ERR_ARG;
    DeviceScratch s;
    const int rc = scratch_for_device(dev, &s);
    if (rc != HP_OK) return rc == HP_ERR_CUDA ? cuda_failure() : rc;

    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned long long *counters = reinterpret_cast<unsigned long long *>(s.base);
    uint32_t *staged = reinterpret_cast<uint32_t *>(s.base + kHeadBytes);
    if (cudaMemsetAsync(counters, 0, 2 * sizeof(unsigned long long), st) != cudaSuccess) return cuda_failure();
    if (n > 0) {
        if (cudaMemcpyAsync(staged, part, sizeof(uint32_t) * (size_t) n, cudaMemcpyHostToDevice, st) != cudaSuccess)
            return cuda_failure();
        const uint64_t want = ((uint64_t) n * 32 + kBlock - 1) / kBlock;
        const uint64_t cap = (uint64_t) s.sms * kBlocksPerSm;
        const unsigned grid = (unsigned) (want < cap ? want : cap);
        k_edge_cut_staged<<<grid, kBlock, 0, st>>>(n, m, d_xadj, d_adj, d_ew, staged, counters);
        if (cudaGetLastError() != cudaSuccess) return HP_ERR_CUDA;  // (cudaGetLastError cleared it)
    }
    unsigned long long host[2] = {0, 0};
    if (cudaMemcpyAsync(host, counters, sizeof(host), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return cuda_failure();
    if (cudaStreamSynchronize(st) != cudaSuccess) return cuda_failure();
    if (host[1] != 0) return HP_ERR_GRAPH;
    // every accepted weight is positive, so the sum of directed entries is a
    // non-negative int64; each undirected edge is counted twice
    *cut = (int64_t) host[0] / 2;
    return HP_OK;
}
