// Diagnostics of the bounded waits (hp_selftest_barrier_timeout, declared in
// include/gpuheipa.h). The cooperative level loops wait for one another at
// grid barriers whose wait is bounded (grid_barrier, common.cuh): when a
// block does not arrive, the others give up after about a second, set an
// error bit and end, and the host reports an error instead of hanging. This
// entry point exercises exactly that path with a block that never arrives, so
// a test can check that the wait ends, that the error bit is reported, and
// that the device stays usable afterwards. No fault, trap or endless loop is
// involved.
#include "../../include/gpuheipa.h"
#include "common.cuh"
#include "context.h"

#include <cuda_runtime.h>

static_assert(HP_DEVERR_SPIN == hp::DEV_ERR_SPIN, "public and device error bits agree");

namespace hp {
namespace {

__global__ void k_barrier_selftest(u32 *bar, u32 *err, u32 absent) {
    if (blockIdx.x == absent) return;  // this block never reaches the barrier
    grid_barrier(bar, err);
}

} // namespace
} // namespace hp

extern "C" int hp_selftest_barrier_timeout(int device, uint32_t blocks, uint32_t *err_bits, double *ms) {
    if (!err_bits || blocks < 2) return HP_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return HP_ERR_ARG;
    }
    if (cudaSetDevice(device) != cudaSuccess) return HP_ERR_CUDA;
    int per_sm = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, hp::k_barrier_selftest, 32, 0) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return HP_ERR_CUDA;
    if ((uint64_t) blocks > (uint64_t) per_sm * (uint64_t) sms) return HP_ERR_ARG;  // must all be resident
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    hp::u32 *d = nullptr;
    int rc = HP_OK;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
        cudaEventCreate(&e1) != cudaSuccess || cudaMalloc(&d, 4 * sizeof(hp::u32)) != cudaSuccess) {
        rc = HP_ERR_CUDA;
    } else {
        hp::u32 *bar = d, *err = d + 2;
        hp::u32 absent = blocks - 1;
        void *args[] = {&bar, &err, &absent};
        hp::u32 h_err = 0;
        float t = 0.f;
        hp::CoopGuard coop(device, s, blocks, (hp::u32) sms);  // cooperative budget until the kernel has completed
        if (cudaMemsetAsync(d, 0, 4 * sizeof(hp::u32), s) != cudaSuccess || cudaEventRecord(e0, s) != cudaSuccess ||
            cudaLaunchCooperativeKernel((const void *) hp::k_barrier_selftest, dim3(blocks), dim3(32), args, 0, s) !=
                cudaSuccess ||
            cudaEventRecord(e1, s) != cudaSuccess ||
            cudaMemcpyAsync(&h_err, err, sizeof(hp::u32), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess || cudaEventElapsedTime(&t, e0, e1) != cudaSuccess) {
            rc = HP_ERR_CUDA;
        } else {
            *err_bits = h_err;
            if (ms) *ms = t;
        }
    }
    cudaGetLastError();
    if (d) cudaFree(d);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) cudaStreamDestroy(s);
    return rc;
}

extern "C" int hp_coop_slot_acquire(int device, int timeout_ms) {
    return hp::CoopSlots::try_acquire_all_for(device, timeout_ms) ? HP_OK : HP_ERR_BUSY;
}

extern "C" int hp_coop_slot_release(int device) {
    hp::CoopSlots::release_all(device);
    return HP_OK;
}
