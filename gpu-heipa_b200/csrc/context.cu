#include "context.h"

#include <chrono>
#include <condition_variable>
#include <map>
#include <mutex>

namespace hp {

std::atomic<unsigned long long> g_kernel_launches{0};
thread_local unsigned long long t_kernel_launches = 0;

static constexpr size_t ALIGN = 256;

static size_t align_up(size_t x) { return (x + ALIGN - 1) & ~(ALIGN - 1); }

void Arena::init(size_t bytes) {
    bytes = align_up(bytes);
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw HpError{HP_ERR_OOM, "device arena of " + std::to_string(bytes) + " bytes could not be allocated: " +
                                      cudaGetErrorString(e)};
    }
    base_ = (char *) p;
    size_ = bytes;
    front_ = 0;
    back_ = bytes;
    peak_ = 0;
}

void Arena::attach(void *p, size_t bytes) {
    // every allocation is ALIGN-aligned (kernels read CSR arrays with 16-byte
    // vector loads), so the base is rounded up to ALIGN
    const uintptr_t at = ((uintptr_t) p + ALIGN - 1) & ~(uintptr_t) (ALIGN - 1);
    const size_t skip = (size_t) (at - (uintptr_t) p);
    bytes = bytes > skip ? bytes - skip : 0;
    base_ = (char *) at;
    size_ = bytes & ~(ALIGN - 1);
    front_ = 0;
    back_ = size_;
    peak_ = 0;
    owns_ = false;
}

void Arena::destroy() {
    if (base_ && owns_) cudaFree(base_);
    base_ = nullptr;
    size_ = front_ = back_ = peak_ = 0;
    owns_ = true;
}

void *Arena::front(size_t bytes) {
    bytes = align_up(bytes == 0 ? 1 : bytes);
    if (front_ + bytes > back_)
        throw HpError{HP_ERR_OOM, "device arena exhausted (front request " + std::to_string(bytes) + " bytes, " +
                                      std::to_string(back_ - front_) + " free of " + std::to_string(size_) + ")"};
    void *p = base_ + front_;
    front_ += bytes;
    if (used() > peak_) peak_ = used();
    return p;
}

void *Arena::back(size_t bytes) {
    bytes = align_up(bytes == 0 ? 1 : bytes);
    if (back_ < front_ + bytes)
        throw HpError{HP_ERR_OOM, "device arena exhausted (scratch request " + std::to_string(bytes) + " bytes, " +
                                      std::to_string(back_ - front_) + " free of " + std::to_string(size_) + ")"};
    back_ -= bytes;
    if (used() > peak_) peak_ = used();
    return base_ + back_;
}

void Ctx::init(int dev, size_t arena_bytes) {
    device = dev;
    HP_CUDA(cudaSetDevice(dev));
    HP_CUDA(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, dev));
    HP_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    HP_CUDA(cudaMalloc(&d_status, sizeof(DevStatus)));
    HP_CUDA(cudaHostAlloc(&h_status, sizeof(DevStatus), cudaHostAllocDefault));
    HP_CUDA(cudaMemsetAsync(d_status, 0, sizeof(DevStatus), stream));
    if (arena_bytes) arena.init(arena_bytes);
}

cudaEvent_t Instr::get_event() {
    if (!pool.empty()) {
        cudaEvent_t e = pool.back();
        pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    HP_CUDA(cudaEventCreate(&e));
    return e;
}

size_t Instr::begin(cudaStream_t s, const char *name, double bytes) {
    if (!enabled || capturing) return SIZE_MAX;
    Rec r;
    r.name = name;
    r.a = get_event();
    r.b = get_event();
    r.bytes = bytes;
    HP_CUDA(cudaEventRecord(r.a, s));
    pending.push_back(r);
    return pending.size() - 1;
}

void Instr::end(cudaStream_t s, size_t idx) {
    if (!enabled || idx >= pending.size()) return;
    HP_CUDA(cudaEventRecord(pending[idx].b, s));
}

KernTimer::KernTimer(Ctx &ctx, const char *name, double bytes) : c(ctx) {
    idx = c.instr.begin(c.stream, name, bytes);
}

KernTimer::~KernTimer() { c.instr.end(c.stream, idx); }

void Instr::resolve() {
    for (Rec &r: pending) {
        float ms = 0.f;
        HP_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
        Total *t = nullptr;
        for (Total &x: totals)
            if (x.name == r.name) t = &x;
        if (!t) {
            totals.push_back(Total{r.name});
            t = &totals.back();
        }
        t->launches += 1;
        t->ms += ms;
        t->bytes += r.bytes;
        if (log.size() < LOG_MAX) log.push_back(Logged{r.name, (double) ms, r.bytes});
        pool.push_back(r.a);
        pool.push_back(r.b);
    }
    pending.clear();
}

void Instr::clear() {
    for (Rec &r: pending) {
        pool.push_back(r.a);
        pool.push_back(r.b);
    }
    pending.clear();
    totals.clear();
    log.clear();
}

void Instr::destroy() {
    clear();
    for (cudaEvent_t e: pool) cudaEventDestroy(e);
    pool.clear();
}

void PhaseProf::add(const char *name, double ms) {
    for (size_t i = 0; i < totals.size(); ++i)
        if (totals[i].first == name) {
            totals[i].second += ms;
            counts[i].second += 1;
            return;
        }
    totals.emplace_back(name, ms);
    counts.emplace_back(name, 1);
}

static double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

ProfScope::ProfScope(Ctx &ctx, const char *nm) : c(ctx), name(nm) {
    if (!c.prof.enabled || c.prof.capturing) return;
    cudaStreamSynchronize(c.stream);
    t0 = now_ms();
}

ProfScope::~ProfScope() {
    if (!c.prof.enabled || c.prof.capturing) return;
    cudaStreamSynchronize(c.stream);
    c.prof.add(name, now_ms() - t0);
}

cudaEvent_t Ctx::event(int slot) {
    if (slot < 0 || slot >= 8) throw HpError{HP_ERR_ARG, "event slot out of range"};
    if (!events[slot]) HP_CUDA(cudaEventCreate(&events[slot]));
    return events[slot];
}

Ctx &Ctx::worker(size_t i) {
    while (workers.size() <= i) {
        std::unique_ptr<Ctx> w(new Ctx());
        try {
            w->init(device, 0);
        } catch (...) {
            w->destroy();
            throw;
        }
        workers.push_back(std::move(w));
    }
    workers[i]->tune = tune;
    return *workers[i];
}

void Ctx::destroy() {
    for (auto &w: workers) w->destroy();
    workers.clear();
    if (stream) cudaStreamSynchronize(stream);
    for (cudaEvent_t &e: events)
        if (e) {
            cudaEventDestroy(e);
            e = nullptr;
        }
    instr.destroy();
    arena.destroy();
    if (d_status) cudaFree(d_status);
    if (h_status) cudaFreeHost(h_status);
    if (stream) cudaStreamDestroy(stream);
    d_status = nullptr;
    h_status = nullptr;
    stream = nullptr;
}

namespace {
std::mutex g_coop_mu;
std::condition_variable g_coop_cv;
// device -> blocks of cooperative grids running; ALL_TAKEN while one caller
// holds the whole budget
std::map<int, unsigned long long> g_coop_used;
constexpr unsigned long long ALL_TAKEN = ~0ull;
inline u32 share_of(u32 blocks, u32 budget) {
    if (budget == 0) budget = 1;
    return blocks == 0 ? 1u : (blocks < budget ? blocks : budget);
}
}  // namespace

void CoopSlots::acquire(int device, u32 blocks, u32 budget) {
    const u32 t = share_of(blocks, budget);
    std::unique_lock<std::mutex> lock(g_coop_mu);
    unsigned long long &used = g_coop_used[device];
    g_coop_cv.wait(lock, [&] { return used != ALL_TAKEN && used + t <= (budget ? budget : 1u); });
    used += t;
}

void CoopSlots::release(int device, u32 blocks, u32 budget) {
    const u32 t = share_of(blocks, budget);
    {
        std::lock_guard<std::mutex> lock(g_coop_mu);
        unsigned long long &used = g_coop_used[device];
        if (used != ALL_TAKEN) used = used >= t ? used - t : 0;
    }
    g_coop_cv.notify_all();
}

bool CoopSlots::try_acquire_all_for(int device, int timeout_ms) {
    std::unique_lock<std::mutex> lock(g_coop_mu);
    unsigned long long &used = g_coop_used[device];
    if (!g_coop_cv.wait_for(lock, std::chrono::milliseconds(timeout_ms < 0 ? 0 : timeout_ms), [&] { return used == 0; }))
        return false;
    used = ALL_TAKEN;
    return true;
}

void CoopSlots::release_all(int device) {
    {
        std::lock_guard<std::mutex> lock(g_coop_mu);
        g_coop_used[device] = 0;
    }
    g_coop_cv.notify_all();
}

void Ctx::zero_status() { HP_CUDA(cudaMemsetAsync(d_status, 0, sizeof(DevStatus), stream)); }

void Ctx::zero_counters() {
    HP_CUDA(cudaMemsetAsync((char *) d_status + sizeof(u32), 0, sizeof(DevStatus) - sizeof(u32), stream));
}

const DevStatus &Ctx::read_status() {
    HP_CUDA(cudaMemcpyAsync(h_status, d_status, sizeof(DevStatus), cudaMemcpyDeviceToHost, stream));
    HP_CUDA(cudaStreamSynchronize(stream));
    return *h_status;
}

void Ctx::sync() { HP_CUDA(cudaStreamSynchronize(stream)); }

void Ctx::check_device_error() {
    const DevStatus &s = read_status();
    if (s.err != 0) throw HpError{HP_ERR_DEVICE, "device reported error bits 0x" + std::to_string(s.err)};
}

} // namespace hp
