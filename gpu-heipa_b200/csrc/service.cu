#include "service.cuh"

#include "../host/initial_partition.h"

namespace hp {

// ---- RegionAlloc -------------------------------------------------------------------

void RegionAlloc::reset(size_t bytes) {
    size_ = bytes;
    free_.clear();
    if (bytes) free_[0] = bytes;
}

bool RegionAlloc::alloc(size_t bytes, size_t &offset) {
    for (auto it = free_.begin(); it != free_.end(); ++it) {
        if (it->second < bytes) continue;
        offset = it->first;
        const size_t rest = it->second - bytes;
        free_.erase(it);
        if (rest) free_[offset + bytes] = rest;
        return true;
    }
    return false;
}

void RegionAlloc::release(size_t offset, size_t bytes) {
    auto it = free_.emplace(offset, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
        it->second += nx->second;
        free_.erase(nx);
    }
    if (it != free_.begin()) {
        auto pv = std::prev(it);
        if (pv->first + pv->second == it->first) {
            pv->second += it->second;
            free_.erase(it);
        }
    }
}

size_t RegionAlloc::largest_free() const {
    size_t b = 0;
    for (const auto &f: free_) b = std::max(b, f.second);
    return b;
}

// ---- Service ---------------------------------------------------------------------------

// A job may be overtaken by later, smaller jobs at most this many times; after
// that nothing else is admitted until it fits (no starvation of large jobs).
constexpr u32 MAX_BYPASS = 64;
constexpr size_t REGION_ALIGN = 4096;

Service::Service(Ctx &owner, char *base, size_t bytes, size_t workers) : device_(owner.device), base_(base) {
    t0_ = std::chrono::steady_clock::now();
    regions_.reset(bytes & ~(REGION_ALIGN - 1));
    if (workers == 0) workers = 1;
    for (size_t w = 0; w < workers; ++w) ctxs_.push_back(&owner.worker(w));
    for (size_t w = 0; w < workers; ++w) threads_.emplace_back([this, w] { worker_main(w); });
}

Service::~Service() {
    {
        std::lock_guard<std::mutex> lk(mu_);
        stop_ = true;
    }
    cv_work_.notify_all();
    for (std::thread &t: threads_) t.join();
}

double Service::now_ms() const {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0_).count();
}

u64 Service::submit(std::shared_ptr<Job> job) {
    job->bytes = (job->bytes + REGION_ALIGN - 1) & ~(REGION_ALIGN - 1);
    u64 id;
    {
        std::lock_guard<std::mutex> lk(mu_);
        id = next_id_++;
        job->t_submit = now_ms();
        jobs_[id] = job;
        queue_.push_back(id);
    }
    cv_work_.notify_one();
    return id;
}

bool Service::is_done(u64 id) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = jobs_.find(id);
    return it == jobs_.end() || it->second->done;
}

std::shared_ptr<Job> Service::wait(u64 id) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = jobs_.find(id);
    if (it == jobs_.end()) return nullptr;
    std::shared_ptr<Job> job = it->second;
    cv_done_.wait(lk, [&] { return job->done; });
    jobs_.erase(id);
    return job;
}

void Service::wait_all() {
    std::unique_lock<std::mutex> lk(mu_);
    cv_done_.wait(lk, [&] { return queue_.empty() && running_ == 0; });
}

void Service::worker_main(size_t w) {
    const bool dev_ok = cudaSetDevice(device_) == cudaSuccess;
    Ctx &c = *ctxs_[w];
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
        u64 id = 0;
        size_t off = 0;
        bool too_large = false;
        cv_work_.wait(lk, [&] {
            for (auto it = queue_.begin(); it != queue_.end(); ++it) {
                Job &j = *jobs_[*it];
                if (j.bytes > regions_.total()) {
                    too_large = true;
                } else if (!regions_.alloc(j.bytes, off)) {
                    // the oldest waiting job blocks later ones once it has
                    // been overtaken often enough
                    if (j.bypassed >= MAX_BYPASS) return false;
                    continue;
                }
                id = *it;
                for (auto jt = queue_.begin(); jt != it; ++jt) ++jobs_[*jt]->bypassed;
                queue_.erase(it);
                return true;
            }
            return stop_ && queue_.empty();
        });
        if (id == 0) return;  // stopping and nothing left
        std::shared_ptr<Job> job = jobs_[id];
        job->t_start = now_ms();
        if (too_large || !dev_ok) {
            job->status = too_large ? HP_ERR_OOM : HP_ERR_DEVICE;
            job->error = too_large ? "request needs more device memory than the service buffer holds"
                                   : "worker could not select the device";
            job->t_end = job->t_start;
            job->done = true;
            cv_done_.notify_all();
            continue;
        }
        ++running_;
        lk.unlock();
        c.arena.attach(base_ + off, job->bytes);
        try {
            c.zero_status();
            job->objective = job->run(c);
            c.sync();
        } catch (const HpError &e) {
            job->status = e.code;
            job->error = e.msg;
        } catch (const std::bad_alloc &) {
            job->status = HP_ERR_OOM;
            job->error = "host allocation failed";
        } catch (const std::exception &e) {
            job->status = HP_ERR_ARG;
            job->error = e.what();
        }
        if (job->status != HP_OK) cudaStreamSynchronize(c.stream);
        c.arena.destroy();  // detaches the slice
        lk.lock();
        regions_.release(off, job->bytes);
        --running_;
        job->t_end = now_ms();
        job->done = true;
        cv_done_.notify_all();
        cv_work_.notify_all();
    }
}

}  // namespace hp
