// Concurrent execution of independent partitioning / mapping requests on one
// GPU: the batched path (a list of graphs) and the serving loop (requests
// that arrive over time). Requests are admitted by a device-memory estimate
// into a region of one preallocated buffer; admitted requests run on worker
// contexts (own host thread, stream and status word each), so the coarsening
// and refinement levels of different requests overlap on the device. Every
// request runs exactly the code of the plain path on its own arena slice, so
// its result does not depend on what else is running.
#pragma once
#include <chrono>
#include <condition_variable>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "context.h"

namespace hp {

// First-fit allocator of byte ranges of one device buffer (host bookkeeping
// only; callers hold the service lock).
class RegionAlloc {
public:
    void reset(size_t bytes);
    bool alloc(size_t bytes, size_t &offset);
    void release(size_t offset, size_t bytes);
    size_t largest_free() const;
    size_t total() const { return size_; }

private:
    size_t size_ = 0;
    std::map<size_t, size_t> free_;  // offset -> length
};

struct Job {
    size_t bytes = 0;                     // arena bytes the request may use
    std::function<s64(Ctx &)> run;        // executes on a worker context; returns the objective
    int status = HP_OK;
    std::string error;
    s64 objective = 0;
    double t_submit = 0, t_start = 0, t_end = 0;  // milliseconds on the service clock
    bool done = false;
    u32 bypassed = 0;  // times a later job was admitted ahead of this one
};

class Service {
public:
    // Serves requests from a device buffer [base, base + bytes) with up to
    // `workers` concurrently running requests; the worker contexts are
    // owner.worker(0 .. workers-1) (created on first use, kept by owner).
    Service(Ctx &owner, char *base, size_t bytes, size_t workers);
    ~Service();
    Service(const Service &) = delete;
    Service &operator=(const Service &) = delete;

    // Queues a job; returns its id. Jobs larger than the whole buffer fail
    // with HP_ERR_OOM when a worker takes them.
    u64 submit(std::shared_ptr<Job> job);
    // Blocks until job `id` is done and returns it (the service forgets it).
    std::shared_ptr<Job> wait(u64 id);
    bool is_done(u64 id);
    void wait_all();
    double now_ms() const;

private:
    void worker_main(size_t w);
    int device_;
    char *base_;
    RegionAlloc regions_;
    std::vector<Ctx *> ctxs_;
    std::vector<std::thread> threads_;
    std::mutex mu_;
    std::condition_variable cv_work_, cv_done_;
    std::deque<u64> queue_;
    std::unordered_map<u64, std::shared_ptr<Job> > jobs_;
    u64 next_id_ = 1;
    size_t running_ = 0;
    bool stop_ = false;
    std::chrono::steady_clock::time_point t0_;
};

}  // namespace hp
