// Many placements on one GPU at once: the batched and served forms.
//
// A single placement is a latency-bound chain of small kernels (about 30 per
// controller iteration) that leaves most of the B200 idle, so throughput comes
// from running many placements at the same time.  The Server keeps a FIFO of
// submitted jobs (each a full adaptive global placement, as mpgp_global_place)
// and a pool of worker threads; each worker runs one job at a time as a
// device-resident Session.  In the batched mode (the default) the running jobs'
// evaluations are gathered into shared rounds (Batch): one launch per kernel
// family carries the iteration of every running job.  Otherwise each session
// launches on its own streams and the jobs' kernels merely overlap.  A job is
// admitted when its estimated device footprint fits in what the memory budget
// has left (continuous batching: a job that arrives while others run joins the
// rounds as soon as a worker and the memory are free).  A job's result does not
// depend on what else runs: every session owns its buffers, every block of a
// batched launch does what the same block of the job's own launch does, and the
// reductions run in a fixed order.
#pragma once

#include <condition_variable>
#include <cstdint>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "mpgp.h"

namespace mpgp {

class Batch;

// Upper bound of the device bytes a Session for this design reserves.
uint64_t estimateSessionBytes(const mpgp_design& design, const mpgp_options& options);

class Server {
public:
    // batched: the running jobs' evaluations share batched launches (Batch);
    // otherwise each job launches its own kernels on its own streams.
    Server(int device, uint64_t memory_budget, int workers, bool batched = true);
    ~Server();
    Server(const Server&) = delete;
    Server& operator=(const Server&) = delete;

    // Copies the design and options; returns the job id.
    int64_t submit(const mpgp_design& design, const mpgp_options& options);
    // Waits up to timeout_seconds (< 0: no limit) for the job; returns whether it is done.
    bool wait(int64_t job, double timeout_seconds);
    // Copies a finished job's outputs out and forgets the job.  Throws the job's
    // failure (as an Error with its status) when it failed.
    void take(int64_t job, double* module_x, double* module_y, mpgp_result* result, mpgp_history_row* history,
              int capacity, mpgp_job_stats* stats);
    [[nodiscard]] mpgp_server_stats stats() const;

private:
    struct Job;
    void work();
    bool admissible(const Job& job) const;

    int device_;
    uint64_t budget_;
    std::unique_ptr<Batch> batch_;
    mutable std::mutex mutex_;
    std::condition_variable ready_;  // queue or admission changed
    std::condition_variable done_;   // a job finished
    std::deque<std::shared_ptr<Job>> queue_;
    std::map<int64_t, std::shared_ptr<Job>> jobs_;
    std::vector<std::thread> workers_;
    bool stopping_ = false;
    int64_t next_id_ = 1;
    uint64_t reserved_ = 0;
    int running_ = 0;
    mpgp_server_stats stats_{};
    double started_ = 0.0;
};

}  // namespace mpgp
