// Iterations of many placements batched into shared launches (the batched and
// served forms).
//
// Each placement keeps its own device-resident Session and Engine, driven by its
// own host thread with the unchanged control law.  When an engine of a Batch
// evaluates, it hands its evaluation plan (Engine::plan: every kernel's
// arguments) to the batch instead of launching it.  The batch thread collects the
// plans that arrive together -- all attached engines, or those that arrived
// within a short window -- uploads their argument blocks in one copy and
// launches each kernel family ONCE over all of them: one scatter, one wirelength
// pass, one metrics pass, one launch per contraction stage (per K split), one
// gather and one reduction for the whole round, instead of about ten launches
// and a host round trip per placement.  Every block of a batched launch does
// exactly what the same block of the placement's own launch would (the kernels
// share one body, see kernels.cuh), so a placement's result is bit-identical to
// its plain run, whatever else is in the batch.
#pragma once

#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "engine.cuh"

namespace mpgp {

struct BatchStats {
    int64_t rounds = 0;        // batched rounds launched
    int64_t evaluations = 0;   // evaluations they carried
    int64_t launches = 0;      // kernel launches of all rounds
    int peak_round = 0;        // most evaluations in one round
    double busy_seconds = 0.0;    // host time from each round's upload to its completion, summed
    double device_seconds = 0.0;  // device time of the rounds (CUDA events around each round), summed
};

class Batch {
public:
    // window_seconds: how long a round waits for the attached engines that have
    // not yet handed in their evaluation before it launches without them.
    Batch(int device, double window_seconds = 300e-6);
    ~Batch();
    Batch(const Batch&) = delete;
    Batch& operator=(const Batch&) = delete;

    [[nodiscard]] cudaStream_t stream() const { return stream_; }
    [[nodiscard]] int device() const { return device_; }
    // An engine takes part in rounds between attach and detach.
    void attach(Engine* engine);
    void detach(Engine* engine);
    // Runs the plan in the next round; returns once the round has completed on the device.
    void evaluate(Engine* engine, const EvalPlan& plan);
    [[nodiscard]] BatchStats stats() const;

private:
    struct Request {
        Engine* engine = nullptr;
        const EvalPlan* plan = nullptr;
        std::atomic<int> done{0};  // set (release) after status and error
        std::string error;
        int status = MPGP_OK;
    };
    void loop();
    void execute(const std::vector<Request*>& round);
    void reserve(std::size_t bytes);

    int device_;
    double window_;
    cudaStream_t stream_ = nullptr;       // the engines' stream: the density chain and the contractions
    cudaStream_t wirelength_ = nullptr;   // the wirelength pass beside it
    cudaStream_t split_ = nullptr;        // the split-1 contraction group beside the split-2 group
    cudaEvent_t split_fork_ = nullptr, split_join_ = nullptr;
    cudaEvent_t fork_ = nullptr, join_ = nullptr;
    cudaEvent_t start_ = nullptr, done_ = nullptr;  // timed: the round's device time
    unsigned char* host_args_ = nullptr;  // pinned staging of a round's argument blocks
    unsigned char* device_args_ = nullptr;
    std::size_t capacity_ = 0;

    mutable std::mutex mutex_;
    std::condition_variable submitted_;
    // Completed rounds, also the futex word the waiting engines sleep on: one wake
    // releases them all at once, and each checks its own request without a lock.
    std::atomic<uint32_t> completed_rounds_{0};
    std::vector<Request*> pending_;
    int attached_ = 0;
    bool stopping_ = false;
    BatchStats stats_;
    std::thread thread_;
};

}  // namespace mpgp
