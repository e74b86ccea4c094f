// Batched rounds of many engines' evaluations (batch.hpp).
#include "batch.hpp"

#include <linux/futex.h>
#include <sys/syscall.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cstring>

#include "common.cuh"
#include "dct_tc.cuh"
#include "field_tc.cuh"

namespace mpgp {

namespace {

std::size_t alignUp(std::size_t value, std::size_t alignment) { return (value + alignment - 1) / alignment * alignment; }

// A round's argument blocks, laid out one after another in one buffer.
struct RoundLayout {
    std::size_t bytes = 0;
    template <typename T>
    std::size_t add(std::size_t count) {
        const std::size_t at = alignUp(bytes, 256);
        bytes = at + std::max<std::size_t>(1, count) * sizeof(T);
        return at;
    }
};

constexpr int kContractionStages = 4;  // forward 1, forward 2, inverse 1, inverse 2
constexpr int kInverseX = 4;           // the banded solve's inverse along x (Engine::contraction)

// The banded field items of a round with one cluster size and share width.
struct FieldGroup {
    FieldShape shape;
    std::vector<FieldItem> items;
    std::size_t at = 0;
};

// Sleeps while *word still holds `seen` (Linux futex; spurious returns are fine).
void futexWait(std::atomic<uint32_t>* word, uint32_t seen) {
    syscall(SYS_futex, reinterpret_cast<uint32_t*>(word), FUTEX_WAIT_PRIVATE, seen, nullptr, nullptr, 0);
}

void futexWakeAll(std::atomic<uint32_t>* word) {
    syscall(SYS_futex, reinterpret_cast<uint32_t*>(word), FUTEX_WAKE_PRIVATE, INT_MAX, nullptr, nullptr, 0);
}

}  // namespace

Batch::Batch(int device, double window_seconds) : device_(device), window_(window_seconds) {
    require(window_seconds >= 0.0, "The batch window must be non-negative.");
    checkCuda(cudaSetDevice(device_), "Select CUDA device");
    checkCuda(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "Create batch stream");
    checkCuda(cudaStreamCreateWithFlags(&wirelength_, cudaStreamNonBlocking), "Create batch wirelength stream");
    checkCuda(cudaStreamCreateWithFlags(&split_, cudaStreamNonBlocking), "Create batch contraction stream");
    checkCuda(cudaEventCreateWithFlags(&split_fork_, cudaEventDisableTiming), "Create batch event");
    checkCuda(cudaEventCreateWithFlags(&split_join_, cudaEventDisableTiming), "Create batch event");
    checkCuda(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming), "Create batch event");
    checkCuda(cudaEventCreateWithFlags(&join_, cudaEventDisableTiming), "Create batch event");
    checkCuda(cudaEventCreate(&start_), "Create batch event");
    checkCuda(cudaEventCreate(&done_), "Create batch event");
    reserve(std::size_t{1} << 20);
    thread_ = std::thread([this] { loop(); });
}

Batch::~Batch() {
    {
        std::lock_guard<std::mutex> lock(mutex_);
        stopping_ = true;
    }
    submitted_.notify_all();
    if (thread_.joinable()) thread_.join();
    cudaSetDevice(device_);
    if (stream_ != nullptr) cudaStreamSynchronize(stream_);
    if (wirelength_ != nullptr) cudaStreamSynchronize(wirelength_);
    if (split_ != nullptr) cudaStreamSynchronize(split_);
    if (split_fork_ != nullptr) cudaEventDestroy(split_fork_);
    if (split_join_ != nullptr) cudaEventDestroy(split_join_);
    if (fork_ != nullptr) cudaEventDestroy(fork_);
    if (join_ != nullptr) cudaEventDestroy(join_);
    if (done_ != nullptr) cudaEventDestroy(done_);
    if (start_ != nullptr) cudaEventDestroy(start_);
    if (host_args_ != nullptr) cudaFreeHost(host_args_);
    if (device_args_ != nullptr) cudaFree(device_args_);
    if (wirelength_ != nullptr) cudaStreamDestroy(wirelength_);
    if (split_ != nullptr) cudaStreamDestroy(split_);
    if (stream_ != nullptr) cudaStreamDestroy(stream_);
}

void Batch::reserve(std::size_t bytes) {
    if (bytes <= capacity_) return;
    const std::size_t grown = std::max(bytes, 2 * capacity_);
    // The previous round has completed (rounds end with a synchronisation), so
    // neither buffer is in use.
    if (host_args_ != nullptr) checkCuda(cudaFreeHost(host_args_), "Free batch staging");
    if (device_args_ != nullptr) checkCuda(cudaFree(device_args_), "Free batch arguments");
    host_args_ = nullptr;
    device_args_ = nullptr;
    capacity_ = 0;
    checkCuda(cudaMallocHost(reinterpret_cast<void**>(&host_args_), grown), "Allocate batch staging");
    checkCuda(cudaMalloc(reinterpret_cast<void**>(&device_args_), grown), "Allocate batch arguments");
    capacity_ = grown;
}

void Batch::attach(Engine* engine) {
    engine->deviceBatches();  // the contraction descriptors the batched launches read
    if (engine->banded()) engine->deviceField();
    std::lock_guard<std::mutex> lock(mutex_);
    ++attached_;
}

void Batch::detach(Engine* /*engine*/) {
    {
        std::lock_guard<std::mutex> lock(mutex_);
        --attached_;
    }
    submitted_.notify_all();  // a round waiting for this engine can start
}

void Batch::evaluate(Engine* engine, const EvalPlan& plan) {
    Request request;
    request.engine = engine;
    request.plan = &plan;
    {
        std::lock_guard<std::mutex> lock(mutex_);
        require(!stopping_, "The batch is shutting down.");
        pending_.push_back(&request);
    }
    submitted_.notify_all();
    // Sleep on the round counter until this request's round has completed.
    for (;;) {
        const uint32_t seen = completed_rounds_.load(std::memory_order_acquire);
        if (request.done.load(std::memory_order_acquire) != 0) break;
        futexWait(&completed_rounds_, seen);
    }
    if (request.status != MPGP_OK) fail(request.status, request.error);
}

BatchStats Batch::stats() const {
    std::lock_guard<std::mutex> lock(mutex_);
    return stats_;
}

void Batch::loop() {
    cudaSetDevice(device_);
    for (;;) {
        std::vector<Request*> round;
        {
            std::unique_lock<std::mutex> lock(mutex_);
            submitted_.wait(lock, [&] { return stopping_ || !pending_.empty(); });
            if (pending_.empty()) return;  // stopping
            // Give the attached engines that have not handed in their evaluation a
            // short window to do so, then launch whatever is there.
            const auto deadline = std::chrono::steady_clock::now() + std::chrono::duration<double>(window_);
            submitted_.wait_until(lock, deadline,
                                  [&] { return stopping_ || static_cast<int>(pending_.size()) >= attached_; });
            round.swap(pending_);
        }
        int status = MPGP_OK;
        std::string error;
        const auto started = std::chrono::steady_clock::now();
        try {
            execute(round);
        } catch (const Error& e) {
            status = e.status();
            error = e.what();
        } catch (const std::exception& e) {
            status = MPGP_ERR_RUNTIME;
            error = e.what();
        }
        const double busy = std::chrono::duration<double>(std::chrono::steady_clock::now() - started).count();
        {
            std::lock_guard<std::mutex> lock(mutex_);
            stats_.rounds += 1;
            stats_.evaluations += static_cast<int64_t>(round.size());
            stats_.peak_round = std::max(stats_.peak_round, static_cast<int>(round.size()));
            stats_.busy_seconds += busy;
        }
        for (Request* r : round) {
            r->status = status;
            r->error = error;
            r->done.store(1, std::memory_order_release);  // the request may be gone after this
        }
        completed_rounds_.fetch_add(1, std::memory_order_acq_rel);
        futexWakeAll(&completed_rounds_);
    }
}

void Batch::execute(const std::vector<Request*>& round) {
    const int n = static_cast<int>(round.size());
    std::vector<int> scatter, metrics, gather;
    std::vector<TcItem> items[kContractionStages][kMaxSplit];
    std::vector<FieldGroup> fields;
    bool mixed_split = false;  // an instance whose stages use different splits (its stages must share a stream)
    int staged = 0;
    for (int i = 0; i < n; ++i) {
        const EvalPlan& p = *round[i]->plan;
        Engine* engine = round[i]->engine;
        if (p.scatter) scatter.push_back(i);
        if (p.metrics) metrics.push_back(i);
        if (p.gather) gather.push_back(i);
        const int total = p.reduce_args.offsets[p.reduce_args.source_count];
        if (total <= p.reduce_args.staged_capacity) staged = std::max(staged, total);
        const TcBatch* device_batches = engine->deviceBatches();
        if (engine->banded()) {
            // The banded launch (as Engine::runDct), then the inverse along x with the
            // last stage of the staged instances.
            const FieldShape& shape = engine->fieldBand().shape;
            if (p.forward || p.gradient) {
                auto group = std::find_if(fields.begin(), fields.end(), [&](const FieldGroup& g) {
                    return g.shape.cluster == shape.cluster && g.shape.share_n == shape.share_n;
                });
                if (group == fields.end()) group = fields.insert(fields.end(), FieldGroup{shape, {}, 0});
                const FieldBand* field = engine->deviceField();
                const FieldMode mode = p.forward ? (p.gradient ? kFieldGradient : kFieldForward) : kFieldInverse;
                for (int b = 0; b < shape.bands; ++b) group->items.push_back(FieldItem{field, b, mode});
            }
            if (p.gradient) {
                const TcBatch& batch = engine->contraction(kInverseX);
                for (int task = 0; task < 2; ++task) {
                    const int tiles = taskTiles(batch, task);
                    for (int tile = 0; tile < tiles; ++tile) {
                        items[kContractionStages - 1][batch.ksplit - 1].push_back(
                            TcItem{device_batches + kInverseX, task, tile});
                    }
                }
            }
            continue;
        }
        for (int stage = 0; stage < kContractionStages; ++stage) {
            mixed_split = mixed_split || engine->contraction(stage).ksplit != engine->contraction(0).ksplit;
            if (stage < 2 ? !p.forward : !p.gradient) continue;
            const TcBatch& batch = engine->contraction(stage);
            const int tasks = stage < 2 ? 1 : 2;
            for (int task = 0; task < tasks; ++task) {
                const int tiles = taskTiles(batch, task);
                for (int tile = 0; tile < tiles; ++tile) {
                    items[stage][batch.ksplit - 1].push_back(TcItem{device_batches + stage, task, tile});
                }
            }
        }
    }

    RoundLayout layout;
    const std::size_t at_scatter = layout.add<ScatterArgs>(scatter.size());
    const std::size_t at_scatter_offsets = layout.add<int>(scatter.size() + 1);
    const std::size_t at_wirelength = layout.add<WirelengthArgs>(static_cast<std::size_t>(n));
    const std::size_t at_wirelength_offsets = layout.add<int>(static_cast<std::size_t>(n) + 1);
    const std::size_t at_metrics = layout.add<MetricsArgs>(metrics.size());
    const std::size_t at_metrics_offsets = layout.add<int>(metrics.size() + 1);
    const std::size_t at_gather = layout.add<GatherArgs>(gather.size());
    const std::size_t at_gather_offsets = layout.add<int>(gather.size() + 1);
    // Reductions: the instances with a gather reduce in its last block (their arguments
    // and pointers to them), the others in the reduction launch.
    std::vector<int> rest;
    for (int i = 0; i < n; ++i) {
        if (!round[i]->plan->gather) rest.push_back(i);
    }
    const std::size_t at_reduce_gather = layout.add<ReduceArgs>(gather.size());
    const std::size_t at_reduce_pointers = layout.add<const ReduceArgs*>(gather.size());
    const std::size_t at_reduce = layout.add<ReduceArgs>(rest.size());
    std::size_t at_items[kContractionStages][kMaxSplit];
    for (int stage = 0; stage < kContractionStages; ++stage) {
        for (int k = 0; k < kMaxSplit; ++k) at_items[stage][k] = layout.add<TcItem>(items[stage][k].size());
    }
    for (FieldGroup& g : fields) g.at = layout.add<FieldItem>(g.items.size());
    reserve(layout.bytes);

    unsigned char* host = host_args_;
    const auto fill = [&](std::size_t at, const std::vector<int>& members, auto args_of, auto blocks_of,
                          std::size_t offsets_at) {
        using Args = std::decay_t<decltype(args_of(*round[0]->plan))>;
        Args* args = reinterpret_cast<Args*>(host + at);
        int* offsets = reinterpret_cast<int*>(host + offsets_at);
        int blocks = 0;
        for (std::size_t j = 0; j < members.size(); ++j) {
            const EvalPlan& p = *round[members[j]]->plan;
            args[j] = args_of(p);
            offsets[j] = blocks;
            blocks += blocks_of(p);
        }
        offsets[members.size()] = blocks;
        return blocks;
    };
    std::vector<int> everyone(static_cast<std::size_t>(n));
    for (int i = 0; i < n; ++i) everyone[static_cast<std::size_t>(i)] = i;
    const int scatter_blocks = fill(
        at_scatter, scatter, [](const EvalPlan& p) { return p.scatter_args; },
        [](const EvalPlan& p) { return p.scatter_blocks; }, at_scatter_offsets);
    const int wirelength_blocks = fill(
        at_wirelength, everyone, [](const EvalPlan& p) { return p.wirelength_args; },
        [](const EvalPlan& p) { return p.wirelength_blocks; }, at_wirelength_offsets);
    const int metrics_blocks = fill(
        at_metrics, metrics, [](const EvalPlan& p) { return p.metrics_args; },
        [](const EvalPlan& p) { return p.metrics_blocks; }, at_metrics_offsets);
    const int gather_blocks = fill(
        at_gather, gather, [](const EvalPlan& p) { return p.gather_args; },
        [](const EvalPlan& p) { return p.gather_blocks; }, at_gather_offsets);
    ReduceArgs* reduce = reinterpret_cast<ReduceArgs*>(host + at_reduce);
    for (std::size_t j = 0; j < rest.size(); ++j) reduce[j] = round[rest[j]]->plan->reduce_args;
    ReduceArgs* reduce_gather = reinterpret_cast<ReduceArgs*>(host + at_reduce_gather);
    const ReduceArgs** reduce_pointers = reinterpret_cast<const ReduceArgs**>(host + at_reduce_pointers);
    for (std::size_t j = 0; j < gather.size(); ++j) {
        reduce_gather[j] = round[gather[j]]->plan->reduce_args;
        reduce_pointers[j] = reinterpret_cast<const ReduceArgs*>(device_args_ + at_reduce_gather) + j;
    }
    for (int stage = 0; stage < kContractionStages; ++stage) {
        for (int k = 0; k < kMaxSplit; ++k) {
            if (!items[stage][k].empty()) {
                std::memcpy(host + at_items[stage][k], items[stage][k].data(), items[stage][k].size() * sizeof(TcItem));
            }
        }
    }
    for (const FieldGroup& g : fields) std::memcpy(host + g.at, g.items.data(), g.items.size() * sizeof(FieldItem));

    unsigned char* dev = device_args_;
    const auto on_device = [&](std::size_t at) { return dev + at; };
    checkCuda(cudaEventRecord(start_, stream_), "Batch start");
    checkCuda(cudaMemcpyAsync(dev, host, layout.bytes, cudaMemcpyHostToDevice, stream_), "Upload batch arguments");
    int64_t launches = 0;
    // The same order as one engine's evaluation (Engine::run): scatter (which forms
    // proposal and lookahead positions), the wirelength pass beside the density
    // chain, metrics, the contractions, then the gather and the reduction.
    if (!scatter.empty()) {
        launchScatterBatch(reinterpret_cast<const ScatterArgs*>(on_device(at_scatter)),
                           reinterpret_cast<const int*>(on_device(at_scatter_offsets)), static_cast<int>(scatter.size()),
                           scatter_blocks, stream_);
        ++launches;
    }
    checkCuda(cudaEventRecord(fork_, stream_), "Batch fork");
    checkCuda(cudaStreamWaitEvent(wirelength_, fork_, 0), "Batch fork");
    if (wirelength_blocks > 0) {
        launchWirelengthBatch(reinterpret_cast<const WirelengthArgs*>(on_device(at_wirelength)),
                              reinterpret_cast<const int*>(on_device(at_wirelength_offsets)), n, wirelength_blocks,
                              wirelength_);
        ++launches;
    }
    checkCuda(cudaEventRecord(join_, wirelength_), "Batch join");
    if (!metrics.empty()) {
        launchMetricsSplitBatch(reinterpret_cast<const MetricsArgs*>(on_device(at_metrics)),
                                reinterpret_cast<const int*>(on_device(at_metrics_offsets)),
                                static_cast<int>(metrics.size()), metrics_blocks, stream_);
        ++launches;
    }
    // The banded field solves, one launch per cluster shape.
    for (const FieldGroup& g : fields) {
        launchFieldBatch(reinterpret_cast<const FieldItem*>(on_device(g.at)), static_cast<int>(g.items.size()), g.shape,
                         stream_);
        ++launches;
    }
    // The contraction stages.  Instances of one K split and of the other are
    // disjoint, so with both present the split-1 group runs on a stream of its own
    // beside the split-2 group (each group's stages stay in order on its stream).
    // Only when every instance uses one split for all its stages: otherwise an
    // instance's stages could land on both streams, and they depend on each other.
    bool both = false;
    for (int stage = 0; stage < kContractionStages && !mixed_split; ++stage) {
        for (int other = 0; other < kContractionStages; ++other) {
            both = both || (!items[stage][0].empty() && !items[other][1].empty());
        }
    }
    if (both) {
        checkCuda(cudaEventRecord(split_fork_, stream_), "Batch split fork");
        checkCuda(cudaStreamWaitEvent(split_, split_fork_, 0), "Batch split fork");
    }
    for (int stage = 0; stage < kContractionStages; ++stage) {
        for (int k = 0; k < kMaxSplit; ++k) {
            if (items[stage][k].empty()) continue;
            launchTcGemmBatch(reinterpret_cast<const TcItem*>(on_device(at_items[stage][k])),
                              static_cast<int>(items[stage][k].size()), k + 1, both && k == 0 ? split_ : stream_);
            ++launches;
        }
    }
    if (both) {
        checkCuda(cudaEventRecord(split_join_, split_), "Batch split join");
        checkCuda(cudaStreamWaitEvent(stream_, split_join_, 0), "Batch split join");
    }
    checkCuda(cudaStreamWaitEvent(stream_, join_, 0), "Batch join");
    if (!gather.empty()) {
        launchGatherBatch(reinterpret_cast<const GatherArgs*>(on_device(at_gather)),
                          reinterpret_cast<const ReduceArgs* const*>(on_device(at_reduce_pointers)),
                          reinterpret_cast<const int*>(on_device(at_gather_offsets)), static_cast<int>(gather.size()),
                          gather_blocks, stream_);
        ++launches;
    }
    if (!rest.empty()) {
        launchReduceBatch(reinterpret_cast<const ReduceArgs*>(on_device(at_reduce)), static_cast<int>(rest.size()),
                          staged, stream_);
        ++launches;
    }
    checkCuda(cudaEventRecord(done_, stream_), "Batch done");
    checkCuda(cudaEventSynchronize(done_), "Batched evaluation on the device");
    float milliseconds = 0.0f;
    checkCuda(cudaEventElapsedTime(&milliseconds, start_, done_), "Batch device time");
    std::lock_guard<std::mutex> lock(mutex_);
    stats_.launches += launches;
    stats_.device_seconds += 1e-3 * static_cast<double>(milliseconds);
}

}  // namespace mpgp
