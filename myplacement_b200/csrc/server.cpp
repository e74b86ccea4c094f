// The batched and served forms (server.hpp).
#include "server.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>

#include "batch.hpp"
#include "common.cuh"
#include "dct_tc.cuh"
#include "session.hpp"

namespace mpgp {

namespace {

double nowSeconds() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

template <typename T>
std::vector<T> copyOf(const T* data, std::size_t count) {
    return data != nullptr ? std::vector<T>(data, data + count) : std::vector<T>();
}

}  // namespace

uint64_t estimateSessionBytes(const mpgp_design& design, const mpgp_options& options) {
    require(design.module_count >= 0 && design.net_count >= 0 && design.pin_count >= 0, "Counts must be non-negative.");
    require(options.bins_x > 0 && options.bins_y > 0, "Bin counts must be positive.");
    uint64_t movable = 0;
    double movable_area = 0.0;
    for (int32_t i = 0; i < design.module_count; ++i) {
        const int32_t flags = design.module_flags != nullptr ? design.module_flags[i] : 0;
        if ((flags & (MPGP_MODULE_FIXED | MPGP_MODULE_TERMINAL)) == 0) {
            ++movable;
            movable_area += design.module_width[i] * design.module_height[i];
        }
    }
    // Fillers (createDensityFillers, GlobalPlacementSupport.cpp:52-103) are cells of
    // about the mean movable size that fill at most t x the row area: bound their
    // count by twice that, and by the option's cap.
    double row_area = 0.0;
    for (int32_t r = 0; r < design.row_count; ++r) {
        row_area += static_cast<double>(design.row_site_count[r]) * design.row_site_spacing[r] * design.row_height[r];
    }
    const double mean_area = movable > 0 ? movable_area / static_cast<double>(movable) : 1.0;
    const double filler_bound = 2.0 * options.target_density * row_area / std::max(mean_area, 1e-9) + 16.0;
    const uint64_t fillers = std::min<uint64_t>(static_cast<uint64_t>(options.maximum_fillers),
                                                static_cast<uint64_t>(std::min(filler_bound, 1e15)));
    const uint64_t particles = movable + fillers;
    const uint64_t pins = static_cast<uint64_t>(design.pin_count);
    const uint64_t nets = static_cast<uint64_t>(design.net_count);
    const uint64_t nx = static_cast<uint64_t>(options.bins_x), ny = static_cast<uint64_t>(options.bins_y);
    const uint64_t bins = nx * ny;
    const uint64_t ldx = static_cast<uint64_t>(paddedLd(options.bins_x));
    const uint64_t ldy = static_cast<uint64_t>(paddedLd(options.bins_y));
    // Twelve split matrices of two fp16 planes: six nx-row and six ny-row ones.
    const uint64_t split = 4ull * 3ull * (nx * ldx + ny * ldy + ny * ldx + nx * ldy);
    // 12 session vectors + sizes, charge, preconditioner, layer, upload scratch (per
    // particle); particle, offset, slot, gradient and a possible static copy (per pin);
    // CSR, weight, work and partials (per net); layers, static charge, source, scale,
    // field, potential (per bin); and the set-up's transient sorting and scanning
    // scratch (per pin and per net), which is freed before the iterations start but
    // must fit while it lives.
    const uint64_t bytes = 256ull * particles + (40ull + 80ull) * pins + (16ull + 48ull) * nets + 64ull * bins + split;
    return bytes + (256ull << 10) /* partials, scalars, rounding of ~60 allocations */;
}

struct Server::Job {
    int64_t id = 0;
    // Owned copy of the design.
    std::vector<double> module_width, module_height, module_x, module_y, net_weight, pin_offset_x, pin_offset_y;
    std::vector<int32_t> module_flags, module_orientation, pin_module;
    std::vector<int64_t> net_pin_start, row_site_count;
    std::vector<double> row_bottom, row_height, row_site_width, row_site_spacing, row_x_start;
    mpgp_design design{};
    mpgp_options options{};
    uint64_t estimate = 0;
    // Outputs.
    std::vector<double> out_x, out_y;
    mpgp_result result{};
    std::vector<mpgp_history_row> history;
    mpgp_job_stats stats{};
    std::string error;
    double submitted = 0.0, started = 0.0, finished = 0.0;
    bool done = false;
};

Server::Server(int device, uint64_t memory_budget, int workers, bool batched) : device_(device) {
    require(workers > 0 && workers <= 256, "A server needs between 1 and 256 workers.");
    int count = 0;
    const cudaError_t status = cudaGetDeviceCount(&count);
    if (status != cudaSuccess || count <= 0) {
        fail(MPGP_ERR_UNAVAILABLE, std::string("CUDA device discovery failed: ") + cudaGetErrorString(status));
    }
    require(device >= 0 && device < count, "Requested CUDA device does not exist on this host.");
    if (memory_budget == 0) {
        checkCuda(cudaSetDevice(device), "Select CUDA device");
        std::size_t free_bytes = 0, total_bytes = 0;
        checkCuda(cudaMemGetInfo(&free_bytes, &total_bytes), "Query free device memory");
        memory_budget = static_cast<uint64_t>(static_cast<double>(free_bytes) * 0.9);
    }
    budget_ = memory_budget;
    if (batched) batch_ = std::make_unique<Batch>(device);
    stats_.batched = batched ? 1 : 0;
    stats_.workers = workers;
    stats_.memory_budget = budget_;
    started_ = nowSeconds();
    workers_.reserve(static_cast<std::size_t>(workers));
    for (int i = 0; i < workers; ++i) workers_.emplace_back([this] { work(); });
}

Server::~Server() {
    {
        std::lock_guard<std::mutex> lock(mutex_);
        stopping_ = true;
    }
    ready_.notify_all();
    for (std::thread& t : workers_) t.join();
    batch_.reset();
}

int64_t Server::submit(const mpgp_design& d, const mpgp_options& o) {
    validateDesign(d);
    auto job = std::make_shared<Job>();
    const std::size_t modules = static_cast<std::size_t>(d.module_count);
    const std::size_t pins = static_cast<std::size_t>(d.pin_count);
    const std::size_t rows = static_cast<std::size_t>(d.row_count);
    job->module_width = copyOf(d.module_width, modules);
    job->module_height = copyOf(d.module_height, modules);
    job->module_x = copyOf(d.module_x, modules);
    job->module_y = copyOf(d.module_y, modules);
    job->module_flags = copyOf(d.module_flags, modules);
    job->module_orientation = copyOf(d.module_orientation, modules);
    job->net_weight = copyOf(d.net_weight, static_cast<std::size_t>(d.net_count));
    job->net_pin_start = copyOf(d.net_pin_start, static_cast<std::size_t>(d.net_count) + 1);
    job->pin_module = copyOf(d.pin_module, pins);
    job->pin_offset_x = copyOf(d.pin_offset_x, pins);
    job->pin_offset_y = copyOf(d.pin_offset_y, pins);
    job->row_bottom = copyOf(d.row_bottom, rows);
    job->row_height = copyOf(d.row_height, rows);
    job->row_site_width = copyOf(d.row_site_width, rows);
    job->row_site_spacing = copyOf(d.row_site_spacing, rows);
    job->row_x_start = copyOf(d.row_x_start, rows);
    job->row_site_count = copyOf(d.row_site_count, rows);
    mpgp_design& v = job->design;
    v = d;
    v.module_width = job->module_width.data();
    v.module_height = job->module_height.data();
    v.module_x = job->module_x.data();
    v.module_y = job->module_y.data();
    v.module_flags = d.module_flags != nullptr ? job->module_flags.data() : nullptr;
    v.module_orientation = d.module_orientation != nullptr ? job->module_orientation.data() : nullptr;
    v.net_weight = job->net_weight.data();
    v.net_pin_start = job->net_pin_start.data();
    v.pin_module = job->pin_module.data();
    v.pin_offset_x = job->pin_offset_x.data();
    v.pin_offset_y = job->pin_offset_y.data();
    v.row_bottom = job->row_bottom.data();
    v.row_height = job->row_height.data();
    v.row_site_width = job->row_site_width.data();
    v.row_site_spacing = job->row_site_spacing.data();
    v.row_x_start = job->row_x_start.data();
    v.row_site_count = job->row_site_count.data();
    job->options = o;
    job->options.cuda_device = device_;
    validateOptions(job->options);
    job->estimate = estimateSessionBytes(job->design, job->options);
    if (job->estimate > budget_) {
        fail(MPGP_ERR_BUDGET, "The job needs about " + std::to_string(job->estimate) +
                                  " device bytes, more than the server's budget of " + std::to_string(budget_) + ".");
    }
    job->history.resize(static_cast<std::size_t>(std::max(0, job->options.iterations)) + 1);
    job->out_x.resize(modules);
    job->out_y.resize(modules);
    {
        std::lock_guard<std::mutex> lock(mutex_);
        require(!stopping_, "The server is shutting down.");
        job->id = next_id_++;
        job->submitted = nowSeconds();
        jobs_[job->id] = job;
        queue_.push_back(job);
        ++stats_.submitted;
    }
    ready_.notify_all();
    return job->id;
}

bool Server::admissible(const Job& job) const {
    return running_ == 0 || reserved_ + job.estimate <= budget_;
}

void Server::work() {
    for (;;) {
        std::shared_ptr<Job> job;
        {
            std::unique_lock<std::mutex> lock(mutex_);
            // FIFO: only the oldest job may start, so a large job is not overtaken forever.
            ready_.wait(lock, [&] { return stopping_ || (!queue_.empty() && admissible(*queue_.front())); });
            if (stopping_) return;
            job = queue_.front();
            queue_.pop_front();
            reserved_ += job->estimate;
            ++running_;
            stats_.peak_running = std::max(stats_.peak_running, running_);
            stats_.peak_reserved = std::max(stats_.peak_reserved, reserved_);
            job->started = nowSeconds();
        }
        int status = MPGP_OK;
        std::string error;
        uint64_t reserved_bytes = 0;
        try {
            checkCuda(cudaSetDevice(device_), "Select CUDA device");
            Session session(job->design, job->options, batch_.get());
            reserved_bytes = session.engine() != nullptr ? session.engine()->reservedBytes() : 0;
            int completed = 0;
            while (!session.step(64, &completed)) {
            }
            session.finish(job->out_x.data(), job->out_y.data(), &job->result, job->history.data(),
                           static_cast<int>(job->history.size()));
        } catch (const Error& e) {
            status = e.status();
            error = e.what();
        } catch (const std::exception& e) {
            status = MPGP_ERR_RUNTIME;
            error = e.what();
        }
        {
            std::lock_guard<std::mutex> lock(mutex_);
            job->finished = nowSeconds();
            job->error = error;
            job->stats.queued_seconds = job->started - job->submitted;
            job->stats.run_seconds = job->finished - job->started;
            job->stats.latency_seconds = job->finished - job->submitted;
            job->stats.estimated_bytes = job->estimate;
            job->stats.reserved_bytes = reserved_bytes;
            job->stats.completed_iterations = job->result.completed_iterations;
            job->stats.status = status;
            job->done = true;
            reserved_ -= job->estimate;
            --running_;
            if (status == MPGP_OK) {
                ++stats_.completed;
                stats_.iterations += job->result.completed_iterations;
            } else {
                ++stats_.failed;
            }
        }
        ready_.notify_all();
        done_.notify_all();
    }
}

bool Server::wait(int64_t id, double timeout_seconds) {
    std::unique_lock<std::mutex> lock(mutex_);
    const auto found = jobs_.find(id);
    require(found != jobs_.end(), "Unknown job " + std::to_string(id) + ".");
    const std::shared_ptr<Job> job = found->second;
    if (timeout_seconds < 0.0) {
        done_.wait(lock, [&] { return job->done; });
        return true;
    }
    return done_.wait_for(lock, std::chrono::duration<double>(timeout_seconds), [&] { return job->done; });
}

void Server::take(int64_t id, double* module_x, double* module_y, mpgp_result* result, mpgp_history_row* history,
                  int capacity, mpgp_job_stats* stats) {
    std::shared_ptr<Job> job;
    {
        std::lock_guard<std::mutex> lock(mutex_);
        const auto found = jobs_.find(id);
        require(found != jobs_.end(), "Unknown job " + std::to_string(id) + ".");
        require(found->second->done, "Job " + std::to_string(id) + " has not finished.");
        job = found->second;
        jobs_.erase(found);
    }
    if (stats != nullptr) *stats = job->stats;
    if (job->stats.status != MPGP_OK) fail(job->stats.status, job->error);
    if (module_x != nullptr) std::copy(job->out_x.begin(), job->out_x.end(), module_x);
    if (module_y != nullptr) std::copy(job->out_y.begin(), job->out_y.end(), module_y);
    if (result != nullptr) *result = job->result;
    if (history != nullptr && capacity > 0) {
        const int rows = std::min(capacity, std::min(job->result.history_count, static_cast<int>(job->history.size())));
        std::copy(job->history.begin(), job->history.begin() + rows, history);
    }
}

mpgp_server_stats Server::stats() const {
    std::lock_guard<std::mutex> lock(mutex_);
    mpgp_server_stats s = stats_;
    s.seconds = nowSeconds() - started_;
    if (batch_) {
        const BatchStats b = batch_->stats();
        s.batch_rounds = b.rounds;
        s.batch_evaluations = b.evaluations;
        s.batch_launches = b.launches;
        s.batch_peak_round = b.peak_round;
        s.batch_busy_seconds = b.busy_seconds;
        s.batch_device_seconds = b.device_seconds;
    }
    return s;
}

}  // namespace mpgp
