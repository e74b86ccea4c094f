// The device engine: resident state of one placement problem and one evaluation
// of the adaptive objective (wirelength, density, field, gradient) per call.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <cstdint>
#include <vector>

#include "dct_tc.cuh"
#include "field_tc.cuh"
#include "kernels.cuh"
#include "setup.hpp"

namespace mpgp {

// Explicit device allocations are counted against a budget before they are made
// (DeviceMemoryBudget, CudaPlacementBackend.cu:60-79).
class DeviceArena {
public:
    explicit DeviceArena(uint64_t limit) : limit_(limit) {}
    ~DeviceArena();
    DeviceArena(const DeviceArena&) = delete;
    DeviceArena& operator=(const DeviceArena&) = delete;

    // Allocations are taken from the device's pool on `stream` (devicePool) once bound;
    // before that, and for an unbound arena, with cudaMalloc.
    void bind(int device, cudaStream_t stream);
    void* allocate(std::size_t bytes, const char* what);
    template <typename T>
    T* array(std::size_t count, const char* what) {
        return static_cast<T*>(allocate(count * sizeof(T), what));
    }
    [[nodiscard]] uint64_t reserved() const { return reserved_; }
    [[nodiscard]] uint64_t headroom() const { return limit_ - std::min(limit_, reserved_); }

private:
    uint64_t limit_;
    uint64_t reserved_ = 0;
    std::vector<void*> blocks_;
    cudaMemPool_t pool_ = nullptr;
    cudaStream_t stream_ = nullptr;
};

struct EvalRequest {
    int mode = kGiven;
    const double2* positions = nullptr;  // kGiven
    const double2* base = nullptr;       // kPropose / kLookahead
    const double2* direction = nullptr;
    const double2* raw_direction = nullptr;
    double2* out_positions = nullptr;
    double step = 0.0;
    double max_displacement = 0.0;
    double smoothing = 1.0;
    bool gradient = false;
    // combined gradient outputs (controller)
    double penalty = 0.0;
    double precond_scale = 1.0;
    double2* raw = nullptr;
    double2* pre = nullptr;
    // split outputs (drop-in backend)
    double2* wire_out = nullptr;
    double2* density_out = nullptr;
    double2* rudy_out = nullptr;
    const double2* prev_positions = nullptr;
    const double2* prev_gradient = nullptr;
    const double2* velocity = nullptr;
    // Work of the previous step folded into this evaluation's gather (kGiven with a
    // gradient): velocity_out = positions - velocity_base (the step just taken; the
    // momentum alignment then uses it) and checkpoint_out = positions.
    const double2* velocity_base = nullptr;
    double2* velocity_out = nullptr;
    double2* checkpoint_out = nullptr;
    bool want_potential = false;
    // The density map, forward field coefficients and energy of the previous
    // evaluation are those of these positions (nothing moved since): keep them and
    // run only the wirelength, the inverse field and the gather.
    bool reuse_density = false;
    // The routability term: RUDY map, energy and (with gradient) its weighted
    // subgradient in the combined gradient.
    bool rudy = false;
    double rudy_weight = 0.0;
};

// RUDY metrics of one evaluation of a grid (RudyMetrics, Rudy.hpp:51-64, and the energy).
struct RudyReport {
    double horizontal_total = 0.0, vertical_total = 0.0;
    double horizontal_mean = 0.0, vertical_mean = 0.0;
    double horizontal_capacity = 0.0, vertical_capacity = 0.0;
    double energy = 0.0, proxy_overflow = 0.0, maximum_utilization = 0.0, p95_utilization = 0.0;
};

struct EvalScalars {
    double v[kScalarCount];
};

// Everything one evaluation launches, with its arguments (Engine::plan).  A plain
// engine launches it on its own streams (Engine::run); a Batch launches the plans
// of many engines together, one batched launch per kernel family.
struct EvalPlan {
    bool scatter = false;
    ScatterArgs scatter_args{};
    int scatter_blocks = 0;
    bool fork_first = false;  // the positions are given: the wirelength pass need not wait for the scatter
    WirelengthArgs wirelength_args{};
    int wirelength_blocks = 0;
    bool rudy = false;
    bool rudy_gradient = false;
    RudyArgs rudy_args{};
    int rudy_blocks = 0;
    bool metrics = false;
    bool metrics_fused = false;
    MetricsArgs metrics_args{};
    int metrics_blocks = 0;
    bool forward = false;       // the two forward contractions (and the source split when not fused)
    bool split_source = false;
    bool gradient = false;      // the two inverse contraction launches
    bool potential = false;
    bool gather = false;
    GatherArgs gather_args{};
    int gather_blocks = 0;
    ReduceArgs reduce_args{};
    int kernels = 0;            // launches of the evaluation (the engine's launch count)
};

class Batch;

// Kernel families timed by the engine's optional event profiler.
enum KernelKind : int {
    kKindScatter = 0,
    kKindWirelength,
    kKindMetrics,
    kKindDctForward,
    kKindDctInverse,
    kKindGather,
    kKindReduce,
    kKindVector,
    kKindDctSplit,
    kKindRudy,
    kKindFieldForward,   // the banded field solve without the inverse passes
    kKindFieldGradient,  // the banded field solve with them
    kKindFieldInverse,   // the banded field solve's inverse passes alone
    kKindCount
};
const char* kernelKindName(int kind);

struct KernelStats {
    int64_t launches[kKindCount] = {};
    double milliseconds[kKindCount] = {};
};

class Engine {
public:
    // With a batch, the engine runs on the batch's stream and its evaluations are
    // launched together with the other engines of the batch (Batch).
    Engine(const Problem& problem, int device, uint64_t budget_bytes, Batch* batch = nullptr);
    // Two-phase construction: the grid's part (streams, the field solve's bases and
    // buffers) needs only the grid, so it can run while the host builds the particles;
    // load() then uploads the problem (whose grid must be this one).
    struct Grid {
        int bins_x = 0, bins_y = 0;
        Rect2 region;
        double target_density = 0.0;
    };
    Engine(const Grid& grid, int device, uint64_t budget_bytes, Batch* batch = nullptr);
    // The problem's upload and device layout, all at once or in two steps: the nets
    // (needing only the pin and net arrays and the movable count), then the particles.
    void load(const Problem& problem);
    void loadNets(const Problem& problem, int64_t movable_count);
    void loadParticles(const Problem& problem);
    ~Engine();
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    // Launches one evaluation on the engine stream and returns its ticket; its scalars
    // are valid after sync(ticket).  Up to kRecords evaluations may be in flight: each
    // publishes into its own record, so a later launch does not overwrite an earlier
    // one's record before the host has read it.  In a batch the evaluation is handed to
    // the batch at sync(), and only one may be in flight.
    uint64_t launch(const EvalRequest& request);
    // The launches of one evaluation (the scalar record's sequence advances), and
    // launching them on the engine's streams.
    EvalPlan plan(const EvalRequest& request);
    void run(const EvalPlan& plan);
    // The engine's contraction batches (forward 1, forward 2, inverse 1, inverse 2 of
    // the staged solve, then the inverse along x of the banded solve) and its banded
    // solve's descriptor, copied to device memory for batched launches; uploaded on first use.
    const TcBatch* deviceBatches();
    const FieldBand* deviceField();
    [[nodiscard]] const TcBatch& contraction(int stage) const;
    // The field solve is banded (field_tc.cu) rather than staged (four contraction launches).
    [[nodiscard]] bool banded() const { return banded_; }
    [[nodiscard]] const FieldBand& fieldBand() const { return field_band_; }
    // Stops taking part in the batch's rounds (the placement has finished); a later
    // evaluation still runs through the batch.
    void leaveBatch();
    // Waits for the evaluation `ticket` (fewer than kRecords launches old) and returns its scalars
    // (scalars it does not compute keep the value of the last evaluation synced before).
    const EvalScalars& sync(uint64_t ticket);
    const EvalScalars& sync() { return sync(launches_issued_); }
    const EvalScalars& evaluate(const EvalRequest& request) { return sync(launch(request)); }
    // Evaluations may be in flight together (not in a batch), up to kRecords.
    [[nodiscard]] bool overlapsEvaluations() const { return batch_ == nullptr; }
    // Evaluation results in the reference's structures.
    void densityMetrics(const EvalScalars& s, bool with_fillers, mpgp_density_metrics& out) const;
    [[nodiscard]] double energy(const EvalScalars& s) const;

    // The routability term (rudy.cu): allocate the RUDY grid(s), freeze capacities,
    // and evaluate a grid's metrics at given positions (calibration, validation, final).
    void enableRudy(const mpgp_options& options);
    [[nodiscard]] bool rudyEnabled() const { return rudy_main_.columns > 0; }
    [[nodiscard]] bool rudyValidationEnabled() const { return rudy_validation_.columns > 0; }
    void setRudyCapacity(bool validation, double horizontal, double vertical);
    void setRudyModel(int model, double temperature);
    [[nodiscard]] double rudyMinimumSpan() const { return rudy_minimum_span_; }
    RudyReport rudyEvaluate(const double2* positions, bool validation);
    [[nodiscard]] int rudyBins() const { return rudy_main_.columns * rudy_main_.rows; }

    // Solves the field of an arbitrary FP64 deviation map (parity hook).
    void fieldSolve(const double* deviation, double* potential, double* field_x, double* field_y);
    // Runs the fixed-point scatter alone at `positions` and copies the three layers out (parity hook).
    void depositLayers(const double2* positions, int64_t* movable, int64_t* macro, int64_t* filler);
    [[nodiscard]] double2* scratchPositions() const { return scratch_positions_; }
    // Failure-detection probe: with polls > 0 every later field contraction waits on a
    // barrier that nothing completes for at most `polls` polls and raises the engine's
    // error flag (the evaluation then fails with MPGP_ERR_TIMEOUT); 0 turns it off.
    void setStallProbe(long long polls);

    [[nodiscard]] double2* newParticleArray(const char* what);
    // `count` zeroed particle arrays from one allocation: out[k] = base + k * stride.
    void newParticleArrays(int count, double2** out, const char* what);
    [[nodiscard]] cudaStream_t stream() const { return stream_; }
    [[nodiscard]] int device() const { return device_; }
    [[nodiscard]] uint64_t reservedBytes() const { return arena_.reserved(); }
    [[nodiscard]] int64_t particleCount() const { return particle_count_; }
    [[nodiscard]] int64_t movableCount() const { return movable_count_; }
    [[nodiscard]] int64_t launches() const { return launches_; }
    [[nodiscard]] const double* precondBase() const { return precond_; }
    void countLaunches(int64_t n) { launches_ += n; }

    // Event profiling: every launch of a family whose bit is set in `families` is
    // bracketed by CUDA events on its stream and its duration is added to the
    // family at sync() (0 turns profiling off).
    void setTiming(uint32_t families);
    [[nodiscard]] const KernelStats& kernelStats() const { return stats_; }
    void resetKernelStats() { stats_ = KernelStats{}; }
    void beginKernel(int kind, cudaStream_t on = nullptr);
    void endKernel(cudaStream_t on = nullptr);
    [[nodiscard]] uint64_t bytesToDevice() const { return h2d_bytes_; }
    [[nodiscard]] uint64_t bytesToHost() const { return d2h_bytes_; }
    void addTransfer(uint64_t to_device, uint64_t to_host) {
        h2d_bytes_ += to_device;
        d2h_bytes_ += to_host;
    }

private:
    struct RudyGrid {
        int columns = 0, rows = 0;
        double bin_w = 0.0, bin_h = 0.0, min_x_span = 0.0, min_y_span = 0.0;
        double capacity_h = 0.0, capacity_v = 0.0;
        unsigned long long* diff = nullptr;
        unsigned long long* horizontal = nullptr;
        unsigned long long* vertical = nullptr;
        double* table = nullptr;
        double* adjoint_h = nullptr;
        double* adjoint_v = nullptr;
        double* utilization = nullptr;
        double* partials = nullptr;
        int blocks = 0;
    };
    void allocateRudyGrid(RudyGrid& grid, int columns, int rows, const char* what);
    [[nodiscard]] RudyArgs rudyArgs(const RudyGrid& grid, const double2* positions, bool with_capacity) const;
    RudyGrid rudy_main_, rudy_validation_;
    int rudy_model_ = 0;
    double rudy_temperature_ = 0.1;
    double rudy_minimum_span_ = 0.25;
    double* rudy_net_weight_ = nullptr;
    double2* rudy_pin_gradient_ = nullptr;
    double* rudy_scalars_ = nullptr;
    double* host_rudy_ = nullptr;
    int wl_net_count_ = 0;
    int wl_pin_count_ = 0;

    void collectTimings();
    void runDct(bool gradient, bool potential, bool forward, bool split_source = true);
    void runBandedField(bool gradient, bool forward, bool split_source);
    void runBandedInverseX(bool gradient, bool potential);
    void runStagedField(bool gradient, bool potential, bool forward, bool split_source);
    void runWirelengthPass(const EvalPlan& p);
    void uploadStatic(const Problem& problem);
    void buildNetLayout(const Problem& problem);
    void buildBasis();

    int device_ = 0;
    Batch* batch_ = nullptr;
    bool owns_stream_ = true;
    bool attached_ = false;
    bool has_pending_ = false;
    EvalPlan batched_plan_{};
    TcBatch* device_batches_ = nullptr;
    cudaStream_t stream_ = nullptr;
    cudaStream_t stream_wl_ = nullptr;  // the wirelength pass overlaps the density chain
    cudaEvent_t fork_ = nullptr;
    cudaEvent_t join_ = nullptr;
    DeviceArena arena_;
    int64_t launches_ = 0;

    int64_t particle_count_ = 0;
    int64_t movable_count_ = 0;
    int bins_x_ = 0, bins_y_ = 0;
    int bin_count_ = 0;
    Rect2 region_;
    double bin_w_ = 0.0, bin_h_ = 0.0, bin_area_ = 0.0;
    double target_density_ = 0.0;
    double static_fixed_sum_ = 0.0, static_dark_sum_ = 0.0, static_placeable_sum_ = 0.0;

    // particles
    double2* size_ = nullptr;
    unsigned char* layer_ = nullptr;
    double* charge_ = nullptr;
    double* precond_ = nullptr;
    double2* scratch_positions_ = nullptr;  // kGiven uploads for the drop-in path

    // netlist
    int* pin_particle_ = nullptr;
    float2* pin_offset_ = nullptr;
    double2* static_pins_ = nullptr;
    int* net_start_ = nullptr;
    float* net_weight_ = nullptr;
    int4* block_work_ = nullptr;
    int wl_blocks_ = 0;
    float2* pin_gradient_ = nullptr;
    int* particle_pin_start_ = nullptr;
    int* pin_slot_ = nullptr;

    // density
    unsigned long long* layers_ = nullptr;
    unsigned long long* totals_ = nullptr;
    double* static_charge_ = nullptr;
    float* source_ = nullptr;

    // field solve: spectral divide, Parseval weights, outputs
    float* spectral_scale_ = nullptr;  // ny x nx
    float* weight_y_ = nullptr;
    float* weight_x_ = nullptr;
    float2* field_ = nullptr;
    float* potential_ = nullptr;

    // tcgen05 split-precision contractions (dct_tc.cu)
    SplitMatrix tc_source_, tc_cx_, tc_cy_, tc_dy_, tc_dxc_, tc_sxwt_, tc_syw_;
    SplitMatrix tc_x1t_, tc_phi_, tc_phit_, tc_t_, tc_ut_;
    TcBatch tc_fwd1_{}, tc_fwd2_{}, tc_inv1_{}, tc_inv2_{}, tc_pot_{};
    // The banded solve where the grid allows it: one banded launch, then the inverse
    // along x of M1 and M2 (tc_invx_) and the potential (tc_potx_).
    bool banded_ = false;
    FieldBand field_band_{};
    FieldBand* device_field_ = nullptr;
    SplitMatrix tc_m1_, tc_m2_;
    TcBatch tc_invx_{}, tc_potx_{};
    int* tc_row_exp_ = nullptr;
    TcScales* tc_scales_ = nullptr;
    int* tc_error_ = nullptr;
    int* host_error_ = nullptr;
    // Evaluation results published by the reduction into mapped pinned memory
    // (ReduceArgs::host_slots), the scalars the current evaluation writes, and
    // the cache of the latest value of every scalar.
    // kRecords records of kRecordSlots slots; launch k publishes into record k % kRecords.
    static constexpr int kRecords = 2;
    static constexpr int kRecordSlots = 2 * (kScalarCount + 1);
    unsigned long long* host_slots_ = nullptr;
    uint32_t record_mask_[kRecords] = {};       // the scalars the record's evaluation writes
    uint32_t record_sequence_[kRecords] = {};   // its sequence (the record's tag)
    uint64_t record_ticket_[kRecords] = {};     // its ticket
    uint64_t launches_issued_ = 0;
    bool nets_loaded_ = false;
    uint64_t synced_ticket_ = 0;
    unsigned long long sequence_ = 0;
    void buildTensorCoreBasis(double max_scale);
    SplitMatrix newSplit(int rows, int cols, const char* what);

    // partials and scalars
    int scatter_blocks_ = 0, metrics_blocks_ = 0, gather_blocks_ = 0, energy_blocks_ = 0;
    bool metrics_fused_ = false;  // metrics pass writes the first contraction's operand planes
    // Second-level (per 32 blocks) wirelength partials and their counters (reduceGroups).
    double* wl_group_ = nullptr;
    unsigned int* wl_counters_ = nullptr;
    // The same second level for the scatter, metrics and gather partials.
    struct Groups {
        int count = 0;
        double* partials = nullptr;
        unsigned int* counters = nullptr;
    };
    Groups sc_groups_, m_groups_, g_groups_;
    Groups newGroups(int blocks, int values, const char* what);
    int wl_groups_ = 0;
    void allocateGroups();
    double* partials_wl_ = nullptr;
    double* partials_sc_ = nullptr;
    double* partials_m_ = nullptr;
    double* partials_e_ = nullptr;
    double* partials_g_ = nullptr;
    double* scalars_ = nullptr;
    EvalScalars* host_scalars_ = nullptr;
    bool last_gradient_ = false;
    bool last_propose_ = false;

    // profiling
    uint32_t timing_mask_ = 0;
    bool open_ = false;
    std::vector<cudaEvent_t> events_;
    std::vector<int> pending_kind_;
    int pending_ = 0;
    KernelStats stats_;
    uint64_t h2d_bytes_ = 0;
    uint64_t d2h_bytes_ = 0;
};

}  // namespace mpgp
