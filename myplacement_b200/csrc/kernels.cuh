// Kernel argument blocks and launchers of the placement engine.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace mpgp {

struct TcScales;

// ---- scalar slots of one evaluation (FP64, reduced on the device) ------------------------
enum Scalar : int {
    kSmooth = 0,      // sum of weighted LSE net lengths
    kHpwl,            // sum of weighted net HPWL
    kPredicted,       // proposal: sum raw_grad . (base - candidate)
    kMaxDisplacement, // proposal: max |base - candidate|
    kOverflowWith,    // density metrics with fillers / without fillers
    kOverflowWithout,
    kChargeWith,
    kChargeWithout,
    kNormalization,
    kDensitySumWith,
    kDensitySumWithout,
    kDensityMaxWith,
    kDensityMaxWithout,
    kEnergy,          // sum phi_hat * rho_hat * w_l * w_k (times bin_area / 2 gives the energy)
    kWireL1,
    kDensityL1,
    kRawNorm2,
    kPreNorm2,
    kDeltaPos2,       // sum |x - x_prev|^2
    kDeltaGrad2,      // sum |g - g_prev|^2 (preconditioned)
    kAlignment,       // sum velocity . g (preconditioned)
    kRudyL1,          // sum |RUDY gradient| over particles (unweighted)
    kRudyEnergy,      // RUDY hotspot energy (with capacity)
    kRudyHorizontal,  // total horizontal / vertical demand
    kRudyVertical,
    kRudyProxy,       // sum of utilisation overflow (divide by bins for the proxy overflow)
    kRudyMaxUtil,     // maximum utilisation
    kScalarCount
};

// ---- wirelength (net-parallel LSE) ---------------------------------------------------
struct WirelengthArgs {
    const double2* positions;     // P particle centres
    const int* pin_particle;      // I' pins in bucket order; < 0: static pin -(s+1)
    const float2* pin_offset;     // I' transformed offsets (movable pins)
    const double2* static_pins;   // S absolute static pin positions
    const int* net_start;         // N'+1 (nets with >= 2 pins, bucket order)
    const float* net_weight;      // N'
    const int4* block_work;       // per block: {lanes per net (1: two-pin nets, 0: warp loop), first net, net count, 0}
    float gamma;
    float inv_gamma;
    const int* pin_slot;          // I': the pin's slot in the particle-ordered gradient array (-1: static)
    float2* pin_gradient;         // particle-ordered slots (written when gradient != 0, movable pins only)
    int gradient;
    double* partials;             // per block: smooth, hpwl
    double* group_partials;       // per 32 blocks: smooth, hpwl (reduceGroups)
    unsigned int* group_counters;
};
void launchWirelength(const WirelengthArgs& args, int blocks, cudaStream_t stream);

// Batched launches (every family below has one): `count` instances' argument blocks
// in device memory, instance k owning launch blocks [offsets[k], offsets[k + 1]) of
// `blocks`; each block does exactly what block (b - offsets[k]) of the instance's own
// launch of offsets[k + 1] - offsets[k] blocks does, so results are those of the plain launch.
void launchWirelengthBatch(const WirelengthArgs* args, const int* offsets, int count, int blocks,
                           cudaStream_t stream);

// The allocation-free wirelength entry (mpgp_wirelength_noalloc): caller-owned
// device arrays in, scratch in a fixed file-scope device array.
constexpr int kNoAllocMaxPins = 1 << 20;
struct NoAllocWirelengthArgs {
    const double* positions;
    const int* net_pin_start;
    const int* pin_particle;
    const double* pin_xy;
    const double* net_weight;
    int net_count;
    int pin_count;
    const int* particle_pin_start;
    const int* particle_pins;
    int particle_count;
    double smoothing;
    double* wire_gradient;
    double* totals;
    void* stream;
};
void launchWirelengthNoAlloc(const NoAllocWirelengthArgs& args);

// ---- density scatter (fixed point) ------------------------------------------------
enum PositionMode : int { kGiven = 0, kPropose = 1, kLookahead = 2 };

struct ScatterArgs {
    int mode;
    int particle_count;
    const double2* positions;   // kGiven: positions to deposit
    const double2* base;        // kPropose / kLookahead: base positions
    const double2* direction;   // kPropose: preconditioned gradient; kLookahead: velocity
    const double2* raw;         // kPropose: raw gradient (predicted reduction)
    double step;                // kPropose: step size; kLookahead: momentum
    double max_displacement;    // kPropose
    double2* out_positions;     // kPropose / kLookahead: the clamped candidate
    const double2* size;        // P (width, height)
    const unsigned char* layer; // P
    double llx, lly, urx, ury;  // region
    double bin_w, bin_h;
    int bins_x, bins_y;
    unsigned long long* layers; // 3 * B fixed-point accumulators (movable, macro, filler)
    unsigned long long* totals; // 3 exact layer totals
    double* partials;           // per block: predicted, max displacement
    double* group_partials;     // per 32 blocks (reduceGroups), when group_counters is set
    unsigned int* group_counters;
};
void launchScatter(const ScatterArgs& args, int blocks, cudaStream_t stream);
void launchScatterBatch(const ScatterArgs* args, const int* offsets, int count, int blocks, cudaStream_t stream);

// ---- density metrics + DCT source --------------------------------------------------
struct MetricsArgs {
    unsigned long long* layers;        // 3 * B, read and reset to zero
    const unsigned long long* totals;  // 3
    const double* static_charge;       // B: t * (fixed + dark), the static part of the charge
    double static_fixed_sum;
    double static_dark_sum;
    double target_density;
    double bin_area;
    int bin_count;
    float* source;                     // B: deviation - mean (FP32 DCT input)
    double* partials;                  // per block: 9 metric partials
    // Fused form: the source is not stored; each row's fp16 planes go straight
    // into the first contraction's operand, with the row exponent from its maximum.
    int columns, rows;
    __half* split_out;
    int split_ld;
    size_t split_plane;
    int* row_exp;
    TcScales* scales;
    double* group_partials;            // per 32 blocks (reduceGroups), when group_counters is set
    unsigned int* group_counters;
};
void launchMetrics(const MetricsArgs& args, int blocks, cudaStream_t stream);
// The fused metrics-and-split pass takes one block per bin row and keeps a
// row's sources in registers: up to kMetricsSplitPerThread bins per thread.
constexpr int kMetricsSplitPerThread = 8;
inline bool metricsSplitFits(int columns) { return columns > 0 && columns <= kMetricsSplitPerThread * 256; }
void launchMetricsSplit(const MetricsArgs& args, cudaStream_t stream);
void launchMetricsSplitBatch(const MetricsArgs* args, const int* offsets, int count, int blocks,
                             cudaStream_t stream);

// ---- RUDY routing-demand map (rudy.cu) -------------------------------------------------
struct RudyArgs {
    const double2* positions;
    const int* pin_particle;      // the wirelength pass's bucketed pins and nets
    const float2* pin_offset;
    const double2* static_pins;
    const int* net_start;
    const double* net_weight;     // FP64 weights in bucket order
    int net_count;
    const int* pin_slot;
    double2* pin_gradient;        // particle-ordered pin slots (gradient pass)
    double llx, lly, urx, ury;    // core region
    double bin_w, bin_h;
    int columns, rows;
    double minimum_x_span, minimum_y_span;
    double inv_unit_h, inv_unit_v;  // fixed point: 2^32 / bin_w, 2^32 / bin_h
    unsigned long long* diff;       // 2 x (rows + 1) x (columns + 1) difference arrays (H, V), zero between uses
    unsigned long long* horizontal; // rows x columns demand maps, written by the prefix pass
    unsigned long long* vertical;
    double capacity_h, capacity_v;  // 0: maps and totals only
    int model;                      // MPGP_RUDY_*
    double temperature;
    double* adjoint_h;
    double* adjoint_v;
    double* utilization;            // per bin max(uh, uv), or null
    double* table;                  // 2 x (rows + 1) x (columns + 1) summed-area tables of the adjoints
    double* partials;               // per block: energy, H total, V total, proxy, max utilisation
};
int rudyBlocks(int count);
void launchRudyDeposit(const RudyArgs& args, cudaStream_t stream);
void launchRudyPrefix(const RudyArgs& args, cudaStream_t stream);
void launchRudyMetrics(const RudyArgs& args, int blocks, cudaStream_t stream);
void launchRudyTables(const RudyArgs& args, cudaStream_t stream);
void launchRudyGradient(const RudyArgs& args, cudaStream_t stream);

// ---- deterministic reduction of all partials into the scalar block ----------------------
// Source row r is partials[r * stride + column]; the producers write their
// partials column-major (partial k of block b at k * grid + b), so stride is 1
// and column is k * grid, and a source's rows are contiguous.
struct ReduceSource {
    const double* partials;
    int rows;    // number of blocks that wrote partials
    int stride;  // doubles between consecutive rows
    int column;  // offset of row 0
    int is_max;
    int target;  // Scalar slot
};
struct ReduceArgs {
    ReduceSource sources[kScalarCount];
    int source_count;
    int offsets[kScalarCount + 1];  // prefix sums of the sources' rows (the staged layout)
    int staged_capacity;            // doubles of dynamic shared memory the reduction kernel has
    double* scalars;             // kScalarCount
    unsigned long long* totals;  // reset to zero after use (may be null)
    // Optional completion record in mapped pinned host memory, written without
    // fences: every scalar travels as two 8-byte words (32 bits of the value and
    // the 32-bit evaluation sequence each), slot kScalarCount carries the sticky
    // device error flag the same way.  An aligned 8-byte store arrives whole, so
    // the host takes a value once both of its words show the current sequence.
    unsigned long long* host_slots;  // 2 * (kScalarCount + 1) words
    const int* device_error;
    unsigned int sequence;
};
static_assert(kScalarCount < 32, "the expected-scalar mask is 32 bits wide");
// One block reduces every source (one warp per source, rows in a fixed order).
constexpr int kReduceThreads = 1024;
constexpr int kReduceStaged = 24576;  // doubles staged in shared memory (192 KiB)
void launchReduce(const ReduceArgs& args, cudaStream_t stream);
// One block per instance; staged_doubles: the largest staging of the instances (shared memory).
void launchReduceBatch(const ReduceArgs* args, int count, int staged_doubles, cudaStream_t stream);

// ---- field gather + gradient combine (the fused update pass) ----------------------------
struct GatherArgs {
    int particle_count;
    int movable_count;
    const double2* positions;
    const int* particle_pin_start;  // M+1: particle i's pin gradients are slots [start[i], start[i+1])
    const float2* pin_gradient;     // particle-ordered slots
    const float2* field;            // B interleaved (Ex, Ey)
    const double* charge;           // P
    const double* precond_base;     // P (nullptr: split mode)
    double llx, lly, urx, ury, inv_bin_w, inv_bin_h;
    int bins_x, bins_y;
    double penalty;
    double precond_scale;           // 1 / density_strength
    double2* raw;                   // combined mode outputs
    double2* pre;
    double2* wire_out;              // split mode outputs (drop-in backend)
    double2* density_out;
    double2* rudy_out;              // split mode, optional: the RUDY subgradient per particle
    const double2* prev_positions;  // optional (step estimate)
    const double2* prev_gradient;
    const double2* velocity;        // optional (momentum alignment)
    const double2* velocity_base;   // optional: velocity_out = positions - velocity_base (the alignment uses it)
    double2* velocity_out;
    double2* checkpoint_out;        // optional: a copy of the positions
    const double2* rudy_gradient;   // optional: RUDY pin slots (particle order), added with rudy_weight
    double rudy_weight;
    double* partials;               // per block: 8 partials (kWireL1 .. kRudyL1)
    double* group_partials;         // per 32 blocks (reduceGroups), when group_counters is set
    unsigned int* group_counters;
};
// With `reduce`, the block that completes the last group fold also reduces the
// evaluation's partials (every source of `reduce`) and publishes them: the gather is
// the evaluation's last kernel, and no reduction launch follows it.
void launchGather(const GatherArgs& args, const ReduceArgs* reduce, int blocks, cudaStream_t stream);
// reduces[k]: instance k's reduction (device memory), or null (a null array: none reduce).
void launchGatherBatch(const GatherArgs* args, const ReduceArgs* const* reduces, const int* offsets, int count,
                       int blocks, cudaStream_t stream);
// The gather's grid: one resident wave of blocks (grid-stride over the particles).
int gatherBlocks(int particle_count);

// ---- small vector kernels ---------------------------------------------------------
// A device-to-device copy of positions as a chained kernel (programmatic launch, no copy engine).
void launchCopyPositions(const double2* source, double2* destination, int count, cudaStream_t stream);
void launchVelocity(const double2* next, const double2* previous, double2* velocity, int count,
                    cudaStream_t stream);


}  // namespace mpgp
