/*
 * mpgp.h -- C ABI of the B200-native global-placement engine (libmpgp.so).
 *
 * The engine evaluates MyPlacement's `adaptive + neumann + course_eplace_v1`
 * global-placement objective on one NVIDIA B200 (sm_100a) and can run the
 * whole adaptive controller with its state resident on the device.
 *
 * Conventions
 *   - Every entry point returns an int status (MPGP_OK == 0) and never throws.
 *     The message of the most recent failure on the calling thread is
 *     available from mpgp_last_error().
 *   - All arrays are caller-owned host memory, plain pointers plus counts.
 *     Positions and gradients are interleaved (x0, y0, x1, y1, ...) doubles,
 *     exactly the layout of std::vector<myplacement::Vec2>.
 *   - A handle is confined to one host thread; its work runs on one CUDA
 *     stream owned by the handle.
 *   - Status codes map onto the reference's error conventions:
 *     MPGP_ERR_INVALID_ARGUMENT  <-> std::invalid_argument
 *     MPGP_ERR_PARSE             <-> myplacement::ParseError (BookShelf input)
 *     MPGP_ERR_RUNTIME / _CUDA / _NON_FINITE / _BUDGET <-> std::runtime_error
 *     MPGP_ERR_UNAVAILABLE       <-> tryCreateCudaPlacementBackend returning
 *                                    nullptr with a populated reason.
 */
#ifndef MPGP_H
#define MPGP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MPGP_ABI_VERSION 1

enum {
    MPGP_OK = 0,
    MPGP_ERR_INVALID_ARGUMENT = 1,
    MPGP_ERR_RUNTIME = 2,
    MPGP_ERR_CUDA = 3,
    MPGP_ERR_BUDGET = 4,
    MPGP_ERR_NON_FINITE = 5,
    MPGP_ERR_UNAVAILABLE = 6,
    MPGP_ERR_TIMEOUT = 7,
    MPGP_ERR_PARSE = 8
};

/* Module flag bits (PlacementDatabase.hpp Module::is_terminal / is_fixed). */
enum { MPGP_MODULE_TERMINAL = 1, MPGP_MODULE_FIXED = 2 };

/* Density layers of a particle (CudaPlacementBackend.cu:789-800: 0/1/2). */
enum { MPGP_LAYER_STANDARD = 0, MPGP_LAYER_MACRO = 1, MPGP_LAYER_FILLER = 2 };

/* Compute backend (GlobalPlacer.hpp:19 ComputeBackend). */
enum { MPGP_BACKEND_CPU = 0, MPGP_BACKEND_CUDA = 1, MPGP_BACKEND_AUTO = 2 };

/* RUDY penalty (Rudy.hpp:16 RudyPenaltyModel). */
enum { MPGP_RUDY_DISABLED = 0, MPGP_RUDY_HINGE_L2 = 1, MPGP_RUDY_SOFTPLUS_L2 = 2, MPGP_RUDY_HINGE_L4 = 3 };

/*
 * A flattened PlacementDatabase (include/myplacement/model/PlacementDatabase.hpp:
 * Module :30-51, Pin :23-28, Net :53-57, SiteRow :59-69).  Pins are listed net
 * by net: the pins of net n are [net_pin_start[n], net_pin_start[n+1]).  Module
 * centres are the `center` field; pin offsets are relative to the centre
 * before the module orientation is applied (transformOffset, PlacementDatabase.cpp:55-68).
 */
typedef struct mpgp_design {
    int32_t module_count;
    const double* module_width;
    const double* module_height;
    const double* module_x;
    const double* module_y;
    const int32_t* module_flags;       /* MPGP_MODULE_* bits */
    const int32_t* module_orientation; /* Orientation enum order N,S,E,W,FN,FS,FE,FW; NULL = all N */
    int32_t net_count;
    const double* net_weight;
    const int64_t* net_pin_start; /* net_count + 1 entries */
    int64_t pin_count;
    const int32_t* pin_module;
    const double* pin_offset_x;
    const double* pin_offset_y;
    int32_t row_count;
    const double* row_bottom;
    const double* row_height;
    const double* row_site_width;
    const double* row_site_spacing;
    const double* row_x_start;
    const int64_t* row_site_count;
} mpgp_design;

/* GlobalPlacementOptions (include/myplacement/placement/GlobalPlacer.hpp:26-80),
 * field for field; mpgp_options_default() fills the reference defaults. */
typedef struct mpgp_options {
    int32_t iterations;
    int32_t bins_x;
    int32_t bins_y;
    int32_t report_interval;
    double target_density;
    double maximum_bin_overflow;
    double initial_smoothing;
    double final_smoothing;
    double maximum_movement_in_bins;
    double penalty_growth;
    int32_t optimizer; /* 1 = adaptive (the only one this engine implements) */
    int32_t maximum_backtracks;
    double backtracking_ratio;
    double armijo_coefficient;
    double maximum_momentum;
    double initial_movement_in_bins;
    double objective_increase_for_density;
    double hpwl_growth_restart_threshold;
    double density_stall_threshold;
    double density_penalty_increase;
    double density_penalty_decrease;
    double minimum_density_penalty;
    double maximum_density_penalty;
    double smoothing_overflow_exponent;
    int32_t feasible_refinement_iterations;
    int32_t pad0;
    uint64_t maximum_fillers;
    uint64_t seed;
    /* RudyOptions (Rudy.hpp:21-40) and the routability schedule. */
    int32_t rudy_columns;
    int32_t rudy_rows;
    double rudy_minimum_span_in_bins;
    double rudy_capacity_factor;
    double rudy_softplus_temperature;
    int32_t rudy_penalty_model;
    int32_t rudy_validation_bins;
    double rudy_validation_capacity_factor;
    double routability_start_overflow;
    double routability_weight_scale;
    int32_t routability_ramp_iterations;
    int32_t density_field_boundary; /* 1 = Neumann (the only boundary the engine implements) */
    int32_t compute_backend;        /* MPGP_BACKEND_* */
    int32_t cuda_device;
    uint64_t maximum_cuda_memory_bytes;
} mpgp_options;

/* DensityMetrics (include/myplacement/metrics/Metrics.hpp:38-47). */
typedef struct mpgp_density_metrics {
    double total_overflow_area;
    double normalized_overflow;
    double maximum_density;
    double average_density;
    double total_charge_area;
    double normalization_area;
    double placeable_area;
    double dark_area;
} mpgp_density_metrics;

/* CudaPlacementEvaluation without the gradient vectors
 * (src/placement/CudaPlacementBackend.hpp:15-23); gradients go to caller arrays. */
typedef struct mpgp_evaluation {
    double hpwl;
    double smooth_wirelength;
    double electrostatic_energy;
    mpgp_density_metrics optimizer_density;
    mpgp_density_metrics design_density;
} mpgp_evaluation;

/* GlobalPlacementIteration (GlobalPlacer.hpp:82-105); the global_history.csv row. */
typedef struct mpgp_history_row {
    int32_t iteration;
    int32_t backtracks;
    double hpwl;
    double overflow;
    double design_overflow;
    double smooth_wirelength;
    double density_energy;
    double objective;
    double penalty;
    double smoothing;
    double step_size;
    double maximum_displacement;
    double gradient_norm;
    double curvature;
    double rudy_energy;
    double rudy_proxy_overflow;
    double rudy_maximum_utilization;
    double rudy_weight;
    int32_t momentum_restarted;
    int32_t accepted;
    int32_t best_checkpoint;
    int32_t rudy_active;
} mpgp_history_row;

/* GlobalPlacementResult (GlobalPlacer.hpp:107-129) minus the history vector. */
typedef struct mpgp_result {
    double hpwl_before;
    double hpwl_after;
    double overflow_before;
    double overflow_after;
    int32_t completed_iterations;
    int32_t accepted_iterations;
    int32_t momentum_restarts;
    int32_t rejected_candidates;
    int32_t best_checkpoint_iteration;
    int32_t restored_best_checkpoint;
    double best_checkpoint_hpwl;
    double best_checkpoint_overflow;
    double elapsed_seconds;
    int32_t compute_backend_used;
    int32_t cuda_device_used;
    uint64_t cuda_reserved_memory_bytes;
    int32_t history_count;
    int32_t evaluations; /* gradient + candidate evaluations performed */
    double rudy_energy_after;
    /* RudyMetrics at the final placement (GlobalPlacementResult::rudy_metrics and
     * rudy_validation_metrics, GlobalPlacer.hpp:107-129); zero when RUDY never activated. */
    double rudy_horizontal_capacity;
    double rudy_vertical_capacity;
    double rudy_proxy_overflow_after;
    double rudy_maximum_utilization_after;
    double rudy_p95_utilization_after;
    double rudy_validation_energy_after;
    double rudy_validation_proxy_overflow_after;
    double rudy_validation_maximum_utilization_after;
    double rudy_validation_p95_utilization_after;
} mpgp_result;

/*
 * The flattened backend layout: what tryCreateCudaPlacementBackend receives
 * (CudaPlacementBackend.hpp:45-48) after buildHostLayout
 * (CudaPlacementBackend.cu:784-839).  Particles are the movable modules in
 * PlacementDatabase::movableModules() order followed by the fillers.  A pin
 * with pin_particle[i] >= 0 sits at particle centre + (pin_x, pin_y) (offset
 * already orientation-transformed); a pin with pin_particle[i] < 0 is static
 * at the absolute position (pin_x, pin_y).  Static bin layers are row-major
 * [row * bins_x + column] physical areas (DensityBin::fixed_area / dark_area).
 */
typedef struct mpgp_layout {
    int64_t particle_count;
    int64_t movable_count;
    const double* particle_width;
    const double* particle_height;
    const int32_t* particle_layer; /* MPGP_LAYER_* */
    const int32_t* particle_pin_count; /* Module::pins.size(); 0 for fillers (preconditioner) */
    int32_t net_count;
    int32_t pad0;
    const double* net_weight;
    const int64_t* net_pin_start;
    int64_t pin_count;
    const int32_t* pin_particle;
    const double* pin_x;
    const double* pin_y;
    int32_t bins_x;
    int32_t bins_y;
    double region_llx;
    double region_lly;
    double region_urx;
    double region_ury;
    double target_density;
    const double* static_fixed_area;
    const double* static_dark_area;
} mpgp_layout;

typedef struct mpgp_backend mpgp_backend;
typedef struct mpgp_session mpgp_session;
typedef struct mpgp_setup mpgp_setup;

/* ---- library ---------------------------------------------------------------- */

/* Replaces cudaPlacementBackendCompiled() (CudaPlacementBackend.hpp:44,
 * CudaPlacementBackend.cu:1152-1154).  Returns 1. */
int mpgp_compiled(void);

/* ABI version of the loaded library (MPGP_ABI_VERSION). */
int mpgp_abi_version(void);

/* Message of the last failure on this thread ("" when none). */
const char* mpgp_last_error(void);

/* Fills the reference defaults of GlobalPlacementOptions (GlobalPlacer.hpp:26-80). */
void mpgp_options_default(mpgp_options* options);

/* ---- drop-in backend: one evaluation per call ---------------------------------- */

/* Replaces tryCreateCudaPlacementBackend (CudaPlacementBackend.hpp:45-48,
 * CudaPlacementBackend.cu:1156-1216).  On a recoverable failure returns
 * MPGP_ERR_UNAVAILABLE and writes the reason (the reference's nullptr + reason). */
int mpgp_backend_create(const mpgp_layout* layout, int device, uint64_t maximum_bytes, mpgp_backend** out,
                        char* reason, size_t reason_capacity);

/* Replaces CudaPlacementBackend::evaluate (CudaPlacementBackend.hpp:32-33,
 * CudaPlacementBackend.cu:921-950).  `positions` holds particle_count (x, y)
 * pairs.  When calculate_gradient != 0 the wire and density gradients (each
 * particle_count (x, y) pairs) are written to the caller's arrays. */
int mpgp_backend_evaluate(mpgp_backend* backend, const double* positions, double smoothing,
                          int calculate_gradient, mpgp_evaluation* out, double* wire_gradient,
                          double* density_gradient);

/* Failure-detection test hook; no counterpart in the reference, which has no
 * device-side waits.  With polls > 0 every field contraction of this backend's
 * later evaluations first waits, for at most `polls` polls, on a barrier that
 * nothing completes: the wait runs out, the contraction raises the backend's
 * error flag and returns before it issues any copy or allocates tensor memory,
 * and the evaluation returns MPGP_ERR_TIMEOUT.  The flag stays raised: every
 * later evaluation of this backend also fails, and a new backend starts clean.
 * 0 turns the hook off. */
int mpgp_backend_set_stall_probe(mpgp_backend* backend, int64_t polls);

/* Replaces CudaPlacementBackend::device() (CudaPlacementBackend.hpp:34). */
int mpgp_backend_device(const mpgp_backend* backend);

/* Replaces CudaPlacementBackend::reservedBytes() (CudaPlacementBackend.hpp:35). */
uint64_t mpgp_backend_reserved_bytes(const mpgp_backend* backend);

/* Replaces ~CudaPlacementBackend (CudaPlacementBackend.hpp:27). */
void mpgp_backend_destroy(mpgp_backend* backend);

/* Parity hook with no behavioural counterpart: copies the three fixed-point
 * dynamic density layers of the last evaluation (movable, macro, filler; each
 * bins_x*bins_y int64 in units of bin_area * 2^-32) to host arrays. */
int mpgp_backend_density_layers(mpgp_backend* backend, int64_t* movable, int64_t* macro, int64_t* filler);

/* Parity hook: solves the Neumann field of `deviation` (bins_x*bins_y doubles)
 * with the engine's DCT contractions, matching ElectrostaticField::solve
 * (ElectrostaticField.cpp:119-133, 205-237).  Any output may be NULL. */
int mpgp_backend_field_solve(mpgp_backend* backend, const double* deviation, double* potential, double* field_x,
                             double* field_y);

/* Parity hook: the RUDY routing-demand proxy of one placement on the backend's
 * nets, as evaluateRudy (Rudy.cpp:227-340) computes it with a fixed capacity.
 * `options` gives rudy_columns, rudy_rows, rudy_minimum_span_in_bins,
 * rudy_penalty_model and rudy_softplus_temperature; the first call fixes the
 * grid and later calls must give the same one.  A zero capacity evaluates the
 * demand alone.  metrics (10 doubles): horizontal and vertical total demand,
 * horizontal and vertical mean demand, horizontal and vertical capacity, proxy
 * overflow, maximum and 95th-percentile utilisation, energy.  With
 * calculate_gradient (positive capacities required) `gradient` receives the
 * subgradient per particle (x, y), zero for fillers, and `energy` the energy of
 * the evaluation that produced it. */
int mpgp_backend_rudy(mpgp_backend* backend, const mpgp_options* options, const double* positions,
                      double horizontal_capacity, double vertical_capacity, int calculate_gradient, double* metrics,
                      double* energy, double* gradient);

/*
 * Allocation-free wirelength and wire gradient.  This entry point has no
 * counterpart in the reference; it exists for callers that own every byte of
 * device memory and cannot let a library call cudaMalloc -- a host framework
 * whose caching allocator or fixed device-memory budget owns the GPU (as the
 * reference's DeviceMemoryBudget does), or a latency-critical loop where the
 * implicit device synchronisation of cudaMalloc/cudaFree is not acceptable.
 *
 * It computes the same log-sum-exp smooth wirelength, HPWL and per-particle
 * wire gradient as one mpgp_backend_evaluate (evaluateSmoothWirelength,
 * AdaptiveGlobalPlacer.cpp:29-82) from caller-owned DEVICE arrays:
 *   positions          particle_count (x, y) doubles
 *   net_pin_start      net_count + 1 int32 offsets into the pins
 *   pin_particle       pin_count int32; < 0 marks a static pin
 *   pin_xy             pin_count (x, y) doubles: the offset from the particle
 *                      centre, or the absolute position of a static pin
 *   net_weight         net_count doubles
 *   particle_pin_start particle_count + 1 int32, particle_pins: the pins of
 *                      each particle (indices into the pin arrays)
 * and writes wire_gradient (particle_count (x, y) doubles) and totals[0] =
 * smooth wirelength, totals[1] = HPWL.  Work is enqueued on `stream` (a
 * cudaStream_t; NULL = the default stream) and is complete when the stream is.
 *
 * Its scratch is one fixed file-scope device array that every GPU loading the
 * library holds until the process exits (8.03 MiB): pin_count may not exceed
 * 1,048,576 (larger inputs return MPGP_ERR_INVALID_ARGUMENT and launch
 * nothing).  The first call on each device looks up that array's device
 * address with the device current; make that first call before any stream
 * capture.  The address is looked up again when the current CUDA context
 * changes (after cudaDeviceReset, or under a caller's own context).  All calls
 * share the one array, and each call clears the pin slots it uses before its
 * net pass: a pin that no net of two or more pins covers (including the pins
 * of a net whose range lies outside [0, pin_count], which is skipped) adds
 * nothing, and a particle takes the gradient of a listed pin only when
 * pin_particle names that particle.  Calls that overlap on the GPU (different
 * streams, or threads) race on the array and must be serialised by the caller.
 * No device memory is allocated or freed.
 */
int mpgp_wirelength_noalloc(const double* positions, const int32_t* net_pin_start, const int32_t* pin_particle,
                            const double* pin_xy, const double* net_weight, int32_t net_count, int32_t pin_count,
                            const int32_t* particle_pin_start, const int32_t* particle_pins,
                            int32_t particle_count, double smoothing, double* wire_gradient, double* totals,
                            void* stream);

/* ---- BookShelf input ----------------------------------------------------------- */

/* BookshelfParser::parseAux (include/myplacement/io/BookshelfParser.hpp:16-19;
 * src/io/BookshelfParser.cpp:313-348 with the readers of :62-278 and
 * validateCounts :280-299): reads the design an .aux file names (.nodes, .scl,
 * .pl, .nets, and .wts when present) into a flattened PlacementDatabase.  The
 * records, values and error texts are the reference reader's, and so is which
 * error comes first; its ParseError is MPGP_ERR_PARSE and the database's
 * std::invalid_argument (duplicate names, negative sizes) is
 * MPGP_ERR_INVALID_ARGUMENT.  The files are read whole and parsed by `threads`
 * host threads (<= 0: one per hardware thread, at most 32); the result does not
 * depend on the thread count.  No GPU is used. */
typedef struct mpgp_bookshelf mpgp_bookshelf;

typedef struct mpgp_bookshelf_view {
    mpgp_design design;               /* arrays owned by the handle; module_orientation is set */
    const char* module_names;         /* the names back to back, no separators */
    const int64_t* module_name_start; /* module_count + 1 offsets into module_names */
    const char* net_names;
    const int64_t* net_name_start;    /* net_count + 1 offsets into net_names */
    const int8_t* pin_direction;      /* PinDirection order: 0 input, 1 output, 2 bidirectional, 3 unknown */
    const int32_t* row_orientation;   /* Orientation order, 8 = unknown */
    int64_t declared_nodes;           /* NumNodes, NumTerminals, NumNets, NumPins as declared; -1 if absent */
    int64_t declared_terminals;
    int64_t declared_nets;
    int64_t declared_pins;
} mpgp_bookshelf_view;

int mpgp_bookshelf_read(const char* aux_path, int32_t threads, mpgp_bookshelf** out);
/* Pointers into the handle, valid until mpgp_bookshelf_destroy. */
int mpgp_bookshelf_get(const mpgp_bookshelf* book, mpgp_bookshelf_view* view);
void mpgp_bookshelf_destroy(mpgp_bookshelf* book);

/* ---- detailed placement ---------------------------------------------------------- */

/* DetailedPlacementMethod (include/myplacement/placement/DetailedPlacer.hpp:14). */
enum { MPGP_DETAILED_NONE = 0, MPGP_DETAILED_ADJACENT_SWAP = 1, MPGP_DETAILED_WINDOW_REORDER = 2 };

/* DetailedPlacementOptions (DetailedPlacer.hpp:23-44) for the device backend;
 * mpgp_detailed_options_default() fills the reference defaults with the
 * window-reorder method. */
typedef struct mpgp_detailed_options {
    int32_t method;
    int32_t passes;
    int32_t window_size;
    int32_t cuda_device;
    uint64_t maximum_net_degree;
    double improvement_epsilon;
    uint64_t maximum_cuda_memory_bytes;
} mpgp_detailed_options;

/* DetailedPlacementResult (DetailedPlacer.hpp:46-57). */
typedef struct mpgp_detailed_result {
    double hpwl_before;
    double hpwl_after;
    double elapsed_seconds;
    uint64_t evaluated_windows;
    uint64_t evaluated_permutations;
    uint64_t accepted_operations;
    int32_t completed_passes;
    int32_t cuda_device_used;
    uint64_t cuda_reserved_memory_bytes;
} mpgp_detailed_result;

void mpgp_detailed_options_default(mpgp_detailed_options* options);

/* tryRunCudaDetailedPlacement (src/placement/CudaDetailedPlacementBackend.hpp:
 * 13-16; src/placement/cuda/CudaDetailedPlacementBackend.cu:491-709): window
 * reordering of four consecutive cells of each row segment, every ordering
 * evaluated on the device, the reference's acceptance rule and order of
 * application, on a legal placement.  The design's module_x / module_y /
 * module_orientation are the placement on entry; the result goes to
 * module_x / module_y / module_orientation (module_count each; orientation
 * may be NULL).  row_orientation (row_count, Orientation order, 8 = unknown;
 * NULL = all N) is the SiteRow orientation a moved cell takes.  Where the
 * reference backend declines (options other than a four-cell window reorder,
 * options out of range, no usable device) the call returns
 * MPGP_ERR_UNAVAILABLE with the reason and changes nothing. */
int mpgp_detailed_place(const mpgp_design* design, const int32_t* row_orientation,
                        const mpgp_detailed_options* options, double* module_x, double* module_y,
                        int32_t* module_orientation, mpgp_detailed_result* result, char* reason,
                        size_t reason_capacity);

/* ---- host setup restated from the reference ----------------------------------- */

/* randomPlacement (src/placement/InitialPlacer.cpp:102-121): writes the module
 * centres (module_count each) after seeding movables uniformly in the core. */
int mpgp_random_placement(const mpgp_design* design, uint64_t seed, double* module_x, double* module_y);

/* The host part of GlobalPlacementSession's constructor (AdaptiveGlobalPlacer.cpp:
 * 114-126): static density (initializeStaticDensity, GlobalPlacementSupport.cpp:21-30),
 * fillers (createDensityFillers, :52-103) and the preconditioner
 * (initializePreconditioner, AdaptiveGlobalPlacer.cpp:358-375).  Host only: it
 * needs no GPU, and mpgp_session_create runs the same code.  Particle queries
 * are in session order (movable modules, then fillers); movable modules report
 * position 0 (their positions are the caller's).  With NULL arrays only the
 * counts are written. */
int mpgp_setup_create(const mpgp_design* design, const mpgp_options* options, mpgp_setup** out);
int mpgp_setup_particles(const mpgp_setup* setup, int64_t* particle_count, int64_t* movable_count, double* x,
                         double* y, double* width, double* height, int32_t* layer, double* preconditioner);
int mpgp_setup_static_density(const mpgp_setup* setup, double* fixed, double* dark);
void mpgp_setup_destroy(mpgp_setup* setup);

/* ---- device-resident adaptive global placement ---------------------------------- */

/* Replaces GlobalPlacer::run (GlobalPlacer.cpp:134-146) ->
 * runAdaptiveGlobalPlacement (AdaptiveGlobalPlacer.cpp:652-953) for
 * compute_backend cuda.  module_x/module_y hold every module centre on input and
 * receive the placed centres.  Up to history_capacity rows are written. */
int mpgp_global_place(const mpgp_design* design, const mpgp_options* options, double* module_x, double* module_y,
                      mpgp_result* result, mpgp_history_row* history, int32_t history_capacity);

/* The same run split into steps, for callers that interleave work or time
 * iterations: create (setup + the two initial evaluations,
 * AdaptiveGlobalPlacer.cpp:656-733), step (up to `iterations` controller
 * iterations; *done becomes 1 after the budget or the early stop), finish
 * (checkpoint restore + final metrics, :930-952). */
int mpgp_session_create(const mpgp_design* design, const mpgp_options* options, mpgp_session** out);
int mpgp_session_step(mpgp_session* session, int32_t iterations, int32_t* completed, int32_t* done);
int mpgp_session_finish(mpgp_session* session, double* module_x, double* module_y, mpgp_result* result,
                        mpgp_history_row* history, int32_t history_capacity);
/* Current particle positions (particle_count (x, y) pairs). */
int mpgp_session_positions(const mpgp_session* session, double* positions);
/* Tracing (no counterpart in the reference, which times only the whole run,
 * AdaptiveGlobalPlacer.cpp:656, 951): every kernel launch of a family whose bit
 * is set in `families` is bracketed by CUDA events on its stream and its device
 * time is accumulated per family (families = 0 turns profiling off; each event
 * pair costs host time, so time only the families of interest).  Families are
 * numbered 0..mpgp_kernel_kind_count()-1. */
int mpgp_kernel_kind_count(void);
const char* mpgp_kernel_kind_name(int kind);
int mpgp_session_set_profiling(mpgp_session* session, uint32_t families);
int mpgp_session_kernel_stats(const mpgp_session* session, int64_t* launches, double* milliseconds,
                              int32_t capacity);
int mpgp_session_reset_kernel_stats(mpgp_session* session);
/* Host<->device bytes the session has copied (setup, positions, scalar read-backs). */
int mpgp_session_transfer_bytes(const mpgp_session* session, uint64_t* to_device, uint64_t* to_host);
/* Number of engine kernel launches issued by this session so far. */
int64_t mpgp_session_kernel_launches(const mpgp_session* session);
/* The CUDA stream the session's work runs on (a cudaStream_t). */
void* mpgp_session_stream(const mpgp_session* session);
void mpgp_session_destroy(mpgp_session* session);

/* ---- batched and served forms ------------------------------------------------
 *
 * No counterpart in the reference, which places one design per process
 * (main.cpp:413, GlobalPlacer::run).  A server runs many independent
 * placements (each exactly mpgp_global_place) at once on one GPU: a FIFO of
 * jobs, `workers` host threads each driving one device-resident session on its
 * own streams, and admission by estimated device footprint against
 * `memory_budget_bytes` (0 = 90 % of the device's free memory).  A job that
 * arrives while others run starts as soon as a worker and the memory are free;
 * its result is the same as when it runs alone. */
typedef struct mpgp_server mpgp_server;

typedef struct mpgp_job_stats {
    double queued_seconds;          /* submit -> start */
    double run_seconds;             /* start -> finish */
    double latency_seconds;         /* submit -> finish */
    uint64_t estimated_bytes;       /* the footprint the admission reserved */
    uint64_t reserved_bytes;        /* device bytes the job's session actually reserved */
    int32_t completed_iterations;
    int32_t status;                 /* MPGP_OK, or the job's failure */
} mpgp_job_stats;

typedef struct mpgp_server_stats {
    int64_t submitted;
    int64_t completed;
    int64_t failed;
    int64_t iterations;             /* controller iterations of completed jobs */
    int32_t workers;
    int32_t peak_running;           /* most jobs on the device at once */
    uint64_t memory_budget;
    uint64_t peak_reserved;         /* largest sum of admitted footprints */
    double seconds;                 /* since the server was created */
    int32_t batched;                /* 1: the running jobs' evaluations share batched launches */
    int32_t batch_peak_round;       /* most evaluations one batched round carried */
    int64_t batch_rounds;           /* batched rounds launched */
    int64_t batch_evaluations;      /* evaluations those rounds carried */
    int64_t batch_launches;         /* kernel launches of those rounds */
    double batch_busy_seconds;      /* host time from each round's upload to its completion, summed */
    double batch_device_seconds;    /* device time of the rounds (CUDA events around each), summed */
} mpgp_server_stats;

/* Upper bound of the device bytes one placement of `design` reserves. */
int mpgp_estimate_bytes(const mpgp_design* design, const mpgp_options* options, uint64_t* bytes);
int mpgp_server_create(int device, uint64_t memory_budget_bytes, int32_t workers, mpgp_server** out);
/* As mpgp_server_create, choosing the mode: batched != 0 gathers the running
 * jobs' evaluations into shared rounds, one launch per kernel family for all of
 * them (mpgp_server_create's mode); batched == 0 lets every job launch its own
 * kernels on its own streams.  The results are the same either way. */
int mpgp_server_create_mode(int device, uint64_t memory_budget_bytes, int32_t workers, int32_t batched,
                            mpgp_server** out);
/* Copies the design and options (options->cuda_device is replaced by the
 * server's device).  A job whose footprint exceeds the budget is refused with
 * MPGP_ERR_BUDGET. */
int mpgp_server_submit(mpgp_server* server, const mpgp_design* design, const mpgp_options* options, int64_t* job);
/* Waits up to timeout_seconds (< 0: without limit); *done = 1 once the job has finished. */
int mpgp_server_wait(mpgp_server* server, int64_t job, double timeout_seconds, int32_t* done);
/* Copies a finished job's outputs (as mpgp_global_place) and releases it; a
 * failed job returns its failure status here. */
int mpgp_server_take(mpgp_server* server, int64_t job, double* module_x, double* module_y, mpgp_result* result,
                     mpgp_history_row* history, int32_t history_capacity, mpgp_job_stats* stats);
int mpgp_server_stats_get(const mpgp_server* server, mpgp_server_stats* stats);
/* Finishes the running jobs, abandons the queued ones, joins the workers. */
void mpgp_server_destroy(mpgp_server* server);

/* ---- autotuning --------------------------------------------------------------
 *
 * No counterpart in the reference.  The K split of the tcgen05 field
 * contractions (how many CTAs of a cluster share one output tile's sum) per
 * contracted length (bins along the summed axis).  The library starts with the
 * table that myplacement_b200/tune.py measured on a B200 (tuned_splits.inc);
 * set replaces it for engines created afterwards (splits 1 or 2; a split whose
 * clusters do not all fit on the GPU at once is not used).  get copies up to
 * `capacity` entries and returns the table's size in *count. */
int mpgp_tuning_set_splits(const int32_t* sizes, const int32_t* splits, int32_t count);
int mpgp_tuning_get_splits(int32_t* sizes, int32_t* splits, int32_t capacity, int32_t* count);

/* The batched form: `count` placements through a server (submit all, take all),
 * in the server's batched mode when batched != 0.  module_x[i] / module_y[i]
 * receive design i's positions; history is not kept. */
int mpgp_batch_place(int32_t count, const mpgp_design* designs, const mpgp_options* options, int device,
                     int32_t workers, int32_t batched, uint64_t memory_budget_bytes, double* const* module_x,
                     double* const* module_y, mpgp_result* results, mpgp_job_stats* job_stats,
                     mpgp_server_stats* server_stats);

#ifdef __cplusplus
}
#endif

#endif /* MPGP_H */
