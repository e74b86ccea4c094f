// Test-oracle infrastructure: only tests/, __graft_entry__.smoke() and the CPU
// baseline legs of bench.py load the libraries built from this file.
//
// A C ABI over the reference's own global-placement code, compiled from the
// unmodified reference sources (oracle/build_oracle.py).  This translation unit
// includes src/placement/AdaptiveGlobalPlacer.cpp so that the reference's
// internal GlobalPlacementSession (AdaptiveGlobalPlacer.cpp:112-389) and
// evaluateSmoothWirelength (:29-82) can be driven one evaluation at a time for
// per-evaluation parity; the same file also provides runAdaptiveGlobalPlacement.
// The flattened design and option structs are the ones the product exposes in
// include/mpgp.h, so both sides read identical inputs.
#include "AdaptiveGlobalPlacer.cpp"

#include "mpgp.h"
#include "myplacement/io/BookshelfParser.hpp"
#include "myplacement/placement/DetailedPlacer.hpp"

#include <cstring>
#include <exception>
#include <random>
#include <string>

namespace {

using namespace myplacement;
using namespace myplacement::detail;

thread_local std::string g_ref_error;

int fail(const std::exception& error) {
    g_ref_error = error.what();
    return dynamic_cast<const std::invalid_argument*>(&error) != nullptr ? MPGP_ERR_INVALID_ARGUMENT
                                                                         : MPGP_ERR_RUNTIME;
}

PlacementDatabase buildDatabase(const mpgp_design* design) {
    PlacementDatabase database;
    for (int32_t index = 0; index < design->module_count; ++index) {
        Module module;
        module.name = "m" + std::to_string(index);
        module.width = design->module_width[index];
        module.height = design->module_height[index];
        module.center = {design->module_x[index], design->module_y[index]};
        module.orientation = design->module_orientation != nullptr
                                 ? static_cast<Orientation>(design->module_orientation[index])
                                 : Orientation::North;
        module.is_terminal = (design->module_flags[index] & MPGP_MODULE_TERMINAL) != 0;
        module.is_fixed = (design->module_flags[index] & MPGP_MODULE_FIXED) != 0;
        database.addModule(std::move(module));
    }
    for (int32_t net_index = 0; net_index < design->net_count; ++net_index) {
        Net net;
        net.name = "n" + std::to_string(net_index);
        net.weight = design->net_weight[net_index];
        const NetId id = database.addNet(std::move(net));
        for (int64_t pin = design->net_pin_start[net_index]; pin < design->net_pin_start[net_index + 1]; ++pin) {
            Pin value;
            value.module = static_cast<ModuleId>(design->pin_module[pin]);
            value.net = id;
            value.offset = {design->pin_offset_x[pin], design->pin_offset_y[pin]};
            database.addPin(value);
        }
    }
    for (int32_t index = 0; index < design->row_count; ++index) {
        SiteRow row;
        row.bottom = design->row_bottom[index];
        row.height = design->row_height[index];
        row.site_width = design->row_site_width[index];
        row.site_spacing = design->row_site_spacing[index];
        row.x_start = design->row_x_start[index];
        row.site_count = static_cast<std::size_t>(design->row_site_count[index]);
        database.rows.push_back(row);
    }
    database.refreshDerivedData();
    return database;
}

GlobalPlacementOptions buildOptions(const mpgp_options* flat) {
    GlobalPlacementOptions options;
    options.iterations = flat->iterations;
    options.bins_x = flat->bins_x;
    options.bins_y = flat->bins_y;
    options.report_interval = flat->report_interval;
    options.target_density = flat->target_density;
    options.maximum_bin_overflow = flat->maximum_bin_overflow;
    options.initial_smoothing = flat->initial_smoothing;
    options.final_smoothing = flat->final_smoothing;
    options.maximum_movement_in_bins = flat->maximum_movement_in_bins;
    options.penalty_growth = flat->penalty_growth;
    options.optimizer = flat->optimizer == 0 ? GlobalOptimizer::Legacy : GlobalOptimizer::Adaptive;
    options.maximum_backtracks = flat->maximum_backtracks;
    options.backtracking_ratio = flat->backtracking_ratio;
    options.armijo_coefficient = flat->armijo_coefficient;
    options.maximum_momentum = flat->maximum_momentum;
    options.initial_movement_in_bins = flat->initial_movement_in_bins;
    options.objective_increase_for_density = flat->objective_increase_for_density;
    options.hpwl_growth_restart_threshold = flat->hpwl_growth_restart_threshold;
    options.density_stall_threshold = flat->density_stall_threshold;
    options.density_penalty_increase = flat->density_penalty_increase;
    options.density_penalty_decrease = flat->density_penalty_decrease;
    options.minimum_density_penalty = flat->minimum_density_penalty;
    options.maximum_density_penalty = flat->maximum_density_penalty;
    options.smoothing_overflow_exponent = flat->smoothing_overflow_exponent;
    options.feasible_refinement_iterations = flat->feasible_refinement_iterations;
    options.maximum_fillers = static_cast<std::size_t>(flat->maximum_fillers);
    options.seed = flat->seed;
    options.rudy_options.columns = flat->rudy_columns;
    options.rudy_options.rows = flat->rudy_rows;
    options.rudy_options.minimum_span_in_bins = flat->rudy_minimum_span_in_bins;
    options.rudy_options.capacity_factor = flat->rudy_capacity_factor;
    options.rudy_options.softplus_temperature = flat->rudy_softplus_temperature;
    options.rudy_options.penalty_model = static_cast<RudyPenaltyModel>(flat->rudy_penalty_model);
    options.rudy_validation_bins = flat->rudy_validation_bins;
    options.rudy_validation_capacity_factor = flat->rudy_validation_capacity_factor;
    options.routability_start_overflow = flat->routability_start_overflow;
    options.routability_weight_scale = flat->routability_weight_scale;
    options.routability_ramp_iterations = flat->routability_ramp_iterations;
    options.density_field_boundary =
        flat->density_field_boundary == 0 ? DensityFieldBoundary::Periodic : DensityFieldBoundary::Neumann;
    options.compute_backend = static_cast<ComputeBackend>(flat->compute_backend);
    options.cuda_device = flat->cuda_device;
    options.maximum_cuda_memory_bytes = static_cast<std::size_t>(flat->maximum_cuda_memory_bytes);
    return options;
}

void copyMetrics(const DensityMetrics& in, mpgp_density_metrics* out) {
    out->total_overflow_area = in.total_overflow_area;
    out->normalized_overflow = in.normalized_overflow;
    out->maximum_density = in.maximum_density;
    out->average_density = in.average_density;
    out->total_charge_area = in.total_charge_area;
    out->normalization_area = in.normalization_area;
    out->placeable_area = in.placeable_area;
    out->dark_area = in.dark_area;
}

struct RefBook {
    PlacementDatabase database;
};

struct RefSession {
    PlacementDatabase database;
    GlobalPlacementOptions options;
    std::vector<DensityFiller> fillers;
    std::unique_ptr<GlobalPlacementSession> session;
};

}  // namespace

extern "C" {

const char* ref_last_error(void) { return g_ref_error.c_str(); }

// Flat view of the reference's randomPlacement (InitialPlacer.cpp:102-121).
// InitialPlacer.cpp needs Eigen, which is absent, so this oracle restates the
// function: mt19937_64(seed) and one uniform_real_distribution draw per axis.
int ref_random_placement(const mpgp_design* design, uint64_t seed, double* module_x, double* module_y) {
    try {
        PlacementDatabase database = buildDatabase(design);
        std::mt19937_64 generator(seed);
        for (const ModuleId id : database.movableModules()) {
            Module& module = database.modules[id];
            const double min_x = database.core_region.ll.x + module.width * 0.5;
            const double max_x = database.core_region.ur.x - module.width * 0.5;
            const double min_y = database.core_region.ll.y + module.height * 0.5;
            const double max_y = database.core_region.ur.y - module.height * 0.5;
            if (min_x <= max_x) {
                std::uniform_real_distribution<double> distribution(min_x, max_x);
                module.center.x = distribution(generator);
            }
            if (min_y <= max_y) {
                std::uniform_real_distribution<double> distribution(min_y, max_y);
                module.center.y = distribution(generator);
            }
            database.clampModuleToCore(id);
        }
        for (std::size_t index = 0; index < database.modules.size(); ++index) {
            module_x[index] = database.modules[index].center.x;
            module_y[index] = database.modules[index].center.y;
        }
        return MPGP_OK;
    } catch (const std::exception& error) {
        return fail(error);
    }
}

// GlobalPlacer::run (GlobalPlacer.cpp:134-146) on the flattened design.
int ref_global_place(const mpgp_design* design, const mpgp_options* flat_options, double* module_x,
                     double* module_y, mpgp_result* result, mpgp_history_row* history, int32_t history_capacity) {
    try {
        PlacementDatabase database = buildDatabase(design);
        const GlobalPlacementOptions options = buildOptions(flat_options);
        const GlobalPlacementResult run = GlobalPlacer().run(database, options);
        for (std::size_t index = 0; index < database.modules.size(); ++index) {
            module_x[index] = database.modules[index].center.x;
            module_y[index] = database.modules[index].center.y;
        }
        std::memset(result, 0, sizeof(*result));
        result->hpwl_before = run.hpwl_before;
        result->hpwl_after = run.hpwl_after;
        result->overflow_before = run.overflow_before;
        result->overflow_after = run.overflow_after;
        result->completed_iterations = run.completed_iterations;
        result->accepted_iterations = run.accepted_iterations;
        result->momentum_restarts = run.momentum_restarts;
        result->rejected_candidates = run.rejected_candidates;
        result->best_checkpoint_iteration = run.best_checkpoint_iteration;
        result->restored_best_checkpoint = run.restored_best_checkpoint ? 1 : 0;
        result->best_checkpoint_hpwl = run.best_checkpoint_hpwl;
        result->best_checkpoint_overflow = run.best_checkpoint_overflow;
        result->elapsed_seconds = run.elapsed_seconds;
        result->compute_backend_used = static_cast<int32_t>(run.compute_backend_used);
        result->cuda_device_used = run.cuda_device_used;
        result->cuda_reserved_memory_bytes = run.cuda_reserved_memory_bytes;
        result->history_count = static_cast<int32_t>(run.history.size());
        result->rudy_energy_after = run.rudy_energy_after;
        result->rudy_horizontal_capacity = run.rudy_metrics.horizontal_capacity;
        result->rudy_vertical_capacity = run.rudy_metrics.vertical_capacity;
        result->rudy_proxy_overflow_after = run.rudy_metrics.proxy_overflow;
        result->rudy_maximum_utilization_after = run.rudy_metrics.maximum_utilization;
        result->rudy_p95_utilization_after = run.rudy_metrics.p95_utilization;
        result->rudy_validation_energy_after = run.rudy_validation_energy_after;
        result->rudy_validation_proxy_overflow_after = run.rudy_validation_metrics.proxy_overflow;
        result->rudy_validation_maximum_utilization_after = run.rudy_validation_metrics.maximum_utilization;
        result->rudy_validation_p95_utilization_after = run.rudy_validation_metrics.p95_utilization;
        const std::size_t rows = std::min<std::size_t>(run.history.size(), static_cast<std::size_t>(
                                                                               std::max(0, history_capacity)));
        for (std::size_t index = 0; index < rows; ++index) {
            const GlobalPlacementIteration& row = run.history[index];
            mpgp_history_row& out = history[index];
            out.iteration = row.iteration;
            out.backtracks = row.backtracks;
            out.hpwl = row.hpwl;
            out.overflow = row.overflow;
            out.design_overflow = row.design_overflow;
            out.smooth_wirelength = row.smooth_wirelength;
            out.density_energy = row.density_energy;
            out.objective = row.objective;
            out.penalty = row.penalty;
            out.smoothing = row.smoothing;
            out.step_size = row.step_size;
            out.maximum_displacement = row.maximum_displacement;
            out.gradient_norm = row.gradient_norm;
            out.curvature = row.curvature;
            out.rudy_energy = row.rudy_energy;
            out.rudy_proxy_overflow = row.rudy_proxy_overflow;
            out.rudy_maximum_utilization = row.rudy_maximum_utilization;
            out.rudy_weight = row.rudy_weight;
            out.momentum_restarted = row.momentum_restarted ? 1 : 0;
            out.accepted = row.accepted ? 1 : 0;
            out.best_checkpoint = row.best_checkpoint ? 1 : 0;
            out.rudy_active = row.rudy_active ? 1 : 0;
        }
        return MPGP_OK;
    } catch (const std::exception& error) {
        return fail(error);
    }
}

// A GlobalPlacementSession (AdaptiveGlobalPlacer.cpp:114-126) on the CPU path.
int ref_session_create(const mpgp_design* design, const mpgp_options* flat_options, void** out) {
    try {
        auto state = std::make_unique<RefSession>();
        state->database = buildDatabase(design);
        state->options = buildOptions(flat_options);
        state->options.compute_backend = ComputeBackend::Cpu;
        validateAdaptiveOptions(state->database, state->options);
        {
            DensityMap static_map(state->database.core_region, state->options.bins_x, state->options.bins_y,
                                  state->options.target_density);
            initializeStaticDensity(static_map, state->database);
            state->fillers = createDensityFillers(state->database, static_map, state->options);
        }
        state->session = std::make_unique<GlobalPlacementSession>(state->database, state->options);
        *out = state.release();
        return MPGP_OK;
    } catch (const std::exception& error) {
        return fail(error);
    }
}

void ref_session_destroy(void* handle) { delete static_cast<RefSession*>(handle); }

int ref_session_counts(void* handle, int64_t* particles, int64_t* movable, int64_t* fillers) {
    auto* state = static_cast<RefSession*>(handle);
    *particles = static_cast<int64_t>(state->session->particleCount());
    *movable = static_cast<int64_t>(state->database.movableModules().size());
    *fillers = static_cast<int64_t>(state->fillers.size());
    return MPGP_OK;
}

// Particle geometry in session order (movable modules, then fillers).
int ref_session_particles(void* handle, double* x, double* y, double* width, double* height, int32_t* layer,
                          int32_t* pin_count) {
    auto* state = static_cast<RefSession*>(handle);
    const std::vector<Vec2> positions = state->session->capturePositions();
    const auto& movable = state->database.movableModules();
    for (std::size_t index = 0; index < positions.size(); ++index) {
        x[index] = positions[index].x;
        y[index] = positions[index].y;
        if (index < movable.size()) {
            const Module& module = state->database.modules[movable[index]];
            width[index] = module.width;
            height[index] = module.height;
            layer[index] = module.is_macro ? MPGP_LAYER_MACRO : MPGP_LAYER_STANDARD;
            pin_count[index] = static_cast<int32_t>(module.pins.size());
        } else {
            const DensityFiller& filler = state->fillers[index - movable.size()];
            width[index] = filler.width;
            height[index] = filler.height;
            layer[index] = MPGP_LAYER_FILLER;
            pin_count[index] = 0;
        }
    }
    return MPGP_OK;
}

// Static layers exactly as initializeStaticDensity builds them (GlobalPlacementSupport.cpp:21-30).
int ref_session_static_density(void* handle, double* fixed, double* dark) {
    auto* state = static_cast<RefSession*>(handle);
    DensityMap map(state->database.core_region, state->options.bins_x, state->options.bins_y,
                   state->options.target_density);
    initializeStaticDensity(map, state->database);
    for (std::size_t index = 0; index < map.bins().size(); ++index) {
        fixed[index] = map.bins()[index].fixed_area;
        dark[index] = map.bins()[index].dark_area;
    }
    return MPGP_OK;
}

// scalars (19 doubles): hpwl, smooth_wirelength, density_energy, objective,
// wire_gradient_l1, density_gradient_l1, raw_gradient_norm, preconditioned_gradient_norm,
// optimizer metrics (8)... design metrics are returned through `design`.
// GlobalPlacementSession::evaluate (AdaptiveGlobalPlacer.cpp:200-268).
int ref_session_evaluate(void* handle, const double* positions, double smoothing, double penalty,
                         double reference_penalty, int calculate_gradient, double* scalars,
                         mpgp_density_metrics* optimizer, mpgp_density_metrics* design, double* raw_gradient,
                         double* preconditioned_gradient) {
    try {
        auto* state = static_cast<RefSession*>(handle);
        const std::size_t count = state->session->particleCount();
        std::vector<Vec2> applied(count);
        for (std::size_t index = 0; index < count; ++index) applied[index] = {positions[2 * index], positions[2 * index + 1]};
        state->session->applyPositions(applied);
        const StateEvaluation evaluation =
            state->session->evaluate(smoothing, penalty, reference_penalty, calculate_gradient != 0);
        scalars[0] = evaluation.metrics.hpwl;
        scalars[1] = evaluation.metrics.smooth_wirelength;
        scalars[2] = evaluation.metrics.density_energy;
        scalars[3] = evaluation.metrics.objective;
        scalars[4] = evaluation.wire_gradient_l1;
        scalars[5] = evaluation.density_gradient_l1;
        scalars[6] = evaluation.raw_gradient_norm;
        scalars[7] = evaluation.preconditioned_gradient_norm;
        copyMetrics(evaluation.metrics.optimizer_density, optimizer);
        copyMetrics(evaluation.metrics.design_density, design);
        if (calculate_gradient != 0) {
            for (std::size_t index = 0; index < count; ++index) {
                raw_gradient[2 * index] = evaluation.raw_gradient[index].x;
                raw_gradient[2 * index + 1] = evaluation.raw_gradient[index].y;
                preconditioned_gradient[2 * index] = evaluation.preconditioned_gradient[index].x;
                preconditioned_gradient[2 * index + 1] = evaluation.preconditioned_gradient[index].y;
            }
        }
        return MPGP_OK;
    } catch (const std::exception& error) {
        return fail(error);
    }
}

// The wire and density parts of one CPU evaluation kept apart, in particle order:
// evaluateSmoothWirelength (AdaptiveGlobalPlacer.cpp:29-82) and the density
// path of GlobalPlacementSession::evaluateDensity (:333-356) with the sampled
// force -charge * E (:236-253).  Layers are returned per bin (any pointer may be NULL).
int ref_session_components(void* handle, const double* positions, double smoothing, double* wire_scalars,
                           double* wire_gradient, double* density_gradient, double* energy, double* movable,
                           double* macro, double* filler, double* potential, double* field_x, double* field_y) {
    try {
        auto* state = static_cast<RefSession*>(handle);
        const std::size_t count = state->session->particleCount();
        std::vector<Vec2> applied(count);
        for (std::size_t index = 0; index < count; ++index) applied[index] = {positions[2 * index], positions[2 * index + 1]};
        state->session->applyPositions(applied);
        const std::vector<Vec2> clamped = state->session->capturePositions();
        const auto& movable_ids = state->database.movableModules();
        for (std::size_t index = movable_ids.size(); index < count; ++index) {
            state->fillers[index - movable_ids.size()].center = clamped[index];
        }

        const SmoothWirelengthEvaluation wire = evaluateSmoothWirelength(state->database, smoothing, true);
        wire_scalars[0] = wire.smooth_wirelength;
        wire_scalars[1] = wire.hpwl;
        for (std::size_t index = 0; index < count; ++index) {
            const Vec2 value = index < movable_ids.size() ? wire.gradient[movable_ids[index]] : Vec2{};
            wire_gradient[2 * index] = value.x;
            wire_gradient[2 * index + 1] = value.y;
        }

        const GlobalPlacementOptions& options = state->options;
        DensityMap map(state->database.core_region, options.bins_x, options.bins_y, options.target_density);
        initializeStaticDensity(map, state->database);
        depositDynamicDensity(map, state->database, state->fillers);
        std::vector<double> deviation;
        buildDensityDeviation(map, deviation);
        ElectrostaticField field(options.bins_x, options.bins_y, state->database.core_region,
                                 DensityFieldBoundary::Neumann);
        field.solve(deviation);
        const double mean = std::accumulate(deviation.begin(), deviation.end(), 0.0) /
                            static_cast<double>(std::max<std::size_t>(1U, deviation.size()));
        double electrostatic = 0.0;
        for (std::size_t index = 0; index < map.bins().size(); ++index) {
            const int column = static_cast<int>(index % static_cast<std::size_t>(map.columns()));
            const int row = static_cast<int>(index / static_cast<std::size_t>(map.columns()));
            electrostatic += 0.5 * (deviation[index] - mean) * field.potentialAt(column, row) *
                             map.bins()[index].region.area();
            if (movable != nullptr) movable[index] = map.bins()[index].movable_area;
            if (macro != nullptr) macro[index] = map.bins()[index].macro_area;
            if (filler != nullptr) filler[index] = map.bins()[index].filler_area;
            if (potential != nullptr) potential[index] = field.potentialAt(column, row);
            if (field_x != nullptr) field_x[index] = field.fieldAt(column, row).x;
            if (field_y != nullptr) field_y[index] = field.fieldAt(column, row).y;
        }
        *energy = std::max(0.0, electrostatic);
        for (std::size_t index = 0; index < count; ++index) {
            double charge = 0.0;
            if (index < movable_ids.size()) {
                charge = densityChargeArea(state->database.modules[movable_ids[index]], options.target_density);
            } else {
                charge = densityChargeArea(state->fillers[index - movable_ids.size()], options.target_density);
            }
            const Vec2 value = field.sampleField(clamped[index]) * (-charge);
            density_gradient[2 * index] = value.x;
            density_gradient[2 * index + 1] = value.y;
        }
        return MPGP_OK;
    } catch (const std::exception& error) {
        return fail(error);
    }
}

// evaluateRudy (Rudy.cpp:227-456) of the session's design at `positions` (applied
// with the session's clamping), with the given grid, model and capacities.
// metrics (10): horizontal/vertical total, horizontal/vertical mean, horizontal/
// vertical capacity, proxy overflow, maximum and p95 utilisation, energy.  The
// gradient is returned in particle order (zero for fillers).
int ref_session_rudy(void* handle, const double* positions, int32_t columns, int32_t rows, double minimum_span,
                     int32_t model, double temperature, double capacity_h, double capacity_v,
                     int calculate_gradient, double* metrics, double* gradient) {
    try {
        auto* state = static_cast<RefSession*>(handle);
        const std::size_t count = state->session->particleCount();
        std::vector<Vec2> applied(count);
        for (std::size_t index = 0; index < count; ++index) applied[index] = {positions[2 * index], positions[2 * index + 1]};
        state->session->applyPositions(applied);
        RudyOptions options = state->options.rudy_options;
        options.columns = columns;
        options.rows = rows;
        options.minimum_span_in_bins = minimum_span;
        options.penalty_model = static_cast<RudyPenaltyModel>(model);
        options.softplus_temperature = temperature;
        const RudyEvaluation r =
            evaluateRudy(state->database, options, RudyCapacity{capacity_h, capacity_v}, calculate_gradient != 0);
        const double values[10] = {r.metrics.horizontal_total_demand, r.metrics.vertical_total_demand,
                                   r.metrics.horizontal_mean_demand,  r.metrics.vertical_mean_demand,
                                   r.metrics.horizontal_capacity,     r.metrics.vertical_capacity,
                                   r.metrics.proxy_overflow,          r.metrics.maximum_utilization,
                                   r.metrics.p95_utilization,         r.energy};
        std::copy(values, values + 10, metrics);
        if (calculate_gradient != 0 && gradient != nullptr) {
            const auto& movable_ids = state->database.movableModules();
            for (std::size_t index = 0; index < count; ++index) {
                const Vec2 value = index < movable_ids.size() && !r.gradient.empty() ? r.gradient[movable_ids[index]]
                                                                                    : Vec2{};
                gradient[2 * index] = value.x;
                gradient[2 * index + 1] = value.y;
            }
        }
        return MPGP_OK;
    } catch (const std::exception& error) {
        return fail(error);
    }
}

// ElectrostaticField::solve + fieldAt/potentialAt (ElectrostaticField.cpp:119-133, 150-162).
int ref_field_solve(int32_t columns, int32_t rows, double llx, double lly, double urx, double ury,
                    const double* deviation, double* potential, double* field_x, double* field_y) {
    try {
        ElectrostaticField field(columns, rows, Rect{{llx, lly}, {urx, ury}}, DensityFieldBoundary::Neumann);
        const std::size_t count = static_cast<std::size_t>(columns) * static_cast<std::size_t>(rows);
        field.solve(std::vector<double>(deviation, deviation + count));
        for (int32_t row = 0; row < rows; ++row) {
            for (int32_t column = 0; column < columns; ++column) {
                const std::size_t index = static_cast<std::size_t>(row) * columns + column;
                potential[index] = field.potentialAt(column, row);
                field_x[index] = field.fieldAt(column, row).x;
                field_y[index] = field.fieldAt(column, row).y;
            }
        }
        return MPGP_OK;
    } catch (const std::exception& error) {
        return fail(error);
    }
}

// ElectrostaticField::sampleField after solve (ElectrostaticField.cpp:135-141, 301-320).
int ref_field_sample(int32_t columns, int32_t rows, double llx, double lly, double urx, double ury,
                     const double* deviation, int64_t point_count, const double* points, double* sampled) {
    try {
        ElectrostaticField field(columns, rows, Rect{{llx, lly}, {urx, ury}}, DensityFieldBoundary::Neumann);
        const std::size_t count = static_cast<std::size_t>(columns) * static_cast<std::size_t>(rows);
        field.solve(std::vector<double>(deviation, deviation + count));
        for (int64_t index = 0; index < point_count; ++index) {
            const Vec2 value = field.sampleField({points[2 * index], points[2 * index + 1]});
            sampled[2 * index] = value.x;
            sampled[2 * index + 1] = value.y;
        }
        return MPGP_OK;
    } catch (const std::exception& error) {
        return fail(error);
    }
}

// A DensityMap built from explicit rectangles (Metrics.cpp:1-119): the
// DensityModelTests case and the scatter edge cases.  rects are
// (llx, lly, urx, ury) quadruples; layer codes follow DensityLayer
// (0 Fixed, 1 Movable, 2 Macro, 3 Filler, 4 Dark).  bins receives 5 doubles per
// bin (fixed, movable, macro, filler, dark); metrics receives with-filler then
// without-filler DensityMetrics.
int ref_density_map(double llx, double lly, double urx, double ury, int32_t columns, int32_t rows,
                    double target_density, int32_t region_count, const double* regions, int32_t rect_count,
                    const double* rects, const int32_t* layers, double* bins, mpgp_density_metrics* metrics) {
    try {
        DensityMap map(Rect{{llx, lly}, {urx, ury}}, columns, rows, target_density);
        if (region_count > 0) {
            std::vector<Rect> placeable;
            for (int32_t index = 0; index < region_count; ++index) {
                placeable.push_back({{regions[4 * index], regions[4 * index + 1]},
                                     {regions[4 * index + 2], regions[4 * index + 3]}});
            }
            map.setPlaceableRegions(placeable);
        }
        for (int32_t index = 0; index < rect_count; ++index) {
            map.addRectangle({{rects[4 * index], rects[4 * index + 1]}, {rects[4 * index + 2], rects[4 * index + 3]}},
                             static_cast<DensityLayer>(layers[index]));
        }
        for (std::size_t index = 0; index < map.bins().size(); ++index) {
            const DensityBin& bin = map.bins()[index];
            bins[5 * index + 0] = bin.fixed_area;
            bins[5 * index + 1] = bin.movable_area;
            bins[5 * index + 2] = bin.macro_area;
            bins[5 * index + 3] = bin.filler_area;
            bins[5 * index + 4] = bin.dark_area;
        }
        copyMetrics(map.metrics(true), &metrics[0]);
        copyMetrics(map.metrics(false), &metrics[1]);
        return MPGP_OK;
    } catch (const std::exception& error) {
        return fail(error);
    }
}

// calculateHpwl / calculateDensity (Metrics.cpp:128-164) on a flattened design.
int ref_design_metrics(const mpgp_design* design, int32_t columns, int32_t rows, double target_density,
                       double* hpwl, mpgp_density_metrics* density) {
    try {
        const PlacementDatabase database = buildDatabase(design);
        *hpwl = calculateHpwl(database).hpwl;
        copyMetrics(calculateDensity(database, columns, rows, target_density), density);
        return MPGP_OK;
    } catch (const std::exception& error) {
        return fail(error);
    }
}

// BookshelfParser::parseAux (src/io/BookshelfParser.cpp:313-348) through the
// reader linked into this library: the reference's own in libref_cpu.so, the
// adapter over libmpgp.so's reader in libref_dropin.so.  ParseError returns
// MPGP_ERR_PARSE.
int ref_bookshelf_read(const char* aux_path, void** out) {
    *out = nullptr;
    try {
        auto book = std::make_unique<RefBook>();
        book->database = BookshelfParser().parseAux(aux_path);
        *out = book.release();
        return MPGP_OK;
    } catch (const ParseError& error) {
        g_ref_error = error.what();
        return MPGP_ERR_PARSE;
    } catch (const std::exception& error) {
        return fail(error);
    }
}

void ref_bookshelf_destroy(void* handle) { delete static_cast<RefBook*>(handle); }

// counts: modules, nets, pins, rows, movable modules; declared: NumNodes,
// NumTerminals, NumNets, NumPins (-1 when absent); regions: core (ll, ur),
// chip (ll, ur), nominal row height.
int ref_bookshelf_counts(void* handle, int64_t* counts, int64_t* declared, double* regions) {
    const PlacementDatabase& d = static_cast<RefBook*>(handle)->database;
    counts[0] = static_cast<int64_t>(d.modules.size());
    counts[1] = static_cast<int64_t>(d.nets.size());
    counts[2] = static_cast<int64_t>(d.pins.size());
    counts[3] = static_cast<int64_t>(d.rows.size());
    counts[4] = static_cast<int64_t>(d.movableModules().size());
    const std::optional<std::size_t>* values[4] = {&d.declared_nodes, &d.declared_terminals, &d.declared_nets,
                                                   &d.declared_pins};
    for (int k = 0; k < 4; ++k) declared[k] = *values[k] ? static_cast<int64_t>(**values[k]) : -1;
    const double r[9] = {d.core_region.ll.x, d.core_region.ll.y, d.core_region.ur.x, d.core_region.ur.y,
                         d.chip_region.ll.x, d.chip_region.ll.y, d.chip_region.ur.x, d.chip_region.ur.y,
                         d.nominalRowHeight()};
    std::memcpy(regions, r, sizeof(r));
    return MPGP_OK;
}

// flags: bit 0 terminal, bit 1 fixed, bit 2 macro.  pin_start / pins: each
// module's pin list (Module::pins).
int ref_bookshelf_modules(void* handle, double* width, double* height, double* x, double* y, int32_t* flags,
                          int32_t* orientation, int64_t* pin_start, int64_t* pins) {
    const PlacementDatabase& d = static_cast<RefBook*>(handle)->database;
    pin_start[0] = 0;
    for (std::size_t m = 0; m < d.modules.size(); ++m) {
        const Module& module = d.modules[m];
        width[m] = module.width;
        height[m] = module.height;
        x[m] = module.center.x;
        y[m] = module.center.y;
        flags[m] = (module.is_terminal ? 1 : 0) | (module.is_fixed ? 2 : 0) | (module.is_macro ? 4 : 0);
        orientation[m] = static_cast<int32_t>(module.orientation);
        pin_start[m + 1] = pin_start[m] + static_cast<int64_t>(module.pins.size());
        for (std::size_t k = 0; k < module.pins.size(); ++k) pins[pin_start[m] + k] = static_cast<int64_t>(module.pins[k]);
    }
    return MPGP_OK;
}

// Nets with their pin lists (Net::pins), and the pins in PlacementDatabase order.
int ref_bookshelf_nets(void* handle, double* weight, int64_t* net_pin_start, int64_t* net_pins, int32_t* pin_module,
                       int64_t* pin_net, double* offset_x, double* offset_y, int32_t* direction) {
    const PlacementDatabase& d = static_cast<RefBook*>(handle)->database;
    net_pin_start[0] = 0;
    for (std::size_t n = 0; n < d.nets.size(); ++n) {
        weight[n] = d.nets[n].weight;
        net_pin_start[n + 1] = net_pin_start[n] + static_cast<int64_t>(d.nets[n].pins.size());
        for (std::size_t k = 0; k < d.nets[n].pins.size(); ++k) {
            net_pins[net_pin_start[n] + k] = static_cast<int64_t>(d.nets[n].pins[k]);
        }
    }
    for (std::size_t p = 0; p < d.pins.size(); ++p) {
        pin_module[p] = static_cast<int32_t>(d.pins[p].module);
        pin_net[p] = static_cast<int64_t>(d.pins[p].net);
        offset_x[p] = d.pins[p].offset.x;
        offset_y[p] = d.pins[p].offset.y;
        direction[p] = static_cast<int32_t>(d.pins[p].direction);
    }
    return MPGP_OK;
}

int ref_bookshelf_rows(void* handle, double* bottom, double* height, double* site_width, double* site_spacing,
                       double* x_start, int64_t* site_count, int32_t* orientation) {
    const PlacementDatabase& d = static_cast<RefBook*>(handle)->database;
    for (std::size_t r = 0; r < d.rows.size(); ++r) {
        bottom[r] = d.rows[r].bottom;
        height[r] = d.rows[r].height;
        site_width[r] = d.rows[r].site_width;
        site_spacing[r] = d.rows[r].site_spacing;
        x_start[r] = d.rows[r].x_start;
        site_count[r] = static_cast<int64_t>(d.rows[r].site_count);
        orientation[r] = static_cast<int32_t>(d.rows[r].orientation);
    }
    return MPGP_OK;
}

// A name's bytes and length (names may hold any byte but blanks, NUL included).
const char* ref_bookshelf_module_name(void* handle, int64_t module, int64_t* length) {
    const std::string& name = static_cast<RefBook*>(handle)->database.modules[static_cast<std::size_t>(module)].name;
    *length = static_cast<int64_t>(name.size());
    return name.data();
}

const char* ref_bookshelf_net_name(void* handle, int64_t net, int64_t* length) {
    const std::string& name = static_cast<RefBook*>(handle)->database.nets[static_cast<std::size_t>(net)].name;
    *length = static_cast<int64_t>(name.size());
    return name.data();
}

// DetailedPlacer::run (src/placement/DetailedPlacer.cpp:262-338) on a flattened
// design with the rows' orientations (NULL: N) and `backend` (0 cpu, 1 cuda,
// 2 auto): the reference's CPU placer, or its CUDA backend in libref_cuda.so, or
// the engine's in libref_dropin.so.  Writes the centres and orientations.
int ref_detailed_place(const mpgp_design* design, const int32_t* row_orientation, const mpgp_detailed_options* flat,
                       int32_t backend, double* x, double* y, int32_t* orientation, mpgp_detailed_result* out) {
    try {
        PlacementDatabase database = buildDatabase(design);
        if (row_orientation != nullptr) {
            for (std::size_t r = 0; r < database.rows.size(); ++r) {
                database.rows[r].orientation = static_cast<Orientation>(row_orientation[r]);
            }
        }
        DetailedPlacementOptions options;
        options.method = static_cast<DetailedPlacementMethod>(flat->method);
        options.passes = flat->passes;
        options.window_size = flat->window_size;
        options.maximum_net_degree = static_cast<std::size_t>(flat->maximum_net_degree);
        options.improvement_epsilon = flat->improvement_epsilon;
        options.compute_backend = static_cast<DetailedPlacementBackend>(backend);
        options.cuda_device = flat->cuda_device;
        options.maximum_cuda_memory_bytes = static_cast<std::size_t>(flat->maximum_cuda_memory_bytes);
        const DetailedPlacementResult result = DetailedPlacer().run(database, options);
        for (std::size_t m = 0; m < database.modules.size(); ++m) {
            x[m] = database.modules[m].center.x;
            y[m] = database.modules[m].center.y;
            orientation[m] = static_cast<int32_t>(database.modules[m].orientation);
        }
        out->hpwl_before = result.hpwl_before;
        out->hpwl_after = result.hpwl_after;
        out->elapsed_seconds = result.elapsed_seconds;
        out->evaluated_windows = result.evaluated_windows;
        out->evaluated_permutations = result.evaluated_permutations;
        out->accepted_operations = result.accepted_operations;
        out->completed_passes = result.completed_passes;
        out->cuda_device_used = result.cuda_device_used;
        out->cuda_reserved_memory_bytes = result.cuda_reserved_memory_bytes;
        return static_cast<int>(result.compute_backend_used) == 1 ? 1 : 0;  // >= 0: the backend used
    } catch (const std::exception& error) {
        g_ref_error = error.what();
        return -(dynamic_cast<const std::invalid_argument*>(&error) != nullptr ? MPGP_ERR_INVALID_ARGUMENT
                                                                              : MPGP_ERR_RUNTIME);
    }
}

}  // extern "C"
