// The adaptive controller of runAdaptiveGlobalPlacement (AdaptiveGlobalPlacer.cpp:
// 652-953) with its vectors resident on the device.
//
// The control law -- smoothing from overflow, the curvature step estimate, the
// Armijo / stable-objective / density-trade acceptance, backtracking, Nesterov
// lookahead with restart, the density-penalty update, best-feasible
// checkpointing and the early stop -- is kept decision for decision and runs
// on the host from about twenty FP64 scalars per evaluation.  Every O(P)
// vector operation of the reference host loops (capturePositions /
// applyPositions, proposeStep, estimateStep, momentumAlignment, the velocity
// and lookahead updates, the gradient combine and preconditioning) is fused
// into the engine's kernels, so positions never leave the device until the
// run finishes.
#include "session.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>
#include <thread>

#include "common.cuh"

namespace mpgp {
namespace {

double clampValue(double value, double lower, double upper) { return std::max(lower, std::min(value, upper)); }

// acceptsCandidate (AdaptiveGlobalPlacer.cpp:521-534).
bool acceptsCandidate(const ObjectiveMetrics& base, const ObjectiveMetrics& candidate, double predicted_reduction,
                      const mpgp_options& o) {
    const double objective_tolerance = std::max(1e-8, std::abs(base.objective) * 1e-10);
    const double armijo_target = base.objective - o.armijo_coefficient * std::max(0.0, predicted_reduction);
    const bool armijo = candidate.objective <= armijo_target + objective_tolerance;
    const bool stable_objective = candidate.objective <= base.objective + objective_tolerance &&
                                  candidate.optimizer.normalized_overflow <= base.optimizer.normalized_overflow * 1.005;
    const double meaningful_density_gain = std::max(1e-4, o.density_stall_threshold * 0.25);
    const bool density_trade =
        candidate.optimizer.normalized_overflow <= base.optimizer.normalized_overflow - meaningful_density_gain &&
        candidate.objective <= base.objective * (1.0 + o.objective_increase_for_density);
    return armijo || stable_objective || density_trade;
}

// updateDensityPenalty (AdaptiveGlobalPlacer.cpp:536-557).
double updateDensityPenalty(double penalty, double reference_penalty, const ObjectiveMetrics& before,
                            const ObjectiveMetrics& after, const mpgp_options& o) {
    const double hpwl_growth = (after.hpwl - before.hpwl) / std::max(before.hpwl, 1.0);
    const double density_improvement = before.optimizer.normalized_overflow - after.optimizer.normalized_overflow;
    const bool density_is_critical = after.optimizer.normalized_overflow > std::max(2.0 * o.maximum_bin_overflow, 0.02);
    if (density_is_critical && density_improvement < o.density_stall_threshold) {
        penalty *= o.density_penalty_increase;
    } else if (!density_is_critical && hpwl_growth > o.hpwl_growth_restart_threshold &&
               density_improvement < o.density_stall_threshold) {
        penalty *= o.density_penalty_decrease;
    } else if (after.optimizer.normalized_overflow > o.maximum_bin_overflow &&
               density_improvement < o.density_stall_threshold) {
        penalty *= o.density_penalty_increase;
    } else if (after.design.normalized_overflow <= o.maximum_bin_overflow) {
        penalty *= o.density_penalty_decrease;
    }
    const double minimum_penalty = std::max(o.minimum_density_penalty, reference_penalty * 0.02);
    const double maximum_penalty = std::max(o.maximum_density_penalty, minimum_penalty * 10.0);
    return clampValue(penalty, minimum_penalty, maximum_penalty);
}

mpgp_history_row makeHistoryRow(int iteration, const ObjectiveMetrics& m, double penalty, double smoothing,
                                double step_size, double maximum_displacement, double gradient_norm, double curvature,
                                int backtracks, bool restarted, bool accepted, bool best_checkpoint, double rudy_weight,
                                bool rudy_active) {
    mpgp_history_row row{};
    row.iteration = iteration;
    row.hpwl = m.hpwl;
    row.overflow = m.optimizer.normalized_overflow;
    row.design_overflow = m.design.normalized_overflow;
    row.smooth_wirelength = m.smooth_wirelength;
    row.density_energy = m.density_energy;
    row.objective = m.objective;
    row.penalty = penalty;
    row.smoothing = smoothing;
    row.step_size = step_size;
    row.maximum_displacement = maximum_displacement;
    row.gradient_norm = gradient_norm;
    row.curvature = curvature;
    row.rudy_energy = m.rudy_energy;
    row.rudy_proxy_overflow = m.rudy_proxy_overflow;
    row.rudy_maximum_utilization = m.rudy_maximum_utilization;
    row.rudy_weight = rudy_weight;
    row.rudy_active = rudy_active ? 1 : 0;
    row.backtracks = backtracks;
    row.momentum_restarted = restarted ? 1 : 0;
    row.accepted = accepted ? 1 : 0;
    row.best_checkpoint = best_checkpoint ? 1 : 0;
    return row;
}

}  // namespace

Session::Session(const mpgp_design& design, const mpgp_options& options, Batch* batch) : options_(options) {
    started_ = std::chrono::steady_clock::now();
    validateDesign(design);
    {
        // validatePublicGlobalOptions + validateAdaptiveOptions.
        validateOptions(options_);
    }
    rudy_requested_ = options_.rudy_penalty_model != MPGP_RUDY_DISABLED;
    derived_ = deriveDesign(design);
    module_x_.assign(design.module_x, design.module_x + design.module_count);
    module_y_.assign(design.module_y, design.module_y + design.module_count);
    module_w_.assign(design.module_width, design.module_width + design.module_count);
    module_h_.assign(design.module_height, design.module_height + design.module_count);
    result_.compute_backend_used = MPGP_BACKEND_CUDA;
    if (derived_.movable.empty()) {  // AdaptiveGlobalPlacer.cpp:653
        empty_ = true;
        done_ = true;
        result_ = mpgp_result{};
        return;
    }
    // The host problem is built on two threads while this one sets up the engine's grid
    // part on the device (the field solve's bases and buffers need only the grid): the
    // pin and net arrays, whose device layout then starts at once, and the static
    // layers, fillers and particle arrays, which are uploaded last.
    std::exception_ptr pins_error, particles_error;
    std::thread pins_thread([&] {
        try {
            buildProblemPins(design, derived_, problem_);
        } catch (...) {
            pins_error = std::current_exception();
        }
    });
    std::thread particles_thread([&] {
        try {
            buildProblemParticles(design, derived_, options_, problem_, fillers_);
        } catch (...) {
            particles_error = std::current_exception();
        }
    });
    struct Join {
        std::thread& t;
        ~Join() {
            if (t.joinable()) t.join();
        }
    } join_pins{pins_thread}, join_particles{particles_thread};
    int device_count = 0;
    const cudaError_t count_status = cudaGetDeviceCount(&device_count);
    if (count_status != cudaSuccess || device_count <= 0) {
        fail(MPGP_ERR_UNAVAILABLE, std::string("CUDA device discovery failed: ") + cudaGetErrorString(count_status));
    }
    require(options_.cuda_device >= 0 && options_.cuda_device < device_count,
            "Requested CUDA device does not exist on this host.");
    const Engine::Grid grid{options_.bins_x, options_.bins_y, derived_.core, options_.target_density};
    engine_ = std::make_unique<Engine>(grid, options_.cuda_device, options_.maximum_cuda_memory_bytes,
                                       rudy_requested_ ? nullptr : batch);
    pins_thread.join();
    if (pins_error) std::rethrow_exception(pins_error);
    engine_->loadNets(problem_, static_cast<int64_t>(derived_.movable.size()));
    particles_thread.join();
    if (particles_error) std::rethrow_exception(particles_error);
    engine_->loadParticles(problem_);
    if (rudy_requested_) engine_->enableRudy(options_);
    result_.cuda_device_used = options_.cuda_device;

    const double bin_w = derived_.core.width() / static_cast<double>(options_.bins_x);
    const double bin_h = derived_.core.height() / static_cast<double>(options_.bins_y);
    min_bin_ = std::min(bin_w, bin_h);
    max_bin_ = std::max(bin_w, bin_h);

    // The controller's twelve particle vectors (positions, lookahead, candidate, previous,
    // velocity, the gradients and the two checkpoints), from one allocation.
    double2* vectors[12] = {};
    engine_->newParticleArrays(12, vectors, "controller vectors");
    cur_ = vectors[0];
    look_ = vectors[1];
    cand_ = vectors[2];
    prev_pos_ = vectors[3];
    velocity_ = vectors[4];
    raw_cur_ = vectors[5];
    pre_cur_ = vectors[6];
    raw_look_ = vectors[7];
    pre_look_ = vectors[8];
    prev_grad_ = vectors[9];
    best_feasible_.positions = vectors[10];
    best_fallback_.positions = vectors[11];
    result_.cuda_reserved_memory_bytes = engine_->reservedBytes();

    // capturePositions (AdaptiveGlobalPlacer.cpp:174-183): movable centres, then fillers.
    const std::size_t particles = static_cast<std::size_t>(engine_->particleCount());
    std::vector<double2> initial(particles);
    for (std::size_t i = 0; i < derived_.movable.size(); ++i) {
        initial[i] = make_double2(module_x_[derived_.movable[i]], module_y_[derived_.movable[i]]);
    }
    for (std::size_t i = 0; i < fillers_.size(); ++i) {
        initial[derived_.movable.size() + i] = make_double2(fillers_[i].x, fillers_[i].y);
    }
    checkCuda(cudaMemcpyAsync(cur_, initial.data(), particles * sizeof(double2), cudaMemcpyHostToDevice,
                              engine_->stream()),
              "Upload initial positions");
    engine_->addTransfer(particles * sizeof(double2), 0);

    // Initial evaluations and the penalty normalisation (AdaptiveGlobalPlacer.cpp:672-733).
    smoothing_ = options_.initial_smoothing * max_bin_;
    StateEval first = evaluateGiven(cur_, true, 1.0, raw_cur_, pre_cur_, false, false);
    result_.hpwl_before = first.m.hpwl;                             // calculateHpwl at the start
    result_.overflow_before = first.m.design.normalized_overflow;   // calculateDensity at the start
    initial_overflow_ = std::max(first.m.optimizer.normalized_overflow, kEpsilon);
    smoothing_ = smoothingFromOverflow(first.m.optimizer.normalized_overflow);
    const double raw_penalty = first.density_l1 > kEpsilon ? first.wire_l1 / first.density_l1 : 1.0;
    penalty_ = clampValue(raw_penalty, options_.minimum_density_penalty, options_.maximum_density_penalty);
    reference_penalty_ = penalty_;
    initial_ = evaluateGiven(cur_, true, penalty_, raw_cur_, pre_cur_, false, false);
    if (rudy_requested_ && initial_.m.design.normalized_overflow <= options_.routability_start_overflow) {
        activateRudy(initial_, false, false);
    }
    last_optimizer_overflow_ = initial_.m.optimizer.normalized_overflow;
    {
        const double count = static_cast<double>(std::max<std::size_t>(1U, particles));
        const double rms = initial_.pre_norm / std::sqrt(count);
        last_step_size_ = (options_.initial_movement_in_bins * min_bin_) / std::max(rms, kEpsilon);
    }
    bool initial_is_best = false;
    considerCheckpoint(cur_, initial_.m, 0, initial_is_best);
    feasible_refinement_iterations_ =
        initial_.m.design.normalized_overflow <= options_.maximum_bin_overflow ? 1 : 0;
}

double Session::smoothingFromOverflow(double overflow) const {
    // AdaptiveGlobalPlacer.cpp:456-462
    const double ratio = clampValue(overflow / std::max(initial_overflow_, kEpsilon), 0.0, 1.0);
    const double annealing = std::pow(ratio, options_.smoothing_overflow_exponent);
    return (options_.final_smoothing + (options_.initial_smoothing - options_.final_smoothing) * annealing) * max_bin_;
}

void Session::fillMetrics(const EvalScalars& s, double penalty, double rudy_weight, StateEval& out) const {
    out.m.hpwl = s.v[kHpwl];
    out.m.smooth_wirelength = s.v[kSmooth];
    out.m.density_energy = engine_->energy(s);
    engine_->densityMetrics(s, true, out.m.optimizer);
    engine_->densityMetrics(s, false, out.m.design);
    out.m.rudy_energy = s.v[kRudyEnergy];
    if (engine_->rudyEnabled()) {
        out.m.rudy_proxy_overflow = s.v[kRudyProxy] / static_cast<double>(engine_->rudyBins());
        out.m.rudy_maximum_utilization = std::max(0.0, s.v[kRudyMaxUtil]);
    }
    out.rudy_l1 = s.v[kRudyL1];
    // GlobalPlacementSession::evaluate objective (AdaptiveGlobalPlacer.cpp:221-222, 294-295).
    out.m.objective = out.m.smooth_wirelength + penalty * out.m.density_energy + rudy_weight * out.m.rudy_energy;
    if (!std::isfinite(out.m.objective) || !std::isfinite(out.m.hpwl)) {
        fail(MPGP_ERR_NON_FINITE, "CUDA adaptive placement objective produced a non-finite value.");
    }
    out.wire_l1 = s.v[kWireL1];
    out.density_l1 = s.v[kDensityL1];
    out.raw_norm = std::sqrt(s.v[kRawNorm2]);
    out.pre_norm = std::sqrt(s.v[kPreNorm2]);
    out.delta_pos2 = s.v[kDeltaPos2];
    out.delta_grad2 = s.v[kDeltaGrad2];
    out.alignment = s.v[kAlignment];
    out.predicted = s.v[kPredicted];
    out.max_displacement = s.v[kMaxDisplacement];
}

EvalRequest Session::givenRequest(double2* positions, bool gradient, double penalty, double2* raw, double2* pre,
                                  bool with_prev, bool with_velocity, bool reuse_density,
                                  double rudy_weight_override) {
    EvalRequest q;
    q.mode = kGiven;
    q.rudy = rudy_active_;
    q.rudy_weight = rudy_weight_override >= 0.0 ? rudy_weight_override : rudy_weight_;
    q.positions = positions;
    q.reuse_density = reuse_density;
    density_cached_ = false;
    q.smoothing = smoothing_;
    q.gradient = gradient;
    q.penalty = penalty;
    q.precond_scale = 1.0 / std::sqrt(1.0 + std::max(0.0, penalty / std::max(reference_penalty_, kEpsilon)));
    q.raw = raw;
    q.pre = pre;
    if (with_prev) {
        q.prev_positions = prev_pos_;
        q.prev_gradient = prev_grad_;
    }
    if (with_velocity) q.velocity = velocity_;
    return q;
}

EvalRequest Session::lookaheadRequest(double momentum, double penalty, double2* raw, double2* pre) {
    density_cached_ = false;
    EvalRequest q;
    q.mode = kLookahead;
    q.rudy = rudy_active_;
    q.rudy_weight = rudy_weight_;
    q.base = cur_;
    q.direction = velocity_;
    q.step = momentum;
    q.out_positions = look_;
    q.smoothing = smoothing_;
    q.gradient = true;
    q.penalty = penalty;
    q.precond_scale = 1.0 / std::sqrt(1.0 + std::max(0.0, penalty / std::max(reference_penalty_, kEpsilon)));
    q.raw = raw;
    q.pre = pre;
    if (has_previous_gradient_) {
        q.prev_positions = prev_pos_;
        q.prev_gradient = prev_grad_;
    }
    return q;
}

StateEval Session::collect(uint64_t ticket, const EvalRequest& q, double penalty) {
    const EvalScalars& s = engine_->sync(ticket);
    ++result_.evaluations;
    StateEval out;
    fillMetrics(s, penalty, q.rudy ? q.rudy_weight : 0.0, out);
    out.raw = q.raw;
    out.pre = q.pre;
    return out;
}

StateEval Session::evaluateGiven(double2* positions, bool gradient, double penalty, double2* raw, double2* pre,
                                 bool with_prev, bool with_velocity, bool reuse_density, double rudy_weight_override) {
    EvalRequest q =
        givenRequest(positions, gradient, penalty, raw, pre, with_prev, with_velocity, reuse_density, rudy_weight_override);
    const uint64_t ticket = launchEvaluation(q);
    return collect(ticket, q, penalty);
}

StateEval Session::evaluateLookahead(double momentum, double penalty, double2* raw, double2* pre) {
    EvalRequest q = lookaheadRequest(momentum, penalty, raw, pre);
    const uint64_t ticket = launchEvaluation(q);
    return collect(ticket, q, penalty);
}

uint64_t Session::launchEvaluation(EvalRequest& q) {
    if (pending_velocity_base_ != nullptr || pending_checkpoint_ != nullptr) {
        if (q.mode == kGiven && q.positions == cur_ && q.gradient && engine_->particleCount() > 0) {
            q.velocity_base = pending_velocity_base_;
            q.velocity_out = pending_velocity_base_ != nullptr ? velocity_ : nullptr;
            q.checkpoint_out = pending_checkpoint_;
            pending_velocity_base_ = nullptr;
            pending_checkpoint_ = nullptr;
        } else {
            flushPending();
        }
    }
    return engine_->launch(q);
}

void Session::flushPending() {
    const int count = static_cast<int>(engine_->particleCount());
    if (pending_velocity_base_ != nullptr) {
        engine_->beginKernel(kKindVector);
        launchVelocity(cur_, pending_velocity_base_, velocity_, count, engine_->stream());
        engine_->endKernel();
        engine_->countLaunches(1);
        pending_velocity_base_ = nullptr;
    }
    if (pending_checkpoint_ != nullptr) {
        launchCopyPositions(cur_, pending_checkpoint_, count, engine_->stream());
        engine_->countLaunches(1);
        pending_checkpoint_ = nullptr;
    }
}

EvalRequest Session::proposalRequest(const double2* base, const double2* pre, const double2* raw, double step,
                                     double max_disp) {
    density_cached_ = false;
    EvalRequest q;
    q.mode = kPropose;
    q.rudy = rudy_active_;
    q.rudy_weight = rudy_weight_;
    q.base = base;
    q.direction = pre;
    q.raw_direction = raw;
    q.step = step;
    q.max_displacement = max_disp;
    q.out_positions = cand_;
    q.smoothing = smoothing_;
    q.gradient = false;
    return q;
}

StateEval Session::evaluateProposal(const double2* base, const StateEval& base_eval, double step, double max_disp,
                                    double penalty) {
    EvalRequest q = proposalRequest(base, base_eval.pre, base_eval.raw, step, max_disp);
    const uint64_t ticket = launchEvaluation(q);
    return collect(ticket, q, penalty);
}

// refreshRudyWeight (AdaptiveGlobalPlacer.cpp:689-698): the weight ramps to its
// target over routability_ramp_iterations accepted iterations.
bool Session::refreshRudyWeight() {
    if (!rudy_active_) return false;
    const double progress =
        std::min(1.0, static_cast<double>(rudy_accepted_age_ + 1) /
                          static_cast<double>(std::max(1, options_.routability_ramp_iterations)));
    const double updated = rudy_target_weight_ * progress;
    const bool changed =
        std::abs(updated - rudy_weight_) > 1e-12 * std::max({1.0, std::abs(updated), std::abs(rudy_weight_)});
    rudy_weight_ = updated;
    return changed;
}

// activateRudy (AdaptiveGlobalPlacer.cpp:699-713 with GlobalPlacementSession::activateRudy
// :149-162 and calibrateRudyCapacity, Rudy.cpp:215-225): capacities frozen from the
// current map, the target weight matched to the wire-plus-density force, and the
// evaluation replaced by one with the routability term.
void Session::activateRudy(StateEval& evaluation, bool with_prev, bool with_velocity) {
    const auto calibrate = [&](bool validation, double factor) {
        const RudyReport raw = engine_->rudyEvaluate(cur_, validation);
        if (!std::isfinite(raw.horizontal_mean) || !std::isfinite(raw.vertical_mean) || raw.horizontal_mean < 0.0 ||
            raw.vertical_mean < 0.0) {
            fail(MPGP_ERR_INVALID_ARGUMENT, "RUDY mean demand must be finite and non-negative.");
        }
        engine_->setRudyCapacity(validation, std::max(kEpsilon, factor * raw.horizontal_mean),
                                 std::max(kEpsilon, factor * raw.vertical_mean));
    };
    calibrate(false, options_.rudy_capacity_factor);
    if (engine_->rudyValidationEnabled()) calibrate(true, options_.rudy_validation_capacity_factor);
    rudy_active_ = true;
    const StateEval probe = evaluateGiven(cur_, true, penalty_, raw_cur_, pre_cur_, with_prev, with_velocity, false, 0.0);
    const double base_l1 = probe.wire_l1 + penalty_ * probe.density_l1;
    rudy_target_weight_ =
        probe.rudy_l1 > kEpsilon ? options_.routability_weight_scale * base_l1 / probe.rudy_l1 : 0.0;
    rudy_accepted_age_ = 0;
    rudy_weight_ = 0.0;
    refreshRudyWeight();
    evaluation = evaluateGiven(cur_, true, penalty_, raw_cur_, pre_cur_, with_prev, with_velocity, false);
}

// refreshCheckpointRudyScore (AdaptiveGlobalPlacer.cpp:598-608).
void Session::refreshCheckpointRudyScore(CheckpointState& checkpoint) {
    if (!checkpoint.found) return;
    const StateEval e = evaluateGiven(checkpoint.positions, false, penalty_, nullptr, nullptr, false, false, false,
                                      rudy_target_weight_);
    checkpoint.rudy_energy = e.m.rudy_energy;
    checkpoint.selection_score = e.m.hpwl + rudy_target_weight_ * e.m.rudy_energy;
}

// A checkpoint of the current positions is copied by the next evaluation's gather;
// any other copy is a kernel of its own.
void Session::copyCheckpoint(double2* positions, double2* destination) {
    if (positions == cur_ && pending_checkpoint_ == nullptr) {
        pending_checkpoint_ = destination;
        return;
    }
    if (pending_checkpoint_ == destination) pending_checkpoint_ = nullptr;  // superseded
    launchCopyPositions(positions, destination, static_cast<int>(engine_->particleCount()), engine_->stream());
    engine_->countLaunches(1);
}

// considerCheckpoint (AdaptiveGlobalPlacer.cpp:559-596); the score adds the routability
// target weight times the RUDY energy.
void Session::considerCheckpoint(double2* positions, const ObjectiveMetrics& m, int iteration, bool& is_new_best) {
    is_new_best = false;
    const double overflow = m.design.normalized_overflow;
    const bool feasible = overflow <= options_.maximum_bin_overflow;
    const double score = m.hpwl + rudy_target_weight_ * m.rudy_energy;
    if (feasible && (!best_feasible_.found || score < best_feasible_.selection_score - 1e-10 ||
                     (std::abs(score - best_feasible_.selection_score) <= 1e-10 && m.hpwl < best_feasible_.hpwl))) {
        copyCheckpoint(positions, best_feasible_.positions);
        best_feasible_.iteration = iteration;
        best_feasible_.hpwl = m.hpwl;
        best_feasible_.overflow = overflow;
        best_feasible_.selection_score = score;
        best_feasible_.rudy_energy = m.rudy_energy;
        best_feasible_.found = true;
        is_new_best = true;
    }
    if (!best_feasible_.found &&
        (!best_fallback_.found || overflow < best_fallback_.overflow - 1e-12 ||
         (std::abs(overflow - best_fallback_.overflow) <= 1e-12 && m.hpwl < best_fallback_.hpwl))) {
        copyCheckpoint(positions, best_fallback_.positions);
        best_fallback_.iteration = iteration;
        best_fallback_.hpwl = m.hpwl;
        best_fallback_.overflow = overflow;
        best_fallback_.selection_score = score;
        best_fallback_.rudy_energy = m.rudy_energy;
        best_fallback_.found = true;
        is_new_best = true;
    }
}

bool Session::step(int iterations, int* completed) {
    int ran = 0;
    while (!done_ && ran < iterations) {
        iterate();
        ++ran;
    }
    if (completed != nullptr) *completed = result_.completed_iterations;
    return done_;
}

// One pass of the loop body of runAdaptiveGlobalPlacement (AdaptiveGlobalPlacer.cpp:735-928).
void Session::iterate() {
    const mpgp_options& o = options_;
    const int iteration = iteration_;
    StateEval current;
    // The momentum lookahead (below) needs nothing from the current evaluation but the
    // go-ahead: when it is likely to run, it is launched right behind the current
    // evaluation, before the host reads that one, and dropped unread if the current
    // evaluation calls for a restart.  Its request and results are those of the
    // sequential order, since no state it reads changes in between.
    const auto momentumOf = [&](int age) {
        return std::min(o.maximum_momentum, static_cast<double>(age) / static_cast<double>(age + 3));
    };
    uint64_t lookahead_ticket = 0;
    EvalRequest lookahead_request;
    if (iteration == 0) {
        current = initial_;
    } else {
        smoothing_ = smoothingFromOverflow(last_optimizer_overflow_);
        if (rudy_active_ && refreshRudyWeight()) has_previous_gradient_ = false;
        EvalRequest q = givenRequest(cur_, true, penalty_, raw_cur_, pre_cur_, has_previous_gradient_, true,
                                     density_cached_, -1.0);
        const uint64_t ticket = launchEvaluation(q);
        const bool speculate = engine_->overlapsEvaluations() && !rudy_requested_ && !rudy_active_ &&
                               objective_worse_streak_ < 2 && momentum_age_ > 0 && !velocity_zero_;
        if (speculate) {
            lookahead_request = lookaheadRequest(momentumOf(momentum_age_), penalty_, raw_look_, pre_look_);
            lookahead_ticket = launchEvaluation(lookahead_request);
        }
        current = collect(ticket, q, penalty_);
    }
    bool rudy_just_activated = false;
    if (rudy_requested_ && !rudy_active_ &&
        current.m.design.normalized_overflow <= o.routability_start_overflow) {
        activateRudy(current, has_previous_gradient_, true);
        refreshCheckpointRudyScore(best_feasible_);
        has_previous_gradient_ = false;
        pending_velocity_base_ = nullptr;  // the velocity restarts from zero
        checkCuda(cudaMemsetAsync(velocity_, 0, sizeof(double2) * static_cast<std::size_t>(engine_->particleCount()),
                                  engine_->stream()),
                  "Clear velocity");
        velocity_zero_ = true;
        rudy_just_activated = true;
    }

    bool restarted = objective_worse_streak_ >= 2 || rudy_just_activated;
    bool momentum_used = false;
    double2* base_positions = cur_;
    const StateEval* base = &current;
    StateEval lookahead;
    if (!restarted && momentum_age_ > 0) {
        const double momentum = momentumOf(momentum_age_);
        const double alignment = velocity_zero_ ? 0.0 : -current.alignment;  // momentumAlignment (:610-617)
        if (alignment <= 0.0) {
            restarted = true;
        } else {
            lookahead = lookahead_ticket != 0 ? collect(lookahead_ticket, lookahead_request, penalty_)
                                              : evaluateLookahead(momentum, penalty_, raw_look_, pre_look_);
            if (lookahead.m.objective > current.m.objective * (1.0 + o.hpwl_growth_restart_threshold)) {
                restarted = true;
            } else {
                base_positions = look_;
                base = &lookahead;
                momentum_used = true;
            }
        }
    }
    if (restarted) {
        base_positions = cur_;
        base = &current;
        momentum_age_ = 0;
        objective_worse_streak_ = 0;
        ++result_.momentum_restarts;
    }

    bool accepted = false;
    bool new_best_checkpoint = false;
    int backtracks = 0;
    double used_step_size = 0.0;
    double used_curvature = 0.0;
    double used_maximum_displacement = 0.0;
    StateEval accepted_eval;

    for (int restart_pass = 0; restart_pass < 2 && !accepted; ++restart_pass) {
        // estimateStep (AdaptiveGlobalPlacer.cpp:470-492).
        const double fallback_step = std::max(last_step_size_, kEpsilon);
        double step_size = fallback_step;
        double curvature = 0.0;
        if (has_previous_gradient_ && base->delta_pos2 > kEpsilon && base->delta_grad2 > kEpsilon) {
            curvature = std::sqrt(base->delta_grad2 / base->delta_pos2);
            step_size = clampValue(1.0 / std::max(curvature, kEpsilon), fallback_step * 0.25, fallback_step * 4.0);
        }
        double candidate_step_size = step_size;
        const double overflow_ratio =
            clampValue(base->m.optimizer.normalized_overflow / std::max(initial_overflow_, kEpsilon), 0.0, 1.0);
        const double maximum_displacement = o.maximum_movement_in_bins * min_bin_ * (0.35 + 0.65 * overflow_ratio);
        for (int attempt = 0; attempt <= o.maximum_backtracks; ++attempt) {
            StateEval candidate = evaluateProposal(base_positions, *base, candidate_step_size, maximum_displacement,
                                                   penalty_);
            if (candidate.predicted <= kEpsilon) break;
            if (acceptsCandidate(base->m, candidate.m, candidate.predicted, o)) {
                accepted = true;
                used_step_size = candidate_step_size;
                used_curvature = curvature;
                used_maximum_displacement = candidate.max_displacement;
                accepted_eval = candidate;
                break;
            }
            ++backtracks;
            ++result_.rejected_candidates;
            candidate_step_size *= o.backtracking_ratio;
        }
        if (accepted || restarted || !momentum_used) break;
        restarted = true;
        ++result_.momentum_restarts;
        momentum_age_ = 0;
        objective_worse_streak_ = 0;
        base_positions = cur_;
        base = &current;
        momentum_used = false;
    }

    const double penalty_used = penalty_;
    if (accepted) {
        // velocity = accepted - current positions, done by the next evaluation (the
        // buffer of the current positions is left alone until then).
        const double2* stepped_from = cur_;
        velocity_zero_ = false;
        last_step_size_ = used_step_size;
        momentum_age_ = restarted ? 0 : momentum_age_ + 1;
        const double hpwl_growth = (accepted_eval.m.hpwl - current.m.hpwl) / std::max(current.m.hpwl, 1.0);
        objective_worse_streak_ = hpwl_growth > o.hpwl_growth_restart_threshold ? objective_worse_streak_ + 1 : 0;
        const double next_penalty = updateDensityPenalty(penalty_, reference_penalty_, current.m, accepted_eval.m, o);
        const bool penalty_changed = std::abs(std::log(next_penalty / std::max(penalty_, kEpsilon))) > 0.01;
        penalty_ = next_penalty;
        const double base_pre_norm = base->pre_norm;
        if (penalty_changed) {
            has_previous_gradient_ = false;
        } else {
            // previous_gradient_positions = base_positions; previous_gradient = base preconditioned gradient.
            if (base_positions == look_) {
                std::swap(prev_pos_, look_);
            } else {
                std::swap(prev_pos_, cur_);
            }
            if (base->pre == pre_look_) {
                std::swap(prev_grad_, pre_look_);
            } else {
                std::swap(prev_grad_, pre_cur_);
            }
            has_previous_gradient_ = true;
        }
        std::swap(cur_, cand_);  // current_positions = accepted positions
        pending_velocity_base_ = stepped_from;
        density_cached_ = true;  // the accepted candidate was the last evaluation
        last_optimizer_overflow_ = accepted_eval.m.optimizer.normalized_overflow;
        considerCheckpoint(cur_, accepted_eval.m, iteration + 1, new_best_checkpoint);
        ++result_.accepted_iterations;
        if (rudy_active_) ++rudy_accepted_age_;
        if (accepted_eval.m.design.normalized_overflow <= o.maximum_bin_overflow) {
            ++feasible_refinement_iterations_;
        } else {
            feasible_refinement_iterations_ = 0;
        }
        history_.push_back(makeHistoryRow(iteration + 1, accepted_eval.m, penalty_used, smoothing_, used_step_size,
                                          used_maximum_displacement, base_pre_norm, used_curvature, backtracks,
                                          restarted, true, new_best_checkpoint, rudy_weight_, rudy_active_));
    } else {
        pending_velocity_base_ = nullptr;  // the velocity restarts from zero
        checkCuda(cudaMemsetAsync(velocity_, 0, sizeof(double2) * static_cast<std::size_t>(engine_->particleCount()),
                                  engine_->stream()),
                  "Clear velocity");
        velocity_zero_ = true;
        momentum_age_ = 0;
        objective_worse_streak_ = 0;
        if (current.m.optimizer.normalized_overflow > o.maximum_bin_overflow) {
            penalty_ = clampValue(penalty_ * o.density_penalty_increase,
                                  std::max(o.minimum_density_penalty, reference_penalty_ * 0.02),
                                  o.maximum_density_penalty);
        }
        last_optimizer_overflow_ = current.m.optimizer.normalized_overflow;
        if (current.m.design.normalized_overflow <= o.maximum_bin_overflow) {
            ++feasible_refinement_iterations_;
        } else {
            feasible_refinement_iterations_ = 0;
        }
        history_.push_back(makeHistoryRow(iteration + 1, current.m, penalty_used, smoothing_, 0.0, 0.0,
                                          current.pre_norm, 0.0, backtracks, restarted, false, false, rudy_weight_,
                                          rudy_active_));
    }
    result_.completed_iterations = iteration + 1;
    ++iteration_;
    if ((iteration >= 20 && feasible_refinement_iterations_ >= o.feasible_refinement_iterations) ||
        iteration_ >= o.iterations) {
        done_ = true;
    }
}

void Session::currentPositions(double* xy) const {
    if (empty_) return;
    const std::size_t particles = static_cast<std::size_t>(engine_->particleCount());
    checkCuda(cudaMemcpyAsync(xy, cur_, particles * sizeof(double2), cudaMemcpyDeviceToHost, engine_->stream()),
              "Download positions");
    checkCuda(cudaStreamSynchronize(engine_->stream()), "Download positions");
}

void Session::finish(double* module_x, double* module_y, mpgp_result* result, mpgp_history_row* history,
                     int capacity) {
    if (!empty_) {
        flushPending();
        const CheckpointState& chosen = best_feasible_.found ? best_feasible_ : best_fallback_;
        double2* final_positions = chosen.found ? chosen.positions : cur_;
        if (chosen.found) {
            result_.restored_best_checkpoint = 1;
            result_.best_checkpoint_iteration = chosen.iteration;
            result_.best_checkpoint_hpwl = chosen.hpwl;
            result_.best_checkpoint_overflow = chosen.overflow;
        }
        const std::size_t particles = static_cast<std::size_t>(engine_->particleCount());
        std::vector<double2> host(particles);
        checkCuda(cudaMemcpyAsync(host.data(), final_positions, particles * sizeof(double2), cudaMemcpyDeviceToHost,
                                  engine_->stream()),
                  "Download final positions");
        checkCuda(cudaStreamSynchronize(engine_->stream()), "Download final positions");
        engine_->addTransfer(0, particles * sizeof(double2));
        // applyPositions (AdaptiveGlobalPlacer.cpp:185-198) for the movable modules.
        const Rect2& core = derived_.core;
        std::vector<double2> clamped(particles);
        for (std::size_t i = 0; i < particles; ++i) {
            const double w = i < derived_.movable.size() ? module_w_[derived_.movable[i]] : fillers_[i - derived_.movable.size()].width;
            const double h = i < derived_.movable.size() ? module_h_[derived_.movable[i]] : fillers_[i - derived_.movable.size()].height;
            const double min_x = core.llx + w * 0.5, max_x = core.urx - w * 0.5;
            const double min_y = core.lly + h * 0.5, max_y = core.ury - h * 0.5;
            clamped[i].x = min_x <= max_x ? clampValue(host[i].x, min_x, max_x) : (core.llx + core.urx) * 0.5;
            clamped[i].y = min_y <= max_y ? clampValue(host[i].y, min_y, max_y) : (core.lly + core.ury) * 0.5;
            if (i < derived_.movable.size()) {
                module_x_[derived_.movable[i]] = clamped[i].x;
                module_y_[derived_.movable[i]] = clamped[i].y;
            }
        }
        // calculateHpwl / calculateDensity at the restored placement (:938-940).
        checkCuda(cudaMemcpyAsync(cand_, clamped.data(), particles * sizeof(double2), cudaMemcpyHostToDevice,
                                  engine_->stream()),
                  "Upload final positions");
        engine_->addTransfer(particles * sizeof(double2), 0);
        const StateEval final_eval = evaluateGiven(cand_, false, penalty_, nullptr, nullptr, false, false);
        result_.hpwl_after = final_eval.m.hpwl;
        result_.overflow_after = final_eval.m.design.normalized_overflow;
        if (rudy_active_) {
            // The RUDY metrics of the final placement (AdaptiveGlobalPlacer.cpp:941-950).
            const RudyReport r = engine_->rudyEvaluate(cand_, false);
            result_.rudy_energy_after = r.energy;
            result_.rudy_horizontal_capacity = r.horizontal_capacity;
            result_.rudy_vertical_capacity = r.vertical_capacity;
            result_.rudy_proxy_overflow_after = r.proxy_overflow;
            result_.rudy_maximum_utilization_after = r.maximum_utilization;
            result_.rudy_p95_utilization_after = r.p95_utilization;
            if (engine_->rudyValidationEnabled()) {
                const RudyReport v = engine_->rudyEvaluate(cand_, true);
                result_.rudy_validation_energy_after = v.energy;
                result_.rudy_validation_proxy_overflow_after = v.proxy_overflow;
                result_.rudy_validation_maximum_utilization_after = v.maximum_utilization;
                result_.rudy_validation_p95_utilization_after = v.p95_utilization;
            }
        }
        result_.cuda_reserved_memory_bytes = engine_->reservedBytes();
        engine_->leaveBatch();
    }
    result_.elapsed_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - started_).count();
    result_.history_count = static_cast<int32_t>(history_.size());
    if (module_x != nullptr && module_y != nullptr) {
        std::copy(module_x_.begin(), module_x_.end(), module_x);
        std::copy(module_y_.begin(), module_y_.end(), module_y);
    }
    if (result != nullptr) *result = result_;
    if (history != nullptr && capacity > 0) {
        const std::size_t rows = std::min<std::size_t>(history_.size(), static_cast<std::size_t>(capacity));
        std::copy(history_.begin(), history_.begin() + static_cast<std::ptrdiff_t>(rows), history);
    }
}

}  // namespace mpgp
