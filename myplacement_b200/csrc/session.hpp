// Device-resident adaptive global placement (one design, one GPU).
#pragma once

#include <chrono>
#include <memory>
#include <vector>

#include "engine.cuh"
#include "setup.hpp"

namespace mpgp {

struct ObjectiveMetrics {
    double hpwl = 0.0;
    double smooth_wirelength = 0.0;
    double density_energy = 0.0;
    double objective = 0.0;
    double rudy_energy = 0.0;
    double rudy_proxy_overflow = 0.0;
    double rudy_maximum_utilization = 0.0;
    mpgp_density_metrics optimizer{};
    mpgp_density_metrics design{};
};

// Host view of one evaluation; the vectors stay on the device.
struct StateEval {
    ObjectiveMetrics m;
    double raw_norm = 0.0;
    double pre_norm = 0.0;
    double wire_l1 = 0.0;
    double density_l1 = 0.0;
    double delta_pos2 = 0.0;
    double delta_grad2 = 0.0;
    double alignment = 0.0;  // sum v . pre
    double rudy_l1 = 0.0;    // |RUDY gradient|_1 over particles (unweighted)
    double predicted = 0.0;
    double max_displacement = 0.0;
    double2* raw = nullptr;
    double2* pre = nullptr;
};

struct CheckpointState {
    double2* positions = nullptr;
    int iteration = 0;
    double hpwl = 0.0;
    double overflow = 0.0;
    double selection_score = 0.0;
    double rudy_energy = 0.0;
    bool found = false;
};

class Session {
public:
    // With a batch, the session's evaluations run in the batch's shared rounds
    // (a routability run, which the batched launches do not cover, runs on its own).
    Session(const mpgp_design& design, const mpgp_options& options, Batch* batch = nullptr);
    // Runs up to `iterations` controller iterations; returns true once the run is done.
    bool step(int iterations, int* completed);
    void finish(double* module_x, double* module_y, mpgp_result* result, mpgp_history_row* history, int capacity);
    [[nodiscard]] int64_t launches() const { return engine_ ? engine_->launches() : 0; }
    [[nodiscard]] void* stream() const { return engine_ ? engine_->stream() : nullptr; }
    [[nodiscard]] bool done() const { return done_; }
    [[nodiscard]] const Problem& problem() const { return problem_; }
    [[nodiscard]] const std::vector<Filler>& fillers() const { return fillers_; }
    [[nodiscard]] const DerivedDesign& derived() const { return derived_; }
    void currentPositions(double* xy) const;
    [[nodiscard]] Engine* engine() const { return engine_.get(); }

private:
    StateEval evaluateGiven(double2* positions, bool gradient, double penalty, double2* raw, double2* pre,
                            bool with_prev, bool with_velocity, bool reuse_density = false,
                            double rudy_weight_override = -1.0);
    StateEval evaluateLookahead(double momentum, double penalty, double2* raw, double2* pre);
    // The requests behind evaluateGiven and evaluateLookahead, and the reading of an
    // evaluation launched earlier (so that two can be in flight).
    EvalRequest givenRequest(double2* positions, bool gradient, double penalty, double2* raw, double2* pre,
                             bool with_prev, bool with_velocity, bool reuse_density, double rudy_weight_override);
    EvalRequest lookaheadRequest(double momentum, double penalty, double2* raw, double2* pre);
    EvalRequest proposalRequest(const double2* base, const double2* pre, const double2* raw, double step,
                                double max_disp);
    StateEval collect(uint64_t ticket, const EvalRequest& request, double penalty);
    // The accepted step's velocity update and checkpoint copy wait for the next
    // evaluation: one at the current positions with a gradient does them in its gather
    // (settlePending hands them to it); before any other evaluation, and before the
    // host reads a checkpoint, flushPending launches them as kernels.
    uint64_t launchEvaluation(EvalRequest& request);
    void flushPending();
    void copyCheckpoint(double2* positions, double2* destination);
    StateEval evaluateProposal(const double2* base, const StateEval& base_eval, double step, double max_disp,
                               double penalty);
    void fillMetrics(const EvalScalars& s, double penalty, double rudy_weight, StateEval& out) const;
    // The routability schedule (AdaptiveGlobalPlacer.cpp:685-719).
    bool refreshRudyWeight();
    void activateRudy(StateEval& evaluation, bool with_prev, bool with_velocity);
    void refreshCheckpointRudyScore(CheckpointState& checkpoint);
    void considerCheckpoint(double2* positions, const ObjectiveMetrics& metrics, int iteration, bool& is_new_best);
    double smoothingFromOverflow(double overflow) const;
    void iterate();

    mpgp_options options_{};
    std::vector<double> module_x_, module_y_;
    std::vector<double> module_w_, module_h_;
    DerivedDesign derived_;
    std::vector<Filler> fillers_;
    Problem problem_;
    std::unique_ptr<Engine> engine_;
    std::chrono::steady_clock::time_point started_;
    bool empty_ = false;
    bool done_ = false;

    double min_bin_ = 0.0, max_bin_ = 0.0;
    double density_strength_base_ = 1.0;

    // device vectors
    double2* cur_ = nullptr;
    double2* look_ = nullptr;
    double2* cand_ = nullptr;
    double2* prev_pos_ = nullptr;
    double2* velocity_ = nullptr;
    double2* raw_cur_ = nullptr;
    double2* pre_cur_ = nullptr;
    double2* raw_look_ = nullptr;
    double2* pre_look_ = nullptr;
    double2* prev_grad_ = nullptr;
    CheckpointState best_feasible_, best_fallback_;

    // controller state (runAdaptiveGlobalPlacement locals, AdaptiveGlobalPlacer.cpp:656-733)
    mpgp_result result_{};
    std::vector<mpgp_history_row> history_;
    double smoothing_ = 0.0;
    double initial_overflow_ = 0.0;
    double penalty_ = 1.0;
    double reference_penalty_ = 1.0;
    double last_optimizer_overflow_ = 0.0;
    double last_step_size_ = 0.0;
    bool has_previous_gradient_ = false;
    int momentum_age_ = 0;
    int objective_worse_streak_ = 0;
    int feasible_refinement_iterations_ = 0;
    int iteration_ = 0;
    StateEval initial_;
    bool velocity_zero_ = true;
    const double2* pending_velocity_base_ = nullptr;  // velocity_ = cur_ - this, not yet done
    double2* pending_checkpoint_ = nullptr;           // a checkpoint of cur_ not yet copied
    // The last evaluation was the accepted candidate now held in cur_, so its
    // density map, field coefficients and energy are still on the device.
    bool density_cached_ = false;
    // RUDY routability term.
    bool rudy_requested_ = false;
    bool rudy_active_ = false;
    int rudy_accepted_age_ = 0;
    double rudy_target_weight_ = 0.0;
    double rudy_weight_ = 0.0;
};

}  // namespace mpgp
