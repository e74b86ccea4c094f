// Drop-in CUDA placement backend for MyPlacement, over the B200 engine's C ABI.
//
// A MyPlacement build links this file (instead of src/placement/cuda/
// CudaPlacementBackend.cu or CudaPlacementBackendStub.cpp) together with
// libmpgp.so.  It provides the three declarations of
// src/placement/CudaPlacementBackend.hpp:
//   cudaPlacementBackendCompiled()            (:44)
//   tryCreateCudaPlacementBackend(...)        (:45-48)
//   CudaPlacementBackend::evaluate / device / reservedBytes (:32-35)
// so GlobalPlacementSession::initializeComputeBackend and evaluateCuda
// (AdaptiveGlobalPlacer.cpp:271-331) drive the engine unchanged.
//
// Data mapping (the reference's buildHostLayout, CudaPlacementBackend.cu:784-839):
//   particles   movable modules in `movable` order, then the fillers; layer 1
//               for macros, 0 for other modules, 2 for fillers; pin counts
//               for the preconditioner (0 for fillers)
//   pins        net by net in net order; a pin of a movable module carries
//               its orientation-transformed offset, any other pin its
//               absolute position and particle -1
//   density     the static map's fixed and dark areas per bin
// Errors keep the reference's conventions: a recoverable creation failure is
// nullptr + reason; an evaluation failure throws std::invalid_argument
// (MPGP_ERR_INVALID_ARGUMENT) or std::runtime_error (everything else).
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "CudaPlacementBackend.hpp"
#include "mpgp.h"

namespace myplacement::detail {
namespace {

[[noreturn]] void raise(int status, const char* what) {
    const std::string message = std::string(what) + ": " + mpgp_last_error();
    if (status == MPGP_ERR_INVALID_ARGUMENT) throw std::invalid_argument(message);
    throw std::runtime_error(message);
}

DensityMetrics toMetrics(const mpgp_density_metrics& m) {
    DensityMetrics out;
    out.total_overflow_area = m.total_overflow_area;
    out.normalized_overflow = m.normalized_overflow;
    out.maximum_density = m.maximum_density;
    out.average_density = m.average_density;
    out.total_charge_area = m.total_charge_area;
    out.normalization_area = m.normalization_area;
    out.placeable_area = m.placeable_area;
    out.dark_area = m.dark_area;
    return out;
}

class EngineBackend final : public CudaPlacementBackend {
public:
    EngineBackend(mpgp_backend* handle, std::size_t particle_count)
        : handle_(handle), particle_count_(particle_count), positions_(2 * particle_count),
          wire_(2 * particle_count), density_(2 * particle_count) {}
    ~EngineBackend() override { mpgp_backend_destroy(handle_); }

    CudaPlacementEvaluation evaluate(const std::vector<Vec2>& particle_positions, double smoothing,
                                     bool calculate_gradient) override {
        if (particle_positions.size() != particle_count_) {
            throw std::invalid_argument("CUDA placement positions do not match the particle count.");
        }
        for (std::size_t i = 0; i < particle_count_; ++i) {
            positions_[2 * i] = particle_positions[i].x;
            positions_[2 * i + 1] = particle_positions[i].y;
        }
        mpgp_evaluation out{};
        const int status = mpgp_backend_evaluate(handle_, positions_.data(), smoothing, calculate_gradient ? 1 : 0,
                                                 &out, wire_.data(), density_.data());
        if (status != MPGP_OK) raise(status, "B200 placement evaluation failed");
        CudaPlacementEvaluation result;
        result.hpwl = out.hpwl;
        result.smooth_wirelength = out.smooth_wirelength;
        result.electrostatic_energy = out.electrostatic_energy;
        result.optimizer_density = toMetrics(out.optimizer_density);
        result.design_density = toMetrics(out.design_density);
        if (calculate_gradient) {
            result.wire_gradient.resize(particle_count_);
            result.density_gradient.resize(particle_count_);
            for (std::size_t i = 0; i < particle_count_; ++i) {
                result.wire_gradient[i] = {wire_[2 * i], wire_[2 * i + 1]};
                result.density_gradient[i] = {density_[2 * i], density_[2 * i + 1]};
            }
        }
        return result;
    }

    [[nodiscard]] int device() const override { return mpgp_backend_device(handle_); }
    [[nodiscard]] std::size_t reservedBytes() const override {
        return static_cast<std::size_t>(mpgp_backend_reserved_bytes(handle_));
    }

private:
    mpgp_backend* handle_;
    std::size_t particle_count_;
    std::vector<double> positions_;
    std::vector<double> wire_;
    std::vector<double> density_;
};

}  // namespace

bool cudaPlacementBackendCompiled() { return mpgp_compiled() != 0; }

std::unique_ptr<CudaPlacementBackend> tryCreateCudaPlacementBackend(
    const PlacementDatabase& database, const std::vector<ModuleId>& movable,
    const std::vector<DensityFiller>& fillers, const DensityMap& static_density,
    const GlobalPlacementOptions& options, std::string& reason) {
    reason.clear();
    if (options.density_field_boundary != DensityFieldBoundary::Neumann) {
        reason = "The CUDA backend currently implements the physical Neumann/DCT field only.";
        return nullptr;
    }
    if (static_density.targetDensity() != options.target_density) {
        reason = "CUDA density map target does not match global-placement options.";
        return nullptr;
    }
    // Particles.
    const std::size_t particle_count = movable.size() + fillers.size();
    std::vector<double> width, height;
    std::vector<int32_t> layer, pin_count;
    width.reserve(particle_count);
    height.reserve(particle_count);
    layer.reserve(particle_count);
    pin_count.reserve(particle_count);
    std::vector<int32_t> module_particle(database.modules.size(), -1);
    for (std::size_t i = 0; i < movable.size(); ++i) {
        const Module& module = database.modules[movable[i]];
        module_particle[movable[i]] = static_cast<int32_t>(i);
        width.push_back(module.width);
        height.push_back(module.height);
        layer.push_back(module.is_macro ? MPGP_LAYER_MACRO : MPGP_LAYER_STANDARD);
        pin_count.push_back(static_cast<int32_t>(module.pins.size()));
    }
    for (const DensityFiller& filler : fillers) {
        width.push_back(filler.width);
        height.push_back(filler.height);
        layer.push_back(MPGP_LAYER_FILLER);
        pin_count.push_back(0);
    }
    // Nets and pins.
    std::vector<double> net_weight;
    std::vector<int64_t> net_pin_start{0};
    std::vector<int32_t> pin_particle;
    std::vector<double> pin_x, pin_y;
    net_weight.reserve(database.nets.size());
    net_pin_start.reserve(database.nets.size() + 1);
    for (const Net& net : database.nets) {
        net_weight.push_back(net.weight);
        for (const PinId pin_id : net.pins) {
            const Pin& pin = database.pins[pin_id];
            const Module& module = database.modules[pin.module];
            const int32_t particle = module_particle[pin.module];
            const Vec2 p = particle >= 0 ? transformOffset(pin.offset, module.orientation) : database.pinPosition(pin_id);
            pin_particle.push_back(particle);
            pin_x.push_back(p.x);
            pin_y.push_back(p.y);
        }
        net_pin_start.push_back(static_cast<int64_t>(pin_particle.size()));
    }
    // Static density.
    const std::size_t bins = static_density.bins().size();
    std::vector<double> fixed(bins), dark(bins);
    for (std::size_t b = 0; b < bins; ++b) {
        fixed[b] = static_density.bins()[b].fixed_area;
        dark[b] = static_density.bins()[b].dark_area;
    }
    mpgp_layout layout{};
    layout.particle_count = static_cast<int64_t>(particle_count);
    layout.movable_count = static_cast<int64_t>(movable.size());
    layout.particle_width = width.data();
    layout.particle_height = height.data();
    layout.particle_layer = layer.data();
    layout.particle_pin_count = pin_count.data();
    layout.net_count = static_cast<int32_t>(net_weight.size());
    layout.net_weight = net_weight.data();
    layout.net_pin_start = net_pin_start.data();
    layout.pin_count = static_cast<int64_t>(pin_particle.size());
    layout.pin_particle = pin_particle.data();
    layout.pin_x = pin_x.data();
    layout.pin_y = pin_y.data();
    layout.bins_x = static_density.columns();
    layout.bins_y = static_density.rows();
    layout.region_llx = static_density.region().ll.x;
    layout.region_lly = static_density.region().ll.y;
    layout.region_urx = static_density.region().ur.x;
    layout.region_ury = static_density.region().ur.y;
    layout.target_density = options.target_density;
    layout.static_fixed_area = fixed.data();
    layout.static_dark_area = dark.data();

    mpgp_backend* handle = nullptr;
    char message[512] = {0};
    const int status = mpgp_backend_create(&layout, options.cuda_device,
                                           static_cast<uint64_t>(options.maximum_cuda_memory_bytes), &handle,
                                           message, sizeof(message));
    if (status != MPGP_OK || handle == nullptr) {
        reason = message[0] != '\0' ? message : mpgp_last_error();
        if (reason.empty()) reason = "The B200 engine could not be created.";
        return nullptr;
    }
    return std::make_unique<EngineBackend>(handle, particle_count);
}

}  // namespace myplacement::detail
