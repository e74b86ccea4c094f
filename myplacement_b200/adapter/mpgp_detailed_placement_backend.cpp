// Drop-in for the reference's CUDA detailed-placement backend:
// myplacement::detail::cudaDetailedPlacementBackendCompiled and
// tryRunCudaDetailedPlacement (src/placement/CudaDetailedPlacementBackend.hpp:9-16)
// over libmpgp.so's mpgp_detailed_place (include/mpgp.h).  Linked in place of
// src/placement/cuda/CudaDetailedPlacementBackend.cu, DetailedPlacer::run with
// the cuda or auto backend reaches the B200 engine; a false return carries the
// engine's reason and leaves the database as it was, as the reference's does.
#include <cstdint>
#include <string>
#include <vector>

#include "CudaDetailedPlacementBackend.hpp"
#include "mpgp.h"

namespace myplacement::detail {

bool cudaDetailedPlacementBackendCompiled() { return mpgp_compiled() != 0; }

bool tryRunCudaDetailedPlacement(PlacementDatabase& database, const DetailedPlacementOptions& options,
                                 DetailedPlacementResult& result, std::string& reason) {
    reason.clear();
    const std::size_t modules = database.modules.size();
    std::vector<double> width(modules), height(modules), x(modules), y(modules);
    std::vector<int32_t> flags(modules), orientation(modules);
    for (std::size_t m = 0; m < modules; ++m) {
        const Module& module = database.modules[m];
        width[m] = module.width;
        height[m] = module.height;
        x[m] = module.center.x;
        y[m] = module.center.y;
        flags[m] = (module.is_terminal ? MPGP_MODULE_TERMINAL : 0) | (module.is_fixed ? MPGP_MODULE_FIXED : 0);
        orientation[m] = static_cast<int32_t>(module.orientation);
    }
    std::vector<double> weight, offset_x, offset_y;
    std::vector<int64_t> pin_start{0};
    std::vector<int32_t> pin_module;
    for (const Net& net : database.nets) {
        weight.push_back(net.weight);
        for (const PinId pin : net.pins) {
            pin_module.push_back(static_cast<int32_t>(database.pins[pin].module));
            offset_x.push_back(database.pins[pin].offset.x);
            offset_y.push_back(database.pins[pin].offset.y);
        }
        pin_start.push_back(static_cast<int64_t>(pin_module.size()));
    }
    std::vector<double> bottom, row_height, site_width, spacing, x_start;
    std::vector<int64_t> sites;
    std::vector<int32_t> row_orientation;
    for (const SiteRow& row : database.rows) {
        bottom.push_back(row.bottom);
        row_height.push_back(row.height);
        site_width.push_back(row.site_width);
        spacing.push_back(row.site_spacing);
        x_start.push_back(row.x_start);
        sites.push_back(static_cast<int64_t>(row.site_count));
        row_orientation.push_back(static_cast<int32_t>(row.orientation));
    }
    mpgp_design design{};
    design.module_count = static_cast<int32_t>(modules);
    design.module_width = width.data();
    design.module_height = height.data();
    design.module_x = x.data();
    design.module_y = y.data();
    design.module_flags = flags.data();
    design.module_orientation = orientation.data();
    design.net_count = static_cast<int32_t>(database.nets.size());
    design.net_weight = weight.data();
    design.net_pin_start = pin_start.data();
    design.pin_count = static_cast<int64_t>(pin_module.size());
    design.pin_module = pin_module.data();
    design.pin_offset_x = offset_x.data();
    design.pin_offset_y = offset_y.data();
    design.row_count = static_cast<int32_t>(database.rows.size());
    design.row_bottom = bottom.data();
    design.row_height = row_height.data();
    design.row_site_width = site_width.data();
    design.row_site_spacing = spacing.data();
    design.row_x_start = x_start.data();
    design.row_site_count = sites.data();

    mpgp_detailed_options flat{};
    flat.method = static_cast<int32_t>(options.method);
    flat.passes = options.passes;
    flat.window_size = options.window_size;
    flat.cuda_device = options.cuda_device;
    flat.maximum_net_degree = options.maximum_net_degree;
    flat.improvement_epsilon = options.improvement_epsilon;
    flat.maximum_cuda_memory_bytes = options.maximum_cuda_memory_bytes;

    std::vector<double> out_x(modules), out_y(modules);
    std::vector<int32_t> out_orientation(modules);
    mpgp_detailed_result out{};
    char why[1024] = {0};
    if (mpgp_detailed_place(&design, row_orientation.data(), &flat, out_x.data(), out_y.data(),
                            out_orientation.data(), &out, why, sizeof(why)) != MPGP_OK) {
        reason = why;
        return false;
    }
    for (std::size_t m = 0; m < modules; ++m) {
        database.modules[m].center = {out_x[m], out_y[m]};
        database.modules[m].orientation = static_cast<Orientation>(out_orientation[m]);
    }
    result = {};
    result.hpwl_before = out.hpwl_before;
    result.hpwl_after = out.hpwl_after;
    result.elapsed_seconds = out.elapsed_seconds;
    result.evaluated_windows = static_cast<std::size_t>(out.evaluated_windows);
    result.evaluated_permutations = static_cast<std::size_t>(out.evaluated_permutations);
    result.accepted_operations = static_cast<std::size_t>(out.accepted_operations);
    result.completed_passes = out.completed_passes;
    result.compute_backend_used = DetailedPlacementBackend::Cuda;
    result.cuda_device_used = out.cuda_device_used;
    result.cuda_reserved_memory_bytes = static_cast<std::size_t>(out.cuda_reserved_memory_bytes);
    return true;
}

}  // namespace myplacement::detail
