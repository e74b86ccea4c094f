// Host setup restated from the reference (see setup.hpp).  Every floating-point
// expression that feeds the static layers, fillers or preconditioner keeps the
// reference's operation order so that the results are bit-identical; this file
// is compiled with -ffp-contract=off.
#include "setup.hpp"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <numeric>
#include <random>
#include <string>
#include <thread>

#include "common.cuh"
#include "workers.hpp"

namespace mpgp {
namespace {

// Rect arithmetic exactly as Geometry.hpp:60-86.
struct R {
    double llx, lly, urx, ury;
    [[nodiscard]] double width() const { return urx - llx; }
    [[nodiscard]] double height() const { return ury - lly; }
    [[nodiscard]] double area() const { return std::max(0.0, width()) * std::max(0.0, height()); }
    [[nodiscard]] R intersection(const R& o) const {
        return {std::max(llx, o.llx), std::max(lly, o.lly), std::min(urx, o.urx), std::min(ury, o.ury)};
    }
    [[nodiscard]] double overlapArea(const R& o) const { return intersection(o).area(); }
};

R moduleRect(double cx, double cy, double w, double h) {
    return {cx - w * 0.5, cy - h * 0.5, cx + w * 0.5, cy + h * 0.5};
}

// transformOffset (PlacementDatabase.cpp:55-68).
void transformOffset(double x, double y, int orientation, double& ox, double& oy) {
    switch (orientation) {
        case 1: ox = -x; oy = -y; return;   // S
        case 2: ox = -y; oy = x; return;    // E
        case 3: ox = y; oy = -x; return;    // W
        case 4: ox = -x; oy = y; return;    // FN
        case 5: ox = x; oy = -y; return;    // FS
        case 6: ox = y; oy = x; return;     // FE
        case 7: ox = -y; oy = -x; return;   // FW
        default: ox = x; oy = y; return;    // N, Unknown
    }
}

int orientationOf(const mpgp_design& design, int module) {
    return design.module_orientation != nullptr ? design.module_orientation[module] : 0;
}

// DensityMap bin rectangles (Metrics.cpp:21-32).
struct Grid {
    R region;
    int columns, rows;
    double bin_width, bin_height;
    Grid(const R& r, int c, int rr) : region(r), columns(c), rows(rr) {
        bin_width = region.width() / static_cast<double>(columns);
        bin_height = region.height() / static_cast<double>(rows);
    }
    [[nodiscard]] R bin(int column, int row) const {
        const double left = region.llx + static_cast<double>(column) * bin_width;
        const double bottom = region.lly + static_cast<double>(row) * bin_height;
        return {left, bottom, left + bin_width, bottom + bin_height};
    }
    void span(const R& clipped, int& c0, int& c1, int& r0, int& r1) const {
        c0 = std::max(0, std::min(columns - 1, static_cast<int>(std::floor((clipped.llx - region.llx) / bin_width))));
        c1 = std::max(0, std::min(columns - 1,
                                  static_cast<int>(std::ceil((clipped.urx - region.llx) / bin_width) - 1.0)));
        r0 = std::max(0, std::min(rows - 1, static_cast<int>(std::floor((clipped.lly - region.lly) / bin_height))));
        r1 = std::max(0, std::min(rows - 1,
                                  static_cast<int>(std::ceil((clipped.ury - region.lly) / bin_height) - 1.0)));
    }
};

bool finite(double value) { return std::isfinite(value); }

// Host threads for a set-up step over `items` elements: one below `from`
// (small designs, many of which the batched and served forms set up at once),
// else up to eight.
Workers setupWorkers(std::size_t items, std::size_t from = std::size_t{1} << 17) {
    if (items < from) return Workers(1);
    return Workers(static_cast<int>(std::min(8u, std::max(1u, std::thread::hardware_concurrency()))));
}

// std::sort's result on several threads: pieces sorted apart, then merged
// pairwise (a sorted sequence of doubles is unique, so it is the same).
void sortAscending(std::vector<double>& values) {
    const Workers workers = setupWorkers(values.size(), std::size_t{1} << 16);
    const std::size_t pieces = static_cast<std::size_t>(workers.threads());
    if (pieces <= 1) {
        std::sort(values.begin(), values.end());
        return;
    }
    std::vector<std::size_t> bound(pieces + 1);
    for (std::size_t k = 0; k <= pieces; ++k) bound[k] = values.size() * k / pieces;
    const auto at = [&](std::size_t k) { return values.begin() + static_cast<std::ptrdiff_t>(bound[k]); };
    workers.run(pieces, [&](std::size_t k) { std::sort(at(k), at(k + 1)); });
    for (std::size_t width = 1; width < pieces; width *= 2) {
        const std::size_t merges = (pieces + 2 * width - 1) / (2 * width);
        workers.run(merges, [&](std::size_t m) {
            const std::size_t first = 2 * width * m;
            const std::size_t middle = std::min(first + width, pieces);
            const std::size_t last = std::min(first + 2 * width, pieces);
            if (middle < last) std::inplace_merge(at(first), at(middle), at(last));
        });
    }
}


// The first index in [0, count) at which `bad` holds, or count; the checks of
// long ranges run on several threads.
template <typename F>
std::size_t firstBad(std::size_t count, const F& bad) {
    std::atomic<std::size_t> first{count};
    setupWorkers(count).blocks(count, 65536, [&](std::size_t b, std::size_t e) {
        for (std::size_t i = b; i < e && i < first.load(std::memory_order_relaxed); ++i) {
            if (!bad(i)) continue;
            std::size_t seen = first.load(std::memory_order_relaxed);
            while (i < seen && !first.compare_exchange_weak(seen, i, std::memory_order_relaxed)) {
            }
            return;
        }
    });
    return first.load();
}

}  // namespace

void defaultOptions(mpgp_options& o) {
    std::memset(&o, 0, sizeof(o));
    o.iterations = 280;
    o.bins_x = 64;
    o.bins_y = 64;
    o.report_interval = 10;
    o.target_density = 0.85;
    o.maximum_bin_overflow = 0.10;
    o.initial_smoothing = 0.75;
    o.final_smoothing = 0.12;
    o.maximum_movement_in_bins = 0.22;
    o.penalty_growth = 1.035;
    o.optimizer = 1;
    o.maximum_backtracks = 6;
    o.backtracking_ratio = 0.5;
    o.armijo_coefficient = 1e-4;
    o.maximum_momentum = 0.92;
    o.initial_movement_in_bins = 0.12;
    o.objective_increase_for_density = 0.002;
    o.hpwl_growth_restart_threshold = 0.02;
    o.density_stall_threshold = 0.002;
    o.density_penalty_increase = 1.05;
    o.density_penalty_decrease = 0.88;
    o.minimum_density_penalty = 1e-4;
    o.maximum_density_penalty = 1e6;
    o.smoothing_overflow_exponent = 1.0;
    o.feasible_refinement_iterations = 12;
    o.maximum_fillers = 50000;
    o.seed = 2026;
    o.rudy_columns = 64;
    o.rudy_rows = 64;
    o.rudy_minimum_span_in_bins = 0.25;
    o.rudy_capacity_factor = 1.00;
    o.rudy_softplus_temperature = 0.10;
    o.rudy_penalty_model = MPGP_RUDY_DISABLED;
    o.rudy_validation_bins = 0;
    o.rudy_validation_capacity_factor = 1.50;
    o.routability_start_overflow = 0.20;
    o.routability_weight_scale = 0.20;
    o.routability_ramp_iterations = 24;
    o.density_field_boundary = 1;
    o.compute_backend = MPGP_BACKEND_CUDA;
    o.cuda_device = 0;
    o.maximum_cuda_memory_bytes = 40ULL * 1024ULL * 1024ULL * 1024ULL;
}

void validateDesign(const mpgp_design& d) {
    require(d.module_count >= 0 && d.net_count >= 0 && d.pin_count >= 0 && d.row_count >= 0,
            "Design counts must be non-negative.");
    require(d.module_count == 0 || (d.module_width && d.module_height && d.module_x && d.module_y && d.module_flags),
            "Design module arrays are missing.");
    require(d.net_pin_start != nullptr, "Design net_pin_start is missing.");
    require(d.net_count == 0 || d.net_weight != nullptr, "Design net weights are missing.");
    require(d.pin_count == 0 || (d.pin_module && d.pin_offset_x && d.pin_offset_y), "Design pin arrays are missing.");
    require(d.row_count == 0 || (d.row_bottom && d.row_height && d.row_site_width && d.row_site_spacing &&
                                 d.row_x_start && d.row_site_count),
            "Design row arrays are missing.");
    require(d.net_pin_start[0] == 0 && d.net_pin_start[d.net_count] == d.pin_count,
            "net_pin_start must begin at 0 and end at pin_count.");
    require(d.pin_count < static_cast<int64_t>(std::numeric_limits<int32_t>::max()),
            "The engine indexes pins with 32-bit integers.");
    // The first net, then the first pin, that fails a check fails with that check's message.
    const std::size_t net = firstBad(static_cast<std::size_t>(d.net_count), [&](std::size_t n) {
        return !(d.net_pin_start[n + 1] >= d.net_pin_start[n]) || !finite(d.net_weight[n]);
    });
    if (net < static_cast<std::size_t>(d.net_count)) {
        require(d.net_pin_start[net + 1] >= d.net_pin_start[net], "net_pin_start must be non-decreasing.");
        require(finite(d.net_weight[net]), "Net weights must be finite.");
    }
    const std::size_t pin = firstBad(static_cast<std::size_t>(d.pin_count), [&](std::size_t p) {
        return !(d.pin_module[p] >= 0 && d.pin_module[p] < d.module_count) || !finite(d.pin_offset_x[p]) ||
               !finite(d.pin_offset_y[p]);
    });
    if (pin < static_cast<std::size_t>(d.pin_count)) {
        require(d.pin_module[pin] >= 0 && d.pin_module[pin] < d.module_count, "Pin refers to an unknown module.");
        require(finite(d.pin_offset_x[pin]) && finite(d.pin_offset_y[pin]), "Pin offsets must be finite.");
    }
    for (int32_t m = 0; m < d.module_count; ++m) {
        require(d.module_width[m] >= 0.0 && d.module_height[m] >= 0.0, "A module cannot have a negative size.");
        require(finite(d.module_width[m]) && finite(d.module_height[m]) && finite(d.module_x[m]) &&
                    finite(d.module_y[m]),
                "Module geometry must be finite.");
    }
    for (int32_t r = 0; r < d.row_count; ++r) {
        require(finite(d.row_bottom[r]) && finite(d.row_height[r]) && finite(d.row_site_spacing[r]) &&
                    finite(d.row_x_start[r]) && d.row_site_count[r] >= 0,
                "SiteRow values must be finite.");
    }
}

void validateOptions(const mpgp_options& o) {
    const bool bad =
        o.iterations <= 0 || o.bins_x < 2 || o.bins_y < 2 || !(o.target_density > 0.0) || o.target_density > 1.0 ||
        o.maximum_bin_overflow < 0.0 || o.initial_smoothing <= 0.0 || o.final_smoothing <= 0.0 ||
        o.maximum_movement_in_bins <= 0.0 || o.initial_movement_in_bins <= 0.0 || o.maximum_backtracks < 0 ||
        o.backtracking_ratio <= 0.0 || o.backtracking_ratio >= 1.0 || o.armijo_coefficient <= 0.0 ||
        o.armijo_coefficient >= 1.0 || o.maximum_momentum < 0.0 || o.maximum_momentum >= 1.0 ||
        o.density_penalty_increase <= 1.0 || o.density_penalty_decrease <= 0.0 || o.density_penalty_decrease >= 1.0 ||
        o.minimum_density_penalty <= 0.0 || o.maximum_density_penalty < o.minimum_density_penalty ||
        o.smoothing_overflow_exponent <= 0.0 || o.feasible_refinement_iterations <= 0 || o.rudy_columns < 2 ||
        o.rudy_rows < 2 || o.rudy_minimum_span_in_bins <= 0.0 || o.rudy_capacity_factor <= 0.0 ||
        o.rudy_softplus_temperature <= 0.0 || o.routability_start_overflow < 0.0 ||
        o.routability_weight_scale < 0.0 || o.routability_ramp_iterations <= 0 || o.rudy_validation_bins < 0 ||
        o.rudy_validation_bins == 1 || !finite(o.rudy_minimum_span_in_bins) || !finite(o.rudy_capacity_factor) ||
        !finite(o.rudy_softplus_temperature) || !finite(o.rudy_validation_capacity_factor) ||
        o.rudy_validation_capacity_factor <= 0.0 || !finite(o.routability_start_overflow) ||
        !finite(o.routability_weight_scale);
    const bool non_finite =
        !finite(o.target_density) || !finite(o.maximum_bin_overflow) || !finite(o.initial_smoothing) ||
        !finite(o.final_smoothing) || !finite(o.maximum_movement_in_bins) || !finite(o.penalty_growth) ||
        !finite(o.backtracking_ratio) || !finite(o.armijo_coefficient) || !finite(o.maximum_momentum) ||
        !finite(o.initial_movement_in_bins) || !finite(o.objective_increase_for_density) ||
        !finite(o.hpwl_growth_restart_threshold) || !finite(o.density_stall_threshold) ||
        !finite(o.density_penalty_increase) || !finite(o.density_penalty_decrease) ||
        !finite(o.minimum_density_penalty) || !finite(o.maximum_density_penalty) ||
        !finite(o.smoothing_overflow_exponent);
    require(!non_finite, "Global placement options contain an unknown mode or non-finite value.");
    require(!bad, "Adaptive global placement options are outside their valid range.");
    require(static_cast<std::size_t>(o.bins_x) <= (std::size_t{1} << 20) / static_cast<std::size_t>(o.bins_y),
            "Density grid exceeds the safe one-million-bin workspace limit.");
    require(static_cast<std::size_t>(o.rudy_columns) <= (std::size_t{1} << 20) / static_cast<std::size_t>(o.rudy_rows),
            "RUDY grid exceeds the safe one-million-bin workspace limit.");
    require(o.optimizer == 1, "The B200 engine implements the adaptive optimizer only.");
    require(o.density_field_boundary == 1, "The B200 engine implements the Neumann (DCT) field only.");
    require(o.maximum_cuda_memory_bytes > 0, "The device memory budget must be non-zero.");
}

DerivedDesign deriveDesign(const mpgp_design& d) {
    DerivedDesign out;
    if (d.row_count > 0) {
        std::vector<double> heights(d.row_height, d.row_height + d.row_count);
        std::sort(heights.begin(), heights.end());
        out.nominal_row_height = heights[heights.size() / 2U];
        const auto rowRect = [&](int r) {
            const double x_end = d.row_x_start[r] + static_cast<double>(d.row_site_count[r]) * d.row_site_spacing[r];
            return R{d.row_x_start[r], d.row_bottom[r], x_end, d.row_bottom[r] + d.row_height[r]};
        };
        R core = rowRect(0);
        for (int r = 0; r < d.row_count; ++r) {
            const R row = rowRect(r);
            core.llx = std::min(core.llx, row.llx);
            core.lly = std::min(core.lly, row.lly);
            core.urx = std::max(core.urx, row.urx);
            core.ury = std::max(core.ury, row.ury);
        }
        out.core = {core.llx, core.lly, core.urx, core.ury};
    }
    const std::size_t modules = static_cast<std::size_t>(d.module_count);
    const std::size_t pins = static_cast<std::size_t>(d.pin_count);
    out.is_fixed.resize(modules);
    out.is_macro.resize(modules);
    out.pin_count.assign(modules, 0);
    // Module flags and the movable list (in module order: each piece's movable
    // modules go after those of the pieces before it), then the pin counts (integer
    // sums, so the pieces' order does not matter), on up to eight host threads.
    const Workers workers = setupWorkers(modules + pins);
    const std::size_t pieces = static_cast<std::size_t>(workers.threads());
    const auto bound = [&](std::size_t k, std::size_t n) { return n * k / pieces; };
    std::vector<std::size_t> movable_in(pieces + 1, 0);
    workers.run(pieces, [&](std::size_t k) {
        std::size_t count = 0;
        for (std::size_t m = bound(k, modules); m < bound(k + 1, modules); ++m) {
            const bool terminal = (d.module_flags[m] & MPGP_MODULE_TERMINAL) != 0;
            const bool fixed = terminal || (d.module_flags[m] & MPGP_MODULE_FIXED) != 0;
            out.is_fixed[m] = fixed ? 1 : 0;
            out.is_macro[m] = (!terminal && out.nominal_row_height > kEpsilon &&
                               std::abs(d.module_height[m] - out.nominal_row_height) > kEpsilon)
                                  ? 1
                                  : 0;
            if (!fixed) ++count;
        }
        movable_in[k + 1] = count;
    });
    for (std::size_t k = 0; k < pieces; ++k) movable_in[k + 1] += movable_in[k];
    out.movable.resize(movable_in[pieces]);
    std::vector<std::vector<int32_t>> counts(pieces > 1 ? pieces : 0);
    workers.run(pieces, [&](std::size_t k) {
        std::size_t at = movable_in[k];
        for (std::size_t m = bound(k, modules); m < bound(k + 1, modules); ++m) {
            if (!out.is_fixed[m]) out.movable[at++] = static_cast<int32_t>(m);
        }
        if (pieces > 1) {
            std::vector<int32_t>& mine = counts[k];
            mine.assign(modules, 0);
            for (std::size_t p = bound(k, pins); p < bound(k + 1, pins); ++p) ++mine[d.pin_module[p]];
        }
    });
    if (pieces <= 1) {
        for (std::size_t p = 0; p < pins; ++p) ++out.pin_count[d.pin_module[p]];
    } else {
        workers.run(pieces, [&](std::size_t k) {
            for (std::size_t m = bound(k, modules); m < bound(k + 1, modules); ++m) {
                int32_t sum = 0;
                for (std::size_t j = 0; j < pieces; ++j) sum += counts[j][m];
                out.pin_count[m] = sum;
            }
        });
    }
    return out;
}

void staticDensity(const mpgp_design& d, const DerivedDesign& derived, int bins_x, int bins_y, double,
                   std::vector<double>& fixed, std::vector<double>& dark) {
    const R region{derived.core.llx, derived.core.lly, derived.core.urx, derived.core.ury};
    require(region.width() >= -kEpsilon && region.height() >= -kEpsilon && region.area() > kEpsilon,
            "DensityMap requires a valid region, positive dimensions, and target density.");
    const Grid grid(region, bins_x, bins_y);
    const std::size_t count = static_cast<std::size_t>(bins_x) * static_cast<std::size_t>(bins_y);
    fixed.assign(count, 0.0);
    dark.assign(count, 0.0);
    // setPlaceableRegions (Metrics.cpp:42-72).
    if (d.row_count > 0) {
        for (int row = 0; row < bins_y; ++row) {
            for (int column = 0; column < bins_x; ++column) {
                dark[static_cast<std::size_t>(row * bins_x + column)] = grid.bin(column, row).area();
            }
        }
        for (int r = 0; r < d.row_count; ++r) {
            const double x_end = d.row_x_start[r] + static_cast<double>(d.row_site_count[r]) * d.row_site_spacing[r];
            const R rect{d.row_x_start[r], d.row_bottom[r], x_end, d.row_bottom[r] + d.row_height[r]};
            const R clipped = rect.intersection(region);
            if (clipped.area() <= kEpsilon) continue;
            int c0, c1, r0, r1;
            grid.span(clipped, c0, c1, r0, r1);
            for (int row = r0; row <= r1; ++row) {
                for (int column = c0; column <= c1; ++column) {
                    dark[static_cast<std::size_t>(row * bins_x + column)] -= clipped.overlapArea(grid.bin(column, row));
                }
            }
        }
        for (int row = 0; row < bins_y; ++row) {
            for (int column = 0; column < bins_x; ++column) {
                double& value = dark[static_cast<std::size_t>(row * bins_x + column)];
                const double tolerance = std::max(1.0, grid.bin(column, row).area()) * 1e-10;
                require(!(value < -tolerance), "Overlapping SiteRows cannot define a density placeable-area mask.");
                value = std::max(0.0, value);
            }
        }
    }
    // Fixed modules into the Fixed layer (addRectangle, Metrics.cpp:74-99).
    for (int32_t m = 0; m < d.module_count; ++m) {
        if (!derived.is_fixed[m]) continue;
        const R clipped = moduleRect(d.module_x[m], d.module_y[m], d.module_width[m], d.module_height[m])
                              .intersection(region);
        if (clipped.area() <= kEpsilon) continue;
        int c0, c1, r0, r1;
        grid.span(clipped, c0, c1, r0, r1);
        for (int row = r0; row <= r1; ++row) {
            for (int column = c0; column <= c1; ++column) {
                const double area = clipped.overlapArea(grid.bin(column, row));
                if (area <= kEpsilon) continue;
                fixed[static_cast<std::size_t>(row * bins_x + column)] += area;
            }
        }
    }
}

std::vector<Filler> createFillers(const mpgp_design& d, const DerivedDesign& derived, const std::vector<double>& fixed,
                                  const std::vector<double>& dark, int, int, const mpgp_options& options) {
    const R core{derived.core.llx, derived.core.lly, derived.core.urx, derived.core.ury};
    double standard_cell_area = 0.0;
    double macro_area = 0.0;
    std::vector<double> areas;
    areas.reserve(derived.movable.size());
    for (const int32_t m : derived.movable) {
        const double area =
            moduleRect(d.module_x[m], d.module_y[m], d.module_width[m], d.module_height[m]).intersection(core).area();
        if (derived.is_macro[m]) {
            macro_area += area;
        } else {
            standard_cell_area += area;
        }
        if (area > kEpsilon) areas.push_back(area);
    }
    // static_density.metrics(false).total_charge_area (Metrics.cpp:101-119 with Metrics.hpp:25-29).
    double static_charge_area = 0.0;
    const double t = options.target_density;
    for (std::size_t index = 0; index < fixed.size(); ++index) {
        const double scaled_area = fixed[index] + 0.0 + dark[index] + 0.0;
        static_charge_area += 0.0 + t * scaled_area;
    }
    const double movable_charge_area = standard_cell_area + t * macro_area;
    const double required_filler_charge_area =
        std::max(0.0, t * core.area() - static_charge_area - movable_charge_area);
    const double filler_area = required_filler_charge_area / std::max(t, kEpsilon);
    if (filler_area <= kEpsilon || areas.empty() || options.maximum_fillers == 0U) return {};

    sortAscending(areas);
    const std::size_t lower = areas.size() / 10U;
    const std::size_t upper = std::max(lower + 1U, areas.size() - areas.size() / 10U);
    const double representative_area =
        std::accumulate(areas.begin() + static_cast<std::ptrdiff_t>(lower),
                        areas.begin() + static_cast<std::ptrdiff_t>(upper), 0.0) /
        static_cast<double>(upper - lower);
    const std::size_t count = std::min<std::size_t>(
        static_cast<std::size_t>(options.maximum_fillers),
        std::max<std::size_t>(1U, static_cast<std::size_t>(std::ceil(filler_area / std::max(representative_area, kEpsilon)))));
    const double area_per_filler = filler_area / static_cast<double>(count);
    const double aspect = std::max(core.width() / core.height(), 0.1);
    const double width = std::sqrt(area_per_filler * aspect);
    const double height = area_per_filler / std::max(width, kEpsilon);

    std::mt19937_64 generator(options.seed ^ 0x9e3779b97f4a7c15ULL);
    std::uniform_real_distribution<double> x_distribution(core.llx + width * 0.5, core.urx - width * 0.5);
    std::uniform_real_distribution<double> y_distribution(core.lly + height * 0.5, core.ury - height * 0.5);
    std::vector<Filler> fillers;
    fillers.reserve(count);
    for (std::size_t index = 0; index < count; ++index) {
        const double x = x_distribution(generator);
        const double y = y_distribution(generator);
        fillers.push_back({x, y, width, height});
    }
    return fillers;
}

// The pin CSR (buildHostLayout, CudaPlacementBackend.cu:815-837): movable pins keep
// their transformed offsets, static pins their absolute positions.
void buildProblemPins(const mpgp_design& d, const DerivedDesign& derived, Problem& problem) {
    std::vector<int32_t> module_particle(static_cast<std::size_t>(d.module_count), -1);
    for (std::size_t index = 0; index < derived.movable.size(); ++index) {
        module_particle[derived.movable[index]] = static_cast<int32_t>(index);
    }
    problem.net_weight.assign(d.net_weight, d.net_weight + d.net_count);
    problem.net_pin_start.assign(d.net_pin_start, d.net_pin_start + d.net_count + 1);
    const std::size_t count = static_cast<std::size_t>(d.pin_count);
    problem.pin_particle.resize(count);
    problem.pin_x.resize(count);
    problem.pin_y.resize(count);
    setupWorkers(count).blocks(count, 65536, [&](std::size_t b, std::size_t e) {
        for (std::size_t p = b; p < e; ++p) {
            const int32_t m = d.pin_module[p];
            double ox, oy;
            transformOffset(d.pin_offset_x[p], d.pin_offset_y[p], orientationOf(d, m), ox, oy);
            const int32_t particle = module_particle[m];
            problem.pin_particle[p] = particle;
            if (particle >= 0) {
                problem.pin_x[p] = ox;
                problem.pin_y[p] = oy;
            } else {
                problem.pin_x[p] = d.module_x[m] + ox;  // pinPosition (PlacementDatabase.cpp:138-142)
                problem.pin_y[p] = d.module_y[m] + oy;
            }
        }
    });
}

void buildProblemParticles(const mpgp_design& d, const DerivedDesign& derived, const mpgp_options& options,
                           Problem& problem, std::vector<Filler>& fillers) {
    problem.bins_x = options.bins_x;
    problem.bins_y = options.bins_y;
    problem.region = derived.core;
    problem.target_density = options.target_density;
    staticDensity(d, derived, options.bins_x, options.bins_y, options.target_density, problem.static_fixed,
                  problem.static_dark);
    fillers = createFillers(d, derived, problem.static_fixed, problem.static_dark, options.bins_x, options.bins_y,
                            options);

    const std::size_t movable = derived.movable.size();
    const std::size_t particles = movable + fillers.size();
    require(particles < static_cast<std::size_t>(std::numeric_limits<int32_t>::max()),
            "The engine indexes particles with 32-bit integers.");
    problem.particle_count = static_cast<int64_t>(particles);
    problem.movable_count = static_cast<int64_t>(movable);
    problem.width.resize(particles);
    problem.height.resize(particles);
    problem.layer.resize(particles);
    problem.charge.resize(particles);
    problem.pin_count.resize(particles);
    problem.precond_base.resize(particles);
    const double t = options.target_density;
    // initializePreconditioner (AdaptiveGlobalPlacer.cpp:358-375): the area sum in module order.
    double total_movable_area = 0.0;
    for (const int32_t m : derived.movable) total_movable_area += d.module_width[m] * d.module_height[m];
    const double average_movable_area =
        total_movable_area / static_cast<double>(std::max<std::size_t>(1U, movable));
    setupWorkers(particles).blocks(particles, 32768, [&](std::size_t b, std::size_t e) {
        for (std::size_t index = b; index < e; ++index) {
            if (index < movable) {
                const int32_t m = derived.movable[index];
                problem.width[index] = d.module_width[m];
                problem.height[index] = d.module_height[m];
                problem.layer[index] = derived.is_macro[m] ? MPGP_LAYER_MACRO : MPGP_LAYER_STANDARD;
                const double area = d.module_width[m] * d.module_height[m];
                problem.charge[index] = derived.is_macro[m] ? t * area : area;  // densityChargeArea (Support.cpp:105-107)
                problem.pin_count[index] = derived.pin_count[m];
            } else {
                const Filler& filler = fillers[index - movable];
                problem.width[index] = filler.width;
                problem.height[index] = filler.height;
                problem.layer[index] = MPGP_LAYER_FILLER;
                problem.charge[index] = t * (filler.width * filler.height);  // Support.cpp:109-111
                problem.pin_count[index] = 0;
            }
            const double area = problem.width[index] * problem.height[index];
            const double area_ratio = std::max(area / std::max(average_movable_area, kEpsilon), 0.1);
            const double pin_factor = std::sqrt(1.0 + static_cast<double>(problem.pin_count[index]));
            const double area_factor = 1.0 + std::sqrt(area_ratio);
            problem.precond_base[index] = 1.0 / (pin_factor * area_factor);
        }
    });
}

Problem buildProblem(const mpgp_design& d, const DerivedDesign& derived, const mpgp_options& options,
                     std::vector<Filler>& fillers) {
    // The pin CSR depends only on the movable list, so a second thread forms it while
    // this one builds the static layers, the fillers and the particle arrays.
    Problem problem;
    std::exception_ptr pins_error;
    std::thread pins([&] {
        try {
            buildProblemPins(d, derived, problem);
        } catch (...) {
            pins_error = std::current_exception();
        }
    });
    struct Join {
        std::thread& t;
        ~Join() {
            if (t.joinable()) t.join();
        }
    } join{pins};
    buildProblemParticles(d, derived, options, problem, fillers);
    pins.join();
    if (pins_error) std::rethrow_exception(pins_error);
    return problem;
}

Problem problemFromLayout(const mpgp_layout& l) {
    require(l.particle_count >= 0 && l.movable_count >= 0 && l.movable_count <= l.particle_count,
            "Layout particle counts are invalid.");
    require(l.particle_count < static_cast<int64_t>(std::numeric_limits<int32_t>::max()) &&
                l.pin_count < static_cast<int64_t>(std::numeric_limits<int32_t>::max()),
            "The engine indexes particles and pins with 32-bit integers.");
    require(l.bins_x >= 2 && l.bins_y >= 2 &&
                static_cast<std::size_t>(l.bins_x) <= (std::size_t{1} << 20) / static_cast<std::size_t>(l.bins_y),
            "Density grid exceeds the safe one-million-bin workspace limit.");
    require(l.target_density > 0.0 && l.target_density <= 1.0, "Target density must be in (0, 1].");
    require(l.region_urx - l.region_llx > 0.0 && l.region_ury - l.region_lly > 0.0, "The region must be non-empty.");
    require(l.net_pin_start != nullptr && l.net_pin_start[0] == 0 && l.net_pin_start[l.net_count] == l.pin_count,
            "net_pin_start must begin at 0 and end at pin_count.");
    Problem problem;
    const std::size_t particles = static_cast<std::size_t>(l.particle_count);
    problem.particle_count = l.particle_count;
    problem.movable_count = l.movable_count;
    problem.width.assign(l.particle_width, l.particle_width + particles);
    problem.height.assign(l.particle_height, l.particle_height + particles);
    problem.layer.assign(l.particle_layer, l.particle_layer + particles);
    problem.pin_count.assign(particles, 0);
    if (l.particle_pin_count != nullptr) problem.pin_count.assign(l.particle_pin_count, l.particle_pin_count + particles);
    problem.charge.resize(particles);
    for (std::size_t i = 0; i < particles; ++i) {
        require(problem.layer[i] >= 0 && problem.layer[i] <= 2, "Particle layer must be 0, 1 or 2.");
        const double area = problem.width[i] * problem.height[i];
        problem.charge[i] = problem.layer[i] == MPGP_LAYER_STANDARD ? area : l.target_density * area;
    }
    problem.net_weight.assign(l.net_weight, l.net_weight + l.net_count);
    problem.net_pin_start.assign(l.net_pin_start, l.net_pin_start + l.net_count + 1);
    const std::size_t pins = static_cast<std::size_t>(l.pin_count);
    problem.pin_particle.assign(l.pin_particle, l.pin_particle + pins);
    problem.pin_x.assign(l.pin_x, l.pin_x + pins);
    problem.pin_y.assign(l.pin_y, l.pin_y + pins);
    for (std::size_t p = 0; p < pins; ++p) {
        require(problem.pin_particle[p] < l.particle_count, "Pin refers to an unknown particle.");
    }
    problem.bins_x = l.bins_x;
    problem.bins_y = l.bins_y;
    problem.region = {l.region_llx, l.region_lly, l.region_urx, l.region_ury};
    problem.target_density = l.target_density;
    const std::size_t bins = static_cast<std::size_t>(l.bins_x) * static_cast<std::size_t>(l.bins_y);
    problem.static_fixed.assign(l.static_fixed_area, l.static_fixed_area + bins);
    problem.static_dark.assign(l.static_dark_area, l.static_dark_area + bins);
    return problem;
}

void randomPlacement(const mpgp_design& d, const DerivedDesign& derived, uint64_t seed, double* module_x,
                     double* module_y) {
    for (int32_t m = 0; m < d.module_count; ++m) {
        module_x[m] = d.module_x[m];
        module_y[m] = d.module_y[m];
    }
    const R core{derived.core.llx, derived.core.lly, derived.core.urx, derived.core.ury};
    std::mt19937_64 generator(seed);
    for (const int32_t m : derived.movable) {
        const double w = d.module_width[m];
        const double h = d.module_height[m];
        const double min_x = core.llx + w * 0.5;
        const double max_x = core.urx - w * 0.5;
        const double min_y = core.lly + h * 0.5;
        const double max_y = core.ury - h * 0.5;
        if (min_x <= max_x) {
            std::uniform_real_distribution<double> distribution(min_x, max_x);
            module_x[m] = distribution(generator);
        }
        if (min_y <= max_y) {
            std::uniform_real_distribution<double> distribution(min_y, max_y);
            module_y[m] = distribution(generator);
        }
        // clampModuleToCore (PlacementDatabase.cpp:202-213).
        if (core.area() <= kEpsilon) continue;
        const double lx = core.llx + w * 0.5, ux = core.urx - w * 0.5;
        const double ly = core.lly + h * 0.5, uy = core.ury - h * 0.5;
        module_x[m] = lx <= ux ? std::max(lx, std::min(module_x[m], ux)) : (core.llx + core.urx) * 0.5;
        module_y[m] = ly <= uy ? std::max(ly, std::min(module_y[m], uy)) : (core.lly + core.ury) * 0.5;
    }
}

}  // namespace mpgp
