// Host-side setup of one global-placement problem: the engine's input model.
//
// A Problem is what the device engine needs: particles (movable modules in
// module order, then density fillers), the netlist flattened to pin CSR, the
// bin grid and the static density layers.  It is built either from the
// drop-in layout (mpgp_layout, i.e. what tryCreateCudaPlacementBackend
// receives) or from a whole design, in which case the reference's session
// setup is restated here operation for operation so that fillers, static
// layers and preconditioner are bit-identical to the reference's.
#pragma once

#include <cstdint>
#include <vector>

#include "mpgp.h"

namespace mpgp {

struct Rect2 {
    double llx = 0.0, lly = 0.0, urx = 0.0, ury = 0.0;
    [[nodiscard]] double width() const { return urx - llx; }
    [[nodiscard]] double height() const { return ury - lly; }
};

struct Problem {
    int64_t particle_count = 0;
    int64_t movable_count = 0;
    std::vector<double> width;         // P
    std::vector<double> height;        // P
    std::vector<int32_t> layer;        // P, MPGP_LAYER_*
    std::vector<double> charge;        // P, densityChargeArea
    std::vector<double> precond_base;  // P, empty for the drop-in backend
    std::vector<int32_t> pin_count;    // P (module pins; 0 for fillers)

    std::vector<double> net_weight;        // N
    std::vector<int64_t> net_pin_start;    // N + 1
    std::vector<int32_t> pin_particle;     // I, -1 for static pins
    std::vector<double> pin_x, pin_y;      // I: transformed offset, or absolute static position

    int bins_x = 0;
    int bins_y = 0;
    Rect2 region;
    double target_density = 0.0;
    std::vector<double> static_fixed;  // B
    std::vector<double> static_dark;   // B
};

// What refreshDerivedData (PlacementDatabase.cpp:162-200) derives from a design.
struct DerivedDesign {
    double nominal_row_height = 0.0;
    Rect2 core;
    std::vector<uint8_t> is_fixed;
    std::vector<uint8_t> is_macro;
    std::vector<int32_t> movable;    // module ids in module order
    std::vector<int32_t> pin_count;  // per module
};

DerivedDesign deriveDesign(const mpgp_design& design);

// Validates the design arrays (sizes, indices, finiteness).
void validateDesign(const mpgp_design& design);

// validateAdaptiveOptions (AdaptiveGlobalPlacer.cpp:413-454) plus the engine's own limits.
void validateOptions(const mpgp_options& options);

// The static density layers of DensityMap after initializeStaticDensity
// (GlobalPlacementSupport.cpp:21-30 -> Metrics.cpp:42-99).
void staticDensity(const mpgp_design& design, const DerivedDesign& derived, int bins_x, int bins_y,
                   double target_density, std::vector<double>& fixed, std::vector<double>& dark);

struct Filler {
    double x, y, width, height;
};

// createDensityFillers (GlobalPlacementSupport.cpp:52-103).
std::vector<Filler> createFillers(const mpgp_design& design, const DerivedDesign& derived,
                                  const std::vector<double>& fixed, const std::vector<double>& dark,
                                  int bins_x, int bins_y, const mpgp_options& options);

// The whole session setup (AdaptiveGlobalPlacer.cpp:114-126 plus buildHostLayout,
// CudaPlacementBackend.cu:784-839).  `fillers` receives the filler geometry.
Problem buildProblem(const mpgp_design& design, const DerivedDesign& derived, const mpgp_options& options,
                     std::vector<Filler>& fillers);
// Its two independent parts, which write disjoint members of `problem` and may run
// on two threads at once: the net and pin arrays (buildHostLayout's CSR part), and
// the grid, the static layers, the fillers and the particle arrays.
void buildProblemPins(const mpgp_design& design, const DerivedDesign& derived, Problem& problem);
void buildProblemParticles(const mpgp_design& design, const DerivedDesign& derived, const mpgp_options& options,
                           Problem& problem, std::vector<Filler>& fillers);

// The drop-in path: a Problem from an mpgp_layout.
Problem problemFromLayout(const mpgp_layout& layout);

// randomPlacement (InitialPlacer.cpp:102-121).
void randomPlacement(const mpgp_design& design, const DerivedDesign& derived, uint64_t seed, double* module_x,
                     double* module_y);

// Fills GlobalPlacementOptions defaults (GlobalPlacer.hpp:26-80).
void defaultOptions(mpgp_options& options);

}  // namespace mpgp
