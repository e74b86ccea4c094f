// Detailed placement by four-cell window reordering, evaluated on the device:
// the reference's CUDA detailed-placement backend (tryRunCudaDetailedPlacement,
// src/placement/CudaDetailedPlacementBackend.hpp:13-16).
#pragma once

#include <string>

#include "mpgp.h"

namespace mpgp {

// Runs the passes on `design` with its positions and orientations, writing the
// result to module_x / module_y / module_orientation (module_count each;
// orientation may be NULL).  Returns false with `reason` where the reference
// backend declines (unsupported options, no device); throws on failures after
// the device work started.
bool detailedPlace(const mpgp_design& design, const int32_t* row_orientation, const mpgp_detailed_options& options,
                   double* module_x, double* module_y, int32_t* module_orientation, mpgp_detailed_result& result,
                   std::string& reason);

}  // namespace mpgp
