// Native BookShelf reader: the records BookshelfParser::parseAux
// (src/io/BookshelfParser.cpp:313-348) builds into a PlacementDatabase, held as
// the flat arrays of mpgp_design plus the names, pin directions, row
// orientations and declared counts.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace mpgp {

struct Bookshelf {
    // Modules in .nodes order (PlacementDatabase::modules).
    std::vector<double> width, height, x, y;  // x, y: the centre (Module::setLowerLeft)
    std::vector<int32_t> flags;               // MPGP_MODULE_TERMINAL | MPGP_MODULE_FIXED
    std::vector<int32_t> orientation;         // Orientation enum order, 8 = Unknown
    std::string module_names;
    std::vector<int64_t> module_name_start;   // modules + 1 offsets into module_names
    // Nets in .nets order; pins net by net (PlacementDatabase::pins).
    std::vector<double> net_weight;
    std::vector<int64_t> net_pin_start;       // nets + 1
    std::string net_names;
    std::vector<int64_t> net_name_start;      // nets + 1
    std::vector<int32_t> pin_module;
    std::vector<double> pin_offset_x, pin_offset_y;
    std::vector<int8_t> pin_direction;        // PinDirection enum order: I, O, B, Unknown
    // SiteRows in .scl order.
    std::vector<double> row_bottom, row_height, row_site_width, row_site_spacing, row_x_start;
    std::vector<int64_t> row_site_count;
    std::vector<int32_t> row_orientation;
    // NumNodes, NumTerminals, NumNets, NumPins as declared; -1 when absent.
    int64_t declared[4] = {-1, -1, -1, -1};
};

// Reads the design named by a BookShelf .aux file.  Same grammar, records and
// error texts as the reference reader: its ParseError becomes Error with
// MPGP_ERR_PARSE, the database's std::invalid_argument (duplicate names,
// negative sizes) MPGP_ERR_INVALID_ARGUMENT.  `threads` <= 0 uses one per
// hardware thread, at most 32; the result does not depend on the thread count.
Bookshelf readBookshelf(const std::string& aux_path, int threads);

}  // namespace mpgp
