// Drop-in for the reference's BookShelf reader: myplacement::BookshelfParser::
// parseAux (include/myplacement/io/BookshelfParser.hpp:16-19) over libmpgp.so's
// native reader (mpgp_bookshelf_read, include/mpgp.h).  Linked in place of
// src/io/BookshelfParser.cpp it returns the PlacementDatabase the reference
// reader builds, and throws ParseError / std::invalid_argument with the same
// texts where the reference reader throws them.
#include <filesystem>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>

#include "mpgp.h"
#include "myplacement/io/BookshelfParser.hpp"

namespace myplacement {

PlacementDatabase BookshelfParser::parseAux(const std::filesystem::path& aux_path) const {
    mpgp_bookshelf* raw = nullptr;
    const int status = mpgp_bookshelf_read(aux_path.c_str(), 0, &raw);
    if (status != MPGP_OK) {
        const std::string message = mpgp_last_error();
        if (status == MPGP_ERR_PARSE) throw ParseError(message);
        if (status == MPGP_ERR_INVALID_ARGUMENT) throw std::invalid_argument(message);
        throw std::runtime_error(message);
    }
    const std::unique_ptr<mpgp_bookshelf, void (*)(mpgp_bookshelf*)> book(raw, mpgp_bookshelf_destroy);
    mpgp_bookshelf_view view;
    if (mpgp_bookshelf_get(book.get(), &view) != MPGP_OK) throw std::runtime_error(mpgp_last_error());
    const mpgp_design& d = view.design;

    PlacementDatabase database;
    database.modules.reserve(static_cast<std::size_t>(d.module_count));
    for (int32_t m = 0; m < d.module_count; ++m) {
        Module module;
        module.name.assign(view.module_names + view.module_name_start[m],
                           view.module_names + view.module_name_start[m + 1]);
        module.width = d.module_width[m];
        module.height = d.module_height[m];
        module.center = {d.module_x[m], d.module_y[m]};
        module.orientation = static_cast<Orientation>(d.module_orientation[m]);
        module.is_terminal = (d.module_flags[m] & MPGP_MODULE_TERMINAL) != 0;
        module.is_fixed = (d.module_flags[m] & MPGP_MODULE_FIXED) != 0;
        database.addModule(std::move(module));
    }
    for (int32_t r = 0; r < d.row_count; ++r) {
        SiteRow row;
        row.bottom = d.row_bottom[r];
        row.height = d.row_height[r];
        row.site_width = d.row_site_width[r];
        row.site_spacing = d.row_site_spacing[r];
        row.x_start = d.row_x_start[r];
        row.site_count = static_cast<std::size_t>(d.row_site_count[r]);
        row.orientation = static_cast<Orientation>(view.row_orientation[r]);
        database.rows.push_back(row);
    }
    database.pins.reserve(static_cast<std::size_t>(d.pin_count));
    database.nets.reserve(static_cast<std::size_t>(d.net_count));
    for (int32_t n = 0; n < d.net_count; ++n) {
        Net net;
        net.name.assign(view.net_names + view.net_name_start[n], view.net_names + view.net_name_start[n + 1]);
        net.weight = d.net_weight[n];
        const NetId id = database.addNet(std::move(net));
        for (int64_t p = d.net_pin_start[n]; p < d.net_pin_start[n + 1]; ++p) {
            Pin pin;
            pin.module = static_cast<ModuleId>(d.pin_module[p]);
            pin.net = id;
            pin.offset = {d.pin_offset_x[p], d.pin_offset_y[p]};
            pin.direction = static_cast<PinDirection>(view.pin_direction[p]);
            database.addPin(pin);
        }
    }
    const auto declared = [](int64_t value) {
        return value >= 0 ? std::optional<std::size_t>(static_cast<std::size_t>(value)) : std::nullopt;
    };
    database.declared_nodes = declared(view.declared_nodes);
    database.declared_terminals = declared(view.declared_terminals);
    database.declared_nets = declared(view.declared_nets);
    database.declared_pins = declared(view.declared_pins);
    database.refreshDerivedData();
    return database;
}

}  // namespace myplacement
