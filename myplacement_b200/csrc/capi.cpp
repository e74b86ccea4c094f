// extern "C" entry points of libmpgp.so (include/mpgp.h).  No exception crosses
// this boundary: each call catches, records the message for mpgp_last_error()
// and returns the status of the failure.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "bookshelf.hpp"
#include "common.cuh"
#include "dct_tc.cuh"
#include "detailed.hpp"
#include "engine.cuh"
#include "mpgp.h"
#include "session.hpp"
#include "server.hpp"
#include "setup.hpp"

namespace {

thread_local std::string g_last_error;

int record(const std::exception& error) {
    g_last_error = error.what();
    if (const auto* e = dynamic_cast<const mpgp::Error*>(&error)) return e->status();
    if (dynamic_cast<const std::bad_alloc*>(&error) != nullptr) return MPGP_ERR_RUNTIME;
    if (dynamic_cast<const std::invalid_argument*>(&error) != nullptr) return MPGP_ERR_INVALID_ARGUMENT;
    return MPGP_ERR_RUNTIME;
}

template <typename F>
int guarded(F&& body) {
    try {
        g_last_error.clear();
        body();
        return MPGP_OK;
    } catch (const std::exception& error) {
        return record(error);
    } catch (...) {
        g_last_error = "unknown failure";
        return MPGP_ERR_RUNTIME;
    }
}

}  // namespace

struct mpgp_backend {
    std::unique_ptr<mpgp::Engine> engine;
    double2* wire = nullptr;
    double2* density = nullptr;
    double2* rudy = nullptr;
    int rudy_columns = 0, rudy_rows = 0;
    int64_t particles = 0;
    std::vector<double2> host;
};

struct mpgp_session {
    std::unique_ptr<mpgp::Session> session;
};

struct mpgp_server {
    std::unique_ptr<mpgp::Server> server;
};

struct mpgp_bookshelf {
    mpgp::Bookshelf book;
};

struct mpgp_setup {
    mpgp::DerivedDesign derived;
    mpgp::Problem problem;
    std::vector<mpgp::Filler> fillers;
};

extern "C" {

int mpgp_compiled(void) { return 1; }

int mpgp_abi_version(void) { return MPGP_ABI_VERSION; }

const char* mpgp_last_error(void) { return g_last_error.c_str(); }

void mpgp_options_default(mpgp_options* options) {
    if (options != nullptr) mpgp::defaultOptions(*options);
}

int mpgp_backend_create(const mpgp_layout* layout, int device, uint64_t maximum_bytes, mpgp_backend** out,
                        char* reason, size_t reason_capacity) {
    const auto write_reason = [&](const std::string& text) {
        if (reason != nullptr && reason_capacity > 0) {
            const std::size_t n = std::min(text.size(), reason_capacity - 1);
            std::memcpy(reason, text.data(), n);
            reason[n] = '\0';
        }
    };
    write_reason("");
    if (out == nullptr || layout == nullptr) {
        g_last_error = "mpgp_backend_create requires a layout and an output handle.";
        write_reason(g_last_error);
        return MPGP_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    // The factory's recoverable failures (CudaPlacementBackend.cu:1156-1216): no
    // device, an absent requested device, or a zero budget give a reason.
    int device_count = 0;
    const cudaError_t status = cudaGetDeviceCount(&device_count);
    if (status != cudaSuccess || device_count <= 0) {
        g_last_error = std::string("CUDA device discovery failed: ") + cudaGetErrorString(status);
        write_reason(g_last_error);
        return MPGP_ERR_UNAVAILABLE;
    }
    if (device < 0 || device >= device_count) {
        g_last_error = "Requested CUDA device does not exist on this host.";
        write_reason(g_last_error);
        return MPGP_ERR_UNAVAILABLE;
    }
    if (maximum_bytes == 0) {
        g_last_error = "CUDA memory limit leaves no allocatable device memory.";
        write_reason(g_last_error);
        return MPGP_ERR_UNAVAILABLE;
    }
    const int rc = guarded([&] {
        auto backend = std::make_unique<mpgp_backend>();
        const mpgp::Problem problem = mpgp::problemFromLayout(*layout);
        backend->engine = std::make_unique<mpgp::Engine>(problem, device, maximum_bytes);
        backend->particles = problem.particle_count;
        backend->wire = backend->engine->newParticleArray("wire gradients");
        backend->density = backend->engine->newParticleArray("density gradients");
        backend->host.resize(static_cast<std::size_t>(problem.particle_count));
        *out = backend.release();
    });
    if (rc != MPGP_OK) {
        write_reason(g_last_error);
        // A creation failure is recoverable for the caller (auto falls back to the CPU).
        return rc == MPGP_ERR_INVALID_ARGUMENT ? rc : MPGP_ERR_UNAVAILABLE;
    }
    return MPGP_OK;
}

int mpgp_backend_evaluate(mpgp_backend* b, const double* positions, double smoothing, int calculate_gradient,
                          mpgp_evaluation* out, double* wire_gradient, double* density_gradient) {
    return guarded([&] {
        mpgp::require(b != nullptr && out != nullptr, "mpgp_backend_evaluate requires a backend and an output.");
        mpgp::require(std::isfinite(smoothing) && smoothing > 0.0,
                      "CUDA global placement requires positive finite smoothing.");
        mpgp::require(b->particles == 0 || positions != nullptr, "CUDA placement positions are missing.");
        mpgp::require(!calculate_gradient || b->particles == 0 || (wire_gradient != nullptr && density_gradient != nullptr),
                      "Gradient outputs are missing.");
        mpgp::Engine& e = *b->engine;
        mpgp::checkCuda(cudaSetDevice(e.device()), "Select CUDA device for evaluation");
        const std::size_t bytes = sizeof(double2) * static_cast<std::size_t>(b->particles);
        for (int64_t i = 0; i < 2 * b->particles; ++i) {
            if (!std::isfinite(positions[i])) {
                mpgp::fail(MPGP_ERR_NON_FINITE, "CUDA placement positions must be finite.");
            }
        }
        if (b->particles > 0) {
            mpgp::checkCuda(cudaMemcpyAsync(e.scratchPositions(), positions, bytes, cudaMemcpyHostToDevice, e.stream()),
                      "Upload CUDA particle positions");
        }
        mpgp::EvalRequest q;
        q.mode = mpgp::kGiven;
        q.positions = e.scratchPositions();
        q.smoothing = smoothing;
        q.gradient = calculate_gradient != 0;
        q.wire_out = b->wire;
        q.density_out = b->density;
        const mpgp::EvalScalars& s = e.evaluate(q);
        out->hpwl = s.v[mpgp::kHpwl];
        out->smooth_wirelength = s.v[mpgp::kSmooth];
        out->electrostatic_energy = e.energy(s);
        e.densityMetrics(s, true, out->optimizer_density);
        e.densityMetrics(s, false, out->design_density);
        if (calculate_gradient && b->particles > 0) {
            mpgp::checkCuda(cudaMemcpyAsync(wire_gradient, b->wire, bytes, cudaMemcpyDeviceToHost, e.stream()),
                      "Download CUDA wire gradients");
            mpgp::checkCuda(cudaMemcpyAsync(density_gradient, b->density, bytes, cudaMemcpyDeviceToHost, e.stream()),
                      "Download CUDA density gradients");
            mpgp::checkCuda(cudaStreamSynchronize(e.stream()), "Synchronize CUDA placement evaluation");
        }
        if (!std::isfinite(out->smooth_wirelength) || !std::isfinite(out->hpwl) ||
            !std::isfinite(out->electrostatic_energy)) {
            mpgp::fail(MPGP_ERR_NON_FINITE, "CUDA global-placement evaluation produced a non-finite metric.");
        }
    });
}

int mpgp_backend_set_stall_probe(mpgp_backend* b, int64_t polls) {
    return guarded([&] {
        mpgp::require(b != nullptr, "mpgp_backend_set_stall_probe requires a backend.");
        mpgp::require(polls >= 0, "The probe's poll count must be non-negative.");
        b->engine->setStallProbe(polls);
    });
}

int mpgp_backend_device(const mpgp_backend* b) { return b != nullptr ? b->engine->device() : -1; }

uint64_t mpgp_backend_reserved_bytes(const mpgp_backend* b) { return b != nullptr ? b->engine->reservedBytes() : 0; }

void mpgp_backend_destroy(mpgp_backend* b) {
    if (b == nullptr) return;
    cudaSetDevice(b->engine->device());
    delete b;
}

int mpgp_backend_density_layers(mpgp_backend* b, int64_t* movable, int64_t* macro, int64_t* filler) {
    return guarded([&] {
        mpgp::require(b != nullptr, "A backend is required.");
        mpgp::checkCuda(cudaSetDevice(b->engine->device()), "Select CUDA device");
        b->engine->depositLayers(b->engine->scratchPositions(), movable, macro, filler);
    });
}

int mpgp_backend_field_solve(mpgp_backend* b, const double* deviation, double* potential, double* field_x,
                             double* field_y) {
    return guarded([&] {
        mpgp::require(b != nullptr && deviation != nullptr, "A backend and a deviation map are required.");
        mpgp::checkCuda(cudaSetDevice(b->engine->device()), "Select CUDA device");
        b->engine->fieldSolve(deviation, potential, field_x, field_y);
    });
}

int mpgp_backend_rudy(mpgp_backend* b, const mpgp_options* options, const double* positions,
                      double horizontal_capacity, double vertical_capacity, int calculate_gradient, double* metrics,
                      double* energy, double* gradient) {
    return guarded([&] {
        mpgp::require(b != nullptr && options != nullptr && metrics != nullptr,
                      "A backend, RUDY options and a metrics output are required.");
        mpgp::require(options->rudy_columns > 0 && options->rudy_rows > 0 &&
                          std::isfinite(options->rudy_minimum_span_in_bins) && options->rudy_minimum_span_in_bins > 0.0 &&
                          std::isfinite(options->rudy_softplus_temperature) && options->rudy_softplus_temperature > 0.0,
                      "RUDY evaluation requires a positive finite grid configuration and penalty model.");
        mpgp::require(static_cast<uint64_t>(options->rudy_columns) * static_cast<uint64_t>(options->rudy_rows) <=
                          1000000ULL,
                      "RUDY grid exceeds the safe one-million-bin workspace limit.");
        mpgp::require(options->rudy_penalty_model >= MPGP_RUDY_DISABLED && options->rudy_penalty_model <= MPGP_RUDY_HINGE_L4,
                      "Unknown RUDY penalty model.");
        mpgp::require(b->particles == 0 || positions != nullptr, "CUDA placement positions are missing.");
        mpgp::require(!calculate_gradient || (horizontal_capacity > 0.0 && vertical_capacity > 0.0 &&
                                              energy != nullptr && (b->particles == 0 || gradient != nullptr)),
                      "A RUDY gradient needs positive capacities and its outputs.");
        mpgp::Engine& e = *b->engine;
        mpgp::checkCuda(cudaSetDevice(e.device()), "Select CUDA device");
        if (b->rudy_columns == 0) {
            mpgp_options grid = *options;
            grid.rudy_validation_bins = 0;
            e.enableRudy(grid);
            b->rudy = e.newParticleArray("RUDY gradients");
            b->rudy_columns = options->rudy_columns;
            b->rudy_rows = options->rudy_rows;
        }
        mpgp::require(b->rudy_columns == options->rudy_columns && b->rudy_rows == options->rudy_rows &&
                          e.rudyMinimumSpan() == options->rudy_minimum_span_in_bins,
                      "The backend's RUDY grid is fixed by its first use.");
        e.setRudyModel(options->rudy_penalty_model, options->rudy_softplus_temperature);
        const std::size_t bytes = sizeof(double2) * static_cast<std::size_t>(b->particles);
        if (b->particles > 0) {
            mpgp::checkCuda(cudaMemcpyAsync(e.scratchPositions(), positions, bytes, cudaMemcpyHostToDevice, e.stream()),
                            "Upload CUDA particle positions");
        }
        e.setRudyCapacity(false, horizontal_capacity, vertical_capacity);
        const mpgp::RudyReport r = e.rudyEvaluate(e.scratchPositions(), false);
        const double values[10] = {r.horizontal_total, r.vertical_total, r.horizontal_mean, r.vertical_mean,
                                   r.horizontal_capacity, r.vertical_capacity, r.proxy_overflow,
                                   r.maximum_utilization, r.p95_utilization, r.energy};
        std::copy(values, values + 10, metrics);
        if (calculate_gradient) {
            mpgp::EvalRequest q;
            q.mode = mpgp::kGiven;
            q.positions = e.scratchPositions();
            q.smoothing = 1.0;
            q.gradient = true;
            q.wire_out = b->wire;
            q.density_out = b->density;
            q.rudy_out = b->rudy;
            q.rudy = true;
            q.rudy_weight = 1.0;
            const mpgp::EvalScalars& s = e.evaluate(q);
            *energy = s.v[mpgp::kRudyEnergy];
            if (b->particles > 0) {
                mpgp::checkCuda(cudaMemcpyAsync(gradient, b->rudy, bytes, cudaMemcpyDeviceToHost, e.stream()),
                                "Download RUDY gradients");
                mpgp::checkCuda(cudaStreamSynchronize(e.stream()), "Synchronize RUDY evaluation");
            }
        }
    });
}

int mpgp_wirelength_noalloc(const double* positions, const int32_t* net_pin_start, const int32_t* pin_particle,
                            const double* pin_xy, const double* net_weight, int32_t net_count, int32_t pin_count,
                            const int32_t* particle_pin_start, const int32_t* particle_pins,
                            int32_t particle_count, double smoothing, double* wire_gradient, double* totals,
                            void* stream) {
    return guarded([&] {
        mpgp::NoAllocWirelengthArgs args{positions,          net_pin_start, pin_particle,   pin_xy,
                                         net_weight,         net_count,     pin_count,      particle_pin_start,
                                         particle_pins,      particle_count, smoothing,     wire_gradient,
                                         totals,             stream};
        mpgp::launchWirelengthNoAlloc(args);
    });
}

int mpgp_bookshelf_read(const char* aux_path, int32_t threads, mpgp_bookshelf** out) {
    return guarded([&] {
        mpgp::require(aux_path != nullptr && out != nullptr, "Arguments are required.");
        *out = nullptr;
        auto b = std::make_unique<mpgp_bookshelf>();
        b->book = mpgp::readBookshelf(aux_path, threads);
        *out = b.release();
    });
}

int mpgp_bookshelf_get(const mpgp_bookshelf* b, mpgp_bookshelf_view* view) {
    return guarded([&] {
        mpgp::require(b != nullptr && view != nullptr, "Arguments are required.");
        const mpgp::Bookshelf& k = b->book;
        *view = mpgp_bookshelf_view{};
        mpgp_design& d = view->design;
        d.module_count = static_cast<int32_t>(k.width.size());
        d.module_width = k.width.data();
        d.module_height = k.height.data();
        d.module_x = k.x.data();
        d.module_y = k.y.data();
        d.module_flags = k.flags.data();
        d.module_orientation = k.orientation.data();
        d.net_count = static_cast<int32_t>(k.net_weight.size());
        d.net_weight = k.net_weight.data();
        d.net_pin_start = k.net_pin_start.data();
        d.pin_count = static_cast<int64_t>(k.pin_module.size());
        d.pin_module = k.pin_module.data();
        d.pin_offset_x = k.pin_offset_x.data();
        d.pin_offset_y = k.pin_offset_y.data();
        d.row_count = static_cast<int32_t>(k.row_bottom.size());
        d.row_bottom = k.row_bottom.data();
        d.row_height = k.row_height.data();
        d.row_site_width = k.row_site_width.data();
        d.row_site_spacing = k.row_site_spacing.data();
        d.row_x_start = k.row_x_start.data();
        d.row_site_count = k.row_site_count.data();
        view->module_names = k.module_names.data();
        view->module_name_start = k.module_name_start.data();
        view->net_names = k.net_names.data();
        view->net_name_start = k.net_name_start.data();
        view->pin_direction = k.pin_direction.data();
        view->row_orientation = k.row_orientation.data();
        view->declared_nodes = k.declared[0];
        view->declared_terminals = k.declared[1];
        view->declared_nets = k.declared[2];
        view->declared_pins = k.declared[3];
    });
}

void mpgp_bookshelf_destroy(mpgp_bookshelf* b) { delete b; }

void mpgp_detailed_options_default(mpgp_detailed_options* options) {
    if (options == nullptr) return;
    // DetailedPlacementOptions (DetailedPlacer.hpp:23-44) with the window reorder
    // selected and device 0.
    options->method = MPGP_DETAILED_WINDOW_REORDER;
    options->passes = 2;
    options->window_size = 4;
    options->cuda_device = 0;
    options->maximum_net_degree = 64;
    options->improvement_epsilon = 1e-9;
    options->maximum_cuda_memory_bytes = 2ULL * 1024ULL * 1024ULL * 1024ULL;
}

int mpgp_detailed_place(const mpgp_design* design, const int32_t* row_orientation,
                        const mpgp_detailed_options* options, double* module_x, double* module_y,
                        int32_t* module_orientation, mpgp_detailed_result* result, char* reason,
                        size_t reason_capacity) {
    std::string why;
    const int status = guarded([&] {
        mpgp::require(design != nullptr && options != nullptr && module_x != nullptr && module_y != nullptr &&
                          result != nullptr,
                      "Arguments are required.");
        mpgp_detailed_result out{};
        if (!mpgp::detailedPlace(*design, row_orientation, *options, module_x, module_y, module_orientation, out,
                                 why)) {
            mpgp::fail(MPGP_ERR_UNAVAILABLE, why);
        }
        *result = out;
    });
    if (status != MPGP_OK && reason != nullptr && reason_capacity > 0) {
        const std::size_t n = std::min(g_last_error.size(), reason_capacity - 1);
        std::memcpy(reason, g_last_error.data(), n);
        reason[n] = '\0';
    }
    return status;
}

int mpgp_random_placement(const mpgp_design* design, uint64_t seed, double* module_x, double* module_y) {
    return guarded([&] {
        mpgp::require(design != nullptr && module_x != nullptr && module_y != nullptr, "Arguments are required.");
        mpgp::validateDesign(*design);
        const mpgp::DerivedDesign derived = mpgp::deriveDesign(*design);
        mpgp::randomPlacement(*design, derived, seed, module_x, module_y);
    });
}

int mpgp_session_create(const mpgp_design* design, const mpgp_options* options, mpgp_session** out) {
    return guarded([&] {
        mpgp::require(design != nullptr && options != nullptr && out != nullptr, "Arguments are required.");
        *out = nullptr;
        auto s = std::make_unique<mpgp_session>();
        s->session = std::make_unique<mpgp::Session>(*design, *options);
        *out = s.release();
    });
}

int mpgp_session_step(mpgp_session* s, int32_t iterations, int32_t* completed, int32_t* done) {
    return guarded([&] {
        mpgp::require(s != nullptr && iterations >= 0, "A session and a non-negative iteration count are required.");
        const bool finished = s->session->step(iterations, completed);
        if (done != nullptr) *done = finished ? 1 : 0;
    });
}

int mpgp_session_finish(mpgp_session* s, double* module_x, double* module_y, mpgp_result* result,
                        mpgp_history_row* history, int32_t history_capacity) {
    return guarded([&] {
        mpgp::require(s != nullptr, "A session is required.");
        s->session->finish(module_x, module_y, result, history, history_capacity);
    });
}

int mpgp_setup_create(const mpgp_design* design, const mpgp_options* options, mpgp_setup** out) {
    return guarded([&] {
        mpgp::require(design != nullptr && options != nullptr && out != nullptr, "Arguments are required.");
        *out = nullptr;
        mpgp::validateDesign(*design);
        mpgp::validateOptions(*options);
        auto setup = std::make_unique<mpgp_setup>();
        setup->derived = mpgp::deriveDesign(*design);
        setup->problem = mpgp::buildProblem(*design, setup->derived, *options, setup->fillers);
        *out = setup.release();
    });
}

int mpgp_setup_particles(const mpgp_setup* s, int64_t* particle_count, int64_t* movable_count, double* x, double* y,
                         double* width, double* height, int32_t* layer, double* preconditioner) {
    return guarded([&] {
        mpgp::require(s != nullptr, "A setup is required.");
        const mpgp::Problem& p = s->problem;
        if (particle_count != nullptr) *particle_count = p.particle_count;
        if (movable_count != nullptr) *movable_count = p.movable_count;
        const std::size_t movable = static_cast<std::size_t>(p.movable_count);
        for (int64_t i = 0; i < p.particle_count; ++i) {
            const std::size_t k = static_cast<std::size_t>(i);
            if (x != nullptr) x[i] = k < movable ? 0.0 : s->fillers[k - movable].x;
            if (y != nullptr) y[i] = k < movable ? 0.0 : s->fillers[k - movable].y;
            if (width != nullptr) width[i] = p.width[k];
            if (height != nullptr) height[i] = p.height[k];
            if (layer != nullptr) layer[i] = p.layer[k];
            if (preconditioner != nullptr) preconditioner[i] = p.precond_base[k];
        }
    });
}

int mpgp_setup_static_density(const mpgp_setup* s, double* fixed, double* dark) {
    return guarded([&] {
        mpgp::require(s != nullptr, "A setup is required.");
        if (fixed != nullptr) std::copy(s->problem.static_fixed.begin(), s->problem.static_fixed.end(), fixed);
        if (dark != nullptr) std::copy(s->problem.static_dark.begin(), s->problem.static_dark.end(), dark);
    });
}

void mpgp_setup_destroy(mpgp_setup* s) { delete s; }

int mpgp_session_positions(const mpgp_session* s, double* positions) {
    return guarded([&] {
        mpgp::require(s != nullptr && positions != nullptr, "A session and an output array are required.");
        s->session->currentPositions(positions);
    });
}

int mpgp_kernel_kind_count(void) { return mpgp::kKindCount; }

const char* mpgp_kernel_kind_name(int kind) { return mpgp::kernelKindName(kind); }

int mpgp_session_set_profiling(mpgp_session* s, uint32_t families) {
    return guarded([&] {
        mpgp::require(s != nullptr, "A session is required.");
        if (s->session->engine() != nullptr) s->session->engine()->setTiming(families);
    });
}

int mpgp_session_reset_kernel_stats(mpgp_session* s) {
    return guarded([&] {
        mpgp::require(s != nullptr, "A session is required.");
        if (s->session->engine() != nullptr) s->session->engine()->resetKernelStats();
    });
}

int mpgp_session_kernel_stats(const mpgp_session* s, int64_t* launches, double* milliseconds, int32_t capacity) {
    return guarded([&] {
        mpgp::require(s != nullptr, "A session is required.");
        const mpgp::Engine* engine = s->session->engine();
        for (int k = 0; k < std::min<int>(capacity, mpgp::kKindCount); ++k) {
            if (launches != nullptr) launches[k] = engine != nullptr ? engine->kernelStats().launches[k] : 0;
            if (milliseconds != nullptr) milliseconds[k] = engine != nullptr ? engine->kernelStats().milliseconds[k] : 0.0;
        }
    });
}

int mpgp_session_transfer_bytes(const mpgp_session* s, uint64_t* to_device, uint64_t* to_host) {
    return guarded([&] {
        mpgp::require(s != nullptr, "A session is required.");
        const mpgp::Engine* engine = s->session->engine();
        if (to_device != nullptr) *to_device = engine != nullptr ? engine->bytesToDevice() : 0;
        if (to_host != nullptr) *to_host = engine != nullptr ? engine->bytesToHost() : 0;
    });
}

int64_t mpgp_session_kernel_launches(const mpgp_session* s) { return s != nullptr ? s->session->launches() : 0; }

void* mpgp_session_stream(const mpgp_session* s) { return s != nullptr ? s->session->stream() : nullptr; }

void mpgp_session_destroy(mpgp_session* s) { delete s; }

int mpgp_global_place(const mpgp_design* design, const mpgp_options* options, double* module_x, double* module_y,
                      mpgp_result* result, mpgp_history_row* history, int32_t history_capacity) {
    return guarded([&] {
        mpgp::require(design != nullptr && options != nullptr && module_x != nullptr && module_y != nullptr,
                      "Arguments are required.");
        mpgp::Session session(*design, *options);
        while (!session.step(64, nullptr)) {
        }
        session.finish(module_x, module_y, result, history, history_capacity);
    });
}


int mpgp_estimate_bytes(const mpgp_design* design, const mpgp_options* options, uint64_t* bytes) {
    return guarded([&] {
        mpgp::require(design != nullptr && options != nullptr && bytes != nullptr, "Arguments are required.");
        *bytes = mpgp::estimateSessionBytes(*design, *options);
    });
}

int mpgp_server_create_mode(int device, uint64_t memory_budget_bytes, int32_t workers, int32_t batched,
                            mpgp_server** out) {
    return guarded([&] {
        mpgp::require(out != nullptr, "An output handle is required.");
        *out = nullptr;
        auto handle = std::make_unique<mpgp_server>();
        handle->server = std::make_unique<mpgp::Server>(device, memory_budget_bytes, workers, batched != 0);
        *out = handle.release();
    });
}

int mpgp_server_create(int device, uint64_t memory_budget_bytes, int32_t workers, mpgp_server** out) {
    return mpgp_server_create_mode(device, memory_budget_bytes, workers, 1, out);
}

int mpgp_server_submit(mpgp_server* s, const mpgp_design* design, const mpgp_options* options, int64_t* job) {
    return guarded([&] {
        mpgp::require(s != nullptr && design != nullptr && options != nullptr && job != nullptr,
                      "Arguments are required.");
        *job = s->server->submit(*design, *options);
    });
}

int mpgp_server_wait(mpgp_server* s, int64_t job, double timeout_seconds, int32_t* done) {
    return guarded([&] {
        mpgp::require(s != nullptr, "A server is required.");
        const bool finished = s->server->wait(job, timeout_seconds);
        if (done != nullptr) *done = finished ? 1 : 0;
    });
}

int mpgp_server_take(mpgp_server* s, int64_t job, double* module_x, double* module_y, mpgp_result* result,
                     mpgp_history_row* history, int32_t history_capacity, mpgp_job_stats* stats) {
    return guarded([&] {
        mpgp::require(s != nullptr, "A server is required.");
        s->server->take(job, module_x, module_y, result, history, history_capacity, stats);
    });
}

int mpgp_server_stats_get(const mpgp_server* s, mpgp_server_stats* stats) {
    return guarded([&] {
        mpgp::require(s != nullptr && stats != nullptr, "Arguments are required.");
        *stats = s->server->stats();
    });
}

void mpgp_server_destroy(mpgp_server* s) { delete s; }

int mpgp_tuning_set_splits(const int32_t* sizes, const int32_t* splits, int32_t count) {
    return guarded([&] {
        mpgp::require(count >= 0 && (count == 0 || (sizes != nullptr && splits != nullptr)),
                      "Sizes and splits are required.");
        mpgp::setTunedSplits(sizes, splits, count);
    });
}

int mpgp_tuning_get_splits(int32_t* sizes, int32_t* splits, int32_t capacity, int32_t* count) {
    return guarded([&] {
        mpgp::require(count != nullptr && capacity >= 0 && (capacity == 0 || (sizes != nullptr && splits != nullptr)),
                      "Output arrays are required.");
        *count = mpgp::tunedSplits(sizes, splits, capacity);
    });
}

int mpgp_batch_place(int32_t count, const mpgp_design* designs, const mpgp_options* options, int device,
                     int32_t workers, int32_t batched, uint64_t memory_budget_bytes, double* const* module_x,
                     double* const* module_y, mpgp_result* results, mpgp_job_stats* job_stats,
                     mpgp_server_stats* server_stats) {
    return guarded([&] {
        mpgp::require(count >= 0 && (count == 0 || (designs != nullptr && options != nullptr)),
                      "Designs and options are required.");
        mpgp::Server server(device, memory_budget_bytes, workers, batched != 0);
        std::vector<int64_t> ids(static_cast<std::size_t>(count));
        for (int32_t i = 0; i < count; ++i) ids[i] = server.submit(designs[i], options[i]);
        int first_failure = MPGP_OK;
        std::string message;
        for (int32_t i = 0; i < count; ++i) {
            server.wait(ids[i], -1.0);
            try {
                server.take(ids[i], module_x != nullptr ? module_x[i] : nullptr,
                            module_y != nullptr ? module_y[i] : nullptr, results != nullptr ? &results[i] : nullptr,
                            nullptr, 0, job_stats != nullptr ? &job_stats[i] : nullptr);
            } catch (const mpgp::Error& e) {
                if (first_failure == MPGP_OK) {
                    first_failure = e.status();
                    message = "job " + std::to_string(i) + ": " + e.what();
                }
            }
        }
        if (server_stats != nullptr) *server_stats = server.stats();
        if (first_failure != MPGP_OK) mpgp::fail(first_failure, message);
    });
}

}  // extern "C"
