// Device engine: allocation, static upload, and the launch sequence of one evaluation.
//
// One evaluation replaces CudaPlacementBackendImpl::evaluate
// (CudaPlacementBackend.cu:921-950) with, on one stream:
//   scatter (+ proposal / lookahead)  ->  wirelength  ->  metrics + source
//   -> DCT forward (2 contractions, spectral epilogue, Parseval energy)
//   [gradient: -> 2 x 2 inverse contractions -> fused field gather + combine]
//   -> scalar reduction
// and one 168-byte scalar read-back, instead of 14 blocking reductions and the
// position / gradient round trips of the reference.
#include "engine.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <atomic>
#include <thread>

#include "batch.hpp"
#include "common.cuh"
#include "ingest.cuh"

namespace mpgp {

cudaMemPool_t devicePool(int device) {
    constexpr int kMaxDevices = 64;
    static std::once_flag once[kMaxDevices];
    static cudaMemPool_t pools[kMaxDevices] = {};
    static cudaError_t status[kMaxDevices] = {};
    require(device >= 0 && device < kMaxDevices, "Device index out of range.");
    std::call_once(once[device], [device] {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        status[device] = cudaMemPoolCreate(&pools[device], &props);
        if (status[device] == cudaSuccess) {
            // Keep freed memory for the next session rather than returning it at every
            // synchronisation.
            uint64_t threshold = ~0ULL;
            status[device] = cudaMemPoolSetAttribute(pools[device], cudaMemPoolAttrReleaseThreshold, &threshold);
        }
    });
    checkCuda(status[device], "Create the device memory pool");
    return pools[device];
}

DeviceArena::~DeviceArena() {
    // The owner has synchronised every stream that used the arrays; the frees are
    // ordered on the legacy stream, which waits for no other non-blocking stream.
    for (void* p : blocks_) {
        if (pool_ != nullptr) {
            cudaFreeAsync(p, nullptr);
        } else {
            cudaFree(p);
        }
    }
}

void DeviceArena::bind(int device, cudaStream_t stream) {
    pool_ = devicePool(device);
    stream_ = stream;
}

void* DeviceArena::allocate(std::size_t bytes, const char* what) {
    bytes = std::max<std::size_t>(bytes, 16);
    bytes = (bytes + 255) & ~static_cast<std::size_t>(255);
    if (bytes > limit_ - std::min(limit_, reserved_)) {
        fail(MPGP_ERR_BUDGET, std::string("CUDA allocation budget exceeded while reserving ") + what +
                                  " (requested " + std::to_string(bytes) + " bytes, reserved " +
                                  std::to_string(reserved_) + " bytes, limit " + std::to_string(limit_) + " bytes).");
    }
    void* p = nullptr;
    if (pool_ != nullptr) {
        checkCuda(cudaMallocFromPoolAsync(&p, bytes, pool_, stream_), what);
    } else {
        checkCuda(cudaMalloc(&p, bytes), what);
    }
    blocks_.push_back(p);
    reserved_ += bytes;
    return p;
}

namespace {

// Bytes copied host -> device by upload() on this thread (the engine's setup traffic).
thread_local uint64_t g_uploaded_bytes = 0;

template <typename T>
void upload(T* device, const std::vector<T>& host, cudaStream_t stream) {
    if (!host.empty()) {
        g_uploaded_bytes += host.size() * sizeof(T);
        checkCuda(cudaMemcpyAsync(device, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice, stream),
                  "upload");
    }
}

}  // namespace

Engine::Engine(const Problem& p, int device, uint64_t budget_bytes, Batch* batch)
    : Engine(Grid{p.bins_x, p.bins_y, p.region, p.target_density}, device, budget_bytes, batch) {
    load(p);
}

Engine::Engine(const Grid& grid, int device, uint64_t budget_bytes, Batch* batch)
    : device_(device), batch_(batch), arena_(budget_bytes) {
    checkCuda(cudaSetDevice(device_), "Select CUDA device");
    if (batch_ != nullptr) {
        require(batch_->device() == device_, "A batch runs on one device.");
        stream_ = batch_->stream();  // every engine of a batch works on the batch's stream
        owns_stream_ = false;
    } else {
        checkCuda(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "Create engine stream");
        checkCuda(cudaStreamCreateWithFlags(&stream_wl_, cudaStreamNonBlocking), "Create wirelength stream");
    }
    arena_.bind(device_, stream_);
    checkCuda(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming), "Create fork event");
    checkCuda(cudaEventCreateWithFlags(&join_, cudaEventDisableTiming), "Create join event");
    bins_x_ = grid.bins_x;
    bins_y_ = grid.bins_y;
    bin_count_ = bins_x_ * bins_y_;
    region_ = grid.region;
    target_density_ = grid.target_density;
    bin_w_ = region_.width() / static_cast<double>(bins_x_);
    bin_h_ = region_.height() / static_cast<double>(bins_y_);
    bin_area_ = (std::max(0.0, region_.width()) * std::max(0.0, region_.height())) / static_cast<double>(bin_count_);
    const uint64_t uploaded_before = g_uploaded_bytes;
    buildBasis();
    h2d_bytes_ += g_uploaded_bytes - uploaded_before;
    // The reduction publishes the scalars and the error flag into mapped pinned
    // memory; the host polls it, with no copy or stream synchronisation on the
    // evaluation's critical path.
    checkCuda(cudaMallocHost(reinterpret_cast<void**>(&host_scalars_), sizeof(EvalScalars)), "pinned scalars");
    std::memset(host_scalars_, 0, sizeof(EvalScalars));
    const std::size_t slot_bytes = static_cast<std::size_t>(kRecords) * kRecordSlots * sizeof(unsigned long long);
    checkCuda(cudaHostAlloc(reinterpret_cast<void**>(&host_slots_), slot_bytes, cudaHostAllocMapped),
              "pinned evaluation record");
    std::memset(host_slots_, 0, slot_bytes);
}

void Engine::load(const Problem& p) {
    loadNets(p, p.movable_count);
    loadParticles(p);
}

void Engine::loadNets(const Problem& p, int64_t movable_count) {
    require(!nets_loaded_, "The engine's nets are loaded once.");
    movable_count_ = movable_count;
    const uint64_t uploaded_before = g_uploaded_bytes;
    buildNetLayout(p);
    h2d_bytes_ += g_uploaded_bytes - uploaded_before;
    nets_loaded_ = true;
}

void Engine::loadParticles(const Problem& p) {
    require(nets_loaded_, "The engine's nets are loaded before its particles.");
    require(p.bins_x == bins_x_ && p.bins_y == bins_y_, "The problem's grid is not the engine's.");
    require(p.movable_count == movable_count_, "The problem's movable count is not the one its nets were laid out for.");
    particle_count_ = p.particle_count;
    const uint64_t uploaded_before = g_uploaded_bytes;
    uploadStatic(p);
    allocateGroups();
    h2d_bytes_ += g_uploaded_bytes - uploaded_before;
    checkCuda(cudaStreamSynchronize(stream_), "Engine setup");
    if (batch_ != nullptr) {
        batch_->attach(this);
        attached_ = true;
    }
}

void Engine::leaveBatch() {
    if (batch_ != nullptr && attached_) {
        attached_ = false;
        batch_->detach(this);
    }
}

Engine::~Engine() {
    leaveBatch();
    if (stream_ != nullptr) {
        cudaStreamSynchronize(stream_);
        if (owns_stream_) cudaStreamDestroy(stream_);
    }
    if (stream_wl_ != nullptr) {
        cudaStreamSynchronize(stream_wl_);
        cudaStreamDestroy(stream_wl_);
    }
    if (fork_ != nullptr) cudaEventDestroy(fork_);
    if (join_ != nullptr) cudaEventDestroy(join_);
    if (host_scalars_ != nullptr) cudaFreeHost(host_scalars_);
    if (host_rudy_ != nullptr) cudaFreeHost(host_rudy_);
    if (host_error_ != nullptr) cudaFreeHost(host_error_);
    if (host_slots_ != nullptr) cudaFreeHost(host_slots_);
    for (cudaEvent_t e : events_) cudaEventDestroy(e);
}

void Engine::newParticleArrays(int count, double2** out, const char* what) {
    // Each array starts on a 256-byte boundary, like a separate allocation would.
    const std::size_t stride = ((static_cast<std::size_t>(std::max<int64_t>(1, particle_count_)) * sizeof(double2) +
                                 255) / 256) * 256 / sizeof(double2);
    double2* base = arena_.array<double2>(stride * static_cast<std::size_t>(count), what);
    checkCuda(cudaMemsetAsync(base, 0, stride * static_cast<std::size_t>(count) * sizeof(double2), stream_), what);
    for (int k = 0; k < count; ++k) out[k] = base + stride * static_cast<std::size_t>(k);
}

double2* Engine::newParticleArray(const char* what) {
    double2* p = arena_.array<double2>(static_cast<std::size_t>(std::max<int64_t>(1, particle_count_)), what);
    checkCuda(cudaMemsetAsync(p, 0, sizeof(double2) * std::max<int64_t>(1, particle_count_), stream_), what);
    return p;
}

void Engine::uploadStatic(const Problem& p) {
    const std::size_t n = static_cast<std::size_t>(std::max<int64_t>(1, particle_count_));
    std::vector<double2> size(static_cast<std::size_t>(particle_count_));
    std::vector<unsigned char> layer(static_cast<std::size_t>(particle_count_));
    for (int64_t i = 0; i < particle_count_; ++i) {
        size[i] = make_double2(p.width[i], p.height[i]);
        layer[i] = static_cast<unsigned char>(p.layer[i]);
    }
    size_ = arena_.array<double2>(n, "particle sizes");
    layer_ = arena_.array<unsigned char>(n, "particle layers");
    charge_ = arena_.array<double>(n, "particle charge areas");
    precond_ = arena_.array<double>(n, "preconditioner");
    scratch_positions_ = arena_.array<double2>(n, "uploaded positions");
    upload(size_, size, stream_);
    upload(layer_, layer, stream_);
    upload(charge_, p.charge, stream_);
    if (!p.precond_base.empty()) upload(precond_, p.precond_base, stream_);

    const std::size_t bins = static_cast<std::size_t>(bin_count_);
    layers_ = arena_.array<unsigned long long>(3 * bins, "fixed-point density layers");
    totals_ = arena_.array<unsigned long long>(4, "density layer totals");
    static_charge_ = arena_.array<double>(bins, "static charge");
    source_ = arena_.array<float>(bins, "density source");
    checkCuda(cudaMemsetAsync(layers_, 0, 3 * bins * sizeof(unsigned long long), stream_), "clear layers");
    checkCuda(cudaMemsetAsync(totals_, 0, 4 * sizeof(unsigned long long), stream_), "clear totals");
    {
        // t * (fixed + dark): the part of every bin's charge area that never moves.
        std::vector<double> static_charge(bins);
        for (std::size_t b = 0; b < bins; ++b) static_charge[b] = target_density_ * (p.static_fixed[b] + p.static_dark[b]);
        upload(static_charge_, static_charge, stream_);
        checkCuda(cudaStreamSynchronize(stream_), "static charge upload");  // the host vector leaves scope
    }
    // Static sums in bin order: DensityMap::metrics (Metrics.cpp:101-119) uses each
    // bin's own rectangle area for the placeable area.
    for (int row = 0; row < bins_y_; ++row) {
        for (int column = 0; column < bins_x_; ++column) {
            const std::size_t b = static_cast<std::size_t>(row) * bins_x_ + column;
            const double left = region_.llx + static_cast<double>(column) * bin_w_;
            const double bottom = region_.lly + static_cast<double>(row) * bin_h_;
            const double area = std::max(0.0, (left + bin_w_) - left) * std::max(0.0, (bottom + bin_h_) - bottom);
            static_fixed_sum_ += p.static_fixed[b];
            static_dark_sum_ += p.static_dark[b];
            static_placeable_sum_ += area - p.static_dark[b];
        }
    }
    scatter_blocks_ = ceilDiv(std::max<int64_t>(1, particle_count_), kThreads);
    gather_blocks_ = gatherBlocks(static_cast<int>(std::min<int64_t>(particle_count_, 1 << 30)));
    metrics_fused_ = metricsSplitFits(bins_x_);
    metrics_blocks_ = metrics_fused_ ? bins_y_ : std::min(ceilDiv(bin_count_, 2 * kThreads), 148 * 2);
    partials_sc_ = arena_.array<double>(2 * static_cast<std::size_t>(scatter_blocks_), "scatter partials");
    partials_m_ = arena_.array<double>(9 * static_cast<std::size_t>(metrics_blocks_), "metric partials");
    partials_g_ = arena_.array<double>(8 * static_cast<std::size_t>(gather_blocks_), "gather partials");
    scalars_ = arena_.array<double>(kScalarCount, "evaluation scalars");
    checkCuda(cudaMemsetAsync(scalars_, 0, kScalarCount * sizeof(double), stream_), "clear scalars");
}

void Engine::buildNetLayout(const Problem& p) {
    // The bucketed layout and the particle pin lists are built on the device
    // (ingest.cu); the host only turns the bucket sizes into the work list.
    const NetLayout layout = buildNetLayoutOnDevice(
        p, static_cast<int>(movable_count_),
        [this](std::size_t bytes, const char* what) { return arena_.allocate(bytes, what); },
        [this]() { return arena_.headroom(); }, stream_);
    pin_particle_ = layout.pin_particle;
    pin_offset_ = layout.pin_offset;
    static_pins_ = layout.static_pins;
    net_start_ = layout.net_start;
    net_weight_ = layout.net_weight;
    rudy_net_weight_ = layout.net_weight64;
    particle_pin_start_ = layout.particle_pin_start;
    pin_slot_ = layout.pin_slot;
    wl_net_count_ = layout.kept_nets;
    wl_pin_count_ = layout.kept_pins;
    // Degree buckets: one thread per two-pin net, G lanes per net for degree <= G,
    // a warp loop above 32.  The blocks run heaviest bucket first, so the long
    // warp-loop nets do not form the kernel's tail.  Each block takes two rounds of
    // its lanes: half the blocks of one round each, and so half the block-end
    // reductions, measured 4% faster a warm iteration (the pass shares the SMs with
    // the field solve, and its blocks' fixed costs held them).
    constexpr int kRounds = 2;
    const int kGroups[6] = {1, 4, 8, 16, 32, 0};
    std::vector<int4> work;
    for (int b = 5; b >= 0; --b) {
        const int group = kGroups[b];
        const int nets_per_block =
            kRounds * (group == 0 ? kThreads / 32 : group == 1 ? kThreads : kThreads / group);
        const int first_net = layout.bucket_first[b];
        const int count = layout.bucket_first[b + 1] - layout.bucket_first[b];
        for (int off = 0; off < count; off += nets_per_block) {
            work.push_back(make_int4(group, first_net + off, std::min(nets_per_block, count - off), 0));
        }
    }
    wl_blocks_ = static_cast<int>(work.size());
    const std::size_t pins = std::max<std::size_t>(1, static_cast<std::size_t>(layout.kept_pins));
    block_work_ = arena_.array<int4>(std::max<std::size_t>(1, work.size()), "wirelength work");
    pin_gradient_ = arena_.array<float2>(pins, "pin gradients");
    partials_wl_ = arena_.array<double>(2 * std::max<std::size_t>(1, work.size()), "wirelength partials");
    upload(block_work_, work, stream_);
    checkCuda(cudaMemsetAsync(pin_gradient_, 0, pins * sizeof(float2), stream_), "clear pin gradients");
    checkCuda(cudaStreamSynchronize(stream_), "net layout upload");
}

void Engine::buildBasis() {
    const int nx = bins_x_, ny = bins_y_;
    const double width = region_.width(), height = region_.height();
    // Spectral divide (ElectrostaticField.cpp:212-221): 1/(4 Nx Ny) / (kx^2 + ky^2), DC removed.
    std::vector<float> scale(static_cast<std::size_t>(ny) * nx);
    const double normalization = 1.0 / (4.0 * static_cast<double>(nx) * static_cast<double>(ny));
    for (int l = 0; l < ny; ++l) {
        const double wave_y = kPi * static_cast<double>(l) / height;
        for (int k = 0; k < nx; ++k) {
            const double wave_x = kPi * static_cast<double>(k) / width;
            const double denominator = wave_x * wave_x + wave_y * wave_y;
            scale[static_cast<std::size_t>(l) * nx + k] =
                denominator <= kEpsilon ? 0.0f : static_cast<float>(normalization / denominator);
        }
    }
    std::vector<float> wy(static_cast<std::size_t>(ny), 1.0f), wx(static_cast<std::size_t>(nx), 1.0f);
    wy[0] = 0.5f;
    wx[0] = 0.5f;
    const std::size_t bins = static_cast<std::size_t>(bin_count_);
    spectral_scale_ = arena_.array<float>(bins, "spectral scale");
    weight_y_ = arena_.array<float>(wy.size(), "Parseval weights");
    weight_x_ = arena_.array<float>(wx.size(), "Parseval weights");
    field_ = arena_.array<float2>(bins, "electric field");
    potential_ = arena_.array<float>(bins, "potential");
    upload(spectral_scale_, scale, stream_);
    upload(weight_y_, wy, stream_);
    upload(weight_x_, wx, stream_);
    double max_scale = 0.0;
    for (float v : scale) max_scale = std::max(max_scale, static_cast<double>(v));
    buildTensorCoreBasis(max_scale);
    checkCuda(cudaStreamSynchronize(stream_), "basis upload");
}

SplitMatrix Engine::newSplit(int rows, int cols, const char* what) {
    SplitMatrix m;
    m.rows = rows;
    m.cols = cols;
    m.ld = paddedLd(cols);
    m.data = arena_.array<__half>(m.elements(), what);
    checkCuda(cudaMemsetAsync(m.data, 0, m.elements() * sizeof(__half), stream_), what);
    return m;
}


void Engine::buildTensorCoreBasis(double max_scale) {
    const int nx = bins_x_, ny = bins_y_;
    TcScales host_scales{};
    enum { kCx = 0, kCy, kDy, kDxc, kSxwt, kSyw };
    tc_cx_ = newSplit(nx, nx, "DCT basis planes");
    tc_cy_ = newSplit(ny, ny, "DCT basis planes");
    tc_dy_ = newSplit(ny, ny, "DCT basis planes");
    tc_dxc_ = newSplit(nx, nx, "DCT basis planes");
    tc_sxwt_ = newSplit(nx, nx, "DST basis planes");
    tc_syw_ = newSplit(ny, ny, "DST basis planes");
    const SplitMatrix basis_planes[kBasisCount] = {tc_cx_, tc_cy_, tc_dy_, tc_dxc_, tc_sxwt_, tc_syw_};
    unsigned long long* ranges = arena_.array<unsigned long long>(2 * kBasisCount, "basis ranges");
    int exponents[kBasisCount] = {};
    double row_l1[kBasisCount] = {};
    buildBasisPlanes(nx, ny, region_.width(), region_.height(), basis_planes, ranges, exponents, row_l1, stream_);
    for (int t = 0; t < kBasisCount; ++t) host_scales.exp_basis[t] = exponents[t];
    tc_source_ = newSplit(ny, nx, "source planes");
    tc_x1t_ = newSplit(nx, ny, "DCT stage planes");
    tc_phi_ = newSplit(ny, nx, "potential coefficient planes");
    tc_phit_ = newSplit(nx, ny, "potential coefficient planes");
    tc_t_ = newSplit(ny, nx, "DCT stage planes");
    tc_ut_ = newSplit(nx, ny, "DCT stage planes");
    tc_row_exp_ = arena_.array<int>(static_cast<std::size_t>(ny), "source plane exponents");
    tc_scales_ = arena_.array<TcScales>(1, "field scales");
    checkCuda(cudaMemcpyAsync(tc_scales_, &host_scales, sizeof(TcScales), cudaMemcpyHostToDevice, stream_),
              "upload field scales");
    checkCuda(cudaStreamSynchronize(stream_), "upload field scales");  // host_scales leaves scope
    tc_error_ = arena_.array<int>(1, "contraction error flag");
    checkCuda(cudaMemsetAsync(tc_error_, 0, sizeof(int), stream_), "clear error flag");
    checkCuda(cudaMallocHost(reinterpret_cast<void**>(&host_error_), sizeof(int)), "pinned error flag");
    *host_error_ = 0;

    // Output bounds |C| <= gain * max |data operand|, with a margin for FP32 rounding.
    constexpr double kMargin = 1.02;
    TcScales* sc = tc_scales_;
    const auto task = [&](TcTask& t, const SplitMatrix& a, const SplitMatrix& b, int m, int n, int k, int mode) {
        std::memset(static_cast<void*>(&t), 0, sizeof(TcTask));
        makeOperandMap(&t.map_a, a, kTileM);
        makeOperandMap(&t.map_b, b, kTileN);
        t.m = m;
        t.n = n;
        t.k = k;
        t.mode = mode;
    };
    // X = S * Cx^T, stored transposed (the K-major B operand of the next contraction).
    task(tc_fwd1_.task[0], tc_source_, tc_cx_, ny, nx, nx, kTcSplitTransposed);
    tc_fwd1_.task[0].row_exp_a = tc_row_exp_;
    tc_fwd1_.task[0].exp_b = &sc->exp_basis[kCx];
    tc_fwd1_.task[0].ref_max = &sc->max_source;
    tc_fwd1_.task[0].gain = static_cast<float>(row_l1[kCx] * kMargin);
    tc_fwd1_.task[0].out_exp = &sc->exp_x;
    tc_fwd1_.task[0].out_max = &sc->max_x;
    tc_fwd1_.task[0].out_t = tc_x1t_.data;
    tc_fwd1_.task[0].out_t_ld = tc_x1t_.ld;
    tc_fwd1_.task[0].out_t_plane = tc_x1t_.plane();
    // rho_hat = Cy * X; epilogue: phi_hat = rho_hat .* scale, stored both ways, + Parseval energy.
    task(tc_fwd2_.task[0], tc_cy_, tc_x1t_, ny, nx, ny, kTcSpectral);
    tc_fwd2_.task[0].exp_a = &sc->exp_basis[kCy];
    tc_fwd2_.task[0].exp_b = &sc->exp_x;
    tc_fwd2_.task[0].ref_max = &sc->max_x;
    tc_fwd2_.task[0].gain = static_cast<float>(row_l1[kCy] * max_scale * kMargin);
    tc_fwd2_.task[0].out_exp = &sc->exp_phi;
    tc_fwd2_.task[0].out_max = &sc->max_phi;
    tc_fwd2_.task[0].clear = &sc->max_source;
    tc_fwd2_.task[0].out = tc_phi_.data;
    tc_fwd2_.task[0].out_ld = tc_phi_.ld;
    tc_fwd2_.task[0].out_plane = tc_phi_.plane();
    tc_fwd2_.task[0].out_t = tc_phit_.data;
    tc_fwd2_.task[0].out_t_ld = tc_phit_.ld;
    tc_fwd2_.task[0].out_t_plane = tc_phit_.plane();
    tc_fwd2_.task[0].scale = spectral_scale_;

    tc_fwd2_.task[0].weight_r = weight_y_;
    tc_fwd2_.task[0].weight_c = weight_x_;
    // T = Dy * phi_hat and U = phi_hat * Dx^T (stored transposed), one launch.
    task(tc_inv1_.task[0], tc_dy_, tc_phit_, ny, nx, ny, kTcSplit);
    tc_inv1_.task[0].exp_a = &sc->exp_basis[kDy];
    tc_inv1_.task[0].exp_b = &sc->exp_phi;
    tc_inv1_.task[0].ref_max = &sc->max_phi;
    tc_inv1_.task[0].gain = static_cast<float>(row_l1[kDy] * kMargin);
    tc_inv1_.task[0].out_exp = &sc->exp_t;
    tc_inv1_.task[0].out = tc_t_.data;
    tc_inv1_.task[0].out_ld = tc_t_.ld;
    tc_inv1_.task[0].out_plane = tc_t_.plane();
    task(tc_inv1_.task[1], tc_phi_, tc_dxc_, ny, nx, nx, kTcSplitTransposed);
    tc_inv1_.task[1].exp_a = &sc->exp_phi;
    tc_inv1_.task[1].exp_b = &sc->exp_basis[kDxc];
    tc_inv1_.task[1].ref_max = &sc->max_phi;
    tc_inv1_.task[1].gain = static_cast<float>(row_l1[kDxc] * kMargin);
    tc_inv1_.task[1].out_exp = &sc->exp_u;
    tc_inv1_.task[1].out_t = tc_ut_.data;
    tc_inv1_.task[1].out_t_ld = tc_ut_.ld;
    tc_inv1_.task[1].out_t_plane = tc_ut_.plane();
    // Ex = T * (Sx diag(kx))^T and Ey = (Sy diag(ky)) * U into the interleaved field, one launch.
    task(tc_inv2_.task[0], tc_t_, tc_sxwt_, ny, nx, nx, kTcField);
    tc_inv2_.task[0].exp_a = &sc->exp_t;
    tc_inv2_.task[0].exp_b = &sc->exp_basis[kSxwt];
    tc_inv2_.task[0].out_f = reinterpret_cast<float*>(field_);
    tc_inv2_.task[0].out_f_ld = 2 * nx;
    tc_inv2_.task[0].out_f_step = 2;
    task(tc_inv2_.task[1], tc_syw_, tc_ut_, ny, nx, ny, kTcField);
    tc_inv2_.task[1].exp_a = &sc->exp_basis[kSyw];
    tc_inv2_.task[1].exp_b = &sc->exp_u;
    tc_inv2_.task[1].out_f = reinterpret_cast<float*>(field_) + 1;
    tc_inv2_.task[1].out_f_ld = 2 * nx;
    tc_inv2_.task[1].out_f_step = 2;
    // Potential (parity hook): phi = T * Dx^T.
    task(tc_pot_.task[0], tc_t_, tc_dxc_, ny, nx, nx, kTcField);
    tc_pot_.task[0].exp_a = &sc->exp_t;
    tc_pot_.task[0].exp_b = &sc->exp_basis[kDxc];
    tc_pot_.task[0].out_f = potential_;
    tc_pot_.task[0].out_f_ld = nx;
    tc_pot_.task[0].out_f_step = 1;
    tc_fwd1_.error_flag = tc_fwd2_.error_flag = tc_inv1_.error_flag = tc_inv2_.error_flag = tc_pot_.error_flag =
        tc_error_;
    // The basis operands never change, so their tiles may be fetched before the
    // contraction waits for its predecessor.
    const auto basis = [&](const int* e) { return e != nullptr && e >= sc->exp_basis && e < sc->exp_basis + 8; };
    for (TcBatch* b : {&tc_fwd1_, &tc_fwd2_, &tc_inv1_, &tc_inv2_, &tc_pot_}) {
        for (TcTask& t : b->task) t.constant_operand = basis(t.exp_a) ? 1 : (basis(t.exp_b) ? 2 : 0);
    }
    tcPlan(tc_fwd1_, 1);
    tcPlan(tc_fwd2_, 1);
    tcPlan(tc_inv1_, 2);
    tcPlan(tc_inv2_, 2);
    tcPlan(tc_pot_, 1);

    // The banded solve (field_tc.cu): Q = S Cx^T, rho_hat = Cy Q, phi_hat, M1 = Dy phi_hat and
    // M2 = Syw phi_hat per band of spectral columns, then Ex = M1 (Sx diag(kx))^T,
    // Ey = M2 Dx^T and the potential M1 Dx^T over all bands.
    // The banded solve for grids taller than kFieldBandedMinRows rows (up to its limits);
    // MPGP_FIELD_SOLVE=staged or =banded chooses for every grid the banded solve takes.
    const char* solve = std::getenv("MPGP_FIELD_SOLVE");
    bool banded = ny > kFieldBandedMinRows;
    if (solve != nullptr && std::strcmp(solve, "staged") == 0) banded = false;
    if (solve != nullptr && std::strcmp(solve, "banded") == 0) banded = true;
    const FieldShape shape = banded ? fieldShape(nx, ny) : FieldShape{};
    banded_ = shape.cluster > 0;
    if (banded_) {
        tc_m1_ = newSplit(ny, nx, "banded field planes");
        tc_m2_ = newSplit(ny, nx, "banded field planes");
        int* band_exp = arena_.array<int>(static_cast<std::size_t>(2 * shape.bands), "banded field exponents");
        FieldBand& f = field_band_;
        makeOperandMap(&f.map_s, tc_source_, kTileM);
        makeOperandMap(&f.map_cx, tc_cx_, shape.share_n);
        makeOperandMap(&f.map_cy, tc_cy_, kTileM);
        makeOperandMap(&f.map_dy, tc_dy_, kTileM);
        makeOperandMap(&f.map_syw, tc_syw_, kTileM);
        f.nx = nx;
        f.ny = ny;
        f.shape = shape;
        f.row_exp = tc_row_exp_;
        f.exp_basis = sc->exp_basis;
        f.scale = spectral_scale_;
        f.m1 = tc_m1_.data;
        f.m2 = tc_m2_.data;
        f.m_ld = tc_m1_.ld;
        f.m_plane = tc_m1_.plane();
        f.m1_exp = band_exp;
        f.m2_exp = band_exp + shape.bands;
        f.gain_dy = static_cast<float>(row_l1[kDy] * kMargin);
        f.gain_syw = static_cast<float>(row_l1[kSyw] * kMargin);
        f.clear = &sc->max_source;
        f.error_flag = tc_error_;
        f.phi_store = arena_.array<unsigned char>(fieldStoreBytes(shape), "kept field coefficients");
        f.phi_records = arena_.array<int>(fieldRecordInts(shape), "kept field coefficient records");
        task(tc_invx_.task[0], tc_m1_, tc_sxwt_, ny, nx, nx, kTcField);
        tc_invx_.task[0].kb_exp_a = f.m1_exp;
        tc_invx_.task[0].exp_b = &sc->exp_basis[kSxwt];
        tc_invx_.task[0].out_f = reinterpret_cast<float*>(field_);
        tc_invx_.task[0].out_f_ld = 2 * nx;
        tc_invx_.task[0].out_f_step = 2;
        task(tc_invx_.task[1], tc_m2_, tc_dxc_, ny, nx, nx, kTcField);
        tc_invx_.task[1].kb_exp_a = f.m2_exp;
        tc_invx_.task[1].exp_b = &sc->exp_basis[kDxc];
        tc_invx_.task[1].out_f = reinterpret_cast<float*>(field_) + 1;
        tc_invx_.task[1].out_f_ld = 2 * nx;
        tc_invx_.task[1].out_f_step = 2;
        task(tc_potx_.task[0], tc_m1_, tc_dxc_, ny, nx, nx, kTcField);
        tc_potx_.task[0].kb_exp_a = f.m1_exp;
        tc_potx_.task[0].exp_b = &sc->exp_basis[kDxc];
        tc_potx_.task[0].out_f = potential_;
        tc_potx_.task[0].out_f_ld = nx;
        tc_potx_.task[0].out_f_step = 1;
        for (TcBatch* b : {&tc_invx_, &tc_potx_}) {
            b->error_flag = tc_error_;
            for (TcTask& t : b->task) t.constant_operand = 2;
        }
        tcPlan(tc_invx_, 2);
        tcPlan(tc_potx_, 1);
    }
    energy_blocks_ = banded_ ? shape.blocks() : tcBlocks(tc_fwd2_, 1);
    partials_e_ = arena_.array<double>(static_cast<std::size_t>(energy_blocks_), "energy partials");
    tc_fwd2_.task[0].energy_partials = partials_e_;
    field_band_.energy_partials = partials_e_;
}

void Engine::setStallProbe(long long polls) {
    for (TcBatch* b : {&tc_fwd1_, &tc_fwd2_, &tc_inv1_, &tc_inv2_, &tc_pot_, &tc_invx_, &tc_potx_}) {
        b->stall_polls = std::max(0LL, polls);
    }
    field_band_.stall_polls = std::max(0LL, polls);
}

const char* kernelKindName(int kind) {
    static const char* names[kKindCount] = {"scatter",     "wirelength",     "metrics",       "dct_forward",
                                            "dct_inverse", "gather",         "reduce",        "vector",
                                            "dct_split",   "rudy",           "field_forward", "field_gradient",
                                            "field_inverse"};
    return kind >= 0 && kind < kKindCount ? names[kind] : "unknown";
}

void Engine::setTiming(uint32_t families) {
    if (families != 0 && events_.empty()) {
        events_.resize(64);
        for (cudaEvent_t& e : events_) checkCuda(cudaEventCreate(&e), "Create profiling event");
        pending_kind_.resize(32);
    }
    timing_mask_ = families;
}

void Engine::beginKernel(int kind, cudaStream_t on) {
    open_ = ((timing_mask_ >> kind) & 1u) != 0;
    if (!open_) return;
    if (pending_ >= static_cast<int>(pending_kind_.size())) collectTimings();
    pending_kind_[pending_] = kind;
    checkCuda(cudaEventRecord(events_[2 * pending_], on != nullptr ? on : stream_), "Record profiling event");
}

void Engine::endKernel(cudaStream_t on) {
    if (!open_) return;
    open_ = false;
    checkCuda(cudaEventRecord(events_[2 * pending_ + 1], on != nullptr ? on : stream_), "Record profiling event");
    ++pending_;
}

void Engine::collectTimings() {
    if (pending_ == 0) return;
    for (int i = 0; i < pending_; ++i) {
        float ms = 0.0f;
        checkCuda(cudaEventSynchronize(events_[2 * i + 1]), "Profiling sync");
        checkCuda(cudaEventElapsedTime(&ms, events_[2 * i], events_[2 * i + 1]), "Profiling elapsed");
        stats_.launches[pending_kind_[i]] += 1;
        stats_.milliseconds[pending_kind_[i]] += static_cast<double>(ms);
    }
    pending_ = 0;
}

// The Neumann field as dense contractions (ElectrostaticField.cpp:205-237):
//   X = S * Cx^T, rho_hat = Cy * X, phi_hat = rho_hat .* scale (+ Parseval energy)
//   gradient: T = Dy * phi_hat, U = phi_hat * Dx^T, Ex = T * (Sx diag(kx))^T, Ey = (Sy diag(ky)) * U
//   potential (parity hook only): phi = T * Dx^T.
Engine::Groups Engine::newGroups(int blocks, int values, const char* what) {
    Groups g;
    g.count = std::max(1, ceilDiv(std::max(1, blocks), 32));
    g.partials = arena_.array<double>(static_cast<std::size_t>(values) * g.count, what);
    const std::size_t counters = static_cast<std::size_t>(g.count) + 1;
    g.counters = arena_.array<unsigned int>(counters, what);
    checkCuda(cudaMemsetAsync(g.counters, 0, counters * sizeof(unsigned int), stream_), what);
    return g;
}

void Engine::allocateGroups() {
    sc_groups_ = newGroups(scatter_blocks_, 2, "scatter group partials");
    m_groups_ = newGroups(metrics_blocks_, 9, "metric group partials");
    g_groups_ = newGroups(gather_blocks_, 8, "gather group partials");
    wl_groups_ = std::max(1, ceilDiv(std::max(1, wl_blocks_), 32));
    wl_group_ = arena_.array<double>(2 * static_cast<std::size_t>(wl_groups_), "wirelength group partials");
    const std::size_t counters = static_cast<std::size_t>(wl_groups_) + 1;
    wl_counters_ = arena_.array<unsigned int>(counters, "wirelength group counters");
    checkCuda(cudaMemsetAsync(wl_counters_, 0, counters * sizeof(unsigned int), stream_), "wirelength group counters");
}

void Engine::runDct(bool gradient, bool potential, bool forward, bool split_source) {
    if (banded_) {
        runBandedField(gradient, forward, split_source);
        runBandedInverseX(gradient, potential);
        return;
    }
    runStagedField(gradient, potential, forward, split_source);
}

void Engine::runBandedField(bool gradient, bool forward, bool split_source) {
    const int nx = bins_x_;
    if (forward && split_source) {
        beginKernel(kKindDctSplit);
        launchSplitSource(source_, tc_source_, nx, tc_row_exp_, tc_scales_, stream_);
        endKernel();
        launches_ += 1;
    }
    // Without the forward flag (the density is that of the previous evaluation) the
    // banded launch runs only the inverse passes, from the coefficients the previous
    // evaluation's launch kept.
    if (forward || gradient) {
        const FieldMode mode = forward ? (gradient ? kFieldGradient : kFieldForward) : kFieldInverse;
        beginKernel(mode == kFieldForward ? kKindFieldForward
                                          : (mode == kFieldGradient ? kKindFieldGradient : kKindFieldInverse));
        launchField(field_band_, mode, stream_);
        endKernel();
        launches_ += 1;
    }
}

void Engine::runBandedInverseX(bool gradient, bool potential) {
    if (!gradient) return;
    beginKernel(kKindDctInverse);
    launchTcGemm(tc_invx_, 2, stream_);
    endKernel();
    launches_ += 1;
    if (potential) {
        beginKernel(kKindDctInverse);
        launchTcGemm(tc_potx_, 1, stream_);
        endKernel();
        launches_ += 1;
    }
}

void Engine::runStagedField(bool gradient, bool potential, bool forward, bool split_source) {
    const int nx = bins_x_;
    if (forward) {
        if (split_source) {
            beginKernel(kKindDctSplit);
            launchSplitSource(source_, tc_source_, nx, tc_row_exp_, tc_scales_, stream_);
            endKernel();
            launches_ += 1;
        }
        beginKernel(kKindDctForward);
        launchTcGemm(tc_fwd1_, 1, stream_);
        endKernel();
        beginKernel(kKindDctForward);
        launchTcGemm(tc_fwd2_, 1, stream_);
        endKernel();
        launches_ += 2;
    }
    if (!gradient) return;
    beginKernel(kKindDctInverse);
    launchTcGemm(tc_inv1_, 2, stream_);
    endKernel();
    beginKernel(kKindDctInverse);
    launchTcGemm(tc_inv2_, 2, stream_);
    endKernel();
    launches_ += 2;
    if (potential) {
        beginKernel(kKindDctInverse);
        launchTcGemm(tc_pot_, 1, stream_);
        endKernel();
        launches_ += 1;
    }
}

EvalPlan Engine::plan(const EvalRequest& q) {
    const int nx = bins_x_, ny = bins_y_;
    const double2* positions = q.mode == kGiven ? q.positions : q.out_positions;
    require(positions != nullptr, "An evaluation needs positions.");
    require(q.smoothing > 0.0 && std::isfinite(q.smoothing), "Global placement requires positive finite smoothing.");
    const bool folds = q.velocity_base != nullptr || q.checkpoint_out != nullptr;
    require(!folds || (q.mode == kGiven && q.gradient && particle_count_ > 0), "Only an evaluation with a gather at "
            "given positions takes the previous step's velocity update and checkpoint copy.");
    require((q.velocity_base == nullptr) == (q.velocity_out == nullptr), "A velocity update needs its output.");
    EvalPlan p;

    ScatterArgs& sa = p.scatter_args;
    sa.mode = q.mode;
    sa.particle_count = static_cast<int>(particle_count_);
    sa.positions = q.positions;
    sa.base = q.base;
    sa.direction = q.direction;
    sa.raw = q.raw_direction;
    sa.step = q.step;
    sa.max_displacement = q.max_displacement;
    sa.out_positions = q.out_positions;
    sa.size = size_;
    sa.layer = layer_;
    sa.llx = region_.llx;
    sa.lly = region_.lly;
    sa.urx = region_.urx;
    sa.ury = region_.ury;
    sa.bin_w = bin_w_;
    sa.bin_h = bin_h_;
    sa.bins_x = nx;
    sa.bins_y = ny;
    sa.layers = layers_;
    sa.totals = totals_;
    sa.partials = partials_sc_;
    sa.group_partials = sc_groups_.partials;
    sa.group_counters = sc_groups_.counters;
    p.scatter = !q.reuse_density && particle_count_ > 0;
    p.scatter_blocks = scatter_blocks_;
    // The wirelength pass needs the positions only: it runs beside the density
    // chain on its own stream (after the scatter when the scatter forms them).
    p.fork_first = q.mode == kGiven;

    WirelengthArgs& wa = p.wirelength_args;
    wa.positions = positions;
    wa.pin_particle = pin_particle_;
    wa.pin_offset = pin_offset_;
    wa.static_pins = static_pins_;
    wa.net_start = net_start_;
    wa.net_weight = net_weight_;
    wa.block_work = block_work_;
    wa.gamma = static_cast<float>(std::max(q.smoothing, kEpsilon));
    wa.inv_gamma = static_cast<float>(1.0 / std::max(q.smoothing, kEpsilon));
    wa.pin_slot = pin_slot_;
    wa.pin_gradient = pin_gradient_;
    wa.gradient = q.gradient ? 1 : 0;
    wa.partials = partials_wl_;
    wa.group_partials = wl_group_;
    wa.group_counters = wl_counters_;
    p.wirelength_blocks = wl_blocks_;
    if (q.rudy) {
        // The routability term runs beside the density chain, after the wirelength pass.
        require(rudy_main_.columns > 0, "RUDY was not enabled for this engine.");
        p.rudy = true;
        p.rudy_gradient = q.gradient;
        p.rudy_args = rudyArgs(rudy_main_, positions, true);
        p.rudy_blocks = rudy_main_.blocks;
    }

    MetricsArgs& ma = p.metrics_args;
    ma.layers = layers_;
    ma.totals = totals_;
    ma.static_charge = static_charge_;
    ma.static_fixed_sum = static_fixed_sum_;
    ma.static_dark_sum = static_dark_sum_;
    ma.target_density = target_density_;
    ma.bin_area = bin_area_;
    ma.bin_count = bin_count_;
    ma.source = source_;
    ma.partials = partials_m_;
    ma.group_partials = m_groups_.partials;
    ma.group_counters = m_groups_.counters;
    int kernels = 1;  // the wirelength pass
    if (!q.reuse_density) {
        p.metrics = true;
        p.metrics_fused = metrics_fused_;
        p.metrics_blocks = metrics_blocks_;
        if (metrics_fused_) {
            ma.columns = nx;
            ma.rows = ny;
            ma.split_out = tc_source_.data;
            ma.split_ld = tc_source_.ld;
            ma.split_plane = tc_source_.plane();
            ma.row_exp = tc_row_exp_;
            ma.scales = tc_scales_;
        }
        kernels += 2;  // scatter, metrics
    }
    p.forward = !q.reuse_density;
    p.split_source = !metrics_fused_;
    p.gradient = q.gradient;
    p.potential = q.gradient && q.want_potential;

    ReduceArgs& ra = p.reduce_args;
    int s = 0;
    const auto add = [&](const double* partials, int rows, int stride, int column, bool is_max, int target) {
        ra.sources[s++] = ReduceSource{partials, rows, stride, column, is_max ? 1 : 0, target};
    };
    add(wl_group_, wl_blocks_ > 0 ? wl_groups_ : 0, 1, 0, false, kSmooth);
    add(wl_group_, wl_blocks_ > 0 ? wl_groups_ : 0, 1, wl_groups_, false, kHpwl);
    // The scatter, metrics and gather partials, folded per 32 blocks by the producers.
    const int scatter_rows = particle_count_ > 0 && q.mode == kPropose ? sc_groups_.count : 0;
    if (!q.reuse_density) {  // otherwise the density scalars of the previous evaluation stand
        add(sc_groups_.partials, scatter_rows, 1, 0, false, kPredicted);
        add(sc_groups_.partials, scatter_rows, 1, sc_groups_.count, true, kMaxDisplacement);
        for (int k = 0; k < 9; ++k) {
            add(m_groups_.partials, m_groups_.count, 1, k * m_groups_.count, k >= 7, kOverflowWith + k);
        }
        add(partials_e_, energy_blocks_, 1, 0, false, kEnergy);
    }
    for (int k = 0; k < 5; ++k) {
        add(rudy_main_.partials, q.rudy ? rudy_main_.blocks : 0, 1, k * rudy_main_.blocks, k == 4, kRudyEnergy + k);
    }
    const bool gather = q.gradient && particle_count_ > 0;
    if (q.gradient) {
        for (int k = 0; k < 8; ++k) {
            add(g_groups_.partials, gather ? g_groups_.count : 0, 1, k * g_groups_.count, false, kWireL1 + k);
        }
    }
    ra.source_count = s;
    ra.offsets[0] = 0;
    for (int k = 0; k < s; ++k) ra.offsets[k + 1] = ra.offsets[k] + ra.sources[k].rows;
    ra.staged_capacity = kReduceStaged;
    ra.scalars = scalars_;
    ra.totals = totals_;
    const uint64_t ticket = ++launches_issued_;
    const int record = static_cast<int>(ticket % kRecords);
    ra.host_slots = host_slots_ + static_cast<std::size_t>(record) * kRecordSlots;
    ra.device_error = tc_error_;
    ra.sequence = static_cast<unsigned int>(++sequence_);
    if (ra.sequence == 0) ra.sequence = static_cast<unsigned int>(++sequence_);  // 0 marks an empty record
    record_sequence_[record] = ra.sequence;
    record_ticket_[record] = ticket;
    record_mask_[record] = 0;
    for (int k = 0; k < s; ++k) record_mask_[record] |= 1U << ra.sources[k].target;
    if (gather) {
        GatherArgs& ga = p.gather_args;
        ga.particle_count = static_cast<int>(particle_count_);
        ga.movable_count = static_cast<int>(movable_count_);
        ga.positions = positions;
        ga.particle_pin_start = particle_pin_start_;
        ga.pin_gradient = pin_gradient_;
        ga.field = field_;
        ga.charge = charge_;
        ga.precond_base = q.wire_out != nullptr ? nullptr : precond_;
        ga.llx = region_.llx;
        ga.lly = region_.lly;
        ga.urx = region_.urx;
        ga.ury = region_.ury;
        ga.inv_bin_w = 1.0 / bin_w_;
        ga.inv_bin_h = 1.0 / bin_h_;
        ga.bins_x = nx;
        ga.bins_y = ny;
        ga.penalty = q.penalty;
        ga.precond_scale = q.precond_scale;
        ga.raw = q.raw;
        ga.pre = q.pre;
        ga.wire_out = q.wire_out;
        ga.density_out = q.density_out;
        ga.rudy_out = q.rudy_out;
        ga.prev_positions = q.prev_positions;
        ga.prev_gradient = q.prev_gradient;
        ga.velocity = q.velocity;
        ga.velocity_base = q.velocity_base;
        ga.velocity_out = q.velocity_out;
        ga.checkpoint_out = q.checkpoint_out;
        ga.rudy_gradient = q.rudy ? rudy_pin_gradient_ : nullptr;
        ga.rudy_weight = q.rudy ? q.rudy_weight : 0.0;
        ga.partials = partials_g_;
        ga.group_partials = g_groups_.partials;
        ga.group_counters = g_groups_.counters;
        p.gather = true;
        p.gather_blocks = gather_blocks_;
        kernels += 1;
    }
    if (!gather) kernels += 1;  // the reduction (a gather reduces in its last block)
    if (q.rudy) kernels += q.gradient ? 7 : 4;
    p.kernels = kernels;
    d2h_bytes_ += static_cast<uint64_t>(s) * sizeof(double) + sizeof(int) + sizeof(unsigned long long);
    last_gradient_ = q.gradient;
    last_propose_ = q.mode == kPropose;
    return p;
}

void Engine::run(const EvalPlan& p) {
    if (p.fork_first) checkCuda(cudaEventRecord(fork_, stream_), "fork");
    if (p.scatter) {
        beginKernel(kKindScatter);
        launchScatter(p.scatter_args, p.scatter_blocks, stream_);
        endKernel();
    }
    if (!p.fork_first) checkCuda(cudaEventRecord(fork_, stream_), "fork");
    // With the banded field solve the wirelength pass is launched after the banded kernel:
    // blocks start in launch order, and the banded kernel's clusters (whole SMs each)
    // would otherwise wait for the wirelength pass's blocks to drain.
    if (!banded_) runWirelengthPass(p);
    if (p.metrics) {
        beginKernel(kKindMetrics);
        if (p.metrics_fused) {
            launchMetricsSplit(p.metrics_args, stream_);
        } else {
            launchMetrics(p.metrics_args, p.metrics_blocks, stream_);
        }
        endKernel();
    }
    if (banded_) {
        runBandedField(p.gradient, p.forward, p.split_source);
        runWirelengthPass(p);
        runBandedInverseX(p.gradient, p.potential);
    } else {
        runStagedField(p.gradient, p.potential, p.forward, p.split_source);
    }
    checkCuda(cudaStreamWaitEvent(stream_, join_, 0), "join");
    if (p.gather) {
        // The gather's last block also reduces and publishes the evaluation.
        beginKernel(kKindGather);
        launchGather(p.gather_args, &p.reduce_args, p.gather_blocks, stream_);
        endKernel();
    } else {
        beginKernel(kKindReduce);
        launchReduce(p.reduce_args, stream_);
        endKernel();
    }
    launches_ += p.kernels;
}

// The wirelength stream's part of an evaluation (after the fork event): the wirelength
// pass and the RUDY kernels, then the join event.
void Engine::runWirelengthPass(const EvalPlan& p) {
    checkCuda(cudaStreamWaitEvent(stream_wl_, fork_, 0), "fork");
    beginKernel(kKindWirelength, stream_wl_);
    launchWirelength(p.wirelength_args, p.wirelength_blocks, stream_wl_);
    endKernel(stream_wl_);
    if (p.rudy) {
        beginKernel(kKindRudy, stream_wl_);
        launchRudyDeposit(p.rudy_args, stream_wl_);
        launchRudyPrefix(p.rudy_args, stream_wl_);
        launchRudyMetrics(p.rudy_args, p.rudy_blocks, stream_wl_);
        if (p.rudy_gradient) {
            launchRudyTables(p.rudy_args, stream_wl_);
            launchRudyGradient(p.rudy_args, stream_wl_);
        }
        endKernel(stream_wl_);
    }
    checkCuda(cudaEventRecord(join_, stream_wl_), "join");
}

uint64_t Engine::launch(const EvalRequest& q) {
    if (batch_ != nullptr) require(!has_pending_, "A batched engine takes one evaluation at a time.");
    EvalPlan p = plan(q);
    if (batch_ != nullptr) {
        require(!p.rudy && !p.potential && (p.metrics_fused || !p.metrics),
                "A batched evaluation supports neither RUDY, the potential, nor grids wider than 2,048 bins.");
        batched_plan_ = p;
        has_pending_ = true;
        return launches_issued_;
    }
    run(p);
    return launches_issued_;
}

const TcBatch* Engine::deviceBatches() {
    if (device_batches_ == nullptr) {
        device_batches_ = arena_.array<TcBatch>(5, "batched contraction descriptors");
        const TcBatch host[5] = {tc_fwd1_, tc_fwd2_, tc_inv1_, tc_inv2_, tc_invx_};
        checkCuda(cudaMemcpyAsync(device_batches_, host, sizeof(host), cudaMemcpyHostToDevice, stream_),
                  "Upload contraction descriptors");
        checkCuda(cudaStreamSynchronize(stream_), "Upload contraction descriptors");  // `host` leaves scope
    }
    return device_batches_;
}

const FieldBand* Engine::deviceField() {
    if (device_field_ == nullptr) {
        device_field_ = arena_.array<FieldBand>(1, "batched field descriptor");
        checkCuda(cudaMemcpyAsync(device_field_, &field_band_, sizeof(FieldBand), cudaMemcpyHostToDevice, stream_),
                  "Upload the field descriptor");
        checkCuda(cudaStreamSynchronize(stream_), "Upload the field descriptor");
    }
    return device_field_;
}

const TcBatch& Engine::contraction(int stage) const {
    switch (stage) {
        case 0: return tc_fwd1_;
        case 1: return tc_fwd2_;
        case 2: return tc_inv1_;
        case 3: return tc_inv2_;
        default: return tc_invx_;
    }
}

const EvalScalars& Engine::sync(uint64_t ticket) {
    const int record = static_cast<int>(ticket % kRecords);
    require(ticket > synced_ticket_ || ticket == launches_issued_, "This evaluation was already read.");
    require(record_ticket_[record] == ticket, "This evaluation's record was reused by a later launch.");
    if (has_pending_) {
        // Batched: the evaluation runs in the batch's next round, which has completed
        // on the device when this returns; the record below is then already complete.
        has_pending_ = false;
        batch_->evaluate(this, batched_plan_);
    }
    // Poll the record until every scalar of this evaluation and the error flag carry
    // its sequence; now and then ask the stream for a fault, so an evaluation that
    // can no longer publish surfaces as an error instead of a hang.
    const unsigned long long tag = static_cast<unsigned long long>(record_sequence_[record]) << 32;
    const uint32_t expected_mask = record_mask_[record];
    const volatile unsigned long long* slots = host_slots_ + static_cast<std::size_t>(record) * kRecordSlots;
    const auto current = [&](int index) { return (slots[index] & 0xffffffff00000000ULL) == tag; };
    const auto complete = [&]() {
        if (!current(2 * kScalarCount)) return false;
        for (uint32_t m = expected_mask; m != 0; m &= m - 1) {
            const int k = __builtin_ctz(m);
            if (!current(2 * k) || !current(2 * k + 1)) return false;
        }
        return true;
    };
    for (uint64_t polls = 1; !complete(); ++polls) {
        if ((polls & 255U) == 0) {
            const cudaError_t status = cudaStreamQuery(stream_);
            if (status == cudaSuccess) {
                std::atomic_thread_fence(std::memory_order_seq_cst);
                if (!complete()) fail(MPGP_ERR_CUDA, "An evaluation ended without publishing its scalars.");
                break;
            }
            if (status != cudaErrorNotReady) checkCuda(status, "Evaluation on the device");
        }
        if (polls > 4096) std::this_thread::yield();
    }
    std::atomic_thread_fence(std::memory_order_acquire);
    for (uint32_t m = expected_mask; m != 0; m &= m - 1) {
        const int k = __builtin_ctz(m);
        const unsigned long long bits = (slots[2 * k] & 0xffffffffULL) | ((slots[2 * k + 1] & 0xffffffffULL) << 32);
        std::memcpy(&host_scalars_->v[k], &bits, sizeof(double));
    }
    synced_ticket_ = std::max(synced_ticket_, ticket);
    // Profiling events are read once no later evaluation is in flight (reading them
    // waits for every recorded event).
    if (ticket == launches_issued_) collectTimings();
    if ((slots[2 * kScalarCount] & 0xffffffffULL) != 0) {
        fail(MPGP_ERR_TIMEOUT, "A tcgen05 field contraction timed out waiting on its pipeline.");
    }
    return *host_scalars_;
}

void Engine::densityMetrics(const EvalScalars& s, bool with, mpgp_density_metrics& out) const {
    out.total_overflow_area = with ? s.v[kOverflowWith] : s.v[kOverflowWithout];
    out.total_charge_area = with ? s.v[kChargeWith] : s.v[kChargeWithout];
    out.normalization_area = s.v[kNormalization];
    out.maximum_density = std::max(0.0, with ? s.v[kDensityMaxWith] : s.v[kDensityMaxWithout]);
    out.average_density = (with ? s.v[kDensitySumWith] : s.v[kDensitySumWithout]) /
                          static_cast<double>(std::max(1, bin_count_));
    out.dark_area = static_dark_sum_;
    out.placeable_area = static_placeable_sum_;
    out.normalized_overflow = out.total_overflow_area / std::max(out.normalization_area, kEpsilon);
}

double Engine::energy(const EvalScalars& s) const { return std::max(0.0, 0.5 * bin_area_ * s.v[kEnergy]); }

void Engine::fieldSolve(const double* deviation, double* potential, double* field_x, double* field_y) {
    // Upload the deviation into the source buffer with its FP64 mean removed
    // (ElectrostaticField.cpp:119-133), then run the same contractions.
    const std::size_t bins = static_cast<std::size_t>(bin_count_);
    double mean = 0.0;
    for (std::size_t i = 0; i < bins; ++i) mean += deviation[i];
    mean /= static_cast<double>(bins);
    std::vector<float> source(bins);
    for (std::size_t i = 0; i < bins; ++i) source[i] = static_cast<float>(deviation[i] - mean);
    upload(source_, source, stream_);
    runDct(true, true, true);
    std::vector<float> p(bins);
    std::vector<float2> f(bins);
    checkCuda(cudaMemcpyAsync(p.data(), potential_, bins * sizeof(float), cudaMemcpyDeviceToHost, stream_), "field");
    checkCuda(cudaMemcpyAsync(f.data(), field_, bins * sizeof(float2), cudaMemcpyDeviceToHost, stream_), "field");
    checkCuda(cudaMemcpyAsync(host_error_, tc_error_, sizeof(int), cudaMemcpyDeviceToHost, stream_),
              "Download contraction status");
    checkCuda(cudaStreamSynchronize(stream_), "field solve");
    collectTimings();
    if (host_error_ != nullptr && *host_error_ != 0) {
        fail(MPGP_ERR_TIMEOUT, "A tcgen05 field contraction timed out waiting on its pipeline.");
    }
    for (std::size_t i = 0; i < bins; ++i) {
        if (potential != nullptr) potential[i] = p[i];
        if (field_x != nullptr) field_x[i] = f[i].x;
        if (field_y != nullptr) field_y[i] = f[i].y;
    }
}

// ---- RUDY (rudy.cu) -------------------------------------------------------------------

void Engine::allocateRudyGrid(RudyGrid& g, int columns, int rows, const char* what) {
    g.columns = columns;
    g.rows = rows;
    g.bin_w = region_.width() / static_cast<double>(columns);
    g.bin_h = region_.height() / static_cast<double>(rows);
    g.min_x_span = rudy_minimum_span_ * g.bin_w;
    g.min_y_span = rudy_minimum_span_ * g.bin_h;
    const std::size_t bins = static_cast<std::size_t>(columns) * static_cast<std::size_t>(rows);
    g.horizontal = arena_.array<unsigned long long>(bins, what);
    g.vertical = arena_.array<unsigned long long>(bins, what);
    g.adjoint_h = arena_.array<double>(bins, what);
    g.adjoint_v = arena_.array<double>(bins, what);
    g.utilization = arena_.array<double>(bins, what);
    const std::size_t padded = static_cast<std::size_t>(columns + 1) * static_cast<std::size_t>(rows + 1);
    g.diff = arena_.array<unsigned long long>(2 * padded, what);
    g.table = arena_.array<double>(2 * padded, what);
    checkCuda(cudaMemsetAsync(g.diff, 0, 2 * padded * sizeof(unsigned long long), stream_), what);
    checkCuda(cudaMemsetAsync(g.table, 0, 2 * padded * sizeof(double), stream_), what);
    g.blocks = std::max(1, std::min(ceilDiv(static_cast<long long>(bins), kThreads), 148 * 2));
    g.partials = arena_.array<double>(5 * static_cast<std::size_t>(g.blocks), what);
    checkCuda(cudaMemsetAsync(g.horizontal, 0, bins * sizeof(unsigned long long), stream_), what);
    checkCuda(cudaMemsetAsync(g.vertical, 0, bins * sizeof(unsigned long long), stream_), what);
    checkCuda(cudaMemsetAsync(g.adjoint_h, 0, bins * sizeof(double), stream_), what);
    checkCuda(cudaMemsetAsync(g.adjoint_v, 0, bins * sizeof(double), stream_), what);
}

void Engine::setRudyModel(int model, double temperature) {
    rudy_model_ = model;
    rudy_temperature_ = temperature;
}

void Engine::enableRudy(const mpgp_options& o) {
    if (rudy_main_.columns > 0) return;
    rudy_model_ = o.rudy_penalty_model;
    rudy_temperature_ = o.rudy_softplus_temperature;
    rudy_minimum_span_ = o.rudy_minimum_span_in_bins;
    allocateRudyGrid(rudy_main_, o.rudy_columns, o.rudy_rows, "RUDY maps");
    if (o.rudy_validation_bins > 0) {
        allocateRudyGrid(rudy_validation_, o.rudy_validation_bins, o.rudy_validation_bins, "RUDY validation maps");
    }
    rudy_pin_gradient_ =
        arena_.array<double2>(std::max<std::size_t>(1, static_cast<std::size_t>(wl_pin_count_)), "RUDY pin gradients");
    rudy_scalars_ = arena_.array<double>(5, "RUDY scalars");
    checkCuda(cudaMallocHost(reinterpret_cast<void**>(&host_rudy_), 5 * sizeof(double)), "pinned RUDY scalars");
    checkCuda(cudaStreamSynchronize(stream_), "RUDY set-up");
}

RudyArgs Engine::rudyArgs(const RudyGrid& g, const double2* positions, bool with_capacity) const {
    RudyArgs a{};
    a.positions = positions;
    a.pin_particle = pin_particle_;
    a.pin_offset = pin_offset_;
    a.static_pins = static_pins_;
    a.net_start = net_start_;
    a.net_weight = rudy_net_weight_;
    a.net_count = wl_net_count_;
    a.pin_slot = pin_slot_;
    a.pin_gradient = rudy_pin_gradient_;
    a.llx = region_.llx;
    a.lly = region_.lly;
    a.urx = region_.urx;
    a.ury = region_.ury;
    a.bin_w = g.bin_w;
    a.bin_h = g.bin_h;
    a.columns = g.columns;
    a.rows = g.rows;
    a.minimum_x_span = g.min_x_span;
    a.minimum_y_span = g.min_y_span;
    a.inv_unit_h = 4294967296.0 / g.bin_w;
    a.inv_unit_v = 4294967296.0 / g.bin_h;
    a.diff = g.diff;
    a.horizontal = g.horizontal;
    a.vertical = g.vertical;
    a.table = g.table;
    a.capacity_h = with_capacity ? g.capacity_h : 0.0;
    a.capacity_v = with_capacity ? g.capacity_v : 0.0;
    a.model = rudy_model_;
    a.temperature = rudy_temperature_;
    a.adjoint_h = g.adjoint_h;
    a.adjoint_v = g.adjoint_v;
    a.utilization = g.utilization;
    a.partials = g.partials;
    return a;
}

void Engine::setRudyCapacity(bool validation, double horizontal, double vertical) {
    RudyGrid& g = validation ? rudy_validation_ : rudy_main_;
    require(g.columns > 0, "RUDY grid is not enabled.");
    g.capacity_h = horizontal;
    g.capacity_v = vertical;
}

RudyReport Engine::rudyEvaluate(const double2* positions, bool validation) {
    const RudyGrid& g = validation ? rudy_validation_ : rudy_main_;
    require(g.columns > 0, "RUDY grid is not enabled.");
    const bool with_capacity = g.capacity_h > 0.0 && g.capacity_v > 0.0;
    const RudyArgs ra = rudyArgs(g, positions, with_capacity);
    launchRudyDeposit(ra, stream_);
    launchRudyPrefix(ra, stream_);
    launchRudyMetrics(ra, g.blocks, stream_);
    ReduceArgs rr{};
    for (int k = 0; k < 5; ++k) rr.sources[k] = ReduceSource{g.partials, g.blocks, 1, k * g.blocks, k == 4 ? 1 : 0, k};
    rr.source_count = 5;
    for (int k = 0; k < 5; ++k) rr.offsets[k + 1] = rr.offsets[k] + g.blocks;
    rr.staged_capacity = kReduceStaged;
    rr.scalars = rudy_scalars_;
    rr.totals = nullptr;
    launchReduce(rr, stream_);
    launches_ += 5;
    checkCuda(cudaMemcpyAsync(host_rudy_, rudy_scalars_, 5 * sizeof(double), cudaMemcpyDeviceToHost, stream_),
              "Download RUDY scalars");
    const std::size_t bins = static_cast<std::size_t>(g.columns) * static_cast<std::size_t>(g.rows);
    std::vector<double> utilization;
    if (with_capacity) {
        utilization.resize(bins);
        checkCuda(cudaMemcpyAsync(utilization.data(), g.utilization, bins * sizeof(double), cudaMemcpyDeviceToHost,
                                  stream_),
                  "Download RUDY utilisation");
    }
    checkCuda(cudaStreamSynchronize(stream_), "RUDY evaluation");
    RudyReport r;
    r.horizontal_total = host_rudy_[1];
    r.vertical_total = host_rudy_[2];
    r.horizontal_mean = r.horizontal_total / static_cast<double>(bins);
    r.vertical_mean = r.vertical_total / static_cast<double>(bins);
    r.horizontal_capacity = with_capacity ? g.capacity_h : 0.0;
    r.vertical_capacity = with_capacity ? g.capacity_v : 0.0;
    if (with_capacity) {
        r.energy = host_rudy_[0];
        r.proxy_overflow = host_rudy_[3] / static_cast<double>(bins);
        r.maximum_utilization = std::max(0.0, host_rudy_[4]);
        // The 95th percentile of the sorted per-bin utilisation (Rudy.cpp:310-314).
        const std::size_t index = static_cast<std::size_t>(
            std::floor(0.95 * static_cast<double>(std::max<std::size_t>(1U, bins - 1U))));
        std::nth_element(utilization.begin(), utilization.begin() + static_cast<std::ptrdiff_t>(index),
                         utilization.end());
        r.p95_utilization = utilization[index];
    }
    return r;
}

void Engine::depositLayers(const double2* positions, int64_t* movable, int64_t* macro, int64_t* filler) {
    // The metrics pass consumes (reads and clears) the layers, so the parity hook
    // runs the scatter alone, copies the three layers out and clears them again.
    ScatterArgs sa{};
    sa.mode = kGiven;
    sa.particle_count = static_cast<int>(particle_count_);
    sa.positions = positions;
    sa.size = size_;
    sa.layer = layer_;
    sa.llx = region_.llx;
    sa.lly = region_.lly;
    sa.urx = region_.urx;
    sa.ury = region_.ury;
    sa.bin_w = bin_w_;
    sa.bin_h = bin_h_;
    sa.bins_x = bins_x_;
    sa.bins_y = bins_y_;
    sa.layers = layers_;
    sa.totals = totals_;
    sa.partials = partials_sc_;
    sa.group_partials = sc_groups_.partials;
    sa.group_counters = sc_groups_.counters;
    beginKernel(kKindScatter);
    launchScatter(sa, particle_count_ > 0 ? scatter_blocks_ : 0, stream_);
    endKernel();
    launches_ += 1;
    const std::size_t bins = static_cast<std::size_t>(bin_count_);
    int64_t* out[3] = {movable, macro, filler};
    for (int k = 0; k < 3; ++k) {
        if (out[k] == nullptr) continue;
        checkCuda(cudaMemcpyAsync(out[k], layers_ + k * bins, bins * sizeof(int64_t), cudaMemcpyDeviceToHost, stream_),
                  "Download density layers");
    }
    checkCuda(cudaMemsetAsync(layers_, 0, 3 * bins * sizeof(unsigned long long), stream_), "clear layers");
    checkCuda(cudaMemsetAsync(totals_, 0, 4 * sizeof(unsigned long long), stream_), "clear totals");
    checkCuda(cudaStreamSynchronize(stream_), "density layers");
    collectTimings();
}

}  // namespace mpgp
