// Net-parallel log-sum-exp wirelength, HPWL and per-pin gradient.
//
// Restates evaluateSmoothWirelength (AdaptiveGlobalPlacer.cpp:29-82) and the
// reference CUDA kernels computeNetBoundsKernel / computeNetSumsKernel /
// computePinGradientKernel (CudaPlacementBackend.cu:209-337) as ONE pass:
//
//   W_e = w_e * ( max x + g ln sum exp((x_i - max x)/g) - min x + g ln sum exp((min x - x_i)/g)
//               + the same in y ),           HPWL_e = w_e * (max x - min x + max y - min y)
//   dW_e/dx_i = w_e * ( exp((x_i - max)/g) / S+ - exp((min - x_i)/g) / S- )
//
// Nets are grouped by degree into buckets.  Two-pin nets (most of a netlist)
// take one thread each and a closed form of the same expressions: with
// d = x_a - x_b and t = exp(-|d|/g), W = |d| + 2 g ln(1 + t) and
// dW/dx_a = -dW/dx_b = w tanh(d / 2g) = w sign(d) (1 - t) / (1 + t).  Larger
// nets take G = 4, 8, 16, 32 lanes (a warp loop above 32); the G lanes of a
// net hold one pin each, so the max/min and the four exponential sums are
// G-wide shuffle reductions and the pin loads of a warp are contiguous.
// Coordinates are taken relative to the net's first pin in FP64 and then
// carried in FP32 (max-shifted exponentials, hardware exp2/log2/reciprocal),
// per-net totals are accumulated in FP64.  The per-pin gradient is written to
// a pin-indexed buffer (no atomics); the particle gather sums it in a fixed
// order, so the wire gradient is deterministic.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <mutex>
#include <string>

#include "common.cuh"
#include "kernels.cuh"

namespace mpgp {
namespace {

struct PinPoint {
    double x, y;
    int particle;
};

__device__ __forceinline__ PinPoint loadPin(const WirelengthArgs& a, int pin) {
    PinPoint p;
    p.particle = a.pin_particle[pin];
    if (p.particle >= 0) {
        const double2 c = a.positions[p.particle];
        const float2 o = a.pin_offset[pin];
        p.x = c.x + static_cast<double>(o.x);
        p.y = c.y + static_cast<double>(o.y);
    } else {
        const double2 s = a.static_pins[-p.particle - 1];
        p.x = s.x;
        p.y = s.y;
    }
    return p;
}

template <int G>
__device__ __forceinline__ float groupMax(float v) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o, G));
    return v;
}

template <int G>
__device__ __forceinline__ float groupMin(float v) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o, G));
    return v;
}

template <int G>
__device__ __forceinline__ float groupSum(float v) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, G);
    return v;
}

// exp(v) for v <= 0 and ln(v) for v >= 1 on the special-function unit.
__device__ __forceinline__ float fastExp(float v) { return __expf(v); }
__device__ __forceinline__ float fastLog(float v) { return __logf(v); }

// One two-pin net.  Two-pin nets lead the layout: net k's pins are 2k and 2k + 1,
// so each of the pin arrays is read as one vector (the arrays start 256-byte aligned).
__device__ __forceinline__ void netPair(const WirelengthArgs& a, int net, double& smooth, double& hpwl) {
    const int2 particle = reinterpret_cast<const int2*>(a.pin_particle)[net];
    const float4 offset = reinterpret_cast<const float4*>(a.pin_offset)[net];
    const int2 slot = a.gradient ? reinterpret_cast<const int2*>(a.pin_slot)[net] : make_int2(0, 0);
    const float weight = a.net_weight[net];
    const auto place = [&](int index, float ox, float oy) {
        PinPoint pin;
        pin.particle = index;
        if (index >= 0) {
            const double2 c = a.positions[index];
            pin.x = c.x + static_cast<double>(ox);
            pin.y = c.y + static_cast<double>(oy);
        } else {
            const double2 s = a.static_pins[-index - 1];
            pin.x = s.x;
            pin.y = s.y;
        }
        return pin;
    };
    const PinPoint p = place(particle.x, offset.x, offset.y);
    const PinPoint q = place(particle.y, offset.z, offset.w);
    const float dx = static_cast<float>(p.x - q.x);
    const float dy = static_cast<float>(p.y - q.y);
    const float ax = fabsf(dx), ay = fabsf(dy);
    const float tx = fastExp(-ax * a.inv_gamma);
    const float ty = fastExp(-ay * a.inv_gamma);
    const float span = ax + ay;
    const float soft = 2.0f * a.gamma * (fastLog(1.0f + tx) + fastLog(1.0f + ty));
    smooth += static_cast<double>(weight) * (static_cast<double>(span) + static_cast<double>(soft));
    hpwl += static_cast<double>(weight) * static_cast<double>(span);
    if (a.gradient) {
        const float gx = copysignf(weight * __fdividef(1.0f - tx, 1.0f + tx), dx);
        const float gy = copysignf(weight * __fdividef(1.0f - ty, 1.0f + ty), dy);
        if (p.particle >= 0) a.pin_gradient[slot.x] = make_float2(gx, gy);
        if (q.particle >= 0) a.pin_gradient[slot.y] = make_float2(-gx, -gy);
    }
}

// Two-pin nets, one thread per net and round; the bucket's pins are consecutive pairs.
__device__ void netPairs(const WirelengthArgs& a, int first, int count, double& smooth, double& hpwl) {
    for (int local = static_cast<int>(threadIdx.x); local < count; local += static_cast<int>(blockDim.x)) {
        netPair(a, first + local, smooth, hpwl);
    }
}

// G lanes per net, degree <= G.
template <int G>
__device__ void netGroups(const WirelengthArgs& a, int first, int count, double& smooth, double& hpwl) {
    constexpr int kPerWarp = 32 / G;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int warps = blockDim.x >> 5;
    const int group = lane / G;
    const int sub = lane % G;
    for (int base = warp * kPerWarp; base < count; base += warps * kPerWarp) {
        const int local = base + group;
        const bool net_ok = local < count;
        int begin = 0, degree = 0;
        float weight = 0.0f;
        if (net_ok) {
            begin = a.net_start[first + local];
            degree = a.net_start[first + local + 1] - begin;
            weight = a.net_weight[first + local];
        }
        const bool pin_ok = net_ok && sub < degree;
        PinPoint p{0.0, 0.0, -1};
        if (pin_ok) p = loadPin(a, begin + sub);
        const double rx = __shfl_sync(0xffffffffu, p.x, lane - sub);
        const double ry = __shfl_sync(0xffffffffu, p.y, lane - sub);
        const float dx = pin_ok ? static_cast<float>(p.x - rx) : 0.0f;
        const float dy = pin_ok ? static_cast<float>(p.y - ry) : 0.0f;
        const float max_x = groupMax<G>(pin_ok ? dx : -FLT_MAX);
        const float min_x = groupMin<G>(pin_ok ? dx : FLT_MAX);
        const float max_y = groupMax<G>(pin_ok ? dy : -FLT_MAX);
        const float min_y = groupMin<G>(pin_ok ? dy : FLT_MAX);
        const float epx = pin_ok ? fastExp((dx - max_x) * a.inv_gamma) : 0.0f;
        const float enx = pin_ok ? fastExp((min_x - dx) * a.inv_gamma) : 0.0f;
        const float epy = pin_ok ? fastExp((dy - max_y) * a.inv_gamma) : 0.0f;
        const float eny = pin_ok ? fastExp((min_y - dy) * a.inv_gamma) : 0.0f;
        const float spx = groupSum<G>(epx);
        const float snx = groupSum<G>(enx);
        const float spy = groupSum<G>(epy);
        const float sny = groupSum<G>(eny);
        if (net_ok && sub == 0) {
            const float span = (max_x - min_x) + (max_y - min_y);
            const float soft = a.gamma * (fastLog(spx) + fastLog(snx) + fastLog(spy) + fastLog(sny));
            smooth += static_cast<double>(weight) * (static_cast<double>(span) + static_cast<double>(soft));
            hpwl += static_cast<double>(weight) * static_cast<double>(span);
        }
        if (a.gradient && pin_ok && p.particle >= 0) {
            const float gx = weight * (__fdividef(epx, spx) - __fdividef(enx, snx));
            const float gy = weight * (__fdividef(epy, spy) - __fdividef(eny, sny));
            a.pin_gradient[a.pin_slot[begin + sub]] = make_float2(gx, gy);
        }
    }
}

// One net of any degree on one warp: three passes over its pins.  `load(pin)`
// returns the pin's position and particle; store(pin, gradient) keeps a
// movable pin's gradient.
template <class Loader, class Store>
__device__ void netOnWarp(const Loader& load, int begin, int end, float weight, float gamma, float inv_gamma,
                          bool gradient, const Store& store, double& smooth, double& hpwl) {
    const int lane = threadIdx.x & 31;
    {
        const PinPoint first_pin = load(begin);
        const double rx = first_pin.x;
        const double ry = first_pin.y;
        float max_x = -FLT_MAX, min_x = FLT_MAX, max_y = -FLT_MAX, min_y = FLT_MAX;
        for (int pin = begin + lane; pin < end; pin += 32) {
            const PinPoint p = load(pin);
            const float dx = static_cast<float>(p.x - rx);
            const float dy = static_cast<float>(p.y - ry);
            max_x = fmaxf(max_x, dx);
            min_x = fminf(min_x, dx);
            max_y = fmaxf(max_y, dy);
            min_y = fminf(min_y, dy);
        }
        max_x = groupMax<32>(max_x);
        min_x = groupMin<32>(min_x);
        max_y = groupMax<32>(max_y);
        min_y = groupMin<32>(min_y);
        float spx = 0.0f, snx = 0.0f, spy = 0.0f, sny = 0.0f;
        for (int pin = begin + lane; pin < end; pin += 32) {
            const PinPoint p = load(pin);
            const float dx = static_cast<float>(p.x - rx);
            const float dy = static_cast<float>(p.y - ry);
            spx += expf((dx - max_x) * inv_gamma);
            snx += expf((min_x - dx) * inv_gamma);
            spy += expf((dy - max_y) * inv_gamma);
            sny += expf((min_y - dy) * inv_gamma);
        }
        spx = groupSum<32>(spx);
        snx = groupSum<32>(snx);
        spy = groupSum<32>(spy);
        sny = groupSum<32>(sny);
        if (lane == 0) {
            const float span = (max_x - min_x) + (max_y - min_y);
            const float soft = gamma * (logf(spx) + logf(snx) + logf(spy) + logf(sny));
            smooth += static_cast<double>(weight) * (static_cast<double>(span) + static_cast<double>(soft));
            hpwl += static_cast<double>(weight) * static_cast<double>(span);
        }
        if (gradient) {
            for (int pin = begin + lane; pin < end; pin += 32) {
                const PinPoint p = load(pin);
                if (p.particle < 0) continue;
                const float dx = static_cast<float>(p.x - rx);
                const float dy = static_cast<float>(p.y - ry);
                const float gx = weight * (expf((dx - max_x) * inv_gamma) / spx - expf((min_x - dx) * inv_gamma) / snx);
                const float gy = weight * (expf((dy - max_y) * inv_gamma) / spy - expf((min_y - dy) * inv_gamma) / sny);
                store(pin, make_float2(gx, gy));
            }
        }
    }
}

struct EnginePinLoader {
    const WirelengthArgs* a;
    __device__ PinPoint operator()(int pin) const { return loadPin(*a, pin); }
};

struct SlotStore {
    const WirelengthArgs* a;
    __device__ void operator()(int pin, float2 g) const { a->pin_gradient[a->pin_slot[pin]] = g; }
};

struct PinStore {
    float2* pin_gradient;
    __device__ void operator()(int pin, float2 g) const { pin_gradient[pin] = g; }
};

// Warp-per-net bucket (degree > 32) of the engine's wirelength pass.
__device__ void netWarps(const WirelengthArgs& a, int first, int count, double& smooth, double& hpwl) {
    const int warp = threadIdx.x >> 5;
    const int warps = blockDim.x >> 5;
    const EnginePinLoader load{&a};
    for (int local = warp; local < count; local += warps) {
        netOnWarp(load, a.net_start[first + local], a.net_start[first + local + 1], a.net_weight[first + local],
                  a.gamma, a.inv_gamma, a.gradient != 0, SlotStore{&a}, smooth, hpwl);
    }
}

// One block of the pass: `block` of `grid` blocks (the launch's, or its instance's in
// a batched launch).
__device__ __forceinline__ void wirelengthBlock(const WirelengthArgs& a, int block, int grid) {
    const int4 work = a.block_work[block];
    double values[2] = {0.0, 0.0};
    switch (work.x) {
        case 1: netPairs(a, work.y, work.z, values[0], values[1]); break;
        case 4: netGroups<4>(a, work.y, work.z, values[0], values[1]); break;
        case 8: netGroups<8>(a, work.y, work.z, values[0], values[1]); break;
        case 16: netGroups<16>(a, work.y, work.z, values[0], values[1]); break;
        case 32: netGroups<32>(a, work.y, work.z, values[0], values[1]); break;
        default: netWarps(a, work.y, work.z, values[0], values[1]); break;
    }
    const bool is_max[2] = {false, false};
    blockReduce<2>(values, is_max);
    if (threadIdx.x == 0) {
        a.partials[block] = values[0];
        a.partials[grid + block] = values[1];
    }
    reduceGroups<2>(a.partials, a.group_partials, a.group_counters, is_max, static_cast<unsigned>(block),
                    static_cast<unsigned>(grid));
}

__global__ void __launch_bounds__(kThreads) wirelengthKernel(WirelengthArgs a) {
    releaseNext();
    waitForPrior();
    wirelengthBlock(a, static_cast<int>(blockIdx.x), static_cast<int>(gridDim.x));
}

__global__ void __launch_bounds__(kThreads) wirelengthBatchKernel(const WirelengthArgs* args, const int* offsets,
                                                                  int count) {
    releaseNext();
    waitForPrior();
    const int3 slot = batchSlot(offsets, count, static_cast<int>(blockIdx.x));
    const WirelengthArgs a = args[slot.x];  // a private copy: stores through its pointers cannot alias it
    wirelengthBlock(a, slot.y, slot.z);
}

}  // namespace

void launchWirelength(const WirelengthArgs& args, int blocks, cudaStream_t stream) {
    if (blocks <= 0) return;
    launchChained("Launch the wirelength pass", wirelengthKernel, dim3(blocks), dim3(kThreads), 0, stream, args);
}

void launchWirelengthBatch(const WirelengthArgs* args, const int* offsets, int count, int blocks,
                           cudaStream_t stream) {
    if (blocks <= 0 || count <= 0) return;
    launchChained("Launch the batched wirelength pass", wirelengthBatchKernel, dim3(blocks), dim3(kThreads), 0,
                  stream, args, offsets, count);
}

// ---- allocation-free variant --------------------------------------------------------
//
// The same per-net LSE pass for callers that own all device memory and cannot
// let the library allocate.  Its only scratch -- the per-pin gradient staging
// buffer and the per-block partial sums -- lives in one file-scope device array
// of fixed size, so the library never calls cudaMalloc for it.  Every GPU that
// loads the library holds this array (8.03 MiB) until the process exits.
namespace {

constexpr int kNoAllocMaxBlocks = 2048;
constexpr std::size_t kNoAllocPinBytes = sizeof(float2) * static_cast<std::size_t>(kNoAllocMaxPins);
constexpr std::size_t kNoAllocScratchBytes = kNoAllocPinBytes + sizeof(double) * 2 * kNoAllocMaxBlocks;
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) unsigned char g_wirelength_scratch[kNoAllocScratchBytes];

std::mutex g_scratch_mutex;
// The array's device address per device, and the ID of the CUDA context it was
// looked up in: a device reset (or a caller's own context) makes a new context,
// in which the old address is no longer valid, so the address is looked up again.
void* g_scratch_address[kNoAllocMaxDevices] = {};
unsigned long long g_scratch_context[kNoAllocMaxDevices] = {};

// The unique ID of the calling thread's current CUDA context (0 if it has none),
// through the driver entry points the runtime exposes (no libcuda link needed).
unsigned long long currentContextId() {
    using GetCurrent = int (*)(void**);
    using GetId = int (*)(void*, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult found{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &found) == cudaSuccess &&
            found == cudaDriverEntryPointSuccess) {
            get_current = reinterpret_cast<GetCurrent>(fn);
        }
        fn = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &fn, cudaEnableDefault, &found) == cudaSuccess &&
            found == cudaDriverEntryPointSuccess) {
            get_id = reinterpret_cast<GetId>(fn);
        }
    });
    void* context = nullptr;
    unsigned long long id = 0;
    if (get_current == nullptr || get_id == nullptr || get_current(&context) != 0 || context == nullptr ||
        get_id(context, &id) != 0) {
        return 0;
    }
    return id;
}

// Pins as the caller lays them out: pin_xy is the offset from the particle
// centre, or the absolute position of a pin whose particle is < 0.
struct CallerPinLoader {
    const double2* positions;
    const int* pin_particle;
    const double2* pin_xy;
    int particle_count;
    __device__ PinPoint operator()(int pin) const {
        PinPoint p;
        p.particle = pin_particle[pin];
        const double2 v = pin_xy[pin];
        if (p.particle >= 0 && p.particle < particle_count) {
            const double2 c = positions[p.particle];
            p.x = c.x + v.x;
            p.y = c.y + v.y;
        } else {
            p.particle = -1;  // static (or an out-of-range index, treated as static)
            p.x = v.x;
            p.y = v.y;
        }
        return p;
    }
};

__global__ void __launch_bounds__(kThreads) noAllocNetKernel(CallerPinLoader load, const int* net_pin_start,
                                                            const double* net_weight, int net_count, int pin_count,
                                                            float gamma, float inv_gamma, unsigned char* scratch) {
    float2* pin_gradient = reinterpret_cast<float2*>(scratch);
    double* partials = reinterpret_cast<double*>(scratch + kNoAllocPinBytes);
    double values[2] = {0.0, 0.0};
    const int warps_total = static_cast<int>((gridDim.x * blockDim.x) >> 5);
    for (int net = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5); net < net_count;
         net += warps_total) {
        const int begin = net_pin_start[net];
        const int end = net_pin_start[net + 1];
        if (begin < 0 || end > pin_count || end < begin) continue;  // malformed CSR: never write outside scratch
        if (end - begin < 2) continue;  // single-pin nets contribute nothing; their slots stay zero
        netOnWarp(load, begin, end, static_cast<float>(net_weight[net]), gamma, inv_gamma, true,
                  PinStore{pin_gradient}, values[0], values[1]);
    }
    const bool is_max[2] = {false, false};
    blockReduce<2>(values, is_max);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x + 0] = values[0];
        partials[2 * blockIdx.x + 1] = values[1];
    }
}

__global__ void __launch_bounds__(kThreads) noAllocParticleKernel(const int* particle_pin_start,
                                                                 const int* particle_pins, const int* pin_particle,
                                                                 int particle_count,
                                                                 int pin_count, const unsigned char* scratch,
                                                                 int net_blocks, double2* wire_gradient,
                                                                 double* totals) {
    const float2* pin_gradient = reinterpret_cast<const float2*>(scratch);
    const double* partials = reinterpret_cast<const double*>(scratch + kNoAllocPinBytes);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < particle_count) {
        double gx = 0.0, gy = 0.0;
        for (int j = particle_pin_start[i]; j < particle_pin_start[i + 1]; ++j) {
            const int pin = particle_pins[j];
            // Only a pin that really belongs to this particle adds its gradient; a pin
            // listed under another particle (or out of range) would read a slot this
            // call did not write for it.
            if (pin < 0 || pin >= pin_count || pin_particle[pin] != i) continue;
            const float2 g = pin_gradient[pin];
            gx += static_cast<double>(g.x);
            gy += static_cast<double>(g.y);
        }
        wire_gradient[i] = make_double2(gx, gy);
    }
    if (blockIdx.x == 0) {  // fixed-order totals of the net pass (deterministic)
        double values[2] = {0.0, 0.0};
        for (int row = threadIdx.x; row < net_blocks; row += blockDim.x) {
            values[0] += partials[2 * row + 0];
            values[1] += partials[2 * row + 1];
        }
        const bool is_max[2] = {false, false};
        blockReduce<2>(values, is_max);
        if (threadIdx.x == 0) {
            totals[0] = values[0];
            totals[1] = values[1];
        }
    }
}

}  // namespace

void launchWirelengthNoAlloc(const NoAllocWirelengthArgs& a) {
    require(a.net_count >= 0 && a.pin_count >= 0 && a.particle_count >= 0, "Counts must be non-negative.");
    if (a.pin_count > kNoAllocMaxPins) {
        fail(MPGP_ERR_INVALID_ARGUMENT, "pin_count " + std::to_string(a.pin_count) +
                                            " exceeds the allocation-free limit of " +
                                            std::to_string(kNoAllocMaxPins) + " pins.");
    }
    require(std::isfinite(a.smoothing) && a.smoothing > 0.0, "Smoothing must be positive and finite.");
    require(a.net_pin_start != nullptr && a.totals != nullptr, "net_pin_start and totals are required.");
    require(a.pin_count == 0 || (a.pin_particle != nullptr && a.pin_xy != nullptr), "Pin arrays are required.");
    require(a.net_count == 0 || a.net_weight != nullptr, "Net weights are required.");
    require(a.particle_count == 0 || (a.positions != nullptr && a.particle_pin_start != nullptr &&
                                      a.particle_pins != nullptr && a.wire_gradient != nullptr),
            "Particle arrays are required.");
    int device = 0;
    checkCuda(cudaGetDevice(&device), "Query the current device");
    require(device >= 0 && device < kNoAllocMaxDevices, "Device index out of range.");
    void* scratch = nullptr;
    {
        // Set-up, once per device and context, with that device current: the
        // host-side name of the array is not a device address, so ask the runtime
        // for it.  The lookup makes the device's primary context current when the
        // thread has none yet, so the context is identified after it.
        const unsigned long long context = currentContextId();
        std::lock_guard<std::mutex> lock(g_scratch_mutex);
        if (g_scratch_address[device] == nullptr || context == 0 || g_scratch_context[device] != context) {
            void* address = nullptr;
            checkCuda(cudaGetSymbolAddress(&address, g_wirelength_scratch), "Locate the wirelength scratch array");
            g_scratch_address[device] = address;
            g_scratch_context[device] = currentContextId();
        }
        scratch = g_scratch_address[device];
    }
    const cudaStream_t stream = static_cast<cudaStream_t>(a.stream);
    const float gamma = static_cast<float>(std::max(a.smoothing, kEpsilon));
    const float inv_gamma = static_cast<float>(1.0 / std::max(a.smoothing, kEpsilon));
    const int net_blocks = std::min(kNoAllocMaxBlocks, std::max(1, ceilDiv(a.net_count, kThreads / 32)));
    const CallerPinLoader load{reinterpret_cast<const double2*>(a.positions), a.pin_particle,
                               reinterpret_cast<const double2*>(a.pin_xy), a.particle_count};
    // Every pin slot of this call starts at zero: a pin that no well-formed net of
    // at least two pins covers (a pin outside every net's range, a net skipped as
    // malformed) then adds nothing, instead of an earlier call's value.
    if (a.pin_count > 0) {
        checkCuda(cudaMemsetAsync(scratch, 0, sizeof(float2) * static_cast<std::size_t>(a.pin_count), stream),
                  "Clear the allocation-free pin slots");
    }
    noAllocNetKernel<<<net_blocks, kThreads, 0, stream>>>(load, a.net_pin_start, a.net_weight, a.net_count,
                                                          a.pin_count, gamma, inv_gamma,
                                                          static_cast<unsigned char*>(scratch));
    checkCuda(cudaGetLastError(), "Launch the allocation-free net pass");
    const int particle_blocks = std::max(1, ceilDiv(a.particle_count, kThreads));
    noAllocParticleKernel<<<particle_blocks, kThreads, 0, stream>>>(
        a.particle_pin_start, a.particle_pins, a.pin_particle, a.particle_count, a.pin_count,
        static_cast<const unsigned char*>(scratch), net_blocks, reinterpret_cast<double2*>(a.wire_gradient),
        a.totals);
    checkCuda(cudaGetLastError(), "Launch the allocation-free particle pass");
}

}  // namespace mpgp
