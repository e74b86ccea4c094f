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
// Nets are grouped by degree into buckets of G = 2, 4, 8, 16, 32 lanes per net
// (a warp loop for degree > 32); the G lanes of a net hold one pin each, so the
// max/min and the four exponential sums are G-wide shuffle reductions and the
// pin loads of a warp are contiguous.  Coordinates are taken relative to the
// net's first pin in FP64 and then carried in FP32 (max-shifted exponentials),
// per-net totals are accumulated in FP64.  The per-pin gradient is written to
// a pin-indexed buffer (no atomics); the particle gather sums it in a fixed
// order, so the wire gradient is deterministic.
#include <cfloat>

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
        const float epx = pin_ok ? expf((dx - max_x) * a.inv_gamma) : 0.0f;
        const float enx = pin_ok ? expf((min_x - dx) * a.inv_gamma) : 0.0f;
        const float epy = pin_ok ? expf((dy - max_y) * a.inv_gamma) : 0.0f;
        const float eny = pin_ok ? expf((min_y - dy) * a.inv_gamma) : 0.0f;
        const float spx = groupSum<G>(epx);
        const float snx = groupSum<G>(enx);
        const float spy = groupSum<G>(epy);
        const float sny = groupSum<G>(eny);
        if (net_ok && sub == 0) {
            const float span = (max_x - min_x) + (max_y - min_y);
            const float soft = a.gamma * (logf(spx) + logf(snx) + logf(spy) + logf(sny));
            smooth += static_cast<double>(weight) * (static_cast<double>(span) + static_cast<double>(soft));
            hpwl += static_cast<double>(weight) * static_cast<double>(span);
        }
        if (a.gradient && pin_ok && p.particle >= 0) {
            const float gx = weight * (epx / spx - enx / snx);
            const float gy = weight * (epy / spy - eny / sny);
            a.pin_gradient[begin + sub] = make_float2(gx, gy);
        }
    }
}

// One warp per net, any degree: three passes over the pins.
__device__ void netWarps(const WirelengthArgs& a, int first, int count, double& smooth, double& hpwl) {
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int warps = blockDim.x >> 5;
    for (int local = warp; local < count; local += warps) {
        const int begin = a.net_start[first + local];
        const int end = a.net_start[first + local + 1];
        const float weight = a.net_weight[first + local];
        const PinPoint first_pin = loadPin(a, begin);
        const double rx = first_pin.x;
        const double ry = first_pin.y;
        float max_x = -FLT_MAX, min_x = FLT_MAX, max_y = -FLT_MAX, min_y = FLT_MAX;
        for (int pin = begin + lane; pin < end; pin += 32) {
            const PinPoint p = loadPin(a, pin);
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
            const PinPoint p = loadPin(a, pin);
            const float dx = static_cast<float>(p.x - rx);
            const float dy = static_cast<float>(p.y - ry);
            spx += expf((dx - max_x) * a.inv_gamma);
            snx += expf((min_x - dx) * a.inv_gamma);
            spy += expf((dy - max_y) * a.inv_gamma);
            sny += expf((min_y - dy) * a.inv_gamma);
        }
        spx = groupSum<32>(spx);
        snx = groupSum<32>(snx);
        spy = groupSum<32>(spy);
        sny = groupSum<32>(sny);
        if (lane == 0) {
            const float span = (max_x - min_x) + (max_y - min_y);
            const float soft = a.gamma * (logf(spx) + logf(snx) + logf(spy) + logf(sny));
            smooth += static_cast<double>(weight) * (static_cast<double>(span) + static_cast<double>(soft));
            hpwl += static_cast<double>(weight) * static_cast<double>(span);
        }
        if (a.gradient) {
            for (int pin = begin + lane; pin < end; pin += 32) {
                const PinPoint p = loadPin(a, pin);
                if (p.particle < 0) continue;
                const float dx = static_cast<float>(p.x - rx);
                const float dy = static_cast<float>(p.y - ry);
                const float gx = weight * (expf((dx - max_x) * a.inv_gamma) / spx - expf((min_x - dx) * a.inv_gamma) / snx);
                const float gy = weight * (expf((dy - max_y) * a.inv_gamma) / spy - expf((min_y - dy) * a.inv_gamma) / sny);
                a.pin_gradient[pin] = make_float2(gx, gy);
            }
        }
    }
}

__global__ void __launch_bounds__(kThreads) wirelengthKernel(WirelengthArgs a) {
    const int4 work = a.block_work[blockIdx.x];
    double values[2] = {0.0, 0.0};
    switch (work.x) {
        case 2: netGroups<2>(a, work.y, work.z, values[0], values[1]); break;
        case 4: netGroups<4>(a, work.y, work.z, values[0], values[1]); break;
        case 8: netGroups<8>(a, work.y, work.z, values[0], values[1]); break;
        case 16: netGroups<16>(a, work.y, work.z, values[0], values[1]); break;
        case 32: netGroups<32>(a, work.y, work.z, values[0], values[1]); break;
        default: netWarps(a, work.y, work.z, values[0], values[1]); break;
    }
    const bool is_max[2] = {false, false};
    blockReduce<2>(values, is_max);
    if (threadIdx.x == 0) {
        a.partials[2 * blockIdx.x + 0] = values[0];
        a.partials[2 * blockIdx.x + 1] = values[1];
    }
}

}  // namespace

void launchWirelength(const WirelengthArgs& args, int blocks, cudaStream_t stream) {
    if (blocks <= 0) return;
    wirelengthKernel<<<blocks, kThreads, 0, stream>>>(args);
}

}  // namespace mpgp
