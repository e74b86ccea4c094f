// RUDY routing-demand map, hotspot penalty and its subgradient on the device.
//
// Restates evaluateRudy (Rudy.cpp:227-456) for the adaptive controller's
// routability term (AdaptiveGlobalPlacer.cpp:149-172, 201-331):
//   deposit   one thread per net: the pin bounding box, expanded to
//             minimum_span_in_bins where a net is thinner (calculateNetBox,
//             Rudy.cpp:120-152), clipped to the core, and its exact rectangle
//             overlap with every covered bin added as horizontal demand
//             w * overlap / y_span and vertical demand w * overlap / x_span.
//             As in the density scatter the terms are quantized to int64 (units
//             of bin_w * 2^-32 and bin_h * 2^-32) and added with integer
//             atomics, so the maps are bit-exact run to run.
//   metrics   one thread per bin: utilisation against the frozen capacities,
//             the penalty model (hinge L2 / softplus L2 / hinge L4,
//             evaluatePenalty Rudy.cpp:83-100), its adjoint, the energy, the
//             proxy overflow, the maximum utilisation and the demand totals
//             (FP64 block partials, reduced in a fixed order); the maps are
//             cleared for the next deposit.
//   gradient  one thread per net: the Clarke subgradient of the overlap map
//             with respect to the four box edges (Rudy.cpp:320-400), split over
//             the pins that sit on each extremal edge (Rudy.cpp:402-452) and
//             written to the pins' particle-ordered slots for the gather.
// Arithmetic is FP64 in the reference's order.
#include <algorithm>
#include <cfloat>
#include <cmath>

#include "common.cuh"
#include "kernels.cuh"

namespace mpgp {
namespace {

struct Box {
    double left, right, bottom, top;
    double raw_left, raw_right, raw_bottom, raw_top;
    double x_span, y_span;
    bool x_physical, y_physical;
};

__device__ __forceinline__ double2 pinPosition(const RudyArgs& a, int pin) {
    const int particle = a.pin_particle[pin];
    if (particle >= 0) {
        const double2 c = a.positions[particle];
        const float2 o = a.pin_offset[pin];
        return make_double2(c.x + static_cast<double>(o.x), c.y + static_cast<double>(o.y));
    }
    return a.static_pins[-particle - 1];
}

__device__ Box netBox(const RudyArgs& a, int begin, int end) {
    Box b;
    b.left = DBL_MAX;
    b.right = -DBL_MAX;
    b.bottom = DBL_MAX;
    b.top = -DBL_MAX;
    for (int pin = begin; pin < end; ++pin) {
        const double2 p = pinPosition(a, pin);
        b.left = fmin(b.left, p.x);
        b.right = fmax(b.right, p.x);
        b.bottom = fmin(b.bottom, p.y);
        b.top = fmax(b.top, p.y);
    }
    const double raw_x_span = b.right - b.left;
    const double raw_y_span = b.top - b.bottom;
    b.raw_left = b.left;
    b.raw_right = b.right;
    b.raw_bottom = b.bottom;
    b.raw_top = b.top;
    b.x_physical = true;
    b.y_physical = true;
    if (raw_x_span < a.minimum_x_span) {
        const double center = (b.left + b.right) * 0.5;
        b.left = center - a.minimum_x_span * 0.5;
        b.right = center + a.minimum_x_span * 0.5;
        b.x_physical = false;
    }
    if (raw_y_span < a.minimum_y_span) {
        const double center = (b.bottom + b.top) * 0.5;
        b.bottom = center - a.minimum_y_span * 0.5;
        b.top = center + a.minimum_y_span * 0.5;
        b.y_physical = false;
    }
    b.x_span = fmax(b.right - b.left, kEpsilon);
    b.y_span = fmax(b.top - b.bottom, kEpsilon);
    return b;
}

__device__ __forceinline__ int startBin(double coordinate, double lower, double length, int count) {
    return max(0, min(count - 1, static_cast<int>(floor((coordinate - lower) / length))));
}

__device__ __forceinline__ int endBin(double coordinate, double lower, double length, int count) {
    return max(0, min(count - 1, static_cast<int>(ceil((coordinate - lower) / length) - 1.0)));
}

__device__ __forceinline__ double overlapLength(double lower_a, double upper_a, double lower_b, double upper_b) {
    return fmax(0.0, fmin(upper_a, upper_b) - fmax(lower_a, lower_b));
}

__device__ __forceinline__ bool approximatelyEqual(double left, double right) {
    return fabs(left - right) <= 1e-10 * fmax(1.0, fmax(fabs(left), fabs(right)));
}

__device__ __forceinline__ double upperDerivative(double upper, double bin_lower, double bin_upper, double overlap) {
    if (upper > bin_lower + kEpsilon && upper < bin_upper - kEpsilon && overlap > kEpsilon) return 1.0;
    if (approximatelyEqual(upper, bin_lower) || approximatelyEqual(upper, bin_upper)) return 0.5;
    return 0.0;
}

__device__ __forceinline__ double lowerDerivative(double lower, double bin_lower, double bin_upper, double overlap) {
    if (lower > bin_lower + kEpsilon && lower < bin_upper - kEpsilon && overlap > kEpsilon) return -1.0;
    if (approximatelyEqual(lower, bin_lower) || approximatelyEqual(lower, bin_upper)) return -0.5;
    return 0.0;
}

__device__ __forceinline__ bool onInteriorGridLine(double coordinate, double lower, double length, int count) {
    const double relative = (coordinate - lower) / length;
    const double nearest = round(relative);
    return nearest > 0.0 && nearest < static_cast<double>(count) && approximatelyEqual(relative, nearest);
}

// Whether the net counts (two or more pins, positive weight) and its clipped box has area.
__device__ __forceinline__ bool clippedRange(const RudyArgs& a, const Box& b, int& c0, int& c1, int& r0, int& r1) {
    const double cl = fmax(b.left, a.llx), cr = fmin(b.right, a.urx);
    const double cb = fmax(b.bottom, a.lly), ct = fmin(b.top, a.ury);
    if (fmax(0.0, cr - cl) * fmax(0.0, ct - cb) <= kEpsilon) return false;
    c0 = startBin(cl, a.llx, a.bin_w, a.columns);
    c1 = endBin(cr, a.llx, a.bin_w, a.columns);
    r0 = startBin(cb, a.lly, a.bin_h, a.rows);
    r1 = endBin(ct, a.lly, a.bin_h, a.rows);
    return true;
}

__global__ void __launch_bounds__(kThreads) rudyDepositKernel(RudyArgs a) {
    releaseNext();
    waitForPrior();
    for (int net = blockIdx.x * blockDim.x + threadIdx.x; net < a.net_count; net += gridDim.x * blockDim.x) {
        const int begin = a.net_start[net];
        const int end = a.net_start[net + 1];
        const double weight = a.net_weight[net];
        if (end - begin < 2 || weight <= 0.0) continue;
        const Box b = netBox(a, begin, end);
        int c0, c1, r0, r1;
        if (!clippedRange(a, b, c0, c1, r0, r1)) continue;
        for (int row = r0; row <= r1; ++row) {
            const double bin_bottom = a.lly + static_cast<double>(row) * a.bin_h;
            const double overlap_y = overlapLength(b.bottom, b.top, bin_bottom, bin_bottom + a.bin_h);
            if (overlap_y <= kEpsilon) continue;
            for (int column = c0; column <= c1; ++column) {
                const double bin_left = a.llx + static_cast<double>(column) * a.bin_w;
                const double overlap = overlapLength(b.left, b.right, bin_left, bin_left + a.bin_w) * overlap_y;
                if (overlap <= kEpsilon) continue;
                const size_t index = static_cast<size_t>(row) * a.columns + column;
                const long long qh = __double2ll_rn(weight * overlap / b.y_span * a.inv_unit_h);
                const long long qv = __double2ll_rn(weight * overlap / b.x_span * a.inv_unit_v);
                atomicAdd(a.horizontal + index, static_cast<unsigned long long>(qh));
                atomicAdd(a.vertical + index, static_cast<unsigned long long>(qv));
            }
        }
    }
}

// evaluatePenalty (Rudy.cpp:83-100): value and derivative of the model at utilisation u.
__device__ __forceinline__ double2 penalty(double u, int model, double temperature) {
    const double overflow = fmax(0.0, u - 1.0);
    if (model == MPGP_RUDY_HINGE_L2) return make_double2(0.5 * overflow * overflow, overflow);
    if (model == MPGP_RUDY_HINGE_L4) {
        const double square = overflow * overflow;
        return make_double2(0.25 * square * square, overflow * square);
    }
    if (model == MPGP_RUDY_SOFTPLUS_L2) {
        const double t = fmax(temperature, kEpsilon);
        const double scaled = (u - 1.0) / t;
        const double softplus = scaled > 30.0 ? scaled : (scaled < -30.0 ? exp(scaled) : log1p(exp(scaled)));
        double sigmoid;
        if (scaled >= 0.0) {
            sigmoid = 1.0 / (1.0 + exp(-scaled));
        } else {
            const double e = exp(scaled);
            sigmoid = e / (1.0 + e);
        }
        const double softened = t * softplus;
        return make_double2(0.5 * softened * softened, softened * sigmoid);
    }
    return make_double2(0.0, 0.0);
}

__global__ void __launch_bounds__(kThreads) rudyMetricsKernel(RudyArgs a) {
    releaseNext();
    waitForPrior();
    const int bins = a.columns * a.rows;
    const double unit_h = 1.0 / a.inv_unit_h, unit_v = 1.0 / a.inv_unit_v;
    const bool with_capacity = a.capacity_h > 0.0 && a.capacity_v > 0.0;
    double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};  // energy, H total, V total, proxy overflow, max utilisation
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < bins; b += gridDim.x * blockDim.x) {
        const double h = static_cast<double>(static_cast<long long>(a.horizontal[b])) * unit_h;
        const double w = static_cast<double>(static_cast<long long>(a.vertical[b])) * unit_v;
        a.horizontal[b] = 0ULL;
        a.vertical[b] = 0ULL;
        v[1] += h;
        v[2] += w;
        if (!with_capacity) continue;
        const double uh = h / a.capacity_h;
        const double uv = w / a.capacity_v;
        const double2 ph = penalty(uh, a.model, a.temperature);
        const double2 pv = penalty(uv, a.model, a.temperature);
        v[0] += (ph.x + pv.x) / static_cast<double>(bins);
        a.adjoint_h[b] = ph.y / (static_cast<double>(bins) * a.capacity_h);
        a.adjoint_v[b] = pv.y / (static_cast<double>(bins) * a.capacity_v);
        v[3] += fmax(0.0, uh - 1.0) + fmax(0.0, uv - 1.0);
        const double u = fmax(uh, uv);
        v[4] = fmax(v[4], u);
        if (a.utilization != nullptr) a.utilization[b] = u;
    }
    const bool is_max[5] = {false, false, false, false, true};
    blockReduce<5>(v, is_max);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < 5; ++k) a.partials[k * gridDim.x + blockIdx.x] = v[k];
    }
}

__global__ void __launch_bounds__(kThreads) rudyGradientKernel(RudyArgs a) {
    releaseNext();
    waitForPrior();
    for (int net = blockIdx.x * blockDim.x + threadIdx.x; net < a.net_count; net += gridDim.x * blockDim.x) {
        const int begin = a.net_start[net];
        const int end = a.net_start[net + 1];
        const double weight = a.net_weight[net];
        Box b{};
        int c0 = 0, c1 = -1, r0 = 0, r1 = -1;
        const bool counted = end - begin >= 2 && weight > 0.0 && (b = netBox(a, begin, end), clippedRange(a, b, c0, c1, r0, r1));
        if (!counted) {
            for (int pin = begin; pin < end; ++pin) {
                if (a.pin_particle[pin] >= 0) a.pin_gradient[a.pin_slot[pin]] = make_double2(0.0, 0.0);
            }
            continue;
        }
        const int g0 = max(0, c0 - (onInteriorGridLine(b.left, a.llx, a.bin_w, a.columns) ? 1 : 0));
        const int g1 = min(a.columns - 1, c1 + (onInteriorGridLine(b.right, a.llx, a.bin_w, a.columns) ? 1 : 0));
        const int h0 = max(0, r0 - (onInteriorGridLine(b.bottom, a.lly, a.bin_h, a.rows) ? 1 : 0));
        const int h1 = min(a.rows - 1, r1 + (onInteriorGridLine(b.top, a.lly, a.bin_h, a.rows) ? 1 : 0));
        double g_left = 0.0, g_right = 0.0, g_bottom = 0.0, g_top = 0.0;
        for (int row = h0; row <= h1; ++row) {
            const double bin_bottom = a.lly + static_cast<double>(row) * a.bin_h;
            const double bin_top = bin_bottom + a.bin_h;
            const double overlap_y = overlapLength(b.bottom, b.top, bin_bottom, bin_top);
            const double d_bottom = lowerDerivative(b.bottom, bin_bottom, bin_top, overlap_y);
            const double d_top = upperDerivative(b.top, bin_bottom, bin_top, overlap_y);
            if (overlap_y <= kEpsilon && d_bottom == 0.0 && d_top == 0.0) continue;
            for (int column = g0; column <= g1; ++column) {
                const double bin_left = a.llx + static_cast<double>(column) * a.bin_w;
                const double bin_right = bin_left + a.bin_w;
                const double overlap_x = overlapLength(b.left, b.right, bin_left, bin_right);
                const double overlap = overlap_x * overlap_y;
                const double d_left = lowerDerivative(b.left, bin_left, bin_right, overlap_x);
                const double d_right = upperDerivative(b.right, bin_left, bin_right, overlap_x);
                if (overlap_x <= kEpsilon && d_left == 0.0 && d_right == 0.0) continue;
                const size_t index = static_cast<size_t>(row) * a.columns + column;
                const double adj_h = a.adjoint_h[index];
                const double adj_v = a.adjoint_v[index];
                const double o_left = d_left * overlap_y;
                const double o_right = d_right * overlap_y;
                const double o_bottom = overlap_x * d_bottom;
                const double o_top = overlap_x * d_top;
                const double x_left = b.x_physical ? overlap / (b.x_span * b.x_span) : 0.0;
                const double x_right = b.x_physical ? -overlap / (b.x_span * b.x_span) : 0.0;
                const double y_bottom = b.y_physical ? overlap / (b.y_span * b.y_span) : 0.0;
                const double y_top = b.y_physical ? -overlap / (b.y_span * b.y_span) : 0.0;
                g_left += adj_h * weight * o_left / b.y_span + adj_v * weight * (o_left / b.x_span + x_left);
                g_right += adj_h * weight * o_right / b.y_span + adj_v * weight * (o_right / b.x_span + x_right);
                g_bottom += adj_h * weight * (o_bottom / b.y_span + y_bottom) + adj_v * weight * o_bottom / b.x_span;
                g_top += adj_h * weight * (o_top / b.y_span + y_top) + adj_v * weight * o_top / b.x_span;
            }
        }
        int n_left = 0, n_right = 0, n_bottom = 0, n_top = 0;
        for (int pin = begin; pin < end; ++pin) {
            const double2 p = pinPosition(a, pin);
            if (approximatelyEqual(p.x, b.x_physical ? b.left : b.raw_left)) ++n_left;
            if (approximatelyEqual(p.x, b.x_physical ? b.right : b.raw_right)) ++n_right;
            if (approximatelyEqual(p.y, b.y_physical ? b.bottom : b.raw_bottom)) ++n_bottom;
            if (approximatelyEqual(p.y, b.y_physical ? b.top : b.raw_top)) ++n_top;
        }
        for (int pin = begin; pin < end; ++pin) {
            if (a.pin_particle[pin] < 0) continue;  // fixed modules take no gradient
            const double2 p = pinPosition(a, pin);
            double gx = 0.0, gy = 0.0;
            if (b.x_physical) {
                if (n_left > 0 && approximatelyEqual(p.x, b.left)) gx += g_left / static_cast<double>(n_left);
                if (n_right > 0 && approximatelyEqual(p.x, b.right)) gx += g_right / static_cast<double>(n_right);
            } else {
                const double center = 0.5 * (g_left + g_right);
                if (n_left > 0 && approximatelyEqual(p.x, b.raw_left)) gx += center / static_cast<double>(n_left);
                if (n_right > 0 && approximatelyEqual(p.x, b.raw_right)) gx += center / static_cast<double>(n_right);
            }
            if (b.y_physical) {
                if (n_bottom > 0 && approximatelyEqual(p.y, b.bottom)) gy += g_bottom / static_cast<double>(n_bottom);
                if (n_top > 0 && approximatelyEqual(p.y, b.top)) gy += g_top / static_cast<double>(n_top);
            } else {
                const double center = 0.5 * (g_bottom + g_top);
                if (n_bottom > 0 && approximatelyEqual(p.y, b.raw_bottom)) gy += center / static_cast<double>(n_bottom);
                if (n_top > 0 && approximatelyEqual(p.y, b.raw_top)) gy += center / static_cast<double>(n_top);
            }
            a.pin_gradient[a.pin_slot[pin]] = make_double2(gx, gy);
        }
    }
}

}  // namespace

int rudyBlocks(int count) { return std::max(1, std::min(ceilDiv(count, kThreads), 148 * 4)); }

void launchRudyDeposit(const RudyArgs& args, cudaStream_t stream) {
    if (args.net_count <= 0) return;
    launchChained("Launch the RUDY deposit", rudyDepositKernel, dim3(rudyBlocks(args.net_count)), dim3(kThreads), 0,
                  stream, args);
}

void launchRudyMetrics(const RudyArgs& args, int blocks, cudaStream_t stream) {
    launchChained("Launch the RUDY metrics", rudyMetricsKernel, dim3(blocks), dim3(kThreads), 0, stream, args);
}

void launchRudyGradient(const RudyArgs& args, cudaStream_t stream) {
    if (args.net_count <= 0) return;
    launchChained("Launch the RUDY gradient", rudyGradientKernel, dim3(rudyBlocks(args.net_count)), dim3(kThreads), 0,
                  stream, args);
}

}  // namespace mpgp
