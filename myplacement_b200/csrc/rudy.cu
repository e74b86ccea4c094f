// RUDY routing-demand map, hotspot penalty and its subgradient on the device.
//
// Restates evaluateRudy (Rudy.cpp:227-456) for the adaptive controller's
// routability term (AdaptiveGlobalPlacer.cpp:149-172, 201-331).  A net's
// rectangle-overlap demand is separable: the overlap of its (expanded, clipped)
// box with bin (c, r) is ox(c) * oy(r), where ox is a partial width in the box's
// first and last columns and the bin width in between, and the same along y.
// So a net's demand is at most 3 x 3 constant blocks, and the passes are:
//   deposit   one thread per net: the pin box, expanded to minimum_span_in_bins
//             where a net is thinner (calculateNetBox, Rudy.cpp:120-152), each
//             block's horizontal demand w * overlap / y_span and vertical demand
//             w * overlap / x_span quantized to int64 (units of bin_w * 2^-32 and
//             bin_h * 2^-32) and added at the block's four corners of a 2-D
//             difference array with integer atomics: at most 72 atomics a net
//             instead of two per covered bin, and the maps stay bit-exact.
//   prefix    two scans (rows, then columns) turn the difference arrays into the
//             demand maps and clear them.
//   metrics   one thread per bin: utilisation against the frozen capacities,
//             the penalty model (hinge L2 / softplus L2 / hinge L4,
//             evaluatePenalty Rudy.cpp:83-100), its adjoint, the energy, the
//             proxy overflow, the maximum utilisation and the demand totals
//             (FP64 block partials, reduced in a fixed order).
//   tables    two scans build summed-area tables of the two adjoints.
//   gradient  one thread per net: the Clarke subgradient with respect to the
//             four box edges (Rudy.cpp:320-400).  An edge's term only involves
//             the one or two columns (rows) its derivative is non-zero in, and
//             the span terms a box-weighted adjoint sum: with the tables each is
//             O(1), not O(box area).  The edge gradients are split over the pins
//             on each extremal edge (Rudy.cpp:402-452) and written to the pins'
//             particle-ordered slots for the gather.
// Arithmetic is FP64; interior bins take the bin width and height as their
// overlap, which the reference's per-bin differences reproduce to the last bit
// or one unit in it.
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

// The parts of a clipped box along one axis: the first cell (partial), the
// interior cells (full), the last cell (partial); lo / hi index ranges and overlaps.
struct AxisParts {
    int count;
    int lo[3], hi[3];
    double overlap[3];
};

__device__ __forceinline__ AxisParts axisParts(double lower, double upper, double origin, double length, int first,
                                               int last) {
    AxisParts p;
    const auto cell = [&](int i) {
        const double begin = origin + static_cast<double>(i) * length;
        return overlapLength(lower, upper, begin, begin + length);
    };
    p.count = 0;
    p.lo[0] = p.hi[0] = first;
    p.overlap[0] = cell(first);
    p.count = 1;
    if (last > first) {
        if (last > first + 1) {
            p.lo[1] = first + 1;
            p.hi[1] = last - 1;
            p.overlap[1] = length;
            p.count = 2;
        }
        p.lo[p.count] = p.hi[p.count] = last;
        p.overlap[p.count] = cell(last);
        ++p.count;
    }
    return p;
}

__device__ __forceinline__ void addCorners(unsigned long long* diff, int stride, int r0, int r1, int c0, int c1,
                                           long long q) {
    if (q == 0) return;
    const unsigned long long up = static_cast<unsigned long long>(q);
    const unsigned long long down = static_cast<unsigned long long>(-q);
    atomicAdd(diff + static_cast<size_t>(r0) * stride + c0, up);
    atomicAdd(diff + static_cast<size_t>(r0) * stride + c1 + 1, down);
    atomicAdd(diff + static_cast<size_t>(r1 + 1) * stride + c0, down);
    atomicAdd(diff + static_cast<size_t>(r1 + 1) * stride + c1 + 1, up);
}

__global__ void __launch_bounds__(kThreads) rudyDepositKernel(RudyArgs a) {
    releaseNext();
    waitForPrior();
    const int stride = a.columns + 1;
    unsigned long long* diff_h = a.diff;
    unsigned long long* diff_v = a.diff + static_cast<size_t>(a.rows + 1) * stride;
    for (int net = blockIdx.x * blockDim.x + threadIdx.x; net < a.net_count; net += gridDim.x * blockDim.x) {
        const int begin = a.net_start[net];
        const int end = a.net_start[net + 1];
        const double weight = a.net_weight[net];
        if (end - begin < 2 || weight <= 0.0) continue;
        const Box b = netBox(a, begin, end);
        int c0, c1, r0, r1;
        if (!clippedRange(a, b, c0, c1, r0, r1)) continue;
        const AxisParts cols = axisParts(b.left, b.right, a.llx, a.bin_w, c0, c1);
        const AxisParts rows = axisParts(b.bottom, b.top, a.lly, a.bin_h, r0, r1);
        for (int i = 0; i < rows.count; ++i) {
            const double overlap_y = rows.overlap[i];
            if (overlap_y <= kEpsilon) continue;
            for (int j = 0; j < cols.count; ++j) {
                const double overlap = cols.overlap[j] * overlap_y;
                if (overlap <= kEpsilon) continue;
                const long long qh = __double2ll_rn(weight * overlap / b.y_span * a.inv_unit_h);
                const long long qv = __double2ll_rn(weight * overlap / b.x_span * a.inv_unit_v);
                addCorners(diff_h, stride, rows.lo[i], rows.hi[i], cols.lo[j], cols.hi[j], qh);
                addCorners(diff_v, stride, rows.lo[i], rows.hi[i], cols.lo[j], cols.hi[j], qv);
            }
        }
    }
}

// Inclusive scan of `length` values (load(i) / store(i, v)) by the whole block,
// in chunks of blockDim.x, always in index order (the sums are deterministic).
template <typename T, class Load, class Store>
__device__ void scanLine(int length, Load load, Store store) {
    __shared__ T warp_sums[32];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int warps = blockDim.x >> 5;
    T carry = T(0);
    for (int base = 0; base < length; base += blockDim.x) {
        const int i = base + static_cast<int>(threadIdx.x);
        T v = i < length ? load(i) : T(0);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const T u = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += u;
        }
        if (lane == 31) warp_sums[warp] = v;
        __syncthreads();
        if (warp == 0) {
            T w = lane < warps ? warp_sums[lane] : T(0);
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const T u = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += u;
            }
            if (lane < warps) warp_sums[lane] = w;
        }
        __syncthreads();
        const T before = warp > 0 ? warp_sums[warp - 1] : T(0);
        if (i < length) store(i, carry + before + v);
        carry += warp_sums[warps - 1];
        __syncthreads();
    }
}

// Difference arrays -> demand maps.  Pass 0 scans each row of both arrays in
// place; pass 1 scans each column, writes the map and clears the array.
__global__ void __launch_bounds__(kThreads) rudyPrefixKernel(RudyArgs a, int pass) {
    releaseNext();
    waitForPrior();
    const int stride = a.columns + 1;
    unsigned long long* diff = a.diff + static_cast<size_t>(blockIdx.y) * (a.rows + 1) * stride;
    unsigned long long* map = blockIdx.y == 0 ? a.horizontal : a.vertical;
    if (pass == 0) {
        unsigned long long* row = diff + static_cast<size_t>(blockIdx.x) * stride;
        scanLine<unsigned long long>(
            stride, [&](int i) { return row[i]; }, [&](int i, unsigned long long v) { row[i] = v; });
    } else {
        const int c = blockIdx.x;
        scanLine<unsigned long long>(
            a.rows + 1,
            [&](int i) {
                const unsigned long long v = diff[static_cast<size_t>(i) * stride + c];
                diff[static_cast<size_t>(i) * stride + c] = 0ULL;
                return v;
            },
            [&](int i, unsigned long long v) {
                if (i < a.rows && c < a.columns) map[static_cast<size_t>(i) * a.columns + c] = v;
            });
    }
}

// Summed-area tables of the two adjoints: table[(r + 1) * (columns + 1) + c + 1]
// = sum over r' <= r, c' <= c (row 0 and column 0 stay zero).
__global__ void __launch_bounds__(kThreads) rudyTableKernel(RudyArgs a, int pass) {
    releaseNext();
    waitForPrior();
    const int stride = a.columns + 1;
    double* table = a.table + static_cast<size_t>(blockIdx.y) * (a.rows + 1) * stride;
    const double* adjoint = blockIdx.y == 0 ? a.adjoint_h : a.adjoint_v;
    if (pass == 0) {
        const int r = blockIdx.x;
        const double* in = adjoint + static_cast<size_t>(r) * a.columns;
        double* out = table + static_cast<size_t>(r + 1) * stride + 1;
        scanLine<double>(a.columns, [&](int i) { return in[i]; }, [&](int i, double v) { out[i] = v; });
    } else {
        const int c = blockIdx.x + 1;
        scanLine<double>(
            a.rows, [&](int i) { return table[static_cast<size_t>(i + 1) * stride + c]; },
            [&](int i, double v) { table[static_cast<size_t>(i + 1) * stride + c] = v; });
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
        const AxisParts cols = axisParts(b.left, b.right, a.llx, a.bin_w, c0, c1);
        const AxisParts rows = axisParts(b.bottom, b.top, a.lly, a.bin_h, r0, r1);
        const int stride = a.columns + 1;
        const double* table_h = a.table;
        const double* table_v = a.table + static_cast<size_t>(a.rows + 1) * stride;
        // Sum of one adjoint over rows [rl, rh] x columns [cl, ch] (inclusive).
        const auto rect = [&](const double* t, int rl, int rh, int cl, int ch) {
            if (rl > rh || cl > ch) return 0.0;
            return t[static_cast<size_t>(rh + 1) * stride + ch + 1] - t[static_cast<size_t>(rl) * stride + ch + 1] -
                   t[static_cast<size_t>(rh + 1) * stride + cl] + t[static_cast<size_t>(rl) * stride + cl];
        };
        // sum over the box's rows of oy(r) * adjoint(c, r), and the same along a row.
        const auto column_sum = [&](const double* t, int c) {
            double sum = 0.0;
            for (int i = 0; i < rows.count; ++i) sum += rows.overlap[i] * rect(t, rows.lo[i], rows.hi[i], c, c);
            return sum;
        };
        const auto row_sum = [&](const double* t, int r) {
            double sum = 0.0;
            for (int j = 0; j < cols.count; ++j) sum += cols.overlap[j] * rect(t, r, r, cols.lo[j], cols.hi[j]);
            return sum;
        };
        // sum over the box of ox(c) oy(r) adjoint(c, r).
        const auto box_sum = [&](const double* t) {
            double sum = 0.0;
            for (int i = 0; i < rows.count; ++i) {
                for (int j = 0; j < cols.count; ++j) {
                    sum += rows.overlap[i] * cols.overlap[j] * rect(t, rows.lo[i], rows.hi[i], cols.lo[j], cols.hi[j]);
                }
            }
            return sum;
        };
        // Edge terms: the columns (rows) next to an edge are the only ones whose
        // derivative can be non-zero; each adds d * (adj_h / y_span + adj_v / x_span)
        // weighted by the other axis' overlaps (Rudy.cpp:360-400).
        double g_left = 0.0, g_right = 0.0, g_bottom = 0.0, g_top = 0.0;
        const auto column_edge = [&](double edge, bool lower) {
            double sum = 0.0;
            const int near = static_cast<int>(floor((edge - a.llx) / a.bin_w));
            for (int c = max(g0, near - 1); c <= min(g1, near + 1); ++c) {
                const double bin_left = a.llx + static_cast<double>(c) * a.bin_w;
                const double bin_right = bin_left + a.bin_w;
                const double overlap_x = overlapLength(b.left, b.right, bin_left, bin_right);
                const double d = lower ? lowerDerivative(edge, bin_left, bin_right, overlap_x)
                                       : upperDerivative(edge, bin_left, bin_right, overlap_x);
                if (d != 0.0) sum += d * (column_sum(table_h, c) / b.y_span + column_sum(table_v, c) / b.x_span);
            }
            return sum;
        };
        const auto row_edge = [&](double edge, bool lower) {
            double sum = 0.0;
            const int near = static_cast<int>(floor((edge - a.lly) / a.bin_h));
            for (int r = max(h0, near - 1); r <= min(h1, near + 1); ++r) {
                const double bin_bottom = a.lly + static_cast<double>(r) * a.bin_h;
                const double bin_top = bin_bottom + a.bin_h;
                const double overlap_y = overlapLength(b.bottom, b.top, bin_bottom, bin_top);
                const double d = lower ? lowerDerivative(edge, bin_bottom, bin_top, overlap_y)
                                       : upperDerivative(edge, bin_bottom, bin_top, overlap_y);
                if (d != 0.0) sum += d * (row_sum(table_h, r) / b.y_span + row_sum(table_v, r) / b.x_span);
            }
            return sum;
        };
        g_left = weight * column_edge(b.left, true);
        g_right = weight * column_edge(b.right, false);
        g_bottom = weight * row_edge(b.bottom, true);
        g_top = weight * row_edge(b.top, false);
        if (b.x_physical) {
            const double span_term = weight * box_sum(table_v) / (b.x_span * b.x_span);
            g_left += span_term;
            g_right -= span_term;
        }
        if (b.y_physical) {
            const double span_term = weight * box_sum(table_h) / (b.y_span * b.y_span);
            g_bottom += span_term;
            g_top -= span_term;
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

void launchRudyPrefix(const RudyArgs& args, cudaStream_t stream) {
    launchChained("Launch the RUDY row scan", rudyPrefixKernel, dim3(args.rows + 1, 2), dim3(kThreads), 0, stream,
                  args, 0);
    launchChained("Launch the RUDY column scan", rudyPrefixKernel, dim3(args.columns + 1, 2), dim3(kThreads), 0,
                  stream, args, 1);
}

void launchRudyTables(const RudyArgs& args, cudaStream_t stream) {
    launchChained("Launch the RUDY adjoint row scan", rudyTableKernel, dim3(args.rows, 2), dim3(kThreads), 0, stream,
                  args, 0);
    launchChained("Launch the RUDY adjoint column scan", rudyTableKernel, dim3(args.columns, 2), dim3(kThreads), 0,
                  stream, args, 1);
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
