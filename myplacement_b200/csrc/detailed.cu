// Detailed placement by window reordering, the orderings evaluated on the
// device: the reference's CUDA detailed-placement backend
// (src/placement/cuda/CudaDetailedPlacementBackend.cu:144-709) with the CPU rule
// it keeps for the windows the device does not take (:328-354).
//
// Each pass cuts the rows into segments of abutting standard cells and the
// segments into windows of four consecutive cells, staggered by two cells on
// odd passes.  One warp evaluates one window: lanes 0..23 each place the cells
// in one of the 24 orders (lexicographic, the order std::next_permutation
// visits) and sum the weighted HPWL of the window's nets; lane 24 sums it for
// the placement as it is.  The sum with fused multiply-adds (what the
// reference's kernel compiles to) picks the best order.
//
// The reference then accepts the windows one after another, each by its host
// arithmetic (products and sums rounded separately) against the placement the
// earlier acceptances left.  A second kernel evaluates that rule
// speculatively: every window's before and after values on the assumption
// that each earlier window decided as the previous round said, for a few
// rounds.  The host walks the windows in the reference's order and takes the
// device's values unless a net of the window belongs to an earlier window
// whose actual decision differed from the assumption; only those windows are
// re-evaluated on the host.  The segment ends the reference keeps on the host
// (two or three cells, every order by its exhaustive rule) go through a tail
// kernel the same way, after the four-cell windows.  The result is the
// reference's exactly.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <string>
#include <vector>

#include "common.cuh"
#include "detailed.hpp"
#include "setup.hpp"
#include "workers.hpp"

namespace mpgp {
namespace {

constexpr int kWindow = 4;
constexpr int kOrders = 24;
constexpr int kCurrentLane = kOrders;  // the lane that evaluates the placement as it is
constexpr int kWindowsPerBlock = 8;
constexpr int kSpeculations = 3;  // rounds of speculative re-decision on the device
constexpr int kOrientationUnknown = 8;
constexpr double kLargest = std::numeric_limits<double>::max();

// Order k (0..n!-1) of n <= 4 cells in lexicographic order (the order
// std::next_permutation visits from 0, 1, ..., n - 1), as 4-bit fields: field
// i is the window cell placed i-th.  The Lehmer digits of k (k / (n-1)!, then
// the remainder's digit for (n-2)!, ...) each pick a field of the cells not yet
// placed (`pool`, packed the same way) and remove it.
__host__ __device__ inline unsigned orderCode(int k, int n = kWindow) {
    unsigned pool = 0x3210u;
    unsigned code = 0u;
    int rest = k;
#pragma unroll
    for (int i = 0; i < kWindow - 1; ++i) {
        if (i >= n - 1) break;
        const int place = n - 1 - i;
        const int factorial = place == 3 ? 6 : place == 2 ? 2 : 1;
        const unsigned d = static_cast<unsigned>(rest / factorial);
        rest %= factorial;
        code |= ((pool >> (4u * d)) & 0xFu) << (4u * static_cast<unsigned>(i));
        pool = (pool & ((1u << (4u * d)) - 1u)) | ((pool >> (4u * (d + 1u))) << (4u * d));
    }
    return code | ((pool & 0xFu) << (4u * static_cast<unsigned>(n - 1)));
}

__host__ __device__ inline int factorialOf(int n) { return n == 4 ? 24 : n == 3 ? 6 : n == 2 ? 2 : 1; }

inline void orderOf(int k, int order[kWindow], int n = kWindow) {
    const unsigned code = orderCode(k, n);
    for (int i = 0; i < n; ++i) order[i] = static_cast<int>((code >> (4u * static_cast<unsigned>(i))) & 0xFu);
}

// alignUp(width, 0, spacing) (DetailedPlacer.cpp:67-70), products and sums
// rounded separately.
__device__ inline double roundedWidthDevice(double width, double spacing) {
    return spacing <= kEpsilon ? width : __dmul_rn(ceil((width - kEpsilon) / spacing), spacing);
}

struct WindowArrays {
    const int4* modules;
    const double* start_x;  // lower-left x of the window's first cell
    const double* bottom;
    const double* spacing;
    const int* net_start;   // windows + 1
    const int* nets;
};

__global__ void __launch_bounds__(32 * kWindowsPerBlock)
    windowOrdersKernel(const double2* __restrict__ center, const double2* __restrict__ size,
                       const int* __restrict__ pin_module, const double2* __restrict__ pin_offset,
                       const int* __restrict__ net_pin_start, const double* __restrict__ net_weight,
                       WindowArrays windows, int window_count, double epsilon, int* __restrict__ best_order,
                       uint8_t* __restrict__ decided, double2* __restrict__ moved_center) {
    const int lane = threadIdx.x & 31;
    const int w = blockIdx.x * kWindowsPerBlock + static_cast<int>(threadIdx.x >> 5);
    if (w >= window_count) return;  // whole warps leave together
    const int4 m4 = windows.modules[w];
    const int module[kWindow] = {m4.x, m4.y, m4.z, m4.w};

    // The window's cells where this lane puts them (registers only: the cell of
    // each slot is picked by comparisons, never by a computed index).
    double cx[kWindow];
    double cy[kWindow];
#pragma unroll
    for (int i = 0; i < kWindow; ++i) {
        const double2 c = center[module[i]];
        cx[i] = c.x;
        cy[i] = c.y;
    }
    if (lane < kOrders) {
        const unsigned code = orderCode(lane);
        double cursor = windows.start_x[w];
        const double bottom = windows.bottom[w];
        const double spacing = windows.spacing[w];
#pragma unroll
        for (int i = 0; i < kWindow; ++i) {
            const unsigned local = (code >> (4u * static_cast<unsigned>(i))) & 0xFu;
            int placed = module[0];
#pragma unroll
            for (int j = 1; j < kWindow; ++j) placed = local == static_cast<unsigned>(j) ? module[j] : placed;
            const double2 s = size[placed];
            const double x = __dadd_rn(cursor, __dmul_rn(s.x, 0.5));
            const double y = __dadd_rn(bottom, __dmul_rn(s.y, 0.5));
#pragma unroll
            for (int j = 0; j < kWindow; ++j) {
                if (local == static_cast<unsigned>(j)) {
                    cx[j] = x;
                    cy[j] = y;
                }
            }
            cursor = __dadd_rn(cursor, roundedWidthDevice(s.x, spacing));
        }
    }

    double fused = 0.0;
    double plain = 0.0;
    if (lane <= kCurrentLane) {
        for (int e = windows.net_start[w]; e < windows.net_start[w + 1]; ++e) {
            const int net = windows.nets[e];
            double fmin_x = kLargest, fmax_x = -kLargest, fmin_y = kLargest, fmax_y = -kLargest;
            double min_x = kLargest, max_x = -kLargest, min_y = kLargest, max_y = -kLargest;
            for (int p = net_pin_start[net]; p < net_pin_start[net + 1]; ++p) {
                const int m = pin_module[p];
                double2 c = center[m];
#pragma unroll
                for (int i = 0; i < kWindow; ++i) {  // a window's cells are distinct: one match at most
                    if (module[i] == m) c = make_double2(cx[i], cy[i]);
                }
                const double2 o = pin_offset[p];
                const double x = c.x + o.x;
                const double y = c.y + o.y;
                fmin_x = fmin(fmin_x, x);
                fmax_x = fmax(fmax_x, x);
                fmin_y = fmin(fmin_y, y);
                fmax_y = fmax(fmax_y, y);
                min_x = x < min_x ? x : min_x;  // std::min / std::max
                max_x = max_x < x ? x : max_x;
                min_y = y < min_y ? y : min_y;
                max_y = max_y < y ? y : max_y;
            }
            const double weight = net_weight[net];
            fused = fma(weight, (fmax_x - fmin_x) + (fmax_y - fmin_y), fused);
            plain = __dadd_rn(plain, __dmul_rn(weight, (max_x - min_x) + (max_y - min_y)));
        }
    }

    // The smallest fused value, the lowest order on ties, to every lane.
    double best = lane < kOrders ? fused : kLargest;
    int index = lane;
    for (int offset = 16; offset > 0; offset >>= 1) {
        const double other = __shfl_xor_sync(0xffffffffu, best, offset);
        const int other_index = __shfl_xor_sync(0xffffffffu, index, offset);
        if (other < best || (other == best && other_index < index)) {
            best = other;
            index = other_index;
        }
    }
    const double before = __shfl_sync(0xffffffffu, plain, kCurrentLane);
    const double after = __shfl_sync(0xffffffffu, plain, index);
    if (lane == 0) {
        best_order[w] = index;
        decided[w] = index > 0 && index < kOrders && after < before - epsilon ? 1 : 0;
    }
    if (lane == index) {  // where the best order puts the window's cells (applyOrder's arithmetic)
#pragma unroll
        for (int i = 0; i < kWindow; ++i) moved_center[module[i]] = make_double2(cx[i], cy[i]);
    }
}

// transformOffset (PlacementDatabase.cpp:55-68).
__host__ __device__ inline double2 transformed(double2 o, int orientation) {
    switch (orientation) {
        case 1: return make_double2(-o.x, -o.y);
        case 2: return make_double2(-o.y, o.x);
        case 3: return make_double2(o.y, -o.x);
        case 4: return make_double2(-o.x, o.y);
        case 5: return make_double2(o.x, -o.y);
        case 6: return make_double2(o.y, o.x);
        case 7: return make_double2(-o.y, -o.x);
        default: return o;
    }
}

// The host's before / after values of every window (its best order against
// its current placement) on the assumption that each earlier window decided as
// `decided_in` says, and the decisions they give.  A cell of an earlier window
// assumed accepted sits where that window's best order puts it, with the
// orientation of its row; every other cell is where the pass found it.  One
// warp per window: each lane takes one net and forms its two terms (products
// rounded separately), and the warp adds them in net order, as the host does.
__global__ void __launch_bounds__(32 * kWindowsPerBlock)
    speculativeValuesKernel(const double2* __restrict__ center, const double2* __restrict__ moved_center,
                            const int* __restrict__ owner, const int8_t* __restrict__ moved_orientation,
                            const double2* __restrict__ raw_offset, const double2* __restrict__ pin_offset,
                            const int* __restrict__ pin_module, const int* __restrict__ net_pin_start,
                            const double* __restrict__ net_weight, WindowArrays windows, int window_count,
                            const int* __restrict__ best_order, double epsilon, const uint8_t* __restrict__ decided_in,
                            uint8_t* __restrict__ decided_out, double* __restrict__ value_before,
                            double* __restrict__ value_after) {
    const int lane = threadIdx.x & 31;
    const int w = blockIdx.x * kWindowsPerBlock + static_cast<int>(threadIdx.x >> 5);
    if (w >= window_count) return;  // whole warps leave together
    const int best = best_order[w];
    if (best <= 0 || best >= kOrders) {
        if (lane == 0) decided_out[w] = 0;
        return;
    }
    const int4 m4 = windows.modules[w];
    const int first = windows.net_start[w];
    const int last = windows.net_start[w + 1];
    double before = 0.0;
    double after = 0.0;
    for (int base = first; base < last; base += 32) {
        double term_before = 0.0;
        double term_after = 0.0;
        const int e = base + lane;
        if (e < last) {
            const int net = windows.nets[e];
            double min_b = kLargest, max_b = -kLargest, min_by = kLargest, max_by = -kLargest;
            double min_a = kLargest, max_a = -kLargest, min_ay = kLargest, max_ay = -kLargest;
            for (int p = net_pin_start[net]; p < net_pin_start[net + 1]; ++p) {
                const int m = pin_module[p];
                double2 offset = pin_offset[p];
                double2 now_c;   // the cell now (before)
                double2 then_c;  // the cell with this window's best order applied (after)
                if (m == m4.x || m == m4.y || m == m4.z || m == m4.w) {
                    now_c = center[m];
                    then_c = moved_center[m];  // its orientation changes only once accepted
                } else {
                    const int j = owner[m];
                    if (j >= 0 && j < w && decided_in[j] != 0) {
                        now_c = moved_center[m];
                        offset = transformed(raw_offset[p], moved_orientation[m]);
                    } else {
                        now_c = center[m];
                    }
                    then_c = now_c;
                }
                const double bx = now_c.x + offset.x;
                const double by = now_c.y + offset.y;
                const double ax = then_c.x + offset.x;
                const double ay = then_c.y + offset.y;
                min_b = bx < min_b ? bx : min_b;
                max_b = max_b < bx ? bx : max_b;
                min_by = by < min_by ? by : min_by;
                max_by = max_by < by ? by : max_by;
                min_a = ax < min_a ? ax : min_a;
                max_a = max_a < ax ? ax : max_a;
                min_ay = ay < min_ay ? ay : min_ay;
                max_ay = max_ay < ay ? ay : max_ay;
            }
            const double weight = net_weight[net];
            term_before = __dmul_rn(weight, (max_b - min_b) + (max_by - min_by));
            term_after = __dmul_rn(weight, (max_a - min_a) + (max_ay - min_ay));
        }
        const int terms = min(32, last - base);
        for (int j = 0; j < terms; ++j) {
            before = __dadd_rn(before, __shfl_sync(0xffffffffu, term_before, j));
            after = __dadd_rn(after, __shfl_sync(0xffffffffu, term_after, j));
        }
    }
    if (lane == 0) {
        value_before[w] = before;
        value_after[w] = after;
        decided_out[w] = after < before - epsilon ? 1 : 0;
    }
}

// The windows the reference keeps on the host (segment ends of two or three
// cells), those with nets to evaluate, in the reference's order.
struct TailArrays {
    const int4* modules;  // unused slots -1
    const int* count;
    const double* start_x;
    const double* bottom;
    const double* spacing;
    const int* net_start;
    const int* nets;
};

// Where each tail window's assumed order (-1: none) puts its cells.
__global__ void __launch_bounds__(256)
    tailPlacementKernel(TailArrays tail, int tail_count, const double2* __restrict__ size,
                        const int8_t* __restrict__ assumed, double2* __restrict__ moved_center) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= tail_count || assumed[t] < 0) return;
    const int n = tail.count[t];
    const int4 m4 = tail.modules[t];
    const int module[kWindow] = {m4.x, m4.y, m4.z, m4.w};
    const unsigned code = orderCode(assumed[t], n);
    double cursor = tail.start_x[t];
    for (int i = 0; i < n; ++i) {
        const unsigned local = (code >> (4u * static_cast<unsigned>(i))) & 0xFu;
        int placed = module[0];
#pragma unroll
        for (int j = 1; j < kWindow; ++j) placed = local == static_cast<unsigned>(j) ? module[j] : placed;
        const double2 s = size[placed];
        moved_center[placed] = make_double2(__dadd_rn(cursor, __dmul_rn(s.x, 0.5)),
                                            __dadd_rn(tail.bottom[t], __dmul_rn(s.y, 0.5)));
        cursor = __dadd_rn(cursor, roundedWidthDevice(s.x, tail.spacing[t]));
    }
}

// optimizeCpuWindow (CudaDetailedPlacementBackend.cu:328-354) for every tail
// window on the assumption that each earlier tail window took the order
// `assumed_in` says: every order in lexicographic order, each taken when it
// beats the best so far by more than epsilon, from the placement as it is.
// Writes the order taken, or -1.  A cell of an earlier tail window assumed
// reordered sits where that order puts it, with its row's orientation; every
// other cell is where the four-cell windows left it.  One warp per window:
// lane k < n! evaluates order k, lane n! the placement as it is, and every lane
// then runs the same selection over the lanes' values in order.
__global__ void __launch_bounds__(32 * kWindowsPerBlock)
    tailOrdersKernel(const double2* __restrict__ center, const int8_t* __restrict__ orientation,
                     const double2* __restrict__ moved_center, const int* __restrict__ owner, int tail_base,
                     const int8_t* __restrict__ moved_orientation, const double2* __restrict__ raw_offset,
                     const double2* __restrict__ size, const int* __restrict__ pin_module,
                     const int* __restrict__ net_pin_start, const double* __restrict__ net_weight, TailArrays tail,
                     int tail_count, double epsilon, const int8_t* __restrict__ assumed_in,
                     int8_t* __restrict__ order_out) {
    const int lane = threadIdx.x & 31;
    const int t = blockIdx.x * kWindowsPerBlock + static_cast<int>(threadIdx.x >> 5);
    if (t >= tail_count) return;  // whole warps leave together
    const int n = tail.count[t];
    const int orders = factorialOf(n);
    const int4 m4 = tail.modules[t];
    const int module[kWindow] = {m4.x, m4.y, m4.z, m4.w};
    double cx[kWindow];
    double cy[kWindow];
    // The window's weighted HPWL with its own cells at (cx, cy).
    const auto value = [&]() {
        double sum = 0.0;
        for (int e = tail.net_start[t]; e < tail.net_start[t + 1]; ++e) {
            const int net = tail.nets[e];
            double min_x = kLargest, max_x = -kLargest, min_y = kLargest, max_y = -kLargest;
            for (int p = net_pin_start[net]; p < net_pin_start[net + 1]; ++p) {
                const int m = pin_module[p];
                double2 c = center[m];
                int turn = orientation[m];
#pragma unroll
                for (int i = 0; i < kWindow; ++i) {
                    if (module[i] == m) c = make_double2(cx[i], cy[i]);
                }
                if (m != module[0] && m != module[1] && m != module[2] && m != module[3]) {
                    const int j = owner[m] - tail_base;
                    if (j >= 0 && j < t && assumed_in[j] >= 0) {
                        c = moved_center[m];
                        turn = moved_orientation[m];
                    }
                }
                const double2 o = transformed(raw_offset[p], turn);
                const double x = c.x + o.x;
                const double y = c.y + o.y;
                min_x = x < min_x ? x : min_x;
                max_x = max_x < x ? x : max_x;
                min_y = y < min_y ? y : min_y;
                max_y = max_y < y ? y : max_y;
            }
            sum = __dadd_rn(sum, __dmul_rn(net_weight[net], (max_x - min_x) + (max_y - min_y)));
        }
        return sum;
    };
#pragma unroll
    for (int i = 0; i < kWindow; ++i) {
        const double2 c = module[i] >= 0 ? center[module[i]] : make_double2(0.0, 0.0);
        cx[i] = c.x;
        cy[i] = c.y;
    }
    if (lane < orders) {
        const unsigned code = orderCode(lane, n);
        double cursor = tail.start_x[t];
        for (int i = 0; i < n; ++i) {
            const unsigned local = (code >> (4u * static_cast<unsigned>(i))) & 0xFu;
            int placed = module[0];
#pragma unroll
            for (int j = 1; j < kWindow; ++j) placed = local == static_cast<unsigned>(j) ? module[j] : placed;
            const double2 s = size[placed];
            const double x = __dadd_rn(cursor, __dmul_rn(s.x, 0.5));
            const double y = __dadd_rn(tail.bottom[t], __dmul_rn(s.y, 0.5));
#pragma unroll
            for (int j = 0; j < kWindow; ++j) {
                if (local == static_cast<unsigned>(j)) {
                    cx[j] = x;
                    cy[j] = y;
                }
            }
            cursor = __dadd_rn(cursor, roundedWidthDevice(s.x, tail.spacing[t]));
        }
    }
    const double mine = lane <= orders ? value() : 0.0;
    double best = __shfl_sync(0xffffffffu, mine, orders);
    int taken = -1;
    for (int k = 0; k < orders; ++k) {
        const double v = __shfl_sync(0xffffffffu, mine, k);
        if (v < best - epsilon) {
            best = v;
            taken = k;
        }
    }
    if (lane == 0) order_out[t] = static_cast<int8_t>(taken);
}

// ---- host ---------------------------------------------------------------------------------

// transformOffset (PlacementDatabase.cpp:55-68).
inline void transform(double x, double y, int orientation, double& ox, double& oy) {
    switch (orientation) {
        case 1: ox = -x; oy = -y; return;
        case 2: ox = -y; oy = x; return;
        case 3: ox = y; oy = -x; return;
        case 4: ox = -x; oy = y; return;
        case 5: ox = x; oy = -y; return;
        case 6: ox = y; oy = x; return;
        case 7: ox = -y; oy = -x; return;
        default: ox = x; oy = y; return;
    }
}

// alignUp(width, 0, spacing) (CudaDetailedPlacementBackend.cu:229-236).
inline double roundedWidth(double width, double spacing) {
    if (spacing <= kEpsilon) return width;
    return 0.0 + std::ceil((width - 0.0 - kEpsilon) / spacing) * spacing;
}

template <typename T>
class DeviceArray {
public:
    DeviceArray() = default;
    DeviceArray(const DeviceArray&) = delete;
    DeviceArray& operator=(const DeviceArray&) = delete;
    ~DeviceArray() {
        if (data_ != nullptr) cudaFree(data_);
    }
    void allocate(std::size_t count, uint64_t& reserved, uint64_t limit, const char* what) {
        const uint64_t bytes = static_cast<uint64_t>(std::max<std::size_t>(count, 1)) * sizeof(T);
        if (bytes > limit - std::min(limit, reserved)) {
            fail(MPGP_ERR_BUDGET, std::string("CUDA detailed-placement budget exceeded while reserving ") + what + ".");
        }
        checkCuda(cudaMalloc(reinterpret_cast<void**>(&data_), bytes), what);
        reserved += bytes;
    }
    void upload(const std::vector<T>& values, cudaStream_t stream) {
        if (!values.empty()) {
            checkCuda(cudaMemcpyAsync(data_, values.data(), values.size() * sizeof(T), cudaMemcpyHostToDevice, stream),
                      "detailed-placement upload");
        }
    }
    void download(std::vector<T>& values, cudaStream_t stream) const {
        if (!values.empty()) {
            checkCuda(cudaMemcpyAsync(values.data(), data_, values.size() * sizeof(T), cudaMemcpyDeviceToHost, stream),
                      "detailed-placement download");
        }
    }
    [[nodiscard]] T* get() const { return data_; }

private:
    T* data_ = nullptr;
};

class Stream {
public:
    Stream() { checkCuda(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate"); }
    ~Stream() { cudaStreamDestroy(stream_); }
    Stream(const Stream&) = delete;
    Stream& operator=(const Stream&) = delete;
    [[nodiscard]] cudaStream_t get() const { return stream_; }

private:
    cudaStream_t stream_ = nullptr;
};

// The placement state the passes change, with the design's fixed data.
struct Placement {
    const mpgp_design& d;
    std::vector<double> cx, cy;
    std::vector<int32_t> orientation;
    std::vector<int32_t> pin_net;
    std::vector<int64_t> module_pin_start;  // module -> its pins, in pin order
    std::vector<int32_t> module_pins;

    explicit Placement(const mpgp_design& design) : d(design) {
        const std::size_t m = static_cast<std::size_t>(d.module_count);
        cx.assign(d.module_x, d.module_x + m);
        cy.assign(d.module_y, d.module_y + m);
        orientation.assign(m, 0);
        if (d.module_orientation != nullptr) orientation.assign(d.module_orientation, d.module_orientation + m);
        pin_net.resize(static_cast<std::size_t>(d.pin_count));
        for (int32_t n = 0; n < d.net_count; ++n) {
            for (int64_t p = d.net_pin_start[n]; p < d.net_pin_start[n + 1]; ++p) pin_net[p] = n;
        }
        module_pin_start.assign(m + 1, 0);
        for (int64_t p = 0; p < d.pin_count; ++p) ++module_pin_start[d.pin_module[p] + 1];
        for (std::size_t k = 0; k < m; ++k) module_pin_start[k + 1] += module_pin_start[k];
        module_pins.resize(static_cast<std::size_t>(d.pin_count));
        std::vector<int64_t> fill(module_pin_start.begin(), module_pin_start.end() - 1);
        for (int64_t p = 0; p < d.pin_count; ++p) module_pins[fill[d.pin_module[p]]++] = static_cast<int32_t>(p);
    }

    [[nodiscard]] double lowerLeftX(int m) const { return cx[m] - d.module_width[m] * 0.5; }
    [[nodiscard]] double lowerLeftY(int m) const { return cy[m] - d.module_height[m] * 0.5; }

    // localHpwl (CudaDetailedPlacementBackend.cu:282-302) with the window's cells
    // at (wx, wy).
    double windowHpwl(const int32_t* modules, int count, const int32_t* nets, int net_count, const double* wx,
                      const double* wy) const {
        double result = 0.0;
        for (int e = 0; e < net_count; ++e) {
            const int32_t net = nets[e];
            double min_x = std::numeric_limits<double>::infinity();
            double max_x = -std::numeric_limits<double>::infinity();
            double min_y = std::numeric_limits<double>::infinity();
            double max_y = -std::numeric_limits<double>::infinity();
            for (int64_t p = d.net_pin_start[net]; p < d.net_pin_start[net + 1]; ++p) {
                const int32_t m = d.pin_module[p];
                double x = cx[m];
                double y = cy[m];
                for (int i = 0; i < count; ++i) {
                    if (modules[i] == m) {
                        x = wx[i];
                        y = wy[i];
                        break;
                    }
                }
                double ox = 0.0;
                double oy = 0.0;
                transform(d.pin_offset_x[p], d.pin_offset_y[p], orientation[m], ox, oy);
                x = x + ox;
                y = y + oy;
                min_x = std::min(min_x, x);
                max_x = std::max(max_x, x);
                min_y = std::min(min_y, y);
                max_y = std::max(max_y, y);
            }
            result += d.net_weight[net] * ((max_x - min_x) + (max_y - min_y));
        }
        return result;
    }

    // centersForOrder (:304-315).
    void centersForOrder(const int32_t* modules, const int* order, int count, double bottom, double spacing,
                         double* wx, double* wy) const {
        double cursor = lowerLeftX(modules[0]);
        for (int i = 0; i < count; ++i) {
            const int local = order[i];
            const int32_t m = modules[local];
            wx[local] = cursor + d.module_width[m] * 0.5;
            wy[local] = bottom + d.module_height[m] * 0.5;
            cursor += roundedWidth(d.module_width[m], spacing);
        }
    }

    // applyOrder (:317-326): setLowerLeft, then the row's orientation when known.
    void applyOrder(const int32_t* modules, const int* order, int count, double bottom, double spacing,
                    int row_orientation) {
        double cursor = lowerLeftX(modules[0]);
        for (int i = 0; i < count; ++i) {
            const int32_t m = modules[order[i]];
            cx[m] = cursor + d.module_width[m] * 0.5;
            cy[m] = bottom + d.module_height[m] * 0.5;
            if (row_orientation != kOrientationUnknown) orientation[m] = row_orientation;
            cursor += roundedWidth(d.module_width[m], spacing);
        }
    }

    // calculateHpwl (Metrics.cpp:128-147): the nets' terms on several threads,
    // summed in net order.
    [[nodiscard]] double hpwl(const Workers& workers) const {
        std::vector<double> term(static_cast<std::size_t>(d.net_count), 0.0);
        workers.blocks(term.size(), 8192, [&](std::size_t b, std::size_t e) {
            for (std::size_t n = b; n < e; ++n) term[n] = netTerm(static_cast<int32_t>(n));
        });
        double result = 0.0;
        for (int32_t n = 0; n < d.net_count; ++n) {
            if (d.net_pin_start[n + 1] - d.net_pin_start[n] >= 2) result += term[n];
        }
        return result;
    }

    // One net's weighted HPWL at the current placement.
    [[nodiscard]] double netTerm(int32_t n) const {
        double min_x = std::numeric_limits<double>::infinity();
        double max_x = -std::numeric_limits<double>::infinity();
        double min_y = std::numeric_limits<double>::infinity();
        double max_y = -std::numeric_limits<double>::infinity();
        for (int64_t p = d.net_pin_start[n]; p < d.net_pin_start[n + 1]; ++p) {
            const int32_t m = d.pin_module[p];
            double ox = 0.0;
            double oy = 0.0;
            transform(d.pin_offset_x[p], d.pin_offset_y[p], orientation[m], ox, oy);
            const double x = cx[m] + ox;
            const double y = cy[m] + oy;
            min_x = std::min(min_x, x);
            max_x = std::max(max_x, x);
            min_y = std::min(min_y, y);
            max_y = std::max(max_y, y);
        }
        return d.net_weight[n] * ((max_x - min_x) + (max_y - min_y));
    }
};

// A window: up to four consecutive cells of a segment and the nets they touch.
struct Windows {
    std::vector<int32_t> row;
    std::vector<int32_t> count;
    std::vector<int32_t> modules;  // kWindow per window (unused slots -1)
    std::vector<int64_t> net_start{0};
    std::vector<int32_t> nets;     // sorted, unique per window
    std::vector<uint8_t> device;   // evaluated on the device (gpu_eligible)

    void clear() {
        row.clear();
        count.clear();
        modules.clear();
        net_start.assign(1, 0);
        nets.clear();
        device.clear();
    }
};

// buildRowSegments (:238-274) and makeWindow (:276-293) for one pass: the
// windows in the reference's order, whichever list they go to.  Rows are
// independent: each sorts its cells (in module order before the sort, as the
// reference collects them, so std::sort leaves ties as the reference's does)
// and cuts its segments and windows on a thread of its own.
void buildWindows(const Placement& s, const std::vector<uint8_t>& standard, int phase, uint64_t maximum_net_degree,
                  const Workers& workers, Windows& out) {
    const mpgp_design& d = s.d;
    out.clear();
    if (d.row_count == 0) return;
    std::vector<std::size_t> sorted_rows(static_cast<std::size_t>(d.row_count));
    std::iota(sorted_rows.begin(), sorted_rows.end(), 0U);
    std::sort(sorted_rows.begin(), sorted_rows.end(),
              [&](std::size_t a, std::size_t b) { return d.row_bottom[a] < d.row_bottom[b]; });
    const auto centre = [&](std::size_t r) { return d.row_bottom[r] + d.row_height[r] * 0.5; };
    const auto nearestRow = [&](double coordinate) {
        const auto it = std::lower_bound(sorted_rows.begin(), sorted_rows.end(), coordinate,
                                         [&](std::size_t r, double value) { return centre(r) < value; });
        if (it == sorted_rows.begin()) return *it;
        if (it == sorted_rows.end()) return sorted_rows.back();
        const std::size_t right = *it;
        const std::size_t left = *(it - 1);
        return std::abs(centre(left) - coordinate) <= std::abs(centre(right) - coordinate) ? left : right;
    };
    constexpr double kSegmentEpsilon = 1e-6;
    const std::size_t modules = static_cast<std::size_t>(d.module_count);
    const std::size_t rows = static_cast<std::size_t>(d.row_count);
    std::vector<int32_t> row_of(modules, -1);
    workers.blocks(modules, 16384, [&](std::size_t b, std::size_t e) {
        for (std::size_t m = b; m < e; ++m) {
            if (standard[m] == 0) continue;
            const std::size_t r = nearestRow(s.cy[m]);
            if (std::abs(s.lowerLeftY(static_cast<int>(m)) - d.row_bottom[r]) <= kSegmentEpsilon) {
                row_of[m] = static_cast<int32_t>(r);
            }
        }
    });
    std::vector<std::size_t> row_start(rows + 1, 0);
    for (const int32_t r : row_of) {
        if (r >= 0) ++row_start[static_cast<std::size_t>(r) + 1];
    }
    for (std::size_t r = 0; r < rows; ++r) row_start[r + 1] += row_start[r];
    std::vector<int32_t> cells(row_start[rows]);
    {
        std::vector<std::size_t> fill(row_start.begin(), row_start.end() - 1);
        for (std::size_t m = 0; m < modules; ++m) {
            if (row_of[m] >= 0) cells[fill[static_cast<std::size_t>(row_of[m])]++] = static_cast<int32_t>(m);
        }
    }

    struct RowWindows {
        std::vector<int32_t> count, modules, nets;
        std::vector<int64_t> net_end;
        std::vector<uint8_t> device;
    };
    std::vector<RowWindows> per_row(rows);
    workers.run(rows, [&](std::size_t r) {
        if (row_start[r + 1] - row_start[r] < 2U) return;
        std::vector<int32_t> row_cells(cells.begin() + static_cast<std::ptrdiff_t>(row_start[r]),
                                       cells.begin() + static_cast<std::ptrdiff_t>(row_start[r + 1]));
        std::sort(row_cells.begin(), row_cells.end(),
                  [&](int32_t a, int32_t b) { return s.lowerLeftX(a) < s.lowerLeftX(b); });
        RowWindows& mine = per_row[r];
        std::vector<int32_t> window_nets;
        const auto emit = [&](std::size_t first, std::size_t size) {
            if (size < 2U) return;
            for (std::size_t start = static_cast<std::size_t>(phase); start + 1U < size; start += kWindow) {
                const std::size_t count = std::min<std::size_t>(kWindow, size - start);
                if (count < 2U) break;
                window_nets.clear();
                for (std::size_t i = 0; i < count; ++i) {
                    const int32_t m = row_cells[first + start + i];
                    for (int64_t k = s.module_pin_start[m]; k < s.module_pin_start[m + 1]; ++k) {
                        window_nets.push_back(s.pin_net[s.module_pins[k]]);
                    }
                }
                std::sort(window_nets.begin(), window_nets.end());
                window_nets.erase(std::unique(window_nets.begin(), window_nets.end()), window_nets.end());
                bool device = count == static_cast<std::size_t>(kWindow) && !window_nets.empty();
                for (const int32_t n : window_nets) {
                    if (static_cast<uint64_t>(d.net_pin_start[n + 1] - d.net_pin_start[n]) > maximum_net_degree) {
                        device = false;
                    }
                }
                mine.count.push_back(static_cast<int32_t>(count));
                for (std::size_t i = 0; i < kWindow; ++i) {
                    mine.modules.push_back(i < count ? row_cells[first + start + i] : -1);
                }
                mine.nets.insert(mine.nets.end(), window_nets.begin(), window_nets.end());
                mine.net_end.push_back(static_cast<int64_t>(mine.nets.size()));
                mine.device.push_back(device ? 1 : 0);
            }
        };
        std::size_t first = 0;
        for (std::size_t i = 1; i < row_cells.size(); ++i) {
            const int32_t previous = row_cells[i - 1];
            const double expected =
                s.lowerLeftX(previous) + roundedWidth(d.module_width[previous], d.row_site_spacing[r]);
            if (std::abs(s.lowerLeftX(row_cells[i]) - expected) > kSegmentEpsilon) {
                emit(first, i - first);
                first = i;
            }
        }
        emit(first, row_cells.size() - first);
    });
    for (std::size_t r = 0; r < rows; ++r) {
        const RowWindows& mine = per_row[r];
        const int64_t base = static_cast<int64_t>(out.nets.size());
        out.row.insert(out.row.end(), mine.count.size(), static_cast<int32_t>(r));
        out.count.insert(out.count.end(), mine.count.begin(), mine.count.end());
        out.modules.insert(out.modules.end(), mine.modules.begin(), mine.modules.end());
        out.nets.insert(out.nets.end(), mine.nets.begin(), mine.nets.end());
        for (const int64_t end : mine.net_end) out.net_start.push_back(base + end);
        out.device.insert(out.device.end(), mine.device.begin(), mine.device.end());
    }
}

}  // namespace

bool detailedPlace(const mpgp_design& d, const int32_t* row_orientation, const mpgp_detailed_options& options,
                   double* module_x, double* module_y, int32_t* module_orientation, mpgp_detailed_result& result,
                   std::string& reason) {
    reason.clear();
    // The checks of tryRunCudaDetailedPlacement (:493-523), without the home
    // server's device allow-list and free-memory reserve.
    if (options.method != MPGP_DETAILED_WINDOW_REORDER || options.window_size != kWindow) {
        reason = "CUDA detailed placement currently supports window reordering with a four-cell window only.";
        return false;
    }
    if (options.passes <= 0 || options.maximum_net_degree < 2U || options.improvement_epsilon < 0.0 ||
        options.maximum_cuda_memory_bytes == 0U) {
        reason = "CUDA detailed-placement options are outside their valid range.";
        return false;
    }
    validateDesign(d);
    for (int32_t m = 0; d.module_orientation != nullptr && m < d.module_count; ++m) {
        require(d.module_orientation[m] >= 0 && d.module_orientation[m] <= kOrientationUnknown,
                "Module orientations must be Orientation values (0-8).");
    }
    for (int32_t r = 0; row_orientation != nullptr && r < d.row_count; ++r) {
        require(row_orientation[r] >= 0 && row_orientation[r] <= kOrientationUnknown,
                "Row orientations must be Orientation values (0-8).");
    }
    int device_count = 0;
    if (cudaGetDeviceCount(&device_count) != cudaSuccess || options.cuda_device < 0 ||
        options.cuda_device >= device_count) {
        cudaGetLastError();
        reason = "Requested CUDA device is unavailable on this host.";
        return false;
    }
    int previous_device = 0;
    cudaGetDevice(&previous_device);
    if (cudaSetDevice(options.cuda_device) != cudaSuccess) {
        cudaGetLastError();
        reason = "Unable to select the requested CUDA device.";
        return false;
    }
    struct RestoreDevice {
        int device;
        ~RestoreDevice() { cudaSetDevice(device); }
    } restore{previous_device};
    cudaDeviceProp properties{};
    if (cudaGetDeviceProperties(&properties, options.cuda_device) != cudaSuccess || properties.major < 6) {
        reason = "Requested CUDA device lacks required double-precision support.";
        return false;
    }
    std::size_t free_bytes = 0;
    std::size_t total_bytes = 0;
    checkCuda(cudaMemGetInfo(&free_bytes, &total_bytes), "cudaMemGetInfo");
    const uint64_t limit = std::min<uint64_t>(options.maximum_cuda_memory_bytes, free_bytes);

    const DerivedDesign derived = deriveDesign(d);
    std::vector<uint8_t> standard(static_cast<std::size_t>(d.module_count));
    for (int32_t m = 0; m < d.module_count; ++m) standard[m] = derived.is_fixed[m] == 0 && derived.is_macro[m] == 0;
    const auto rowOrientation = [&](int r) { return row_orientation != nullptr ? row_orientation[r] : 0; };

    const Workers workers = Workers::all(16);
    Placement s(d);
    result = mpgp_detailed_result{};
    result.hpwl_before = s.hpwl(workers);
    result.cuda_device_used = options.cuda_device;
    const auto started = std::chrono::steady_clock::now();

    // Device copies of the design: sizes, pin modules and net CSR once; centres
    // and orientation-transformed pin offsets at the start of every pass.
    const std::size_t modules = static_cast<std::size_t>(d.module_count);
    const std::size_t pins = static_cast<std::size_t>(d.pin_count);
    const std::size_t nets = static_cast<std::size_t>(d.net_count);
    const std::size_t window_capacity = modules / kWindow + 1;
    uint64_t reserved = 0;
    DeviceArray<double2> center, moved_center, size, pin_offset, raw_offset;
    DeviceArray<int> pin_module, net_pin_start, owner;
    DeviceArray<int8_t> moved_orientation;
    DeviceArray<double> net_weight;
    DeviceArray<int4> window_modules;
    DeviceArray<double> window_start, window_bottom, window_spacing, value_before, value_after;
    DeviceArray<int> window_net_start, window_nets, best_order;
    DeviceArray<uint8_t> decided[2];
    center.allocate(modules, reserved, limit, "CUDA detailed module centers");
    moved_center.allocate(modules, reserved, limit, "CUDA detailed moved centers");
    owner.allocate(modules, reserved, limit, "CUDA detailed window owners");
    moved_orientation.allocate(modules, reserved, limit, "CUDA detailed moved orientations");
    size.allocate(modules, reserved, limit, "CUDA detailed module sizes");
    pin_offset.allocate(pins, reserved, limit, "CUDA detailed pin offsets");
    raw_offset.allocate(pins, reserved, limit, "CUDA detailed raw pin offsets");
    pin_module.allocate(pins, reserved, limit, "CUDA detailed pin modules");
    net_pin_start.allocate(nets + 1, reserved, limit, "CUDA detailed net offsets");
    net_weight.allocate(nets, reserved, limit, "CUDA detailed net weights");
    window_modules.allocate(window_capacity, reserved, limit, "CUDA detailed window modules");
    window_start.allocate(window_capacity, reserved, limit, "CUDA detailed window start x");
    window_bottom.allocate(window_capacity, reserved, limit, "CUDA detailed window bottoms");
    window_spacing.allocate(window_capacity, reserved, limit, "CUDA detailed window spacing");
    window_net_start.allocate(window_capacity + 1, reserved, limit, "CUDA detailed window net offsets");
    window_nets.allocate(std::max<std::size_t>(pins, 1), reserved, limit, "CUDA detailed window net ids");
    best_order.allocate(window_capacity, reserved, limit, "CUDA detailed best orders");
    value_before.allocate(window_capacity, reserved, limit, "CUDA detailed window values");
    value_after.allocate(window_capacity, reserved, limit, "CUDA detailed window values");
    decided[0].allocate(window_capacity, reserved, limit, "CUDA detailed decisions");
    decided[1].allocate(window_capacity, reserved, limit, "CUDA detailed decisions");
    const std::size_t tail_capacity = modules / 2 + 1;  // every window holds two cells at least
    DeviceArray<int4> tail_modules;
    DeviceArray<int> tail_count, tail_net_start;
    DeviceArray<double> tail_start, tail_bottom, tail_spacing;
    DeviceArray<int8_t> tail_decided[2], orientation_now;
    tail_modules.allocate(tail_capacity, reserved, limit, "CUDA detailed tail windows");
    tail_count.allocate(tail_capacity, reserved, limit, "CUDA detailed tail windows");
    tail_start.allocate(tail_capacity, reserved, limit, "CUDA detailed tail windows");
    tail_bottom.allocate(tail_capacity, reserved, limit, "CUDA detailed tail windows");
    tail_spacing.allocate(tail_capacity, reserved, limit, "CUDA detailed tail windows");
    tail_net_start.allocate(tail_capacity + 1, reserved, limit, "CUDA detailed tail window net offsets");
    tail_decided[0].allocate(tail_capacity, reserved, limit, "CUDA detailed tail orders");
    tail_decided[1].allocate(tail_capacity, reserved, limit, "CUDA detailed tail orders");
    orientation_now.allocate(modules, reserved, limit, "CUDA detailed orientations");
    result.cuda_reserved_memory_bytes = reserved;

    Stream stream;
    {
        std::vector<double2> sizes(modules);
        for (std::size_t m = 0; m < modules; ++m) sizes[m] = make_double2(d.module_width[m], d.module_height[m]);
        const std::vector<int> modules_of_pins(d.pin_module, d.pin_module + pins);
        std::vector<int> starts(nets + 1);
        for (std::size_t n = 0; n <= nets; ++n) starts[n] = static_cast<int>(d.net_pin_start[n]);
        const std::vector<double> weights(d.net_weight, d.net_weight + nets);
        std::vector<double2> raw(pins);
        for (std::size_t q = 0; q < pins; ++q) raw[q] = make_double2(d.pin_offset_x[q], d.pin_offset_y[q]);
        raw_offset.upload(raw, stream.get());
        size.upload(sizes, stream.get());
        pin_module.upload(modules_of_pins, stream.get());
        net_pin_start.upload(starts, stream.get());
        net_weight.upload(weights, stream.get());
        checkCuda(cudaStreamSynchronize(stream.get()), "detailed-placement upload");
    }

    Windows windows;
    std::vector<double2> host_center(modules);
    std::vector<double2> host_offset(pins);
    std::vector<int4> host_modules;
    std::vector<double> host_start, host_bottom, host_spacing, before, after;
    std::vector<int> host_net_start, host_nets, best, host_owner(modules);
    std::vector<int8_t> host_moved_orientation(modules);
    std::vector<uint8_t> assumed, divergent(nets);
    std::vector<int4> tail_host_modules;
    std::vector<int> tail_host_count, tail_host_net_start, tail_host_nets, tail_of_window;
    std::vector<double> tail_host_start, tail_host_bottom, tail_host_spacing;
    std::vector<int8_t> tail_result, tail_assumed, host_orientation_now(modules);
    for (int pass = 0; pass < options.passes; ++pass) {
        buildWindows(s, standard, (pass % 2) * (kWindow / 2), options.maximum_net_degree, workers, windows);
        const std::size_t total = windows.row.size();
        host_modules.clear();
        host_start.clear();
        host_bottom.clear();
        host_spacing.clear();
        host_net_start.assign(1, 0);
        host_nets.clear();
        std::vector<std::size_t> on_device;
        for (std::size_t k = 0; k < total; ++k) {
            if (windows.device[k] == 0) continue;
            on_device.push_back(k);
            const int32_t* m = &windows.modules[k * kWindow];
            host_modules.push_back(make_int4(m[0], m[1], m[2], m[3]));
            host_start.push_back(s.lowerLeftX(m[0]));
            host_bottom.push_back(d.row_bottom[windows.row[k]]);
            host_spacing.push_back(d.row_site_spacing[windows.row[k]]);
            for (int64_t e = windows.net_start[k]; e < windows.net_start[k + 1]; ++e) host_nets.push_back(windows.nets[e]);
            host_net_start.push_back(static_cast<int>(host_nets.size()));
        }
        const std::size_t count = on_device.size();
        require(count <= window_capacity && host_nets.size() <= std::max<std::size_t>(pins, 1),
                "Detailed-placement window arrays exceed their capacity.");
        // The host-rule windows with nets to evaluate (optimizeCpuWindow returns
        // at once for the others).
        tail_host_modules.clear();
        tail_host_count.clear();
        tail_host_start.clear();
        tail_host_bottom.clear();
        tail_host_spacing.clear();
        tail_host_net_start.assign(1, 0);
        tail_host_nets.clear();
        tail_of_window.assign(total, -1);
        for (std::size_t k = 0; k < total; ++k) {
            if (windows.device[k] != 0 || windows.net_start[k + 1] == windows.net_start[k]) continue;
            bool too_wide = false;
            for (int64_t e = windows.net_start[k]; e < windows.net_start[k + 1]; ++e) {
                const int32_t net = windows.nets[e];
                too_wide |= static_cast<uint64_t>(d.net_pin_start[net + 1] - d.net_pin_start[net]) >
                            options.maximum_net_degree;
            }
            if (too_wide) continue;
            tail_of_window[k] = static_cast<int>(tail_host_count.size());
            const int32_t* m = &windows.modules[k * kWindow];
            tail_host_modules.push_back(make_int4(m[0], m[1], m[2], m[3]));
            tail_host_count.push_back(windows.count[k]);
            tail_host_start.push_back(s.lowerLeftX(m[0]));
            tail_host_bottom.push_back(d.row_bottom[windows.row[k]]);
            tail_host_spacing.push_back(d.row_site_spacing[windows.row[k]]);
            for (int64_t e = windows.net_start[k]; e < windows.net_start[k + 1]; ++e) {
                tail_host_nets.push_back(windows.nets[e]);
            }
            tail_host_net_start.push_back(static_cast<int>(tail_host_nets.size()));
        }
        const std::size_t tails = tail_host_count.size();
        require(tails <= tail_capacity && tail_host_nets.size() <= std::max<std::size_t>(pins, 1),
                "Detailed-placement tail window arrays exceed their capacity.");
        if (count > 0 || tails > 0) {
            // Owners: device window j as j, tail window t as count + t; and the
            // orientation a moved cell takes.
            std::fill(host_owner.begin(), host_owner.end(), -1);
            for (std::size_t m = 0; m < modules; ++m) host_moved_orientation[m] = static_cast<int8_t>(s.orientation[m]);
            const auto own = [&](std::size_t k, int value) {
                const int32_t* m = &windows.modules[k * kWindow];
                const int r = windows.row[k];
                for (int i = 0; i < windows.count[k]; ++i) {
                    host_owner[m[i]] = value;
                    if (rowOrientation(r) != kOrientationUnknown) {
                        host_moved_orientation[m[i]] = static_cast<int8_t>(rowOrientation(r));
                    }
                }
            };
            for (std::size_t j = 0; j < count; ++j) own(on_device[j], static_cast<int>(j));
            for (std::size_t k = 0; k < total; ++k) {
                if (tail_of_window[k] >= 0) own(k, static_cast<int>(count) + tail_of_window[k]);
            }
            owner.upload(host_owner, stream.get());
            moved_orientation.upload(host_moved_orientation, stream.get());
        }
        best.assign(count, 0);
        before.assign(count, 0.0);
        after.assign(count, 0.0);
        assumed.assign(count, 0);
        if (count > 0) {
            for (std::size_t m = 0; m < modules; ++m) host_center[m] = make_double2(s.cx[m], s.cy[m]);
            workers.blocks(pins, 65536, [&](std::size_t b, std::size_t e) {
                for (std::size_t p = b; p < e; ++p) {
                    double ox = 0.0;
                    double oy = 0.0;
                    transform(d.pin_offset_x[p], d.pin_offset_y[p], s.orientation[d.pin_module[p]], ox, oy);
                    host_offset[p] = make_double2(ox, oy);
                }
            });
            center.upload(host_center, stream.get());
            pin_offset.upload(host_offset, stream.get());
            window_modules.upload(host_modules, stream.get());
            window_start.upload(host_start, stream.get());
            window_bottom.upload(host_bottom, stream.get());
            window_spacing.upload(host_spacing, stream.get());
            window_net_start.upload(host_net_start, stream.get());
            window_nets.upload(host_nets, stream.get());
            const WindowArrays arrays{window_modules.get(), window_start.get(), window_bottom.get(),
                                      window_spacing.get(), window_net_start.get(), window_nets.get()};
            const int n = static_cast<int>(count);
            const unsigned blocks = static_cast<unsigned>((count + kWindowsPerBlock - 1) / kWindowsPerBlock);
            windowOrdersKernel<<<blocks, 32 * kWindowsPerBlock, 0, stream.get()>>>(
                center.get(), size.get(), pin_module.get(), pin_offset.get(), net_pin_start.get(), net_weight.get(),
                arrays, n, options.improvement_epsilon, best_order.get(), decided[0].get(), moved_center.get());
            checkCuda(cudaGetLastError(), "windowOrdersKernel launch");
            // Each iteration re-decides every window on the previous iteration's
            // decisions; the last one's input is the assumption its values rest on.
            int in = 0;
            for (int iteration = 0; iteration < kSpeculations; ++iteration, in ^= 1) {
                speculativeValuesKernel<<<blocks, 32 * kWindowsPerBlock, 0, stream.get()>>>(
                    center.get(), moved_center.get(), owner.get(), moved_orientation.get(), raw_offset.get(),
                    pin_offset.get(), pin_module.get(), net_pin_start.get(), net_weight.get(), arrays, n,
                    best_order.get(), options.improvement_epsilon, decided[in].get(), decided[in ^ 1].get(),
                    value_before.get(), value_after.get());
                checkCuda(cudaGetLastError(), "speculativeValuesKernel launch");
            }
            best_order.download(best, stream.get());
            decided[in ^ 1].download(assumed, stream.get());
            value_before.download(before, stream.get());
            value_after.download(after, stream.get());
            checkCuda(cudaStreamSynchronize(stream.get()), "windowOrdersKernel");
        }

        // The device's windows in order (:649-677), then the host's (:680-688).
        std::fill(divergent.begin(), divergent.end(), 0);
        double wx[kWindow];
        double wy[kWindow];
        for (std::size_t j = 0; j < count; ++j) {
            const std::size_t k = on_device[j];
            ++result.evaluated_windows;
            result.evaluated_permutations += kOrders;
            const int order_index = best[j];
            if (order_index <= 0 || order_index >= kOrders) continue;
            const int32_t* m = &windows.modules[k * kWindow];
            const int32_t* window_nets_k = &windows.nets[windows.net_start[k]];
            const int net_count = static_cast<int>(windows.net_start[k + 1] - windows.net_start[k]);
            int order[kWindow];
            orderOf(order_index, order);
            const int r = windows.row[k];
            // The device's values rest on the assumed decisions of the earlier
            // windows; they are exact unless one whose cells sit on these nets
            // decided otherwise.
            double value_now = before[j];
            double value_then = after[j];
            bool stale = false;
            for (int e = 0; e < net_count && !stale; ++e) stale = divergent[window_nets_k[e]] != 0;
            if (stale) {
                for (int i = 0; i < kWindow; ++i) {
                    wx[i] = s.cx[m[i]];
                    wy[i] = s.cy[m[i]];
                }
                value_now = s.windowHpwl(m, kWindow, window_nets_k, net_count, wx, wy);
                s.centersForOrder(m, order, kWindow, d.row_bottom[r], d.row_site_spacing[r], wx, wy);
                value_then = s.windowHpwl(m, kWindow, window_nets_k, net_count, wx, wy);
            }
            const bool accept = value_then < value_now - options.improvement_epsilon;
            if (accept) {
                s.applyOrder(m, order, kWindow, d.row_bottom[r], d.row_site_spacing[r], rowOrientation(r));
                ++result.accepted_operations;
            }
            if (accept != (assumed[j] != 0)) {
                for (int e = 0; e < net_count; ++e) divergent[window_nets_k[e]] = 1;
            }
        }
        // The host-rule windows: evaluated on the device the same speculative
        // way, from the placement the four-cell windows left.
        tail_result.assign(tails, -1);
        tail_assumed.assign(tails, -1);
        if (tails > 0) {
            for (std::size_t m = 0; m < modules; ++m) {
                host_center[m] = make_double2(s.cx[m], s.cy[m]);
                host_orientation_now[m] = static_cast<int8_t>(s.orientation[m]);
            }
            center.upload(host_center, stream.get());
            orientation_now.upload(host_orientation_now, stream.get());
            tail_modules.upload(tail_host_modules, stream.get());
            tail_count.upload(tail_host_count, stream.get());
            tail_start.upload(tail_host_start, stream.get());
            tail_bottom.upload(tail_host_bottom, stream.get());
            tail_spacing.upload(tail_host_spacing, stream.get());
            tail_net_start.upload(tail_host_net_start, stream.get());
            window_nets.upload(tail_host_nets, stream.get());
            checkCuda(cudaMemsetAsync(tail_decided[0].get(), 0xFF, tails, stream.get()), "tail orders");
            const TailArrays tail{tail_modules.get(), tail_count.get(), tail_start.get(), tail_bottom.get(),
                                  tail_spacing.get(), tail_net_start.get(), window_nets.get()};
            const int n = static_cast<int>(tails);
            const unsigned blocks = static_cast<unsigned>((tails + 255) / 256);
            const unsigned warp_blocks = static_cast<unsigned>((tails + kWindowsPerBlock - 1) / kWindowsPerBlock);
            int in = 0;
            for (int iteration = 0; iteration < kSpeculations; ++iteration, in ^= 1) {
                if (iteration > 0) {
                    tailPlacementKernel<<<blocks, 256, 0, stream.get()>>>(tail, n, size.get(), tail_decided[in].get(),
                                                                         moved_center.get());
                    checkCuda(cudaGetLastError(), "tailPlacementKernel launch");
                }
                tailOrdersKernel<<<warp_blocks, 32 * kWindowsPerBlock, 0, stream.get()>>>(
                    center.get(), orientation_now.get(), moved_center.get(), owner.get(), static_cast<int>(count),
                    moved_orientation.get(), raw_offset.get(), size.get(), pin_module.get(), net_pin_start.get(),
                    net_weight.get(), tail, n, options.improvement_epsilon, tail_decided[in].get(),
                    tail_decided[in ^ 1].get());
                checkCuda(cudaGetLastError(), "tailOrdersKernel launch");
            }
            tail_decided[in].download(tail_result, stream.get());
            tail_decided[in ^ 1].download(tail_assumed, stream.get());
            checkCuda(cudaStreamSynchronize(stream.get()), "tailOrdersKernel");
        }
        std::fill(divergent.begin(), divergent.end(), 0);
        for (std::size_t k = 0; k < total; ++k) {
            if (windows.device[k] != 0) continue;
            ++result.evaluated_windows;
            const int t = tail_of_window[k];
            if (t < 0) continue;  // no nets, or one above the degree limit: nothing to evaluate
            // optimizeCpuWindow (:328-354).
            const int32_t* m = &windows.modules[k * kWindow];
            const int n = windows.count[k];
            const int32_t* window_nets_k = &windows.nets[windows.net_start[k]];
            const int net_count = static_cast<int>(windows.net_start[k + 1] - windows.net_start[k]);
            const int r = windows.row[k];
            result.evaluated_permutations += static_cast<uint64_t>(factorialOf(n));
            bool stale = false;
            for (int e = 0; e < net_count && !stale; ++e) stale = divergent[window_nets_k[e]] != 0;
            int taken = tail_result[t];
            if (stale) {
                for (int i = 0; i < n; ++i) {
                    wx[i] = s.cx[m[i]];
                    wy[i] = s.cy[m[i]];
                }
                double best_value = s.windowHpwl(m, n, window_nets_k, net_count, wx, wy);
                taken = -1;
                for (int candidate = 0; candidate < factorialOf(n); ++candidate) {
                    int order[kWindow];
                    orderOf(candidate, order, n);
                    s.centersForOrder(m, order, n, d.row_bottom[r], d.row_site_spacing[r], wx, wy);
                    const double value = s.windowHpwl(m, n, window_nets_k, net_count, wx, wy);
                    if (value < best_value - options.improvement_epsilon) {
                        best_value = value;
                        taken = candidate;
                    }
                }
            }
            if (taken >= 0) {
                int order[kWindow];
                orderOf(taken, order, n);
                s.applyOrder(m, order, n, d.row_bottom[r], d.row_site_spacing[r], rowOrientation(r));
                ++result.accepted_operations;
            }
            if (taken != tail_assumed[t]) {
                for (int e = 0; e < net_count; ++e) divergent[window_nets_k[e]] = 1;
            }
        }
        result.completed_passes = pass + 1;
    }
    result.hpwl_after = s.hpwl(workers);
    result.elapsed_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - started).count();
    std::copy(s.cx.begin(), s.cx.end(), module_x);
    std::copy(s.cy.begin(), s.cy.end(), module_y);
    if (module_orientation != nullptr) std::copy(s.orientation.begin(), s.orientation.end(), module_orientation);
    return true;
}

}  // namespace mpgp
