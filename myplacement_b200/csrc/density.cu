// Course-ePlace density: fixed-point scatter and the per-bin metrics pass.
//
// scatter: restates DensityMap::addRectangle (Metrics.cpp:74-99) for every
// particle (depositDynamicDensity, GlobalPlacementSupport.cpp:32-40; the
// reference CUDA depositParticlesKernel, CudaPlacementBackend.cu:339-375).  The
// overlap of a particle with each covered bin is computed in FP32 bin units and
// quantized to int64 in units of bin_area * 2^-32, then added with integer
// atomics, so the map is bit-exact run to run and equal to the fixed-point CPU
// oracle (oracle/density_fixed.c).  Every floating-point operation uses an
// explicitly rounded intrinsic, so no fused multiply-add can change a bit.
// The same pass optionally forms the particle positions first: the
// backtracking proposal (proposeStep, AdaptiveGlobalPlacer.cpp:494-519) or the
// Nesterov lookahead (:776-780), both clamped to the core
// (clampCenterToRegion, GlobalPlacementSupport.cpp:11-19).
//
// metrics: restates buildDensityMetricsKernel + collectDensityMetrics
// (CudaPlacementBackend.cu:377-398, 1022-1038) and DensityMap::metrics
// (Metrics.cpp:101-119), reads-and-clears the fixed-point layers and writes the
// mean-free FP32 source of the Poisson solve (ElectrostaticField.cpp:119-133);
// the mean comes from the exact integer layer totals of the scatter.
#include <algorithm>

#include "common.cuh"
#include "dct_tc.cuh"
#include "kernels.cuh"
#include "split.cuh"

namespace mpgp {
namespace {

__device__ __forceinline__ double clampIndex(double value, int upper) {
    return value < 0.0 ? 0.0 : (value > static_cast<double>(upper) ? static_cast<double>(upper) : value);
}

__device__ __forceinline__ double clampCenter(double value, double size, double low, double high) {
    const double lo = __dadd_rn(low, __dmul_rn(size, 0.5));
    const double hi = __dsub_rn(high, __dmul_rn(size, 0.5));
    return lo <= hi ? fmax(lo, fmin(value, hi)) : __dmul_rn(__dadd_rn(low, high), 0.5);
}

// One block of the scatter: particles block * 256 .. of the launch (or of its
// instance in a batched launch), each adding its fixed-point overlaps to the map
// with integer atomics (the map is L2-resident, so the atomics stay in L2).
__device__ __forceinline__ void scatterBlock(const ScatterArgs& a, int block, int grid) {
    const int i = block * static_cast<int>(blockDim.x) + static_cast<int>(threadIdx.x);
    double predicted = 0.0;
    double displacement = 0.0;
    long long totals[3] = {0, 0, 0};
    if (i < a.particle_count) {
        double2 c;
        const double2 size = a.size[i];
        if (a.mode == kGiven) {
            c = a.positions[i];
        } else {
            const double2 base = a.base[i];
            const double2 dir = a.direction[i];
            double dx, dy;
            if (a.mode == kPropose) {
                dx = dir.x * (-a.step);
                dy = dir.y * (-a.step);
                const double norm = sqrt(dx * dx + dy * dy);
                if (norm > a.max_displacement) {
                    const double s = a.max_displacement / norm;
                    dx = dx * s;
                    dy = dy * s;
                }
            } else {
                dx = dir.x * a.step;
                dy = dir.y * a.step;
            }
            c.x = clampCenter(base.x + dx, size.x, a.llx, a.urx);
            c.y = clampCenter(base.y + dy, size.y, a.lly, a.ury);
            a.out_positions[i] = c;
            if (a.mode == kPropose) {
                const double2 raw = a.raw[i];
                const double ax = base.x - c.x;
                const double ay = base.y - c.y;
                predicted = raw.x * ax + raw.y * ay;
                displacement = sqrt(ax * ax + ay * ay);
            }
        }
        // Fixed-point deposit (oracle/density_fixed.c).
        const double half_w = __dmul_rn(size.x, 0.5);
        const double half_h = __dmul_rn(size.y, 0.5);
        const double l = fmax(a.llx, __dsub_rn(c.x, half_w));
        const double r = fmin(a.urx, __dadd_rn(c.x, half_w));
        const double b = fmax(a.lly, __dsub_rn(c.y, half_h));
        const double t = fmin(a.ury, __dadd_rn(c.y, half_h));
        if (__dmul_rn(fmax(0.0, __dsub_rn(r, l)), fmax(0.0, __dsub_rn(t, b))) > 1e-9) {
            const double gl = __ddiv_rn(__dsub_rn(l, a.llx), a.bin_w);
            const double gr = __ddiv_rn(__dsub_rn(r, a.llx), a.bin_w);
            const double gb = __ddiv_rn(__dsub_rn(b, a.lly), a.bin_h);
            const double gt = __ddiv_rn(__dsub_rn(t, a.lly), a.bin_h);
            const int c0 = static_cast<int>(clampIndex(floor(gl), a.bins_x - 1));
            const int c1 = static_cast<int>(clampIndex(__dsub_rn(ceil(gr), 1.0), a.bins_x - 1));
            const int r0 = static_cast<int>(clampIndex(floor(gb), a.bins_y - 1));
            const int r1 = static_cast<int>(clampIndex(__dsub_rn(ceil(gt), 1.0), a.bins_y - 1));
            const float fl = __double2float_rn(__dsub_rn(gl, static_cast<double>(c0)));
            const float fr = __double2float_rn(__dsub_rn(gr, static_cast<double>(c0)));
            const float fb = __double2float_rn(__dsub_rn(gb, static_cast<double>(r0)));
            const float ft = __double2float_rn(__dsub_rn(gt, static_cast<double>(r0)));
            const int code = a.layer[i];
            unsigned long long* target = a.layers + static_cast<size_t>(code) * a.bins_x * a.bins_y;
            long long sum = 0;
            for (int row = r0; row <= r1; ++row) {
                const float fi = static_cast<float>(row - r0);
                const float oy = fmaxf(0.0f, __fsub_rn(fminf(ft, __fadd_rn(fi, 1.0f)), fmaxf(fb, fi)));
                for (int column = c0; column <= c1; ++column) {
                    const float fj = static_cast<float>(column - c0);
                    const float ox = fmaxf(0.0f, __fsub_rn(fminf(fr, __fadd_rn(fj, 1.0f)), fmaxf(fl, fj)));
                    const long long q = __float2ll_rn(__fmul_rn(__fmul_rn(ox, oy), kFixedOne));
                    if (q != 0) {
                        atomicAdd(target + static_cast<size_t>(row) * a.bins_x + column,
                                  static_cast<unsigned long long>(q));
                        sum += q;
                    }
                }
            }
            totals[code] = sum;
        }
    }
    // Exact integer totals of each layer (for the mean removal) and the proposal scalars.
    __shared__ long long block_totals[3];
    if (threadIdx.x < 3) block_totals[threadIdx.x] = 0;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const long long w = warpSumI64(totals[k]);
        if ((threadIdx.x & 31) == 0 && w != 0) {
            atomicAdd(reinterpret_cast<unsigned long long*>(&block_totals[k]), static_cast<unsigned long long>(w));
        }
    }
    double values[2] = {predicted, displacement};
    const bool is_max[2] = {false, true};
    blockReduce<2>(values, is_max);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            if (block_totals[k] != 0) atomicAdd(a.totals + k, static_cast<unsigned long long>(block_totals[k]));
        }
        if (a.partials != nullptr) {
            a.partials[block] = values[0];
            a.partials[grid + block] = values[1];
        }
    }
    if (a.partials != nullptr && a.group_counters != nullptr) {
        reduceGroups<2>(a.partials, a.group_partials, a.group_counters, is_max, static_cast<unsigned>(block),
                        static_cast<unsigned>(grid));
    }
}

__global__ void __launch_bounds__(kThreads) scatterKernel(ScatterArgs a) {
    releaseNext();
    waitForPrior();
    scatterBlock(a, static_cast<int>(blockIdx.x), static_cast<int>(gridDim.x));
}

__global__ void __launch_bounds__(kThreads) scatterBatchKernel(const ScatterArgs* args, const int* offsets,
                                                               int count) {
    releaseNext();
    waitForPrior();
    const int3 slot = batchSlot(offsets, count, static_cast<int>(blockIdx.x));
    const ScatterArgs a = args[slot.x];
    scatterBlock(a, slot.y, slot.z);
}

// One bin's metric terms (DensityBin::chargeArea / normalizationArea, Metrics.hpp:25-35).
struct BinTerms {
    double t, unit, capacity, inv_area, mean;
    __device__ void add(unsigned long long qm, unsigned long long qc, unsigned long long qf, double static_charge,
                        double (&v)[9], float& source) const {
        const double movable = static_cast<double>(static_cast<long long>(qm)) * unit;
        const double macro = static_cast<double>(static_cast<long long>(qc)) * unit;
        const double filler = static_cast<double>(static_cast<long long>(qf)) * unit;
        const double without = movable + t * macro + static_charge;  // chargeArea(t, false)
        const double with = without + t * filler;                    // chargeArea(t, true)
        const double density_with = with * inv_area;
        const double density_without = without * inv_area;
        v[0] += fmax(0.0, with - capacity);
        v[1] += fmax(0.0, without - capacity);
        v[2] += with;
        v[3] += without;
        v[4] += movable + t * macro;  // normalizationArea
        v[5] += density_with;
        v[6] += density_without;
        v[7] = fmax(v[7], density_with);
        v[8] = fmax(v[8], density_without);
        source = static_cast<float>((density_with - t) - mean);
    }
};

__global__ void __launch_bounds__(kThreads) metricsKernel(MetricsArgs a) {
    releaseNext();
    waitForPrior();
    BinTerms terms;
    terms.t = a.target_density;
    terms.unit = a.bin_area * kFixedUnit;
    terms.capacity = terms.t * a.bin_area;
    terms.inv_area = 1.0 / a.bin_area;
    // Mean of the density deviation from the exact layer totals.
    const double movable_sum = static_cast<double>(static_cast<long long>(a.totals[0])) * terms.unit;
    const double macro_sum = static_cast<double>(static_cast<long long>(a.totals[1])) * terms.unit;
    const double filler_sum = static_cast<double>(static_cast<long long>(a.totals[2])) * terms.unit;
    const double charge_total =
        movable_sum + terms.t * (a.static_fixed_sum + macro_sum + a.static_dark_sum + filler_sum);
    terms.mean = charge_total / (a.bin_area * static_cast<double>(a.bin_count)) - terms.t;

    double v[9] = {0, 0, 0, 0, 0, 0, 0, -1.0e308, -1.0e308};
    const int bins = a.bin_count;
    unsigned long long* qm = a.layers;
    unsigned long long* qc = a.layers + bins;
    unsigned long long* qf = a.layers + 2 * static_cast<size_t>(bins);
    const int stride = gridDim.x * blockDim.x;
    if ((bins & 1) == 0) {
        // Two bins per step: 16-byte loads of every layer, stores of zeros and the source pair.
        for (int pair = blockIdx.x * blockDim.x + threadIdx.x; pair < bins / 2; pair += stride) {
            const ulonglong2 m = reinterpret_cast<const ulonglong2*>(qm)[pair];
            const ulonglong2 c = reinterpret_cast<const ulonglong2*>(qc)[pair];
            const ulonglong2 f = reinterpret_cast<const ulonglong2*>(qf)[pair];
            const double2 st = reinterpret_cast<const double2*>(a.static_charge)[pair];
            const ulonglong2 zero = make_ulonglong2(0ULL, 0ULL);
            reinterpret_cast<ulonglong2*>(qm)[pair] = zero;
            reinterpret_cast<ulonglong2*>(qc)[pair] = zero;
            reinterpret_cast<ulonglong2*>(qf)[pair] = zero;
            float2 out;
            terms.add(m.x, c.x, f.x, st.x, v, out.x);
            terms.add(m.y, c.y, f.y, st.y, v, out.y);
            reinterpret_cast<float2*>(a.source)[pair] = out;
        }
    } else {
        for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < bins; b += stride) {
            const unsigned long long m = qm[b], c = qc[b], f = qf[b];
            qm[b] = 0ULL;
            qc[b] = 0ULL;
            qf[b] = 0ULL;
            terms.add(m, c, f, a.static_charge[b], v, a.source[b]);
        }
    }
    const bool is_max[9] = {false, false, false, false, false, false, false, true, true};
    blockReduce<9>(v, is_max);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < 9; ++k) a.partials[k * gridDim.x + blockIdx.x] = v[k];
    }
    if (a.group_counters != nullptr) {
        reduceGroups<9>(a.partials, a.group_partials, a.group_counters, is_max, blockIdx.x, gridDim.x);
    }
}

// The metrics pass fused with the source split of the field solve: one block
// per bin row forms the row's sources in registers (they are never stored),
// takes the row maximum for the row's plane exponent (splitSourceKernel's rule)
// and writes the fp16 hi / lo planes of the first contraction's operand.
__device__ __forceinline__ void metricsSplitBlock(const MetricsArgs& a, int block, int grid) {
    BinTerms terms;
    terms.t = a.target_density;
    terms.unit = a.bin_area * kFixedUnit;
    terms.capacity = terms.t * a.bin_area;
    terms.inv_area = 1.0 / a.bin_area;
    const double movable_sum = static_cast<double>(static_cast<long long>(a.totals[0])) * terms.unit;
    const double macro_sum = static_cast<double>(static_cast<long long>(a.totals[1])) * terms.unit;
    const double filler_sum = static_cast<double>(static_cast<long long>(a.totals[2])) * terms.unit;
    const double charge_total =
        movable_sum + terms.t * (a.static_fixed_sum + macro_sum + a.static_dark_sum + filler_sum);
    terms.mean = charge_total / (a.bin_area * static_cast<double>(a.bin_count)) - terms.t;
    if (block == 0 && threadIdx.x == 0) {
        a.scales->max_x = 0u;
        a.scales->max_phi = 0u;
    }

    const int row = block;
    const int cols = a.columns;
    const size_t base = static_cast<size_t>(row) * cols;
    const int bins = a.bin_count;
    unsigned long long* qm = a.layers + base;
    unsigned long long* qc = a.layers + bins + base;
    unsigned long long* qf = a.layers + 2 * static_cast<size_t>(bins) + base;
    const double* st = a.static_charge + base;
    double v[9] = {0, 0, 0, 0, 0, 0, 0, -1.0e308, -1.0e308};
    float out[kMetricsSplitPerThread];
    float top = 0.0f;
    const bool pairs = (cols & 1) == 0;
    if (pairs) {
#pragma unroll
        for (int j = 0; j < kMetricsSplitPerThread / 2; ++j) {
            const int pair = static_cast<int>(threadIdx.x) + j * kThreads;
            out[2 * j] = 0.0f;
            out[2 * j + 1] = 0.0f;
            if (pair < cols / 2) {
                const ulonglong2 m = reinterpret_cast<const ulonglong2*>(qm)[pair];
                const ulonglong2 c = reinterpret_cast<const ulonglong2*>(qc)[pair];
                const ulonglong2 f = reinterpret_cast<const ulonglong2*>(qf)[pair];
                const double2 s = reinterpret_cast<const double2*>(st)[pair];
                const ulonglong2 zero = make_ulonglong2(0ULL, 0ULL);
                reinterpret_cast<ulonglong2*>(qm)[pair] = zero;
                reinterpret_cast<ulonglong2*>(qc)[pair] = zero;
                reinterpret_cast<ulonglong2*>(qf)[pair] = zero;
                terms.add(m.x, c.x, f.x, s.x, v, out[2 * j]);
                terms.add(m.y, c.y, f.y, s.y, v, out[2 * j + 1]);
                top = fmaxf(top, fmaxf(fabsf(out[2 * j]), fabsf(out[2 * j + 1])));
            }
        }
    } else {
#pragma unroll
        for (int j = 0; j < kMetricsSplitPerThread; ++j) {
            const int c = static_cast<int>(threadIdx.x) + j * kThreads;
            out[j] = 0.0f;
            if (c < cols) {
                const unsigned long long m = qm[c], cm = qc[c], f = qf[c];
                qm[c] = 0ULL;
                qc[c] = 0ULL;
                qf[c] = 0ULL;
                terms.add(m, cm, f, st[c], v, out[j]);
                top = fmaxf(top, fabsf(out[j]));
            }
        }
    }
    __shared__ float warp_top[kThreads / 32];
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int offset = 16; offset > 0; offset >>= 1) top = fmaxf(top, __shfl_xor_sync(0xffffffffu, top, offset));
    if (lane == 0) warp_top[threadIdx.x >> 5] = top;
    __syncthreads();
    top = 0.0f;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) top = fmaxf(top, warp_top[w]);
    const int e = exponentOf(top) - kPlaneTop;
    if (threadIdx.x == 0) {
        a.row_exp[row] = e;
        atomicMax(&a.scales->max_source, __float_as_uint(top));
    }
    const float inv_scale = static_cast<float>(pow2(-e));
    __half* hi = a.split_out + static_cast<size_t>(row) * a.split_ld;
    __half* lo = hi + a.split_plane;
    if (pairs) {
#pragma unroll
        for (int j = 0; j < kMetricsSplitPerThread / 2; ++j) {
            const int pair = static_cast<int>(threadIdx.x) + j * kThreads;
            if (pair < cols / 2) {
                __half h0, l0, h1, l1;
                splitScaled(out[2 * j], inv_scale, h0, l0);
                splitScaled(out[2 * j + 1], inv_scale, h1, l1);
                reinterpret_cast<uint32_t*>(hi)[pair] = packHalves(h0, h1);
                reinterpret_cast<uint32_t*>(lo)[pair] = packHalves(l0, l1);
            }
        }
    } else {
#pragma unroll
        for (int j = 0; j < kMetricsSplitPerThread; ++j) {
            const int c = static_cast<int>(threadIdx.x) + j * kThreads;
            if (c < cols) splitScaled(out[j], inv_scale, hi[c], lo[c]);
        }
    }
    const bool is_max[9] = {false, false, false, false, false, false, false, true, true};
    blockReduce<9>(v, is_max);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < 9; ++k) a.partials[k * grid + block] = v[k];
    }
    if (a.group_counters != nullptr) {
        reduceGroups<9>(a.partials, a.group_partials, a.group_counters, is_max, static_cast<unsigned>(block),
                        static_cast<unsigned>(grid));
    }
}

__global__ void __launch_bounds__(kThreads) metricsSplitKernel(MetricsArgs a) {
    releaseNext();
    waitForPrior();
    metricsSplitBlock(a, static_cast<int>(blockIdx.x), static_cast<int>(gridDim.x));
}

__global__ void __launch_bounds__(kThreads) metricsSplitBatchKernel(const MetricsArgs* args, const int* offsets,
                                                                    int count) {
    releaseNext();
    waitForPrior();
    const int3 slot = batchSlot(offsets, count, static_cast<int>(blockIdx.x));
    const MetricsArgs a = args[slot.x];
    metricsSplitBlock(a, slot.y, slot.z);
}

__global__ void velocityKernel(const double2* next, const double2* previous, double2* velocity, int count) {
    releaseNext();
    waitForPrior();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const double2 n = next[i];
    const double2 p = previous[i];
    velocity[i] = make_double2(n.x - p.x, n.y - p.y);
}

// Copies `count` positions (a checkpoint of the controller's placement).
__global__ void copyPositionsKernel(const double2* source, double2* destination, int count) {
    releaseNext();
    waitForPrior();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        destination[i] = source[i];
    }
}

}  // namespace

void launchScatter(const ScatterArgs& args, int blocks, cudaStream_t stream) {
    if (blocks <= 0) return;
    launchChained("Launch the density scatter", scatterKernel, dim3(blocks), dim3(kThreads), 0, stream, args);
}

void launchMetrics(const MetricsArgs& args, int blocks, cudaStream_t stream) {
    launchChained("Launch the density metrics", metricsKernel, dim3(blocks), dim3(kThreads), 0, stream, args);
}

void launchMetricsSplit(const MetricsArgs& args, cudaStream_t stream) {
    if (args.rows <= 0) return;
    launchChained("Launch the density metrics and source split", metricsSplitKernel, dim3(args.rows),
                  dim3(kThreads), 0, stream, args);
}

void launchScatterBatch(const ScatterArgs* args, const int* offsets, int count, int blocks, cudaStream_t stream) {
    if (blocks <= 0 || count <= 0) return;
    launchChained("Launch the batched density scatter", scatterBatchKernel, dim3(blocks), dim3(kThreads), 0, stream,
                  args, offsets, count);
}

void launchMetricsSplitBatch(const MetricsArgs* args, const int* offsets, int count, int blocks,
                             cudaStream_t stream) {
    if (blocks <= 0 || count <= 0) return;
    launchChained("Launch the batched density metrics and source split", metricsSplitBatchKernel, dim3(blocks),
                  dim3(kThreads), 0, stream, args, offsets, count);
}

void launchCopyPositions(const double2* source, double2* destination, int count, cudaStream_t stream) {
    if (count <= 0) return;
    int device = 0, sms = 0;
    checkCuda(cudaGetDevice(&device), "Query the current device");
    checkCuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "Query the SM count");
    const int blocks = std::max(1, std::min(ceilDiv(count, kThreads), 4 * sms));
    launchChained("Launch the checkpoint copy", copyPositionsKernel, dim3(blocks), dim3(kThreads), 0, stream, source,
                  destination, count);
}

void launchVelocity(const double2* next, const double2* previous, double2* velocity, int count, cudaStream_t stream) {
    if (count <= 0) return;
    launchChained("Launch the velocity update", velocityKernel, dim3(ceilDiv(count, kThreads)), dim3(kThreads), 0,
                  stream, next, previous, velocity, count);
}

}  // namespace mpgp
