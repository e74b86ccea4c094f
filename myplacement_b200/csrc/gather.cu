// The fused per-particle pass of a gradient evaluation, and the scalar reduction.
//
// gather: for each particle, in one pass,
//   wire     = sum of its pins' LSE gradients, which the wirelength pass wrote
//              into consecutive slots (fixed pin order: deterministic)
//   density  = -charge * E(position)  -- bilinear sample of the DCT field with
//              the Neumann mirror parity (sampleWithParity / reflectIndex,
//              ElectrostaticField.cpp:289-320; CudaPlacementBackend.cu:158-192, 575-591)
//   raw      = wire + penalty * density [+ rudy_weight * RUDY, summed over the pins' slots]
//   pre      = raw * precond_base / density_strength
// and the FP64 block partials the controller needs: |wire|_1, |density|_1,
// |raw|^2, |pre|^2 (GlobalPlacementSession::evaluateCuda, AdaptiveGlobalPlacer.cpp:
// 308-330), the curvature terms |x - x_prev|^2 and |pre - pre_prev|^2
// (estimateStep, :470-492) and the momentum alignment sum v . pre (:610-617).
// In split mode (the drop-in backend) it writes the wire and density
// gradients separately instead, as CudaPlacementBackend::evaluate returns them.
//
// reduce: folds every kernel's per-block partials into the evaluation's
// scalar block in a fixed order (deterministic) and clears the integer layer
// totals for the next scatter.
#include <algorithm>
#include <mutex>

#include "common.cuh"
#include "kernels.cuh"

namespace mpgp {
namespace {

// Field sample with mirror parity; positions are already clamped to the region,
// so one reflection step at most is needed on each side.
__device__ __forceinline__ double2 sampleField(const GatherArgs& a, double x, double y) {
    x = fmax(a.llx, fmin(x, a.urx));
    y = fmax(a.lly, fmin(y, a.ury));
    const double gx = (x - a.llx) * a.inv_bin_w - 0.5;
    const double gy = (y - a.lly) * a.inv_bin_h - 0.5;
    const double fx = floor(gx);
    const double fy = floor(gy);
    const int left = static_cast<int>(fx);
    const int bottom = static_cast<int>(fy);
    const double tx = gx - fx;
    const double ty = gy - fy;
    double ex[4], ey[4];
#pragma unroll
    for (int corner = 0; corner < 4; ++corner) {
        int column = left + (corner & 1);
        int row = bottom + (corner >> 1);
        double sx = 1.0, sy = 1.0;
        if (column < 0) { column = -column - 1; sx = -sx; }
        if (column >= a.bins_x) { column = 2 * a.bins_x - column - 1; sx = -sx; }
        if (row < 0) { row = -row - 1; sy = -sy; }
        if (row >= a.bins_y) { row = 2 * a.bins_y - row - 1; sy = -sy; }
        // Positions are clamped to the region, so one reflection suffices; keep the
        // index in range even for non-finite input.
        column = min(max(column, 0), a.bins_x - 1);
        row = min(max(row, 0), a.bins_y - 1);
        const float2 f = a.field[static_cast<size_t>(row) * a.bins_x + column];
        ex[corner] = sx * static_cast<double>(f.x);  // Ex is odd in x
        ey[corner] = sy * static_cast<double>(f.y);  // Ey is odd in y
    }
    const double lower_x = ex[0] * (1.0 - tx) + ex[1] * tx;
    const double upper_x = ex[2] * (1.0 - tx) + ex[3] * tx;
    const double lower_y = ey[0] * (1.0 - tx) + ey[1] * tx;
    const double upper_y = ey[2] * (1.0 - tx) + ey[3] * tx;
    return make_double2(lower_x * (1.0 - ty) + upper_x * ty, lower_y * (1.0 - ty) + upper_y * ty);
}

// One scalar into the host record: low and high 32 bits, each beside the sequence.
__device__ __forceinline__ void publishScalar(unsigned long long* slots, int target, double value,
                                              unsigned int sequence) {
    const unsigned long long bits = static_cast<unsigned long long>(__double_as_longlong(value));
    const unsigned long long tag = static_cast<unsigned long long>(sequence) << 32;
    volatile unsigned long long* slot = reinterpret_cast<volatile unsigned long long*>(slots) + 2 * target;
    slot[0] = tag | (bits & 0xffffffffULL);
    slot[1] = tag | (bits >> 32);
}

// Thread 0 resets the layer totals and publishes the error flag.
__device__ __forceinline__ void finishReduce(const ReduceArgs& a) {
    if (threadIdx.x != 0) return;
    if (a.totals != nullptr) {
        a.totals[0] = 0ULL;
        a.totals[1] = 0ULL;
        a.totals[2] = 0ULL;
    }
    if (a.host_slots != nullptr) {
        const unsigned int error = static_cast<unsigned int>(*reinterpret_cast<const volatile int*>(a.device_error));
        const unsigned long long tag = static_cast<unsigned long long>(a.sequence) << 32;
        reinterpret_cast<volatile unsigned long long*>(a.host_slots)[2 * kScalarCount] = tag | error;
    }
}

// Every source of `a` reduced by the calling block: warp w takes sources w,
// w + warps, ... (four at a time, their first rows loaded together); lane l
// sums rows l, l + 32, ... in order, then a fixed shuffle tree, so the scalars
// do not depend on timing.  With a completion record, the scalars and the
// error flag are also published to host memory.
__device__ void reduceAllSources(const ReduceArgs& a) {
    constexpr int kSourcesPerWarp = 4;  // sources a warp handles per pass, loads issued together
    constexpr int kRowsPerLane = 4;     // rows lane + 32 j prefetched per source
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int warps = blockDim.x >> 5;
    for (int first = warp; first < a.source_count; first += warps * kSourcesPerWarp) {
        double x[kSourcesPerWarp][kRowsPerLane];
#pragma unroll
        for (int i = 0; i < kSourcesPerWarp; ++i) {
            const int s = first + i * warps;
            const ReduceSource src = s < a.source_count ? a.sources[s] : ReduceSource{nullptr, 0, 0, 0, 0, 0};
#pragma unroll
            for (int j = 0; j < kRowsPerLane; ++j) {
                const int row = lane + 32 * j;
                x[i][j] = row < src.rows ? __ldcg(src.partials + static_cast<size_t>(row) * src.stride + src.column)
                                         : (src.is_max ? -1.0e308 : 0.0);
            }
        }
#pragma unroll
        for (int i = 0; i < kSourcesPerWarp; ++i) {
            const int s = first + i * warps;
            if (s >= a.source_count) break;
            const ReduceSource src = a.sources[s];
            double value = src.is_max ? -1.0e308 : 0.0;
#pragma unroll
            for (int j = 0; j < kRowsPerLane; ++j) value = src.is_max ? fmax(value, x[i][j]) : value + x[i][j];
            for (int row = lane + 32 * kRowsPerLane; row < src.rows; row += 32) {
                const double y = __ldcg(src.partials + static_cast<size_t>(row) * src.stride + src.column);
                value = src.is_max ? fmax(value, y) : value + y;
            }
            value = src.is_max ? warpMax(value) : warpSum(value);
            if (lane == 0) {
                const double result = src.rows > 0 ? value : 0.0;
                a.scalars[src.target] = result;
                if (a.host_slots != nullptr) publishScalar(a.host_slots, src.target, result, a.sequence);
            }
        }
    }
    finishReduce(a);
}

__device__ __forceinline__ void gatherBlock(const GatherArgs& a, const ReduceArgs* reduce, int block, int grid) {
    double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    // Grid-stride over the particles (one resident wave), each thread in ascending order.
    for (int i = block * blockDim.x + threadIdx.x; i < a.particle_count; i += grid * blockDim.x) {
        double wx = 0.0, wy = 0.0, rx_rudy = 0.0, ry_rudy = 0.0;
        if (i < a.movable_count) {
            const int begin = a.particle_pin_start[i];
            const int end = a.particle_pin_start[i + 1];
            for (int j = begin; j < end; ++j) {
                const float2 g = a.pin_gradient[j];
                wx += static_cast<double>(g.x);
                wy += static_cast<double>(g.y);
            }
            if (a.rudy_gradient != nullptr) {
                for (int j = begin; j < end; ++j) {
                    const double2 g = a.rudy_gradient[j];
                    rx_rudy += g.x;
                    ry_rudy += g.y;
                }
                v[7] += fabs(rx_rudy) + fabs(ry_rudy);
            }
        }
        const double2 p = a.positions[i];
        if (a.checkpoint_out != nullptr) a.checkpoint_out[i] = p;
        double2 step = make_double2(0.0, 0.0);
        if (a.velocity_base != nullptr) {
            const double2 b = a.velocity_base[i];
            step = make_double2(p.x - b.x, p.y - b.y);
            a.velocity_out[i] = step;
        }
        const double2 e = sampleField(a, p.x, p.y);
        const double q = a.charge[i];
        const double dx = -q * e.x;
        const double dy = -q * e.y;
        v[0] += fabs(wx) + fabs(wy);
        v[1] += fabs(dx) + fabs(dy);
        if (a.precond_base == nullptr) {
            a.wire_out[i] = make_double2(wx, wy);
            a.density_out[i] = make_double2(dx, dy);
            if (a.rudy_out != nullptr) a.rudy_out[i] = make_double2(rx_rudy, ry_rudy);
        } else {
            const double rx = wx + dx * a.penalty + rx_rudy * a.rudy_weight;
            const double ry = wy + dy * a.penalty + ry_rudy * a.rudy_weight;
            const double s = a.precond_base[i] * a.precond_scale;
            const double px = rx * s;
            const double py = ry * s;
            a.raw[i] = make_double2(rx, ry);
            a.pre[i] = make_double2(px, py);
            v[2] += rx * rx + ry * ry;
            v[3] += px * px + py * py;
            if (a.prev_positions != nullptr) {
                const double2 pp = a.prev_positions[i];
                const double2 pg = a.prev_gradient[i];
                const double ax = p.x - pp.x, ay = p.y - pp.y;
                const double gx = px - pg.x, gy = py - pg.y;
                v[4] += ax * ax + ay * ay;
                v[5] += gx * gx + gy * gy;
            }
            if (a.velocity != nullptr) {
                const double2 vel = a.velocity_base != nullptr ? step : a.velocity[i];
                v[6] += vel.x * px + vel.y * py;
            }
        }
    }
    const bool is_max[8] = {false, false, false, false, false, false, false, false};
    blockReduce<8>(v, is_max);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a.partials[k * grid + block] = v[k];
    }
    if (a.group_counters != nullptr) {
        const int state = reduceGroups<8>(a.partials, a.group_partials, a.group_counters, is_max,
                                          static_cast<unsigned>(block), static_cast<unsigned>(grid));
        // The block that folded the last group: every partial of the evaluation is in
        // place (the gather runs last), so it reduces and publishes them itself.
        if (state == 2 && reduce != nullptr) reduceAllSources(*reduce);
    }
}

__global__ void __launch_bounds__(kThreads) gatherKernel(GatherArgs a, ReduceArgs reduce, int with_reduce) {
    releaseNext();
    waitForPrior();
    gatherBlock(a, with_reduce ? &reduce : nullptr, static_cast<int>(blockIdx.x), static_cast<int>(gridDim.x));
}

__global__ void __launch_bounds__(kThreads) gatherBatchKernel(const GatherArgs* args, const ReduceArgs* const* reduces,
                                                              const int* offsets, int count) {
    releaseNext();
    waitForPrior();
    const int3 slot = batchSlot(offsets, count, static_cast<int>(blockIdx.x));
    const GatherArgs a = args[slot.x];
    gatherBlock(a, reduces != nullptr ? reduces[slot.x] : nullptr, slot.y, slot.z);
}

// The scalar reduction as its own kernel: every partial of every source is
// first staged in shared memory with all loads in flight together (eight per
// thread at a time), then warp w sums sources w, w + 32, ... from shared memory,
// lane l taking rows l, l + 32, ... in order and a fixed shuffle tree.
__device__ __forceinline__ void reduceBlock(const ReduceArgs& a) {
    extern __shared__ double staged[];
    const int total = a.offsets[a.source_count];
    if (total > a.staged_capacity) {
        reduceAllSources(a);
        return;
    }
    // The source table in shared memory: lanes look up different sources at once,
    // which the parameter bank would serialise.
    __shared__ const double* base_of[kScalarCount];
    __shared__ int stride_of[kScalarCount];
    __shared__ int offset_of[kScalarCount + 1];
    if (threadIdx.x < a.source_count) {
        const ReduceSource src = a.sources[threadIdx.x];
        base_of[threadIdx.x] = src.partials + src.column;
        stride_of[threadIdx.x] = src.stride;
    }
    if (threadIdx.x <= a.source_count) offset_of[threadIdx.x] = a.offsets[threadIdx.x];
    __syncthreads();
    constexpr int kBatch = 8;
    int s = 0;  // the source of element e; e only grows, so the search resumes where it stopped
    for (int base = threadIdx.x; base < total; base += kBatch * kReduceThreads) {
        double x[kBatch];
#pragma unroll
        for (int j = 0; j < kBatch; ++j) {
            const int e = base + j * kReduceThreads;
            x[j] = 0.0;
            if (e < total) {
                while (e >= offset_of[s + 1]) ++s;
                x[j] = __ldcg(base_of[s] + static_cast<size_t>(e - offset_of[s]) * stride_of[s]);
            }
        }
#pragma unroll
        for (int j = 0; j < kBatch; ++j) {
            const int e = base + j * kReduceThreads;
            if (e < total) staged[e] = x[j];
        }
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    for (int s = threadIdx.x >> 5; s < a.source_count; s += kReduceThreads / 32) {
        const ReduceSource& src = a.sources[s];
        const int first = offset_of[s];
        double value = src.is_max ? -1.0e308 : 0.0;
        for (int row = lane; row < src.rows; row += 32) {
            const double y = staged[first + row];
            value = src.is_max ? fmax(value, y) : value + y;
        }
        value = src.is_max ? warpMax(value) : warpSum(value);
        if (lane == 0) {
            const double result = src.rows > 0 ? value : 0.0;
            a.scalars[src.target] = result;
            if (a.host_slots != nullptr) publishScalar(a.host_slots, src.target, result, a.sequence);
        }
    }
    finishReduce(a);
}

__global__ void __launch_bounds__(kReduceThreads) reduceKernel(ReduceArgs a) {
    releaseNext();
    waitForPrior();
    reduceBlock(a);
}

// One block per instance, each with the shared memory of the largest staging.
__global__ void __launch_bounds__(kReduceThreads) reduceBatchKernel(const ReduceArgs* args) {
    releaseNext();
    waitForPrior();
    reduceBlock(args[blockIdx.x]);
}

void configureReduce() {
    constexpr int kMaxDevices = 64;
    static std::once_flag once[kMaxDevices];
    static cudaError_t attribute[kMaxDevices] = {};
    int device = 0;
    checkCuda(cudaGetDevice(&device), "Query the current device");
    require(device >= 0 && device < kMaxDevices, "Device index out of range.");
    std::call_once(once[device], [device] {
        attribute[device] = cudaFuncSetAttribute(reduceKernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 kReduceStaged * static_cast<int>(sizeof(double)));
        if (attribute[device] == cudaSuccess) {
            attribute[device] = cudaFuncSetAttribute(reduceBatchKernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                     kReduceStaged * static_cast<int>(sizeof(double)));
        }
    });
    checkCuda(attribute[device], "Configure the scalar reduction");
}

}  // namespace

int gatherBlocks(int particle_count) {
    int per_sm = 0, sms = 0, device = 0;
    checkCuda(cudaGetDevice(&device), "Query the current device");
    checkCuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "Query the SM count");
    checkCuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gatherKernel, kThreads, 0), "Gather occupancy");
    return std::max(1, std::min(ceilDiv(std::max(1, particle_count), kThreads), std::max(1, per_sm) * sms));
}

void launchGather(const GatherArgs& args, const ReduceArgs* reduce, int blocks, cudaStream_t stream) {
    if (blocks <= 0) return;
    require(reduce == nullptr || args.group_counters != nullptr, "A gather that reduces needs its group counters.");
    const ReduceArgs empty{};
    launchChained("Launch the field gather", gatherKernel, dim3(blocks), dim3(kThreads), 0, stream, args,
                  reduce != nullptr ? *reduce : empty, reduce != nullptr ? 1 : 0);
}

void launchReduce(const ReduceArgs& args, cudaStream_t stream) {
    if (args.source_count <= 0) return;
    configureReduce();
    const int total = args.offsets[args.source_count];
    const size_t smem = total <= args.staged_capacity ? static_cast<size_t>(total) * sizeof(double) : 0;
    launchChained("Launch the scalar reduction", reduceKernel, dim3(1), dim3(kReduceThreads), smem, stream, args);
}

void launchGatherBatch(const GatherArgs* args, const ReduceArgs* const* reduces, const int* offsets, int count,
                       int blocks, cudaStream_t stream) {
    if (blocks <= 0 || count <= 0) return;
    launchChained("Launch the batched field gather", gatherBatchKernel, dim3(blocks), dim3(kThreads), 0, stream, args,
                  reduces, offsets, count);
}

void launchReduceBatch(const ReduceArgs* args, int count, int staged_doubles, cudaStream_t stream) {
    if (count <= 0) return;
    configureReduce();
    const size_t smem = static_cast<size_t>(std::max(0, std::min(staged_doubles, kReduceStaged))) * sizeof(double);
    launchChained("Launch the batched scalar reduction", reduceBatchKernel, dim3(count), dim3(kReduceThreads), smem,
                  stream, args);
}

}  // namespace mpgp
