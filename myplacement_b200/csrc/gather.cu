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

__global__ void __launch_bounds__(kThreads) gatherKernel(GatherArgs a) {
    releaseNext();
    waitForPrior();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (i < a.particle_count) {
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
                v[7] = fabs(rx_rudy) + fabs(ry_rudy);
            }
        }
        const double2 p = a.positions[i];
        const double2 e = sampleField(a, p.x, p.y);
        const double q = a.charge[i];
        const double dx = -q * e.x;
        const double dy = -q * e.y;
        v[0] = fabs(wx) + fabs(wy);
        v[1] = fabs(dx) + fabs(dy);
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
            v[2] = rx * rx + ry * ry;
            v[3] = px * px + py * py;
            if (a.prev_positions != nullptr) {
                const double2 pp = a.prev_positions[i];
                const double2 pg = a.prev_gradient[i];
                const double ax = p.x - pp.x, ay = p.y - pp.y;
                const double gx = px - pg.x, gy = py - pg.y;
                v[4] = ax * ax + ay * ay;
                v[5] = gx * gx + gy * gy;
            }
            if (a.velocity != nullptr) {
                const double2 vel = a.velocity[i];
                v[6] = vel.x * px + vel.y * py;
            }
        }
    }
    const bool is_max[8] = {false, false, false, false, false, false, false, false};
    blockReduce<8>(v, is_max);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a.partials[8 * blockIdx.x + k] = v[k];
    }
}

__global__ void __launch_bounds__(kThreads) reduceKernel(ReduceArgs a) {
    releaseNext();
    waitForPrior();
    const int s = blockIdx.x;
    if (s >= a.source_count) {
        return;
    }
    const ReduceSource src = a.sources[s];
    double value = src.is_max ? -1.0e308 : 0.0;
    for (int row = threadIdx.x; row < src.rows; row += blockDim.x) {
        const double x = src.partials[static_cast<size_t>(row) * src.stride + src.column];
        value = src.is_max ? fmax(value, x) : value + x;
    }
    double values[1] = {value};
    const bool is_max[1] = {src.is_max != 0};
    blockReduce<1>(values, is_max);
    if (threadIdx.x == 0) {
        a.scalars[src.target] = src.rows > 0 ? values[0] : 0.0;
        if (s == 0 && a.totals != nullptr) {
            a.totals[0] = 0ULL;
            a.totals[1] = 0ULL;
            a.totals[2] = 0ULL;
        }
    }
}

}  // namespace

void launchGather(const GatherArgs& args, int blocks, cudaStream_t stream) {
    if (blocks <= 0) return;
    launchChained("Launch the field gather", gatherKernel, dim3(blocks), dim3(kThreads), 0, stream, args);
}

void launchReduce(const ReduceArgs& args, cudaStream_t stream) {
    if (args.source_count <= 0) return;
    launchChained("Launch the scalar reduction", reduceKernel, dim3(args.source_count), dim3(kThreads), 0, stream,
                  args);
}

}  // namespace mpgp
