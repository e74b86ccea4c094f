/*
 * Test-oracle infrastructure: loaded only by tests/, __graft_entry__.smoke()
 * and bench.py's CPU baseline legs; never linked into the product.
 *
 * Fixed-point restatement of the course-ePlace dynamic density deposit:
 * DensityMap::addRectangle (src/metrics/Metrics.cpp:74-99) applied per particle
 * by depositDynamicDensity (src/placement/GlobalPlacementSupport.cpp:32-40),
 * i.e. the reference CUDA depositParticlesKernel
 * (src/placement/cuda/CudaPlacementBackend.cu:339-375).
 *
 * The arithmetic below is the specification the device scatter reproduces bit
 * for bit (compile with -ffp-contract=off; no fused multiply-add anywhere):
 *
 *   per particle, FP64:
 *     l = max(x0, cx - 0.5 w), r = min(x1, cx + 0.5 w)   (same for y)
 *     skip when max(0, r - l) * max(0, t - b) <= 1e-9     (Rect::area <= kEpsilon)
 *     gl = (l - x0) / bw, gr = (r - x0) / bw               (bin units)
 *     c0 = clamp(floor(gl), 0, nx - 1), c1 = clamp(ceil(gr) - 1, 0, nx - 1)
 *     fl = (float)(gl - c0), fr = (float)(gr - c0)         (same for rows)
 *   per covered bin (j = c - c0, i = r - r0), FP32:
 *     ox = max(0, min(fr, j + 1) - max(fl, j)), oy likewise
 *     q  = llrint(ox * oy * 2^32)                          (round to nearest even)
 *   layer[bin] += q  (int64; bin area units of 2^-32).
 *
 * Integer sums are independent of the order in which particles are visited,
 * so any parallel schedule that computes the same q per (particle, bin) gives
 * an identical map.
 */
#include <math.h>
#include <stdint.h>

#define MPGP_FIXED_ONE 4294967296.0f /* 2^32 */

static double clamp_index(double value, int upper) {
    if (value < 0.0) return 0.0;
    if (value > (double)upper) return (double)upper;
    return value;
}

/* Deposits one particle into `layer` (nx*ny int64, row-major). */
static void deposit(double cx, double cy, double w, double h, double x0, double y0, double x1, double y1,
                    int nx, int ny, double bw, double bh, int64_t* layer) {
    const double l = fmax(x0, cx - w * 0.5);
    const double r = fmin(x1, cx + w * 0.5);
    const double b = fmax(y0, cy - h * 0.5);
    const double t = fmin(y1, cy + h * 0.5);
    if (fmax(0.0, r - l) * fmax(0.0, t - b) <= 1e-9) return;
    const double gl = (l - x0) / bw;
    const double gr = (r - x0) / bw;
    const double gb = (b - y0) / bh;
    const double gt = (t - y0) / bh;
    const int c0 = (int)clamp_index(floor(gl), nx - 1);
    const int c1 = (int)clamp_index(ceil(gr) - 1.0, nx - 1);
    const int r0 = (int)clamp_index(floor(gb), ny - 1);
    const int r1 = (int)clamp_index(ceil(gt) - 1.0, ny - 1);
    const float fl = (float)(gl - (double)c0);
    const float fr = (float)(gr - (double)c0);
    const float fb = (float)(gb - (double)r0);
    const float ft = (float)(gt - (double)r0);
    for (int row = r0; row <= r1; ++row) {
        const float i = (float)(row - r0);
        const float oy = fmaxf(0.0f, fminf(ft, i + 1.0f) - fmaxf(fb, i));
        for (int column = c0; column <= c1; ++column) {
            const float j = (float)(column - c0);
            const float ox = fmaxf(0.0f, fminf(fr, j + 1.0f) - fmaxf(fl, j));
            const float area = ox * oy;
            const int64_t q = (int64_t)llrintf(area * MPGP_FIXED_ONE);
            if (q != 0) layer[(int64_t)row * nx + column] += q;
        }
    }
}

/*
 * Deposits `count` particles into the movable / macro / filler layers
 * (layer codes 0 / 1 / 2).  Layers are accumulated into (callers zero them).
 * Returns 0, or -1 on invalid arguments.
 */
int oracle_deposit(int64_t count, const double* x, const double* y, const double* width, const double* height,
                   const int32_t* layer_code, double x0, double y0, double x1, double y1, int32_t nx, int32_t ny,
                   int64_t* movable, int64_t* macro, int64_t* filler) {
    if (nx <= 0 || ny <= 0 || !(x1 > x0) || !(y1 > y0)) return -1;
    const double bw = (x1 - x0) / (double)nx;
    const double bh = (y1 - y0) / (double)ny;
    for (int64_t p = 0; p < count; ++p) {
        int64_t* target = layer_code[p] == 0 ? movable : (layer_code[p] == 1 ? macro : filler);
        deposit(x[p], y[p], width[p], height[p], x0, y0, x1, y1, nx, ny, bw, bh, target);
    }
    return 0;
}

/* Deposits arbitrary rectangles (llx, lly, urx, ury) into one layer: the
 * clipped-rectangle edge cases of Metrics.cpp:74-99. */
int oracle_deposit_rects(int64_t count, const double* rects, double x0, double y0, double x1, double y1, int32_t nx,
                         int32_t ny, int64_t* layer) {
    if (nx <= 0 || ny <= 0 || !(x1 > x0) || !(y1 > y0)) return -1;
    const double bw = (x1 - x0) / (double)nx;
    const double bh = (y1 - y0) / (double)ny;
    for (int64_t p = 0; p < count; ++p) {
        const double* rect = rects + 4 * p;
        const double w = rect[2] - rect[0];
        const double h = rect[3] - rect[1];
        deposit(rect[0] + w * 0.5, rect[1] + h * 0.5, w, h, x0, y0, x1, y1, nx, ny, bw, bh, layer);
    }
    return 0;
}
