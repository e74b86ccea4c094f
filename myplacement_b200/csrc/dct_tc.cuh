// tcgen05 split-precision contractions (dct_tc.cu): operands, tasks, launchers.
#pragma once

#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <vector>

namespace mpgp {

// Operands are stored as two fp16 planes of a power-of-two scaled value:
// x * 2^-e = hi + 2^-11 lo, |x * 2^-e| <= 2^kPlaneTop, hi = fp16(x * 2^-e),
// lo = fp16((x * 2^-e - hi) * 2^11).
constexpr int kSplit = 2;
constexpr int kPlaneTop = 14;  // log2 of the largest scaled magnitude (fp16 max is 65504)
constexpr int kTileM = 128;    // UMMA M = TMEM lanes
constexpr int kTileN = 64;     // UMMA N = accumulator columns per CTA
constexpr int kBlockK = 64;    // fp16 elements per 128-byte swizzled row
constexpr int kStages = 3;
constexpr int kMaxSplit = 2;   // largest K split (cluster size)
constexpr int kMaxKbExponents = 32;  // K-blocks of a contraction whose A carries one exponent per K-block

// A row-major matrix stored as kSplit fp16 planes; ld is a multiple of kBlockK
// and the padding columns are zero.
struct SplitMatrix {
    __half* data = nullptr;
    int rows = 0;
    int cols = 0;
    int ld = 0;
    [[nodiscard]] size_t plane() const { return static_cast<size_t>(rows) * ld; }
    [[nodiscard]] size_t elements() const { return static_cast<size_t>(kSplit) * plane(); }
};

inline int paddedLd(int cols) { return ((cols + kBlockK - 1) / kBlockK) * kBlockK; }

enum TcMode : int {
    kTcSplit = 0,            // C -> split planes, row-major
    kTcSplitTransposed = 1,  // C^T -> split planes
    kTcSpectral = 2,         // phi = C .* scale -> split planes (row-major and transposed) + Parseval energy
    kTcField = 3,            // C -> FP32 (strided)
};

// Device-resident scale bookkeeping of one field solve.  Magnitudes are the bit
// patterns of non-negative floats (ordered like the floats, so atomicMax works).
struct TcScales {
    unsigned max_source;  // max |S|            (split kernel; cleared by the spectral contraction)
    unsigned max_x;       // max |S Cx^T|       (first contraction; cleared by the split kernel)
    unsigned max_phi;     // max |phi_hat|      (spectral contraction; cleared by the split kernel)
    int exp_x;            // plane exponents written by the producing contraction
    int exp_phi;
    int exp_t;
    int exp_u;
    int exp_basis[8];     // fixed exponents of the basis operands
};

// C (m x n) = A (m x k) * B (n x k)^T with A and B K-major split operands.
// A value of C is sum * 2^(exp_a + exp_b [+ row_exp_a[row]]).
struct alignas(64) TcTask {
    CUtensorMap map_a;
    CUtensorMap map_b;
    int m, n, k;
    int mode;
    int constant_operand;  // 1: A, 2: B is a fixed basis matrix (loaded before the dependency wait); 0: none
    const int* exp_a;      // exponent of A, or null when row_exp_a or kb_exp_a is given
    const int* row_exp_a;  // per-row exponents of A
    const int* kb_exp_a;   // exponents of A per K-block (at most kMaxKbExponents), or null
    const int* exp_b;
    // Output planes: exponent = exponent_of(ref_max * gain) - kPlaneTop, published
    // in out_exp by block 0; the actual max |C| is folded into out_max.
    const unsigned* ref_max;
    float gain;
    int* out_exp;
    unsigned* out_max;
    unsigned* clear;  // block 0 zeroes this magnitude (chain bookkeeping), or null
    __half* out;
    int out_ld;
    size_t out_plane;
    __half* out_t;
    int out_t_ld;
    size_t out_t_plane;
    float* out_f;
    int out_f_ld;
    int out_f_step;
    const float* scale;
    const float* weight_r;
    const float* weight_c;

    double* energy_partials;  // one per CTA of the launch (tcBlocks)
};

// One launch: up to two independent tasks (grid.y), each output tile computed by
// a cluster of `ksplit` CTAs that split its K range (tcPlan chooses ksplit).
struct alignas(64) TcBatch {
    TcTask task[2];
    int* error_flag;
    int ksplit;
    // Failure-detection probe (0 = off): every CTA first waits, for at most this many
    // polls, on an mbarrier that nothing completes, raises error_flag when the wait
    // runs out and returns before it issues any copy or allocates tensor memory.
    long long stall_polls;
};

// One cluster's work in a batched launch: output tile `tile` of task `task` of
// `batch` (a TcBatch in device memory, whose tensor maps the TMA reads there).
struct TcItem {
    const TcBatch* batch;
    int task;
    int tile;
};
// Output tiles of task i of a batch.
int taskTiles(const TcBatch& batch, int task);
// Launches `count` items (clusters of `ksplit` CTAs) from device memory.
void launchTcGemmBatch(const TcItem* items, int count, int ksplit, cudaStream_t stream);

void makeOperandMap(CUtensorMap* map, const SplitMatrix& m, int box_rows);
// Chooses the K split of a batch: the tuned split of its contracted length when
// one is set and its clusters all fit on the GPU at once, else the largest cluster
// size whose clusters all fit.  Call after the tasks are filled in.
void tcPlan(TcBatch& batch, int task_count);
// The tuned splits (contracted length -> split), compiled in from tuned_splits.inc;
// set replaces the whole table (engines planned afterwards use it).
void setTunedSplits(const int* sizes, const int* splits, int count);
// Copies up to `capacity` entries out; returns the table's size.
int tunedSplits(int* sizes, int* splits, int capacity);
// CTAs of one task row of the launch (the count of energy partials a spectral task writes).
int tcBlocks(const TcBatch& batch, int task_count);
void launchTcGemm(const TcBatch& batch, int task_count, cudaStream_t stream);
// Host split of FP64 values into the planes of x * 2^-exponent; returns the exponent.
int splitHost(const std::vector<double>& values, int rows, int cols, int ld, std::vector<__half>& planes);

// The six basis operands of the field solve, built on the device (FP64 values,
// split into planes with one exponent per matrix):
//   0 cx[k][c]   = 2 cos(pi k (2c+1) / 2nx)                 DCT-II along x
//   1 cy[l][r]   = 2 cos(pi l (2r+1) / 2ny)                 DCT-II along y
//   2 dy[r][l]   = 2 cos(pi l (2r+1) / 2ny), 1 for l = 0    DCT-III along y
//   3 dxc[c][k]  = 2 cos(pi k (2c+1) / 2nx), 1 for k = 0    DCT-III along x
//   4 sxwt[c][k] = (pi k / width) 2 sin(pi k (2c+1) / 2nx)  DST-III along x times the wave number
//   5 syw[r][l]  = (pi l / height) 2 sin(pi l (2r+1) / 2ny) DST-III along y times the wave number
// The planes go to out[t]; exponents[t] and max_row_l1[t] (the largest row sum
// of |values|, which bounds |A x| / max |x|) come back to the host.
constexpr int kBasisCount = 6;
void buildBasisPlanes(int nx, int ny, double width, double height, const SplitMatrix (&out)[kBasisCount],
                      unsigned long long* scratch, int (&exponents)[kBasisCount],
                      double (&max_row_l1)[kBasisCount], cudaStream_t stream);
// Splits the FP32 source S with one exponent per row (row_exp), folds max |S| into
// scales->max_source and clears the magnitudes the forward contractions fold into.
void launchSplitSource(const float* source, const SplitMatrix& out, int cols, int* row_exp, TcScales* scales,
                       cudaStream_t stream);

}  // namespace mpgp
