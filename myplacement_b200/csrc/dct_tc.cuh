// tcgen05 split-precision contractions (dct_tc.cu): operands, tasks, launchers.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <vector>

namespace mpgp {

#ifndef MPGP_SPLIT_PLANES
#define MPGP_SPLIT_PLANES 3
#endif
constexpr int kSplit = MPGP_SPLIT_PLANES;  // bf16 planes per operand (x = hi + mid + lo)
constexpr int kTileM = 128;  // UMMA M = TMEM lanes
constexpr int kTileN = 64;   // UMMA N = accumulator columns per CTA
constexpr int kBlockK = 64;  // bf16 elements per 128-byte swizzled row
constexpr int kStages = 3;

// A row-major matrix stored as kSplit bf16 planes; ld is a multiple of kBlockK
// and the padding columns are zero.
struct SplitMatrix {
    __nv_bfloat16* data = nullptr;
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

// C (m x n) = A (m x k) * B (n x k)^T with A and B K-major split operands.
struct alignas(64) TcTask {
    CUtensorMap map_a;
    CUtensorMap map_b;
    int m, n, k;
    int mode;
    __nv_bfloat16* out;
    int out_ld;
    size_t out_plane;
    __nv_bfloat16* out_t;
    int out_t_ld;
    size_t out_t_plane;
    float* out_f;
    int out_f_ld;
    int out_f_step;
    const float* scale;
    const float* weight_r;
    const float* weight_c;
    double* energy_partials;
};

struct alignas(64) TcBatch {
    TcTask task[2];
    int* error_flag;
    unsigned long long* trace;  // development timeline of CTA (0, 0), or null
};

void makeOperandMap(CUtensorMap* map, const SplitMatrix& m, int box_rows);
void launchTcGemm(const TcBatch& batch, int task_count, cudaStream_t stream);
int tcTiles(int m, int n);
int tcSmemBytes();
void splitHost(const std::vector<double>& values, int rows, int cols, int ld, std::vector<__nv_bfloat16>& planes);
void launchSplitSource(const float* source, const SplitMatrix& out, int cols, cudaStream_t stream);

}  // namespace mpgp
