// Banded field solve (field_tc.cu): per band of 64 spectral columns, one cluster
// runs the forward DCT along x and y, the spectral divide with its Parseval
// energy and, for a gradient, the inverse transforms along y; the inverse along x
// is one ordinary contraction launch (dct_tc.cu) over the bands' outputs.
#pragma once

#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "dct_tc.cuh"

namespace mpgp {

// The tallest grid the banded solve takes: its clusters hold every row of the band.
constexpr int kFieldMaxRows = 512;
// The widest: the inverse along x carries one exponent per band (kMaxKbExponents).
constexpr int kFieldMaxColumns = kBlockK * kMaxKbExponents;
// By default only grids taller than this take the banded solve: on smaller grids its
// clusters hold whole SMs for little work, and batched rounds of many small
// placements ran faster with the staged solve.
constexpr int kFieldBandedMinRows = 256;

struct FieldShape {
    int m_blocks = 0;  // 128-row blocks of the y range
    int shares = 0;    // CTAs per band and row block
    int share_n = 0;   // spectral columns per CTA (64 / shares)
    int cluster = 0;   // CTAs per cluster: m_blocks * shares (0: the grid is too tall)
    int bands = 0;     // 64-column bands of the spectral x range
    [[nodiscard]] int blocks() const { return bands * cluster; }
};
// The banded solve's shape for an nx x ny grid (cluster 0 beyond kFieldMaxRows x kFieldMaxColumns).
FieldShape fieldShape(int nx, int ny);

// What a banded launch runs.
enum FieldMode : int {
    kFieldForward = 0,   // passes 0-1: phi_hat (kept in phi_store) and the energy partials
    kFieldGradient = 1,  // passes 0-3: also M1 and M2
    kFieldInverse = 2,   // passes 2-3 only, from the phi_hat the last forward launch kept
};

// One grid's banded solve.  With S the split source (ny x nx), Cx, Cy the DCT-II
// bases, Dy the DCT-III basis and Syw the wave-number-weighted DST-III basis along
// y (dct_tc.cuh), the cluster of band b computes for kx in b:
//   Q = S Cx^T, rho_hat = Cy Q, phi_hat = rho_hat .* scale, the energy partials,
//   and with a gradient M1 = Dy phi_hat and M2 = Syw phi_hat,
// written as split planes with one exponent per band (m1_exp[b], m2_exp[b]).
struct alignas(64) FieldBand {
    CUtensorMap map_s;    // S planes, 128-row boxes
    CUtensorMap map_cx;   // Cx planes, share_n-row boxes
    CUtensorMap map_cy;   // Cy planes, 128-row boxes
    CUtensorMap map_dy;   // Dy planes, 128-row boxes
    CUtensorMap map_syw;  // Syw planes, 128-row boxes
    int nx = 0, ny = 0;
    FieldShape shape;
    const int* row_exp = nullptr;    // per-row exponents of S
    const int* exp_basis = nullptr;  // TcScales::exp_basis
    const float* scale = nullptr;    // spectral scale [ny][nx]
    double* energy_partials = nullptr;  // one per CTA (shape.blocks())
    __half* m1 = nullptr;
    __half* m2 = nullptr;
    int m_ld = 0;
    size_t m_plane = 0;
    int* m1_exp = nullptr;
    int* m2_exp = nullptr;
    // phi_hat^T of the last forward launch, per band and share in the layout the
    // inverse passes read it in (fieldStoreBytes), and per producing CTA its plane
    // exponent and tile maximum ([band][share][row block][4] ints).
    unsigned char* phi_store = nullptr;
    int* phi_records = nullptr;
    float gain_dy = 0.0f;   // bounds |Dy x| <= gain_dy max |x| (row L1 norm with a margin)
    float gain_syw = 0.0f;
    unsigned* clear = nullptr;  // a magnitude block 0 zeroes (chain bookkeeping), or null
    int* error_flag = nullptr;
    // Failure-detection probe, as TcBatch::stall_polls.
    long long stall_polls = 0;
};

// Bytes of FieldBand::phi_store and ints of FieldBand::phi_records for a shape.
size_t fieldStoreBytes(const FieldShape& shape);
size_t fieldRecordInts(const FieldShape& shape);

void launchField(const FieldBand& band, FieldMode mode, cudaStream_t stream);

// One cluster's work in a batched launch: band `band` of the grid `field` (a
// FieldBand in device memory) in mode `mode` (a FieldMode).
struct FieldItem {
    const FieldBand* field;
    int band;
    int mode;
};
// Launches `count` items, all of grids of one shape's cluster size and share
// width (`shape`), from device memory.
void launchFieldBatch(const FieldItem* items, int count, const FieldShape& shape, cudaStream_t stream);

}  // namespace mpgp
