// Dense FP32 contractions for the Neumann DCT/DST field (SIMT CUDA-core path).
//
// The reference solves the field with FFTW r2r plans (ElectrostaticField.cpp:
// 164-182, 205-237) or cuFFT Z2Z emulation (CudaPlacementBackend.cu:407-545,
// 679-742).  Here each 1-D transform is a dense basis matrix and each 2-D
// transform is two contractions, C = A * B, batched two at a time.  The
// spectral divide phi_hat = rho_hat / (4 Nx Ny (kx^2 + ky^2)) and the
// Parseval energy sum are fused into the epilogue of the second forward
// contraction.  This file is the portable FP32 form; dct_tc.cu holds the
// tcgen05 tensor-core form.
#include "common.cuh"
#include "kernels.cuh"

namespace mpgp {
namespace {

constexpr int kTile = 64;
constexpr int kDepth = 16;

struct GemmBatch {
    GemmTask task[2];
    int count;
};

__global__ void __launch_bounds__(256) gemmKernel(GemmBatch batch) {
    const GemmTask& t = batch.task[blockIdx.z];
    const int tiles_n = (t.n + kTile - 1) / kTile;
    const int tiles_m = (t.m + kTile - 1) / kTile;
    const int tile = blockIdx.x;
    if (tile >= tiles_m * tiles_n) return;
    const int m0 = (tile / tiles_n) * kTile;
    const int n0 = (tile % tiles_n) * kTile;
    __shared__ __align__(16) float As[kDepth][kTile];
    __shared__ __align__(16) float Bs[kDepth][kTile];
    const int tid = threadIdx.x;
    const int ty = tid / 16;
    const int tx = tid % 16;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < t.k; k0 += kDepth) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int e = tid + 256 * j;
            const int row = e / kDepth;
            const int col = e % kDepth;
            const int gr = m0 + row;
            const int gc = k0 + col;
            As[col][row] = (gr < t.m && gc < t.k) ? t.a[static_cast<size_t>(gr) * t.lda + gc] : 0.0f;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int e = tid + 256 * j;
            const int row = e / kTile;
            const int col = e % kTile;
            const int gr = k0 + row;
            const int gc = n0 + col;
            Bs[row][col] = (gr < t.k && gc < t.n) ? t.b[static_cast<size_t>(gr) * t.ldb + gc] : 0.0f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kDepth; ++kk) {
            const float4 av = *reinterpret_cast<const float4*>(&As[kk][ty * 4]);
            const float4 bv = *reinterpret_cast<const float4*>(&Bs[kk][tx * 4]);
            const float a4[4] = {av.x, av.y, av.z, av.w};
            const float b4[4] = {bv.x, bv.y, bv.z, bv.w};
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a4[i], b4[j], acc[i][j]);
        }
        __syncthreads();
    }
    double energy = 0.0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int r = m0 + ty * 4 + i;
        if (r >= t.m) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int c = n0 + tx * 4 + j;
            if (c >= t.n) continue;
            float value = acc[i][j];
            if (t.scale != nullptr) {
                const float phi = value * t.scale[static_cast<size_t>(r) * t.n + c];
                energy += static_cast<double>(phi) * static_cast<double>(value) *
                          static_cast<double>(t.weight_r[r]) * static_cast<double>(t.weight_c[c]);
                value = phi;
            }
            t.c[static_cast<size_t>(r) * t.ldc + static_cast<size_t>(c) * t.c_step] = value;
        }
    }
    if (t.energy_partials != nullptr) {
        double values[1] = {energy};
        const bool is_max[1] = {false};
        blockReduce<1>(values, is_max);
        if (threadIdx.x == 0) t.energy_partials[tile] = values[0];
    }
}

}  // namespace

int gemmBlocks(const GemmTask& task) {
    return ((task.m + kTile - 1) / kTile) * ((task.n + kTile - 1) / kTile);
}

void launchGemm(const GemmTask* tasks, int task_count, cudaStream_t stream) {
    GemmBatch batch{};
    int blocks = 0;
    for (int i = 0; i < task_count; ++i) {
        batch.task[i] = tasks[i];
        blocks = blocks > gemmBlocks(tasks[i]) ? blocks : gemmBlocks(tasks[i]);
    }
    batch.count = task_count;
    gemmKernel<<<dim3(blocks, 1, task_count), 256, 0, stream>>>(batch);
}

}  // namespace mpgp
