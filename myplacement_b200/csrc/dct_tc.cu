// Split-precision tcgen05 contractions for the Neumann DCT/DST field (sm_100a).
//
// The field solve of ElectrostaticField::solveNeumann (ElectrostaticField.cpp:
// 205-237) is six dense contractions C = A * B^T (see engine.cu runDct).  Each
// operand is stored as kSplit bf16 planes whose sum carries ~8 * kSplit bits of
// the FP32 value (x = hi + mid + lo); a contraction accumulates the cross
// products whose combined order is below kSplit (hh, hm, mh, hl, lh, mm for
// three planes), smallest first.
//
// Per CTA: one 128 x kTileN output tile and six warps.
//   warp 0 lane 0  TMA producer: K-blocks of 64 elements of every plane of A
//                  and B into a kStages-deep shared-memory ring (3-D tensor
//                  maps: K, rows, plane; 128-byte swizzle; zero fill past edges).
//   warp 1 lane 0  tcgen05.mma issuer: the products of one K-block into one of
//                  two TMEM accumulators (double-buffered), restarted every
//                  K-block; tcgen05.commit releases the smem stage and
//                  publishes the partial.
//   warps 2-5      read each partial with tcgen05.ld (warp w owns TMEM lanes
//                  32 * (w % 4) .. +31, i.e. tile rows) and sum the partials in
//                  FP64 registers, which keeps the accumulation error of long K
//                  chains at FP64 level; then the fused epilogue: re-split into
//                  bf16 planes (plain or transposed), or the spectral divide with
//                  the Parseval energy partials, or FP32 field stores.
// Every mbarrier wait is bounded: on a timeout the CTA raises the error flag,
// drains the copies it issued, frees its TMEM and returns.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "common.cuh"
#include "dct_tc.cuh"

namespace mpgp {
namespace {

constexpr int kTcThreads = 192;
constexpr int kStageBytes = kSplit * (kTileM + kTileN) * kBlockK * 2;
constexpr int kSmemBytes = kStages * kStageBytes + 1024 /* alignment slack */ + 256 /* barriers */;
constexpr uint32_t kTmemColumns = 2 * kTileN;  // two partial accumulators
constexpr long kSpinLimit = 1L << 22;
constexpr int kTilePitch = kTileN + 1;  // floats per staged row (odd pitch: no bank conflicts)
static_assert(kTileM * kTilePitch * 4 <= kStages * kStageBytes, "the staged tile must fit in the ring");

__device__ __forceinline__ unsigned long long nowNs() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}
#define TC_TRACE(slot) \
    do { if (batch.trace != nullptr && blockIdx.x == 0 && blockIdx.y == 0) batch.trace[(slot)] = nowNs(); } while (0)

__device__ __forceinline__ uint32_t smemAddress(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbarInit(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbarExpectTx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbarArrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbarTryWait(uint32_t bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done != 0;
}

// Bounded wait; false (and the error flag raised) after kSpinLimit polls.
__device__ __forceinline__ bool mbarWait(uint32_t bar, uint32_t parity, int* error_flag) {
    for (long i = 0; i < kSpinLimit; ++i) {
        if (mbarTryWait(bar, parity)) return true;
    }
    if (error_flag != nullptr) atomicExch(error_flag, 1);
    return false;
}

__device__ __forceinline__ void tmaLoad3d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int x, int y, int z) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y), "r"(z)
        : "memory");
}

// UMMA shared-memory descriptor: K-major, 128-byte swizzle, 8-row groups 1024 B apart.
__device__ __forceinline__ uint64_t smemDescriptor(uint32_t address) {
    return static_cast<uint64_t>((address >> 4) & 0x3FFFu) | (1ull << 16) | (64ull << 32) | (1ull << 46) |
           (2ull << 61);
}

// Instruction descriptor: BF16 x BF16 -> F32, both K-major, M = 128, N = kTileN.
constexpr uint32_t kInstrDescriptor =
    (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(kTileN >> 3) << 17) |
    (static_cast<uint32_t>(kTileM >> 4) << 24);

__device__ __forceinline__ void ummaF16(uint32_t tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem), "l"(a), "l"(b), "r"(kInstrDescriptor), "r"(accumulate));
}

__device__ __forceinline__ void ummaCommit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tmemLoad16(uint32_t address, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(address));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// x = sum of kSplit bf16 pieces, largest first.
template <typename T>
__device__ __forceinline__ void splitValue(T x, __nv_bfloat16 (&piece)[kSplit]) {
    T rest = x;
#pragma unroll
    for (int p = 0; p < kSplit; ++p) {
        piece[p] = __float2bfloat16_rn(static_cast<float>(rest));
        rest = rest - static_cast<T>(__bfloat162float(piece[p]));
    }
}

// Cross products of planes kept by the split (a-plane, b-plane), smallest order first.
__device__ __forceinline__ void planePair(int product, int& pa, int& pb) {
    if (kSplit == 2) {
        const int a[3] = {1, 0, 0};
        const int b[3] = {0, 1, 0};
        pa = a[product];
        pb = b[product];
    } else {
        const int a[6] = {2, 0, 1, 1, 0, 0};
        const int b[6] = {0, 2, 1, 0, 1, 0};
        pa = a[product];
        pb = b[product];
    }
}
constexpr int kProducts = kSplit == 2 ? 3 : 6;

__global__ void __launch_bounds__(kTcThreads, 1) tcGemmKernel(const __grid_constant__ TcBatch batch) {
    const TcTask& t = batch.task[blockIdx.y];
    const int tiles_n = (t.n + kTileN - 1) / kTileN;
    const int tiles_m = (t.m + kTileM - 1) / kTileM;
    if (static_cast<int>(blockIdx.x) >= tiles_m * tiles_n) return;
    const int m0 = (blockIdx.x / tiles_n) * kTileM;
    const int n0 = (blockIdx.x % tiles_n) * kTileN;
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    if (threadIdx.x == 0) TC_TRACE(51);

    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    uint64_t* barriers = reinterpret_cast<uint64_t*>(smem + kStages * kStageBytes);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(barriers + 2 * kStages + 4);
    volatile int* failed = reinterpret_cast<volatile int*>(tmem_slot + 1);
    const uint32_t full0 = smemAddress(barriers);
    const uint32_t empty0 = smemAddress(barriers + kStages);
    const uint32_t partial0 = smemAddress(barriers + 2 * kStages);
    const uint32_t consumed0 = smemAddress(barriers + 2 * kStages + 2);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smemAddress(tmem_slot)),
                     "r"(kTmemColumns));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 32) {
        *failed = 0;
        for (int s = 0; s < kStages; ++s) {
            mbarInit(full0 + 8 * s, 1);
            mbarInit(empty0 + 8 * s, 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbarInit(partial0 + 8 * b, 1);
            mbarInit(consumed0 + 8 * b, 4);  // one arrival per epilogue warp
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    const int k_blocks = (t.k + kBlockK - 1) / kBlockK;
    double energy = 0.0;
    if (threadIdx.x == 0) TC_TRACE(0);

    if (warp == 0) {
        if (lane == 0) {
            // TMA producer.
            bool ok = true;
            int issued = 0;
            for (int kb = 0; kb < k_blocks && ok; ++kb) {
                const int s = kb % kStages;
                if (kb >= kStages) ok = mbarWait(empty0 + 8 * s, ((kb / kStages) - 1) & 1, batch.error_flag);
                if (!ok) break;
                unsigned char* stage = smem + s * kStageBytes;
                if (kb < 16) TC_TRACE(1 + kb);
                mbarExpectTx(full0 + 8 * s, kStageBytes);
                for (int p = 0; p < kSplit; ++p) {
                    tmaLoad3d(smemAddress(stage + p * kTileM * kBlockK * 2), &t.map_a, full0 + 8 * s, kb * kBlockK,
                              m0, p);
                    tmaLoad3d(smemAddress(stage + kSplit * kTileM * kBlockK * 2 + p * kTileN * kBlockK * 2),
                              &t.map_b, full0 + 8 * s, kb * kBlockK, n0, p);
                }
                issued = kb + 1;
            }
            if (!ok) {
                // Drain: wait (bounded) for every issued stage so no copy lands after exit.
                for (int kb = max(0, issued - kStages); kb < issued; ++kb) {
                    mbarWait(full0 + 8 * (kb % kStages), (kb / kStages) & 1, nullptr);
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // tcgen05.mma issuer: K-block kb accumulates into buffer kb % 2 from zero.
            for (int kb = 0; kb < k_blocks; ++kb) {
                const int s = kb % kStages;
                const int buffer = kb & 1;
                if (kb >= 2 && !mbarWait(consumed0 + 8 * buffer, ((kb >> 1) - 1) & 1, batch.error_flag)) break;
                if (!mbarWait(full0 + 8 * s, (kb / kStages) & 1, batch.error_flag)) break;
                if (kb < 16) TC_TRACE(17 + kb);
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t stage = smemAddress(smem + s * kStageBytes);
                const uint32_t a_base = stage;
                const uint32_t b_base = stage + kSplit * kTileM * kBlockK * 2;
                const uint32_t accumulator = tmem + static_cast<uint32_t>(buffer * kTileN);
#pragma unroll
                for (int kk = 0; kk < kBlockK / 16; ++kk) {
#pragma unroll
                    for (int product = 0; product < kProducts; ++product) {
                        int pa, pb;
                        planePair(product, pa, pb);
                        const uint64_t da = smemDescriptor(a_base + pa * kTileM * kBlockK * 2 + kk * 32);
                        const uint64_t db = smemDescriptor(b_base + pb * kTileN * kBlockK * 2 + kk * 32);
                        ummaF16(accumulator, da, db, (kk > 0 || product > 0) ? 1u : 0u);
                    }
                }
                ummaCommit(empty0 + 8 * s);
                ummaCommit(partial0 + 8 * buffer);
            }
        }
    } else {
        // Epilogue warps: FP64 sum of the K-block partials, then the fused output.
        const int quarter = warp & 3;
        const int row = m0 + quarter * 32 + lane;
        const uint32_t lane_base = tmem + (static_cast<uint32_t>(quarter * 32) << 16);
        double acc[kTileN];
#pragma unroll
        for (int j = 0; j < kTileN; ++j) acc[j] = 0.0;
        bool ok = true;
        for (int kb = 0; kb < k_blocks; ++kb) {
            const int buffer = kb & 1;
            ok = __all_sync(0xffffffffu, mbarWait(partial0 + 8 * buffer, (kb >> 1) & 1, batch.error_flag) ? 1 : 0) != 0;
            if (!ok) break;
            if (warp == 2 && lane == 0 && kb < 16) TC_TRACE(33 + kb);
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int c0 = 0; c0 < kTileN; c0 += 16) {
                float v[16];
                tmemLoad16(lane_base + static_cast<uint32_t>(buffer * kTileN + c0), v);
#pragma unroll
                for (int j = 0; j < 16; ++j) acc[c0 + j] += static_cast<double>(v[j]);
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbarArrive(consumed0 + 8 * buffer);
        }
        // Stage the tile in shared memory (the ring is idle once the last partial has
        // been read).  FP32 keeps 24 bits, as many as the three bf16 output planes hold.
        (void)row;
        float* tile = reinterpret_cast<float*>(smem);
        const int local_row = quarter * 32 + lane;
        if (ok) {
#pragma unroll
            for (int j = 0; j < kTileN; ++j) tile[local_row * kTilePitch + j] = static_cast<float>(acc[j]);
        } else {
            *failed = 1;
        }
    }
    __syncwarp();
    __syncthreads();
    float* tile = reinterpret_cast<float*>(smem);  // [kTileM][kTilePitch], staged by the epilogue warps
    const bool tile_ok = *failed == 0 && k_blocks > 0;
    // Output passes with all six warps, four independent elements per thread; a
    // warp's lanes run along the contiguous dimension of the destination.
    if (tile_ok && t.mode != kTcSplitTransposed) {
        // Row-major pass: lane <-> column, four rows per thread.
        for (int g = threadIdx.x; g < kTileM * kTileN / 4; g += kTcThreads) {
            const int c = g % kTileN;
            const int r0 = (g / kTileN) * 4;
            const int gcol = n0 + c;
            if (gcol >= t.n) continue;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int r = r0 + i;
                const int grow = m0 + r;
                if (grow >= t.m) continue;
                float value = tile[r * kTilePitch + c];
                if (t.mode == kTcSpectral) {
                    const float phi = value * t.scale[static_cast<size_t>(grow) * t.n + gcol];
                    energy += static_cast<double>(phi) * static_cast<double>(value) *
                              static_cast<double>(t.weight_r[grow] * t.weight_c[gcol]);
                    value = phi;
                    tile[r * kTilePitch + c] = phi;
                }
                if (t.mode == kTcField) {
                    t.out_f[static_cast<size_t>(grow) * t.out_f_ld + static_cast<size_t>(gcol) * t.out_f_step] = value;
                    continue;
                }
                __nv_bfloat16 piece[kSplit];
                splitValue(value, piece);
                __nv_bfloat16* out = t.out + static_cast<size_t>(grow) * t.out_ld + gcol;
#pragma unroll
                for (int p = 0; p < kSplit; ++p) out[static_cast<size_t>(p) * t.out_plane] = piece[p];
            }
        }
    }
    if (tile_ok && (t.mode == kTcSplitTransposed || t.mode == kTcSpectral)) {
        if (t.mode == kTcSpectral) __syncthreads();  // the row-major pass rewrote the tile with phi
        // Transposed pass: lane <-> row, four columns per thread.
        for (int g = threadIdx.x; g < kTileM * kTileN / 4; g += kTcThreads) {
            const int r = g % kTileM;
            const int c0 = (g / kTileM) * 4;
            const int grow = m0 + r;
            if (grow >= t.m) continue;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int c = c0 + i;
                const int gcol = n0 + c;
                if (gcol >= t.n) continue;
                __nv_bfloat16 piece[kSplit];
                splitValue(tile[r * kTilePitch + c], piece);
                __nv_bfloat16* out = t.out_t + static_cast<size_t>(gcol) * t.out_t_ld + grow;
#pragma unroll
                for (int p = 0; p < kSplit; ++p) out[static_cast<size_t>(p) * t.out_t_plane] = piece[p];
            }
        }
    }
    if (threadIdx.x == 64) TC_TRACE(49);
    if (t.mode == kTcSpectral && t.energy_partials != nullptr) {
        double values[1] = {energy};
        const bool is_max[1] = {false};
        blockReduce<1>(values, is_max);
        if (threadIdx.x == 0) t.energy_partials[blockIdx.x] = values[0];
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemColumns));
    }
    if (threadIdx.x == 0) TC_TRACE(50);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no -lcuda).
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encoder() {
    static std::once_flag once;
    static EncodeTiled fn = nullptr;
    static cudaError_t status = cudaSuccess;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult query{};
        status = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &query);
        if (status == cudaSuccess && query == cudaDriverEntryPointSuccess) fn = reinterpret_cast<EncodeTiled>(p);
    });
    if (fn == nullptr) fail(MPGP_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable from the CUDA driver.");
    return fn;
}

__global__ void splitSourceKernel(const float* source, int rows, int cols, __nv_bfloat16* out, int ld,
                                  size_t plane) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows * cols) return;
    const int r = i / cols;
    const int c = i % cols;
    __nv_bfloat16 piece[kSplit];
    splitValue(source[i], piece);
    __nv_bfloat16* dst = out + static_cast<size_t>(r) * ld + c;
#pragma unroll
    for (int p = 0; p < kSplit; ++p) dst[static_cast<size_t>(p) * plane] = piece[p];
}

}  // namespace

int tcSmemBytes() { return kSmemBytes; }

void makeOperandMap(CUtensorMap* map, const SplitMatrix& m, int box_rows) {
    require(m.ld % kBlockK == 0 && m.rows > 0 && m.data != nullptr, "Split operand layout is invalid.");
    const cuuint64_t dims[3] = {static_cast<cuuint64_t>(m.ld), static_cast<cuuint64_t>(m.rows),
                                static_cast<cuuint64_t>(kSplit)};
    const cuuint64_t strides[2] = {static_cast<cuuint64_t>(m.ld) * 2,
                                   static_cast<cuuint64_t>(m.ld) * static_cast<cuuint64_t>(m.rows) * 2};
    const cuuint32_t box[3] = {static_cast<cuuint32_t>(kBlockK), static_cast<cuuint32_t>(box_rows), 1};
    const cuuint32_t element_strides[3] = {1, 1, 1};
    const CUresult result =
        encoder()(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, m.data, dims, strides, box, element_strides,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (result != CUDA_SUCCESS) {
        fail(MPGP_ERR_CUDA, "cuTensorMapEncodeTiled failed with status " + std::to_string(static_cast<int>(result)));
    }
}

int tcTiles(int m, int n) { return ((m + kTileM - 1) / kTileM) * ((n + kTileN - 1) / kTileN); }

void launchTcGemm(const TcBatch& batch, int task_count, cudaStream_t stream) {
    static std::once_flag once;
    static cudaError_t attribute = cudaSuccess;
    std::call_once(once, [] {
        attribute = cudaFuncSetAttribute(tcGemmKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
    });
    checkCuda(attribute, "Configure the tcgen05 contraction kernel");
    int blocks = 0;
    for (int i = 0; i < task_count; ++i) blocks = std::max(blocks, tcTiles(batch.task[i].m, batch.task[i].n));
    tcGemmKernel<<<dim3(blocks, task_count), kTcThreads, kSmemBytes, stream>>>(batch);
}

// Host split of FP64 values into kSplit bf16 planes (basis matrices).
void splitHost(const std::vector<double>& values, int rows, int cols, int ld, std::vector<__nv_bfloat16>& planes) {
    planes.assign(static_cast<size_t>(kSplit) * rows * ld, __float2bfloat16_rn(0.0f));
    for (int r = 0; r < rows; ++r) {
        for (int c = 0; c < cols; ++c) {
            double rest = values[static_cast<size_t>(r) * cols + c];
            for (int p = 0; p < kSplit; ++p) {
                const __nv_bfloat16 piece = __float2bfloat16_rn(static_cast<float>(rest));
                planes[static_cast<size_t>(p) * rows * ld + static_cast<size_t>(r) * ld + c] = piece;
                rest -= static_cast<double>(__bfloat162float(piece));
            }
        }
    }
}

void launchSplitSource(const float* source, const SplitMatrix& out, int cols, cudaStream_t stream) {
    const int count = out.rows * cols;
    if (count <= 0) return;
    splitSourceKernel<<<ceilDiv(count, kThreads), kThreads, 0, stream>>>(
        source, out.rows, cols, out.data, out.ld, static_cast<size_t>(out.rows) * out.ld);
}

}  // namespace mpgp
