// Split-precision tcgen05 contractions for the Neumann DCT/DST field (sm_100a).
//
// The field solve of ElectrostaticField::solveNeumann (ElectrostaticField.cpp:
// 205-237) is six dense contractions C = A * B^T (engine.cu runDct).
//
// Precision: each operand x is scaled by a power of two 2^-e (so that the
// scaled magnitudes stay below 2^14) and stored as two fp16 planes,
// hi = fp16(x 2^-e) and lo = fp16((x 2^-e - hi) 2^11), which carry ~22 bits;
// lo is kept at the magnitude of x so that it does not fall into the fp16
// subnormal range, which the tensor cores flush.  A contraction accumulates
// hi*hi in one TMEM accumulator and hi*lo + lo*hi in a second one, combined as
// main + 2^-11 corr (the error-corrected fp16 split of Ootomo and Yokota,
// "Recovering single precision accuracy from Tensor Cores while surpassing the
// FP32 theoretical peak performance", IJHPCA 2022); the dropped lo*lo term is
// ~2^-22 relative.  Partials are restarted every K-block and summed in FP64
// registers, which keeps the accumulation error of long K chains at FP64 level.  Plane
// exponents follow the data: the source gets one exponent per row, every later
// stage a bound from the measured maximum of its input (TcScales).
//
// A 128 x kTileN output tile is computed by a cluster of `ksplit` (at most
// kMaxSplit) CTAs, each owning a contiguous share of the K-blocks, so that a
// 512 x 512 contraction (32 tiles) spreads over more SMs.  Per CTA, six warps:
//   warp 0 lane 0  TMA producer: K-blocks of 64 elements of both planes of A
//                  and B into a kStages-deep shared-memory ring (3-D tensor
//                  maps: K, rows, plane; 128-byte swizzle; zero fill past edges).
//   warp 1 lane 0  tcgen05.mma issuer: the three products of one K-block into
//                  one of two TMEM accumulator pairs (double-buffered),
//                  restarted every K-block; tcgen05.commit releases the smem
//                  stage and publishes the partial.
//   warps 2-5      read each partial with tcgen05.ld (warp w owns TMEM lanes
//                  32 * (w % 4) .. +31, i.e. tile rows), sum the partials in
//                  FP64 registers and park the FP64 tile in shared memory.
// CTA r of a cluster owns rows r * 128 / ksplit .. of the tile: every peer
// sends it those parked rows with one bulk shared-to-shared copy (completion
// on an mbarrier of the owner), and the owner sums the ksplit pieces in a
// fixed order (the result does not depend on scheduling), then runs the fused
// epilogue with all six warps and 16-byte stores: re-split into planes (plain
// or transposed), the spectral divide with the Parseval energy partials, or
// FP32 field stores.  Every mbarrier wait is bounded: on a timeout the CTA
// raises the error flag, drains the copies it issued and frees its TMEM; a
// failed CTA still sends its (flagged) rows, so its peers never wait on it.
#include <cuda.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "common.cuh"
#include "split.cuh"
#include "dct_tc.cuh"
#include "tc_ptx.cuh"

namespace mpgp {
namespace {

using namespace tc;

constexpr int kTcThreads = 192;
constexpr int kStageBytes = kSplit * (kTileM + kTileN) * kBlockK * 2;
constexpr int kRingBytes = kStages * kStageBytes;
constexpr int kParkPitch = kTileN + 2;  // doubles per parked row: 64 values, the failure flag, padding
constexpr int kParkBytes = kTileM * kParkPitch * 8;
constexpr int kTilePitch = kTileN + 1;  // floats per staged row (odd pitch: no bank conflicts)
constexpr int kStagedOffset = kParkBytes;
constexpr int kReceiveOffset = kRingBytes;
constexpr int kBarrierOffset = kReceiveOffset + kParkBytes;
constexpr int kPrefetchOffset = kBarrierOffset + 256;  // epilogue inputs fetched right after the dependency wait
constexpr int kPrefetchInts = 4 + kTileM + kMaxKbExponents;  // exp_a, exp_b, out_exp, -, the tile's row exponents,
                                                              // then A's per-K-block exponents
constexpr int kSmemBytes = kPrefetchOffset + kPrefetchInts * 4 + 1024 /* alignment slack */;
constexpr uint32_t kTmemColumns = 4 * kTileN;  // two buffers x (main, correction) accumulators
constexpr uint32_t kInstrDescriptor = instrDescriptor(kTileN);
constexpr uint32_t kPairDescriptor = instrDescriptor(2 * kTileN);  // A x [B_hi; B_lo]
static_assert(kStagedOffset + kTileM * kTilePitch * 4 <= kRingBytes, "the parked and staged tiles must fit in the ring");
static_assert((kParkPitch * 8) % 16 == 0, "parked rows must keep 16-byte alignment for the bulk copies");
static_assert(kTileM % (8 * kMaxSplit) == 0, "every split owns whole 8-row groups");


// One CTA of the cluster that computes output tile `tile_index` of task `t`;
// `local_block` = tile_index * ksplit + the CTA's rank (its energy partial and,
// for block 0, the task's bookkeeping).  The caller has released its successor.
__device__ __forceinline__ void tcTile(const TcBatch& batch, const TcTask& t, int tile_index, int local_block) {
    const int ksplit = batch.ksplit;
    const int tiles_n = (t.n + kTileN - 1) / kTileN;
    const int tiles_m = (t.m + kTileM - 1) / kTileM;
    // The whole cluster shares the tile, so the whole cluster leaves together.
    if (tile_index >= tiles_m * tiles_n) return;
    if (batch.stall_polls > 0) {
        // Failure-detection probe: a bounded wait on a barrier that nothing completes.
        // Every CTA of every cluster takes this path before any cluster barrier, copy
        // or TMEM allocation, so nothing is in flight when it returns.
        __shared__ __align__(8) uint64_t probe;
        if (threadIdx.x == 0) {
            mbarInit(smemAddress(&probe), 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            bool done = false;
            for (long long i = 0; i < batch.stall_polls && !done; ++i) done = mbarTryWait(smemAddress(&probe), 0);
            if (!done) atomicExch(batch.error_flag, 1);
        }
        waitForPrior();  // the grid completes only after its predecessor, as on the normal path
        __syncthreads();
        return;
    }
    const int split = static_cast<int>(clusterRank());
    const int m0 = (tile_index / tiles_n) * kTileM;
    const int n0 = (tile_index % tiles_n) * kTileN;
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int k_blocks_total = (t.k + kBlockK - 1) / kBlockK;
    const int per_split = (k_blocks_total + ksplit - 1) / ksplit;
    const int kb_begin = min(k_blocks_total, split * per_split);
    const int k_blocks = min(k_blocks_total, kb_begin + per_split) - kb_begin;
    const int rows_per = kTileM / ksplit;
    const int row_begin = split * rows_per;
    const uint32_t slice_bytes = static_cast<uint32_t>(rows_per * kParkPitch * 8);

    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    uint64_t* barriers = reinterpret_cast<uint64_t*>(smem + kBarrierOffset);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(barriers + 2 * kStages + 5);
    const uint32_t full0 = smemAddress(barriers);
    const uint32_t empty0 = smemAddress(barriers + kStages);
    const uint32_t partial0 = smemAddress(barriers + 2 * kStages);
    const uint32_t consumed0 = smemAddress(barriers + 2 * kStages + 2);
    const uint32_t received = smemAddress(barriers + 2 * kStages + 4);
    // In the idle ring after the K-loop: the parked FP64 rows [kTileM][kParkPitch] and the
    // staged FP32 tile [kTileM][kTilePitch]; past the ring: the rows the peers send,
    // [ksplit][rows_per][kParkPitch].
    const uint32_t parked_s = smemAddress(smem);
    const uint32_t staged_s = smemAddress(smem + kStagedOffset);
    const uint32_t incoming_s = smemAddress(smem + kReceiveOffset);

    if (threadIdx.x == 32) {
        for (int s = 0; s < kStages; ++s) {
            mbarInit(full0 + 8 * s, 1);
            mbarInit(empty0 + 8 * s, 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbarInit(partial0 + 8 * b, 1);
            mbarInit(consumed0 + 8 * b, 4);  // one arrival per epilogue warp
        }
        // The rows the peers send; its phase completes once they have all landed.
        mbarInit(received, 1);
        mbarExpectTx(received, static_cast<uint32_t>(ksplit - 1) * slice_bytes);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    clusterArrive();  // this CTA's barriers are initialised; peers wait for it before sending
    // The spectral scale of this CTA's output rows (a fixed table) goes to the slot of
    // the receive area that no peer writes (a CTA's own split), before the wait.
    float* scale_tile = reinterpret_cast<float*>(smem + kReceiveOffset +
                                                 static_cast<size_t>(split) * rows_per * kParkPitch * 8);
    if (t.mode == kTcSpectral && threadIdx.x >= 64) {
        // The four epilogue warps, eight loads in flight per thread.
        constexpr int kBatch = 8;
        const int count = rows_per * kTileN;
        for (int base = static_cast<int>(threadIdx.x) - 64; base < count; base += kBatch * (kTcThreads - 64)) {
            float v[kBatch];
#pragma unroll
            for (int j = 0; j < kBatch; ++j) {
                const int e = base + j * (kTcThreads - 64);
                const int grow = m0 + row_begin + e / kTileN;
                const int gcol = n0 + e % kTileN;
                v[j] = e < count && grow < t.m && gcol < t.n ? __ldg(t.scale + static_cast<size_t>(grow) * t.n + gcol)
                                                             : 0.0f;
            }
#pragma unroll
            for (int j = 0; j < kBatch; ++j) {
                const int e = base + j * (kTcThreads - 64);
                if (e < count) scale_tile[e] = v[j];
            }
        }
    }
    // The first stages' basis tiles do not depend on the previous kernels: issue them
    // now, so that only the data operand's latency follows the dependency wait.
    const int prefetched = t.constant_operand != 0 ? min(k_blocks, kStages) : 0;
    if (warp == 0 && lane == 0) {
        for (int kb = 0; kb < prefetched; ++kb) {
            unsigned char* stage = smem + kb * kStageBytes;
            const int k0 = (kb_begin + kb) * kBlockK;
            mbarExpectTx(full0 + 8 * kb, kStageBytes);
            if (t.constant_operand == 1) {
                tmaLoad3d(smemAddress(stage), &t.map_a, full0 + 8 * kb, k0, m0, 0);
            } else {
                tmaLoad3d(smemAddress(stage + kSplit * kTileM * kBlockK * 2), &t.map_b, full0 + 8 * kb, k0, n0, 0);
            }
        }
    }
    waitForPrior();   // the operands and scale bookkeeping come from the previous kernels

    if (warp == 0) {
        if (lane == 0) {
            // TMA producer (starts while warp 1 allocates TMEM).
            bool ok = true;
            int issued = 0;
            for (int kb = 0; kb < k_blocks && ok; ++kb) {
                const int s = kb % kStages;
                if (kb >= kStages) ok = mbarWait(empty0 + 8 * s, ((kb / kStages) - 1) & 1, batch.error_flag);
                if (!ok) break;
                unsigned char* stage = smem + s * kStageBytes;
                const int k0 = (kb_begin + kb) * kBlockK;
                const bool early = kb < prefetched;  // its basis tile is already on the way
                if (!early) mbarExpectTx(full0 + 8 * s, kStageBytes);
                // One box per operand carries both planes (a TMA instruction costs about the
                // same whatever its size, so fewer and larger boxes stream faster).
                if (!early || t.constant_operand != 1) {
                    tmaLoad3d(smemAddress(stage), &t.map_a, full0 + 8 * s, k0, m0, 0);
                }
                if (!early || t.constant_operand != 2) {
                    tmaLoad3d(smemAddress(stage + kSplit * kTileM * kBlockK * 2), &t.map_b, full0 + 8 * s, k0, n0, 0);
                }
                issued = kb + 1;
            }
            if (!ok) {
                // Drain: wait (bounded) for every issued stage so no copy lands after exit.
                for (int kb = max(0, issued - kStages); kb < issued; ++kb) {
                    mbarWait(full0 + 8 * (kb % kStages), (kb / kStages) & 1, nullptr);
                }
            }
        } else {
            // The epilogue's scalar inputs (written by the previous kernels), fetched
            // now so that their latency hides behind the main loop.
            int* early = reinterpret_cast<int*>(smem + kPrefetchOffset);
            if (lane == 1) {
                early[0] = t.exp_a != nullptr ? *t.exp_a : 0;
                early[1] = *t.exp_b;
                early[2] = t.mode != kTcField ? planeExponent(t.ref_max, t.gain) : 0;
            }
            if (t.row_exp_a != nullptr) {
                for (int r = lane - 1; r < rows_per; r += 31) {
                    early[4 + r] = __ldg(t.row_exp_a + min(m0 + row_begin + r, t.m - 1));
                }
            }
        }
        __syncwarp();
        clusterWait();
    } else if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smemAddress(tmem_slot)),
                     "r"(kTmemColumns));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        asm volatile("bar.sync 2, 160;" ::: "memory");  // TMEM address -> epilogue warps
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(tmem_slot);
        if (lane == 0) {
            // tcgen05.mma issuer: K-block kb accumulates into buffer kb % 2 from zero.
            for (int kb = 0; kb < k_blocks; ++kb) {
                const int s = kb % kStages;
                const int buffer = kb & 1;
                if (kb >= 2 && !mbarWait(consumed0 + 8 * buffer, ((kb >> 1) - 1) & 1, batch.error_flag)) break;
                if (!mbarWait(full0 + 8 * s, (kb / kStages) & 1, batch.error_flag)) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t stage = smemAddress(smem + s * kStageBytes);
                const uint32_t a_base = stage;
                const uint32_t b_base = stage + kSplit * kTileM * kBlockK * 2;
                const uint32_t main_acc = tmem + static_cast<uint32_t>(buffer * 2 * kTileN);
                const uint32_t corr_acc = main_acc + kTileN;
#pragma unroll
                for (int kk = 0; kk < kBlockK / 16; ++kk) {
                    // [B_hi; B_lo] are consecutive rows of the stage: one product of A_hi with
                    // both (2 kTileN columns) writes main and the first correction term
                    // (corr_acc follows main_acc); A_lo B_hi completes the correction.
                    const uint64_t a_hi = smemDescriptor(a_base + kk * 32);
                    const uint64_t a_lo = smemDescriptor(a_base + kTileM * kBlockK * 2 + kk * 32);
                    const uint64_t b_both = smemDescriptor(b_base + kk * 32);
                    ummaF16(main_acc, a_hi, b_both, kPairDescriptor, kk > 0 ? 1u : 0u);
                    ummaF16(corr_acc, a_lo, b_both, kInstrDescriptor, 1u);
                }
                ummaCommit(empty0 + 8 * s);
                ummaCommit(partial0 + 8 * buffer);
            }
        }
        __syncwarp();
        clusterWait();
    } else {
        // Epilogue warps: FP64 sum of this split's K-block partials, parked in shared memory.
        asm volatile("bar.sync 2, 160;" ::: "memory");
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(tmem_slot);
        const int quarter = warp & 3;
        const uint32_t lane_base = tmem + (static_cast<uint32_t>(quarter * 32) << 16);
        // A's per-K-block exponents, staged for the epilogue warps.
        int* kb_exp = reinterpret_cast<int*>(smem + kPrefetchOffset) + 4 + kTileM;
        if (t.kb_exp_a != nullptr) {
            for (int kb = static_cast<int>(threadIdx.x) - 64; kb < k_blocks; kb += 128) {
                kb_exp[kb] = t.kb_exp_a[kb_begin + kb];
            }
            asm volatile("bar.sync 1, 128;" ::: "memory");
        }
        double acc[kTileN];
#pragma unroll
        for (int j = 0; j < kTileN; ++j) acc[j] = 0.0;
        bool ok = true;
        for (int kb = 0; kb < k_blocks; ++kb) {
            const int buffer = kb & 1;
            ok = __all_sync(0xffffffffu, mbarWait(partial0 + 8 * buffer, (kb >> 1) & 1, batch.error_flag) ? 1 : 0) != 0;
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (t.kb_exp_a != nullptr) {
                // A K-block of A with an exponent of its own: its partial carries that scale.
                const double k_scale = pow2(kb_exp[kb]);
#pragma unroll
                for (int c0 = 0; c0 < kTileN; c0 += 16) {
                    uint32_t main_part[16], corr_part[16];
                    tmemLoad16(lane_base + static_cast<uint32_t>(buffer * 2 * kTileN + c0), main_part);
                    tmemLoad16(lane_base + static_cast<uint32_t>(buffer * 2 * kTileN + kTileN + c0), corr_part);
                    tmemWait(main_part, corr_part);
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const double part = static_cast<double>(__uint_as_float(main_part[j])) +
                                            static_cast<double>(__uint_as_float(corr_part[j])) *
                                                (1.0 / static_cast<double>(kLoShift));
                        acc[c0 + j] += part * k_scale;
                    }
                }
            } else {
#pragma unroll
                for (int c0 = 0; c0 < kTileN; c0 += 16) {
                    uint32_t main_part[16], corr_part[16];
                    tmemLoad16(lane_base + static_cast<uint32_t>(buffer * 2 * kTileN + c0), main_part);
                    tmemLoad16(lane_base + static_cast<uint32_t>(buffer * 2 * kTileN + kTileN + c0), corr_part);
                    tmemWait(main_part, corr_part);
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        acc[c0 + j] += static_cast<double>(__uint_as_float(main_part[j])) +
                                       static_cast<double>(__uint_as_float(corr_part[j])) *
                                           (1.0 / static_cast<double>(kLoShift));
                    }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbarArrive(consumed0 + 8 * buffer);
        }
        // The ring is idle once the last partial has been read (or was never used).
        const int local_row = quarter * 32 + lane;
        double* row = reinterpret_cast<double*>(smem) + local_row * kParkPitch;
#pragma unroll
        for (int j = 0; j < kTileN; j += 2) *reinterpret_cast<double2*>(row + j) = make_double2(acc[j], acc[j + 1]);
        row[kTileN] = ok ? 0.0 : 1.0;  // failure flag travels with the rows
        row[kTileN + 1] = 0.0;
        asm volatile("bar.sync 1, 128;" ::: "memory");  // the epilogue warps' rows are all parked
        clusterWait();
        if (threadIdx.x == 64 && ksplit > 1) {
            // Send every peer the rows it owns; wait until the copies have read them.
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            for (int owner = 0; owner < ksplit; ++owner) {
                if (owner == split) continue;
                const uint32_t src = parked_s + static_cast<uint32_t>(owner * rows_per * kParkPitch * 8);
                const uint32_t dst =
                    clusterAddress(incoming_s + static_cast<uint32_t>(split * rows_per * kParkPitch * 8), owner);
                bulkToPeer(dst, src, slice_bytes, clusterAddress(received, owner));
            }
            asm volatile("cp.async.bulk.commit_group;" ::: "memory");
            asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
        }
    }
    __syncthreads();

    bool tile_ok = mbarWait(received, 0, batch.error_flag);
    tile_ok = __syncthreads_and(tile_ok ? 1 : 0) != 0;
    for (int s = 0; s < ksplit && tile_ok; ++s) {
        const uint32_t piece = s == split ? parked_s + static_cast<uint32_t>(row_begin * kParkPitch * 8)
                                          : incoming_s + static_cast<uint32_t>(s * rows_per * kParkPitch * 8);
        tile_ok = loadShared2(piece + kTileN * 8).x == 0.0;
    }
    if (!tile_ok && threadIdx.x == 0) atomicExch(batch.error_flag, 1);

    // Fused sum and output, one (row, eight columns) unit per thread and pass: the
    // fixed-order sum over the splits, the unscaling, then the row-major output
    // (planes, field, or spectral divide + planes) and the staged copy for the
    // transposed pass.
    const int* early = reinterpret_cast<const int*>(smem + kPrefetchOffset);
    const int exp_a = early[0];
    const int exp_b = early[1];
    const bool split_out = t.mode != kTcField;
    const int out_exp = early[2];
    const float inv_scale = static_cast<float>(pow2(-out_exp));
    const bool staging = t.mode == kTcSplitTransposed || t.mode == kTcSpectral;
    double energy = 0.0;
    float magnitude = 0.0f;
    if (tile_ok) {
        for (int u = threadIdx.x; u < rows_per * (kTileN / 8); u += kTcThreads) {
            // Lanes run down the rows: their shared-memory rows are a pitch apart,
            // so the pieces' 16-byte loads and the staged stores hit distinct banks.
            const int r_local = u % rows_per;
            const int c0 = (u / rows_per) * 8;
            const int r = row_begin + r_local;
            const int grow = m0 + r;
            const int gcol0 = n0 + c0;
            const bool row_in = grow < t.m;
            const int valid = row_in ? max(0, min(8, t.n - gcol0)) : 0;
            // Global inputs first, so their latency overlaps the shared-memory sum.
            const int shift = exp_b + (t.row_exp_a != nullptr ? early[4 + r_local] : exp_a);
            float sc[8];
            if (t.mode == kTcSpectral) {
                // The spectral divide (ElectrostaticField.cpp:212-221), from the staged table.
                const float4 lo4 = *reinterpret_cast<const float4*>(scale_tile + r_local * kTileN + c0);
                const float4 hi4 = *reinterpret_cast<const float4*>(scale_tile + r_local * kTileN + c0 + 4);
                sc[0] = lo4.x;
                sc[1] = lo4.y;
                sc[2] = lo4.z;
                sc[3] = lo4.w;
                sc[4] = hi4.x;
                sc[5] = hi4.y;
                sc[6] = hi4.z;
                sc[7] = hi4.w;
            }
            double sum[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) sum[i] = 0.0;
            for (int s = 0; s < ksplit; ++s) {
                const uint32_t piece =
                    (s == split ? parked_s + static_cast<uint32_t>((r * kParkPitch + c0) * 8)
                                : incoming_s + static_cast<uint32_t>(((s * rows_per + r_local) * kParkPitch + c0) * 8));
#pragma unroll
                for (int i = 0; i < 8; i += 2) {
                    const double2 p = loadShared2(piece + i * 8);
                    sum[i] += p.x;
                    sum[i + 1] += p.y;
                }
            }
            const double unscale = pow2(shift);
            float v[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) v[i] = static_cast<float>(sum[i] * unscale);
            if (t.mode == kTcSpectral) {
                const double wr = parsevalWeight(grow);
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const float phi = v[i] * sc[i];
                    if (i < valid) {
                        energy += static_cast<double>(phi) * static_cast<double>(v[i]) * wr * parsevalWeight(gcol0 + i);
                    }
                    v[i] = phi;
                }
            }
            if (staging) {
#pragma unroll
                for (int i = 0; i < 8; ++i) storeShared(staged_s + static_cast<uint32_t>((r * kTilePitch + c0 + i) * 4), v[i]);
            }
            if (valid == 0) continue;
            if (t.mode == kTcField) {
                float* dst = t.out_f + static_cast<size_t>(grow) * t.out_f_ld + static_cast<size_t>(gcol0) * t.out_f_step;
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    if (i < valid) dst[static_cast<size_t>(i) * t.out_f_step] = v[i];
                }
                continue;
            }
            if (t.mode == kTcSplitTransposed) {
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    if (i < valid) magnitude = fmaxf(magnitude, fabsf(v[i]));
                }
                continue;
            }
            // kTcSplit and kTcSpectral: row-major planes.
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                if (i < valid) magnitude = fmaxf(magnitude, fabsf(v[i]));
            }
            __half* hi = t.out + static_cast<size_t>(grow) * t.out_ld + gcol0;
            if (valid == 8) {
                storeSplit8(v, inv_scale, hi, hi + t.out_plane);
            } else {
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    if (i < valid) splitScaled(v[i], inv_scale, hi[i], hi[i + t.out_plane]);
                }
            }
        }
    }
    if (staging) {
        __syncthreads();
        // Transposed pass: eight consecutive rows of one column per thread.
        const int groups = rows_per / 8;
        for (int g = threadIdx.x; g < groups * kTileN && tile_ok; g += kTcThreads) {
            const int r0 = row_begin + (g / kTileN) * 8;  // lanes along the columns: conflict-free reads
            const int c = g % kTileN;
            const int grow0 = m0 + r0;
            const int gcol = n0 + c;
            if (gcol >= t.n || grow0 >= t.m) continue;
            const int valid = min(8, t.m - grow0);
            float v[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) v[i] = loadShared(staged_s + static_cast<uint32_t>(((r0 + i) * kTilePitch + c) * 4));
            __half* hi = t.out_t + static_cast<size_t>(gcol) * t.out_t_ld + grow0;
            if (valid == 8) {
                storeSplit8(v, inv_scale, hi, hi + t.out_t_plane);
            } else {
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    if (i < valid) splitScaled(v[i], inv_scale, hi[i], hi[i + t.out_t_plane]);
                }
            }
        }
    }
    if (split_out) {
        double values[2] = {energy, static_cast<double>(magnitude)};
        const bool is_max[2] = {false, true};
        blockReduce<2>(values, is_max);
        if (threadIdx.x == 0) {
            if (t.mode == kTcSpectral && t.energy_partials != nullptr) t.energy_partials[local_block] = values[0];
            if (t.out_max != nullptr) atomicMax(t.out_max, __float_as_uint(static_cast<float>(values[1])));
            if (local_block == 0) {
                if (t.out_exp != nullptr) *t.out_exp = out_exp;
                if (t.clear != nullptr) *t.clear = 0u;
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 1) {
        const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(tmem_slot);
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemColumns));
    }
}

__global__ void __launch_bounds__(kTcThreads, 1) tcGemmKernel(const __grid_constant__ TcBatch batch) {
    releaseNext();
    tcTile(batch, batch.task[blockIdx.y], static_cast<int>(blockIdx.x) / batch.ksplit, static_cast<int>(blockIdx.x));
}

// Batched: cluster c computes items[c] (an instance's batch, task and tile); every
// item's batch has the launch's K split.
__global__ void __launch_bounds__(kTcThreads, 1) tcGemmBatchKernel(const TcItem* items, int ksplit) {
    releaseNext();
    const TcItem item = items[blockIdx.x / static_cast<unsigned>(ksplit)];
    const TcBatch& batch = *item.batch;
    if (threadIdx.x == 0) {
        // The tensor maps live in global memory here (uploaded by a copy, possibly into
        // memory an earlier engine's maps used): make the TMA proxy see their current bytes.
        const TcTask& t = batch.task[item.task];
        asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(&t.map_a) : "memory");
        asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(&t.map_b) : "memory");
    }
    tcTile(batch, batch.task[item.task], item.tile,
           item.tile * ksplit + static_cast<int>(blockIdx.x % static_cast<unsigned>(ksplit)));
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

// One warp per source row: the row's exponent from its maximum, then its planes.
__global__ void splitSourceKernel(const float* source, int rows, int cols, __half* out, int ld, size_t plane,
                                  int* row_exp, TcScales* scales) {
    releaseNext();
    waitForPrior();
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        scales->max_x = 0u;
        scales->max_phi = 0u;
    }
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= rows) return;
    const float* src = source + static_cast<size_t>(row) * cols;
    float top = 0.0f;
    for (int c = lane; c < cols; c += 32) top = fmaxf(top, fabsf(src[c]));
#pragma unroll
    for (int offset = 16; offset > 0; offset >>= 1) top = fmaxf(top, __shfl_xor_sync(0xffffffffu, top, offset));
    const int e = exponentOf(top) - kPlaneTop;
    if (lane == 0) {
        row_exp[row] = e;
        atomicMax(&scales->max_source, __float_as_uint(top));
    }
    const float inv_scale = static_cast<float>(pow2(-e));
    __half* dst = out + static_cast<size_t>(row) * ld;
    for (int c = lane; c < cols; c += 32) splitScaled(src[c], inv_scale, dst[c], dst[c + plane]);
}

// The shared-memory attribute is per device: set it once on each device that launches.
void configureKernel() {
    constexpr int kMaxDevices = 64;
    static std::once_flag once[kMaxDevices];
    static cudaError_t attribute[kMaxDevices] = {};
    int device = 0;
    checkCuda(cudaGetDevice(&device), "Query the current device");
    require(device >= 0 && device < kMaxDevices, "Device index out of range.");
    std::call_once(once[device], [device] {
        attribute[device] = cudaFuncSetAttribute(tcGemmKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
        if (attribute[device] == cudaSuccess) {
            attribute[device] =
                cudaFuncSetAttribute(tcGemmBatchKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
        }
    });
    checkCuda(attribute[device], "Configure the tcgen05 contraction kernel");
}

int batchTiles(const TcBatch& batch, int task_count) {
    int tiles = 0;
    for (int i = 0; i < task_count; ++i) {
        const TcTask& t = batch.task[i];
        tiles = std::max(tiles, ((t.m + kTileM - 1) / kTileM) * ((t.n + kTileN - 1) / kTileN));
    }
    return tiles;
}

cudaLaunchConfig_t launchConfig(dim3 grid, int ksplit, cudaStream_t stream, cudaLaunchAttribute* attribute) {
    cudaLaunchConfig_t config{};
    config.gridDim = grid;
    config.blockDim = dim3(kTcThreads);
    config.dynamicSmemBytes = kSmemBytes;
    config.stream = stream;
    attribute[0].id = cudaLaunchAttributeClusterDimension;
    attribute[0].val.clusterDim.x = static_cast<unsigned>(ksplit);
    attribute[0].val.clusterDim.y = 1;
    attribute[0].val.clusterDim.z = 1;
    attribute[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attribute[1].val.programmaticStreamSerializationAllowed = 1;
    config.attrs = attribute;
    config.numAttrs = 2;
    return config;
}

}  // namespace

void makeOperandMap(CUtensorMap* map, const SplitMatrix& m, int box_rows) {
    require(m.ld % kBlockK == 0 && m.rows > 0 && m.data != nullptr, "Split operand layout is invalid.");
    const cuuint64_t dims[3] = {static_cast<cuuint64_t>(m.ld), static_cast<cuuint64_t>(m.rows),
                                static_cast<cuuint64_t>(kSplit)};
    const cuuint64_t strides[2] = {static_cast<cuuint64_t>(m.ld) * 2,
                                   static_cast<cuuint64_t>(m.ld) * static_cast<cuuint64_t>(m.rows) * 2};
    const cuuint32_t box[3] = {static_cast<cuuint32_t>(kBlockK), static_cast<cuuint32_t>(box_rows),
                               static_cast<cuuint32_t>(kSplit)};  // both planes: [plane][row][64 halves]
    const cuuint32_t element_strides[3] = {1, 1, 1};
    const CUresult result =
        encoder()(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 3, m.data, dims, strides, box, element_strides,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (result != CUDA_SUCCESS) {
        fail(MPGP_ERR_CUDA, "cuTensorMapEncodeTiled failed with status " + std::to_string(static_cast<int>(result)));
    }
}

namespace {

// The autotuned K splits (tuned_splits.inc), replaceable at run time (mpgp_tuning_set_splits).
std::mutex g_split_mutex;
std::vector<std::pair<int, int>>& splitTable() {
    static std::vector<std::pair<int, int>> table = {
        std::pair<int, int>{0, 0},  // (no tuned size is 0; keeps the initialiser list non-empty)
#include "tuned_splits.inc"
    };
    return table;
}

// The tuned split for a contraction over k, or 0 when k is not in the table.
int tunedSplit(int k) {
    std::lock_guard<std::mutex> lock(g_split_mutex);
    for (const auto& entry : splitTable()) {
        if (entry.first == k && entry.first > 0) return entry.second;
    }
    return 0;
}

}  // namespace

void setTunedSplits(const int* sizes, const int* splits, int count) {
    for (int i = 0; i < count; ++i) {
        require(sizes[i] > 0 && (splits[i] == 1 || splits[i] == 2), "A tuned split is 1 or 2 for a positive size.");
    }
    std::lock_guard<std::mutex> lock(g_split_mutex);
    auto& table = splitTable();
    table.assign(1, std::pair<int, int>{0, 0});
    for (int i = 0; i < count; ++i) table.emplace_back(sizes[i], splits[i]);
}

int tunedSplits(int* sizes, int* splits, int capacity) {
    std::lock_guard<std::mutex> lock(g_split_mutex);
    int count = 0;
    for (const auto& entry : splitTable()) {
        if (entry.first <= 0) continue;
        if (count < capacity) {
            sizes[count] = entry.first;
            splits[count] = entry.second;
        }
        ++count;
    }
    return count;
}

namespace {

// Clusters of `ksplit` CTAs the GPU holds at once (-1 when the query fails); the
// answer depends only on the device and the cluster size, so it is asked once.
int activeClusters(int ksplit) {
    constexpr int kMaxDevices = 64;
    static std::mutex mutex;
    static int known[kMaxDevices][kMaxSplit + 1] = {};  // 0: not asked yet
    int device = 0;
    checkCuda(cudaGetDevice(&device), "Query the current device");
    require(device >= 0 && device < kMaxDevices && ksplit >= 1 && ksplit <= kMaxSplit, "Device index out of range.");
    std::lock_guard<std::mutex> lock(mutex);
    int& answer = known[device][ksplit];
    if (answer == 0) {
        cudaLaunchAttribute attribute[2] = {};
        cudaLaunchConfig_t config = launchConfig(dim3(static_cast<unsigned>(ksplit)), ksplit, nullptr, attribute);
        int clusters = 0;
        if (cudaOccupancyMaxActiveClusters(&clusters, tcGemmKernel, &config) != cudaSuccess) {
            (void)cudaGetLastError();
            clusters = -1;
        }
        answer = clusters == 0 ? -1 : clusters;
    }
    return answer;
}

// The largest split whose clusters of a batch of `tiles` tiles still fit on the GPU at once.
int fittingSplit(int tiles, int k_blocks) {
    int best = 1;
    for (int ksplit = 2; ksplit <= kMaxSplit && ksplit <= k_blocks; ksplit *= 2) {
        const int clusters = activeClusters(ksplit);
        if (clusters < 0 || tiles > clusters) break;  // the split would no longer run in one wave
        best = ksplit;
    }
    return best;
}

}  // namespace

void tcPlan(TcBatch& batch, int task_count) {
    configureKernel();
    const int tiles = batchTiles(batch, task_count) * task_count;
    int k_blocks = 0;
    int k = 0;
    for (int i = 0; i < task_count; ++i) {
        const int kb = (batch.task[i].k + kBlockK - 1) / kBlockK;
        k_blocks = i == 0 ? kb : std::min(k_blocks, kb);
        k = std::max(k, batch.task[i].k);
    }
    for (int i = 0; i < task_count; ++i) {
        const TcTask& t = batch.task[i];
        require(t.kb_exp_a == nullptr || (t.k + kBlockK - 1) / kBlockK <= kMaxKbExponents,
                "A contraction with per-K-block exponents has too many K-blocks.");
    }
    const int fitting = fittingSplit(tiles, k_blocks);
    const int tuned = tunedSplit(k);
    // The tuned split where it is allowed (it divides the K blocks among at most as
    // many CTAs as fit in one wave), else the largest split that fits.
    batch.ksplit = tuned > 0 && tuned <= fitting ? tuned : fitting;
}

int tcBlocks(const TcBatch& batch, int task_count) {
    (void)task_count;
    return batchTiles(batch, task_count) * batch.ksplit;
}

int taskTiles(const TcBatch& batch, int task) {
    const TcTask& t = batch.task[task];
    return ((t.m + kTileM - 1) / kTileM) * ((t.n + kTileN - 1) / kTileN);
}

void launchTcGemmBatch(const TcItem* items, int count, int ksplit, cudaStream_t stream) {
    if (count <= 0) return;
    configureKernel();
    require(ksplit >= 1 && ksplit <= kMaxSplit && (ksplit & (ksplit - 1)) == 0,
            "Contraction K split must be a power of two up to kMaxSplit.");
    cudaLaunchAttribute attribute[2] = {};
    const cudaLaunchConfig_t config =
        launchConfig(dim3(static_cast<unsigned>(count * ksplit)), ksplit, stream, attribute);
    checkCuda(cudaLaunchKernelEx(&config, tcGemmBatchKernel, items, ksplit),
              "Launch the batched tcgen05 contraction kernel");
}

void launchTcGemm(const TcBatch& batch, int task_count, cudaStream_t stream) {
    configureKernel();
    require(batch.ksplit >= 1 && batch.ksplit <= kMaxSplit && (batch.ksplit & (batch.ksplit - 1)) == 0,
            "Contraction K split must be a power of two up to kMaxSplit.");
    cudaLaunchAttribute attribute[2] = {};
    const cudaLaunchConfig_t config =
        launchConfig(dim3(static_cast<unsigned>(tcBlocks(batch, task_count)), static_cast<unsigned>(task_count)),
                     batch.ksplit, stream, attribute);
    checkCuda(cudaLaunchKernelEx(&config, tcGemmKernel, batch), "Launch the tcgen05 contraction kernel");
}

int splitHost(const std::vector<double>& values, int rows, int cols, int ld, std::vector<__half>& planes) {
    double top = 0.0;
    for (double v : values) top = std::max(top, std::fabs(v));
    int e = 0;
    if (top > 0.0) {
        const double m = std::frexp(top, &e);
        if (m == 0.5) e -= 1;
    }
    e -= kPlaneTop;
    planes.assign(static_cast<size_t>(kSplit) * rows * ld, __float2half_rn(0.0f));
    for (int r = 0; r < rows; ++r) {
        for (int c = 0; c < cols; ++c) {
            const double y = std::ldexp(values[static_cast<size_t>(r) * cols + c], -e);
            const __half hi = __double2half(y);
            const __half lo = __double2half((y - static_cast<double>(__half2float(hi))) * 2048.0);
            planes[static_cast<size_t>(r) * ld + c] = hi;
            planes[static_cast<size_t>(rows) * ld + static_cast<size_t>(r) * ld + c] = lo;
        }
    }
    return e;
}

// Basis value t at (row i, column j); n is the transform length of matrix t.
__device__ double basisValue(int t, int i, int j, int nx, int ny, double width, double height) {
    const bool along_x = t == 0 || t == 3 || t == 4;
    const int n = along_x ? nx : ny;
    const int freq = t <= 1 ? i : j;
    const int pos = t <= 1 ? j : i;
    const double turn = static_cast<double>((static_cast<long long>(freq) * (2 * pos + 1)) % (4LL * n)) /
                        (2.0 * static_cast<double>(n));  // the angle over pi
    if (t <= 1) return 2.0 * cospi(turn);
    if (t <= 3) return freq == 0 ? 1.0 : 2.0 * cospi(turn);
    if (freq == 0) return 0.0;
    const double wave = 3.141592653589793 * static_cast<double>(freq) / (along_x ? width : height);
    return wave * 2.0 * sinpi(turn);
}

struct BasisShape {
    int nx, ny;
    double width, height;
};

// Pass 1: per matrix, the largest |value| and the largest row sum of |values|
// (non-negative doubles compare like their bit patterns, so atomicMax is exact).
__global__ void __launch_bounds__(kThreads) basisRangeKernel(BasisShape b, unsigned long long* scratch) {
    const int t = blockIdx.y;
    const int n = (t == 0 || t == 3 || t == 4) ? b.nx : b.ny;
    const int i = blockIdx.x;
    if (i >= n) return;
    double values[2] = {0.0, 0.0};  // row sum, row max
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const double v = fabs(basisValue(t, i, j, b.nx, b.ny, b.width, b.height));
        values[0] += v;
        values[1] = fmax(values[1], v);
    }
    const bool is_max[2] = {false, true};
    blockReduce<2>(values, is_max);
    if (threadIdx.x == 0) {
        atomicMax(scratch + t, static_cast<unsigned long long>(__double_as_longlong(values[1])));
        atomicMax(scratch + kBasisCount + t, static_cast<unsigned long long>(__double_as_longlong(values[0])));
    }
}

struct BasisPlanes {
    __half* data[kBasisCount];
    int ld[kBasisCount];
    size_t plane[kBasisCount];
    int exponent[kBasisCount];
};

// Pass 2: the planes, as splitHost forms them.
__global__ void __launch_bounds__(kThreads) basisPlanesKernel(BasisShape b, BasisPlanes p) {
    const int t = blockIdx.y;
    const int n = (t == 0 || t == 3 || t == 4) ? b.nx : b.ny;
    const int i = blockIdx.x;
    if (i >= n) return;
    const double inv_scale = pow2(-p.exponent[t]);
    __half* hi = p.data[t] + static_cast<size_t>(i) * p.ld[t];
    __half* lo = hi + p.plane[t];
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const double y = basisValue(t, i, j, b.nx, b.ny, b.width, b.height) * inv_scale;
        const __half h = __double2half(y);
        hi[j] = h;
        lo[j] = __double2half((y - static_cast<double>(__half2float(h))) * 2048.0);
    }
}

void buildBasisPlanes(int nx, int ny, double width, double height, const SplitMatrix (&out)[kBasisCount],
                      unsigned long long* scratch, int (&exponents)[kBasisCount],
                      double (&max_row_l1)[kBasisCount], cudaStream_t stream) {
    const BasisShape shape{nx, ny, width, height};
    const dim3 grid(static_cast<unsigned>(std::max(nx, ny)), kBasisCount);
    checkCuda(cudaMemsetAsync(scratch, 0, 2 * kBasisCount * sizeof(unsigned long long), stream), "basis ranges");
    basisRangeKernel<<<grid, kThreads, 0, stream>>>(shape, scratch);
    checkCuda(cudaGetLastError(), "Launch the basis range pass");
    unsigned long long ranges[2 * kBasisCount] = {};
    checkCuda(cudaMemcpyAsync(ranges, scratch, sizeof(ranges), cudaMemcpyDeviceToHost, stream), "basis ranges");
    checkCuda(cudaStreamSynchronize(stream), "basis ranges");
    BasisPlanes planes{};
    for (int t = 0; t < kBasisCount; ++t) {
        double top = 0.0, row = 0.0;
        std::memcpy(&top, &ranges[t], sizeof(double));
        std::memcpy(&row, &ranges[kBasisCount + t], sizeof(double));
        int e = 0;
        if (top > 0.0) {
            const double m = std::frexp(top, &e);
            if (m == 0.5) e -= 1;
        }
        exponents[t] = e - kPlaneTop;
        max_row_l1[t] = row;
        planes.data[t] = out[t].data;
        planes.ld[t] = out[t].ld;
        planes.plane[t] = out[t].plane();
        planes.exponent[t] = exponents[t];
    }
    basisPlanesKernel<<<grid, kThreads, 0, stream>>>(shape, planes);
    checkCuda(cudaGetLastError(), "Launch the basis plane pass");
}

void launchSplitSource(const float* source, const SplitMatrix& out, int cols, int* row_exp, TcScales* scales,
                       cudaStream_t stream) {
    if (out.rows <= 0) return;
    const int rows_per_block = kThreads / 32;
    launchChained("Launch the source split", splitSourceKernel, dim3(ceilDiv(out.rows, rows_per_block)),
                  dim3(kThreads), 0, stream, source, out.rows, cols, out.data, out.ld, out.plane(), row_exp, scales);
}

}  // namespace mpgp
