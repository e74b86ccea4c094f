// Banded tcgen05 field solve (sm_100a): the forward DCT, the spectral divide and
// the inverse transforms along y of ElectrostaticField::solveNeumann
// (ElectrostaticField.cpp:205-237) for one band of 64 spectral columns per cluster.
//
// A two-dimensional transform C_y X C_x^T restricted to spectral columns kx in a
// band needs only the rows of C_x in that band: Q = S C_x[band]^T is a ny x 64
// slab, and rho_hat[:, band] = C_y Q needs only that slab.  Likewise the inverse
// along y, M = D_y phi_hat[:, band], needs only the band's coefficients.  So one
// cluster per band runs the three contraction passes with no data from any other
// cluster; only the inverse along x, which sums over every band, is left to a
// second launch.  Inside the cluster, CTA (i, h) owns rows 128 i .. 128 i + 127 and
// the share h of the band's columns (share_n of them):
//   pass 0  Q[rows i, share h]      = S[rows i, :] Cx[share h, :]^T  (K = x)
//   pass 1  rho_hat[rows i, share h] = Cy[rows i, :] Q[:, share h]   (K = y)
//   pass 2  M1[rows i, share h]     = Dy[rows i, :] phi_hat[:, share h]  (K = ky)
//   pass 3  M2[rows i, share h]     = Syw[rows i, :] phi_hat[:, share h]
// Pass 1 and 2 contract over all rows, so their B operand (Q^T, phi_hat^T) is
// gathered: every CTA writes its 128 x share_n result, split into fp16 planes,
// straight into the K-major 128-byte-swizzled layout of that operand in its own
// shared memory, then copies it (one bulk shared-to-shared copy) into the same place
// in the CTAs of the other row blocks of its share.  Each producer splits with its
// own exponent, taken from its tile's maximum; the exponent travels with the tile,
// and the consumer restarts its accumulation at every K-block anyway, so it scales
// each K-block's partial by its producer's exponent in the FP64 sum.
//
// Warp roles and the arithmetic follow dct_tc.cu: warp 0 lane 0 issues TMA loads
// into a three-stage ring (the basis and source tiles), warp 1 lane 0 issues the
// three products of the error-corrected fp16 split per K-step into double-buffered
// TMEM accumulators, warps 2-5 sum the K-block partials in FP64 registers and run
// each pass's epilogue.  The ring runs across the passes, so the next pass's basis
// tiles load while the current epilogue runs.  Every mbarrier wait is bounded; a
// CTA whose wait runs out raises the error flag and still writes and sends its
// tiles, so its peers never wait on it.  The cluster barriers are reached by every
// thread of every CTA on every path.
#include <cuda.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "common.cuh"
#include "field_tc.cuh"
#include "split.cuh"
#include "tc_ptx.cuh"

namespace mpgp {
namespace {

using namespace tc;

constexpr int kFieldThreads = 192;
constexpr int kMaxShareN = 32;
constexpr int kMaxRowBlocks = kFieldMaxRows / kTileM;
constexpr int kMaxCluster = 8;
constexpr int kFieldStages = 3;
constexpr int kATileBytes = kSplit * kTileM * kBlockK * 2;        // 32 KB: one 128 x 64 tile, both planes
constexpr int kAPlaneBytes = kTileM * kBlockK * 2;
constexpr int kBTileMaxBytes = kSplit * kMaxShareN * kBlockK * 2;  // 8 KB
constexpr int kFieldStageBytes = kATileBytes + kBTileMaxBytes;
constexpr int kGatherOffset = kFieldStages * kFieldStageBytes;
constexpr int kGatherBytes = 2 * kMaxRowBlocks * kBTileMaxBytes;  // the gathered B operand, every K-block
constexpr int kScalePitch = kMaxShareN + 1;                        // floats per staged scale row (odd: no bank conflicts)
constexpr int kScaleOffset = kGatherOffset + kGatherBytes;         // the spectral scale of the CTA's tile
constexpr int kRecordOffset = kScaleOffset + kTileM * kScalePitch * 4;  // [2][kMaxRowBlocks] 16-byte exponent records
constexpr int kPhiMaxOffset = kRecordOffset + 2 * kMaxRowBlocks * 16;  // [kMaxCluster] floats
constexpr int kReduceOffset = kPhiMaxOffset + kMaxCluster * 4;         // float [2][4], double [4]
constexpr int kFieldBarrierOffset = kReduceOffset + 64;
constexpr int kFieldBarriers = 2 * kFieldStages + 6;
constexpr int kFieldSmemBytes = kFieldBarrierOffset + kFieldBarriers * 8 + 16 + 1024 /* alignment slack */;
static_assert(kGatherOffset % 1024 == 0 && kATileBytes % 1024 == 0, "swizzled tiles must stay 1024-byte aligned");
static_assert(kReduceOffset % 8 == 0, "the reduction slots hold doubles");
static_assert(kFieldSmemBytes <= 227 * 1024, "the banded solve must fit one CTA's shared memory");

__device__ __forceinline__ int planeExponentOf(float top) {
    return min(120, max(-120, exponentOf(top) - kPlaneTop));
}

__device__ __forceinline__ void storeRemote(uint32_t cluster_address, float v) {
    asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(cluster_address), "f"(v) : "memory");
}

__device__ __forceinline__ void epilogueSync() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

// The maximum of `v` over the 128 epilogue threads (slot: four floats of shared memory).
__device__ __forceinline__ float epilogueMax(float v, float* slot, int quarter) {
#pragma unroll
    for (int offset = 16; offset > 0; offset >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, offset));
    if ((threadIdx.x & 31) == 0) slot[quarter] = v;
    epilogueSync();
    return fmaxf(fmaxf(slot[0], slot[1]), fmaxf(slot[2], slot[3]));
}

// Writes one row r of a 128 x N result, split with 2^-e, as column r of the
// gathered K-major operand: K-block 2 i + r / 64, element r % 64 of each of the N
// operand rows (128-byte swizzle: 16-byte chunk c of row n sits at chunk c ^ (n % 8)).
template <int N>
__device__ __forceinline__ void writeGathered(unsigned char* gathered, int i, int r, const float (&v)[N],
                                              float inv_scale) {
    constexpr int kTile = kSplit * N * kBlockK * 2;
    unsigned char* tile = gathered + (2 * i + (r >> 6)) * kTile;
    const int kk = r & 63;
#pragma unroll
    for (int n = 0; n < N; ++n) {
        __half hi, lo;
        splitScaled(v[n], inv_scale, hi, lo);
        const int offset = n * 128 + ((((kk >> 3) ^ (n & 7))) << 4) + (kk & 7) * 2;
        *reinterpret_cast<__half*>(tile + offset) = hi;
        *reinterpret_cast<__half*>(tile + N * 128 + offset) = lo;
    }
}

// One CTA of the cluster of band `band` in mode `mode` (FieldMode); `local_block`
// indexes its energy partial.  The caller has released its successor.
template <int N>
__device__ __forceinline__ void fieldBand(const FieldBand& f, int band, int mode, int local_block) {
    constexpr int kBTile = kSplit * N * kBlockK * 2;
    constexpr uint32_t kDescriptor = instrDescriptor(N);
    constexpr uint32_t kPairDescriptor = instrDescriptor(2 * N);  // A x [B_hi; B_lo]: main and first correction
    constexpr uint32_t kTmemColumns = 4 * N < 32 ? 32 : 4 * N;
    const FieldShape& shape = f.shape;
    if (f.stall_polls > 0) {
        // Failure-detection probe: a bounded wait on a barrier that nothing completes.
        // Every CTA of every cluster takes this path before any cluster barrier, copy
        // or TMEM allocation, so nothing is in flight when it returns.
        __shared__ __align__(8) uint64_t probe;
        if (threadIdx.x == 0) {
            mbarInit(smemAddress(&probe), 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            bool done = false;
            for (long long k = 0; k < f.stall_polls && !done; ++k) done = mbarTryWait(smemAddress(&probe), 0);
            if (!done) atomicExch(f.error_flag, 1);
        }
        waitForPrior();
        __syncthreads();
        return;
    }
    const int rank = static_cast<int>(clusterRank());
    const int shares = shape.shares;
    const int row_blocks = shape.m_blocks;
    const int i = rank / shares;
    const int h = rank % shares;
    const int kx0 = band * kBlockK + h * N;
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int s1 = (f.nx + kBlockK - 1) / kBlockK;  // pass 0 K-blocks (x)
    const int s2 = 2 * row_blocks;                   // pass 1-3 K-blocks (y, ky)
    const bool forward = mode != kFieldInverse;
    const bool gradient = mode != kFieldForward;
    // Ring steps: pass 0 (s1 K-blocks), then s2 per later pass; an inverse launch starts at pass 2.
    const int steps = forward ? s1 + s2 + (gradient ? 2 * s2 : 0) : 2 * s2;
    const int pass1_step = forward ? s1 : -1;
    const int pass2_step = forward ? s1 + s2 : 0;
    const auto decode = [&](int step, int& pass, int& kb) {
        if (forward && step < s1) {
            pass = 0;
            kb = step;
            return;
        }
        const int t = forward ? step - s1 : step + s2;
        pass = 1 + t / s2;
        kb = t % s2;
    };
    const uint32_t push_bytes = static_cast<uint32_t>(2 * kBTile);
    // This share's slot of the kept phi_hat^T and of its records.
    unsigned char* const store = f.phi_store + static_cast<size_t>(band * shares + h) * s2 * kBTile;
    int* const store_records = f.phi_records + static_cast<size_t>(band * shares + h) * row_blocks * 4;

    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    unsigned char* gathered = smem + kGatherOffset;
    int* records = reinterpret_cast<int*>(smem + kRecordOffset);  // [2][kMaxRowBlocks][4]
    float* phi_max = reinterpret_cast<float*>(smem + kPhiMaxOffset);
    float* reduce_f = reinterpret_cast<float*>(smem + kReduceOffset);
    double* reduce_d = reinterpret_cast<double*>(smem + kReduceOffset + 32);
    uint64_t* barriers = reinterpret_cast<uint64_t*>(smem + kFieldBarrierOffset);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(barriers + kFieldBarriers);
    const uint32_t full0 = smemAddress(barriers);
    const uint32_t empty0 = smemAddress(barriers + kFieldStages);
    const uint32_t partial0 = smemAddress(barriers + 2 * kFieldStages);
    const uint32_t consumed0 = smemAddress(barriers + 2 * kFieldStages + 2);
    const uint32_t received_q = smemAddress(barriers + 2 * kFieldStages + 4);
    const uint32_t received_phi = smemAddress(barriers + 2 * kFieldStages + 5);
    const uint32_t gathered_s = smemAddress(gathered);
    const uint32_t records_s = smemAddress(records);

    if (threadIdx.x == 32) {
        for (int s = 0; s < kFieldStages; ++s) {
            mbarInit(full0 + 8 * s, 1);
            mbarInit(empty0 + 8 * s, 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbarInit(partial0 + 8 * b, 1);
            mbarInit(consumed0 + 8 * b, 4);  // one arrival per epilogue warp
        }
        // A gathered operand is complete once the four epilogue warps have written this
        // CTA's tile and every other row block's tile has landed.
        const uint32_t incoming = static_cast<uint32_t>(row_blocks - 1) * (push_bytes + 16);
        mbarInit(received_q, 5);
        mbarExpectTx(received_q, incoming);
        if (forward) {
            mbarInit(received_phi, 5);
            mbarExpectTx(received_phi, incoming);
        } else {
            mbarInit(received_phi, 1);  // the loader's arrival with the kept operand's bytes
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    clusterArrive();  // this CTA's barriers are initialised; peers wait for it before sending

    // The first ring stages' basis tiles do not depend on the previous kernels: Cx
    // (pass 0's B) for a forward launch, Dy (pass 2's A, whole stages) for an inverse one.
    const int prefetched = min(kFieldStages, forward ? s1 : s2);
    if (warp == 0 && lane == 0) {
        for (int step = 0; step < prefetched; ++step) {
            const uint32_t stage = smemAddress(smem + step * kFieldStageBytes);
            if (forward) {
                mbarExpectTx(full0 + 8 * step, static_cast<uint32_t>(kATileBytes + kBTile));
                tmaLoad3d(stage + kATileBytes, &f.map_cx, full0 + 8 * step, step * kBlockK, kx0, 0);
            } else {
                mbarExpectTx(full0 + 8 * step, static_cast<uint32_t>(kATileBytes));
                tmaLoad3d(stage, &f.map_dy, full0 + 8 * step, step * kBlockK, i * kTileM, 0);
            }
        }
    }
    // The spectral scale of each epilogue thread's row (a fixed table), staged in shared
    // memory: epilogue warp q loads rows 32 q .. 32 q + 31 of the tile, a row per
    // 32 / N-lane group and pass, and reads back only its own rows.
    const int quarter = warp & 3;
    const int r = quarter * 32 + lane;
    const int row = i * kTileM + r;
    float* scale = reinterpret_cast<float*>(smem + kScaleOffset) + r * kScalePitch;
    if (warp >= 2) {
        constexpr int kRowsPerPass = 32 / N;
        const int j = lane % N;
        const int kx = kx0 + j;
        float v[32 / kRowsPerPass];
#pragma unroll
        for (int k = 0; k < 32 / kRowsPerPass; ++k) {
            const int rr = k * kRowsPerPass + lane / N;
            const int grow = i * kTileM + quarter * 32 + rr;
            v[k] = grow < f.ny && kx < f.nx ? __ldg(f.scale + static_cast<size_t>(grow) * f.nx + kx) : 0.0f;
        }
        float* tile = reinterpret_cast<float*>(smem + kScaleOffset);
#pragma unroll
        for (int k = 0; k < 32 / kRowsPerPass; ++k) {
            const int rr = k * kRowsPerPass + lane / N;
            tile[(quarter * 32 + rr) * kScalePitch + j] = v[k];
        }
        __syncwarp();
    }
    waitForPrior();  // the source planes and their row exponents come from the previous kernels
    clusterWait();
    if (forward && gradient && warp < 2) clusterArrive();  // the second cluster barrier: see the spectral epilogue

    if (warp == 0) {
        if (lane == 0) {
            if (!forward) {
                // The kept phi_hat^T of this share (every row block's K-blocks) and its records.
                mbarExpectTx(received_phi, static_cast<uint32_t>(s2 * kBTile + row_blocks * 16));
                bulkFromGlobal(gathered_s, store, static_cast<uint32_t>(s2 * kBTile), received_phi);
                bulkFromGlobal(records_s + 16 * kMaxRowBlocks, store_records, static_cast<uint32_t>(row_blocks * 16),
                               received_phi);
            }
            bool ok = true;
            int issued = 0;
            for (int step = 0; step < steps && ok; ++step) {
                const int slot = step % kFieldStages;
                if (step >= kFieldStages) ok = mbarWait(empty0 + 8 * slot, ((step / kFieldStages) - 1) & 1, f.error_flag);
                if (!ok) break;
                const uint32_t stage = smemAddress(smem + slot * kFieldStageBytes);
                const uint32_t full = full0 + 8 * slot;
                const bool early = step < prefetched;  // its basis tile is already on the way
                int pass, kb;
                decode(step, pass, kb);
                if (pass == 0) {
                    if (!early) {
                        mbarExpectTx(full, static_cast<uint32_t>(kATileBytes + kBTile));
                        tmaLoad3d(stage + kATileBytes, &f.map_cx, full, step * kBlockK, kx0, 0);
                    }
                    tmaLoad3d(stage, &f.map_s, full, step * kBlockK, i * kTileM, 0);
                } else if (!early) {
                    const CUtensorMap* map = pass == 1 ? &f.map_cy : (pass == 2 ? &f.map_dy : &f.map_syw);
                    mbarExpectTx(full, static_cast<uint32_t>(kATileBytes));
                    tmaLoad3d(stage, map, full, kb * kBlockK, i * kTileM, 0);
                }
                issued = step + 1;
            }
            if (!ok) {
                // Drain: wait (bounded) for every issued stage so no copy lands after exit.
                for (int step = max(0, issued - kFieldStages); step < issued; ++step) {
                    mbarWait(full0 + 8 * (step % kFieldStages), (step / kFieldStages) & 1, nullptr);
                }
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smemAddress(tmem_slot)),
                     "r"(kTmemColumns));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        asm volatile("bar.sync 2, 160;" ::: "memory");  // TMEM address -> epilogue warps
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(tmem_slot);
        if (lane == 0) {
            // A partial covers a pair of K-blocks (2 p, 2 p + 1) of a pass: one producer's
            // tile of a gathered operand, so one exponent.
            int partial = 0;
            for (int step = 0; step < steps; ++step) {
                const int slot = step % kFieldStages;
                int pass, kb;
                decode(step, pass, kb);
                const int count = pass == 0 ? s1 : s2;
                const bool opens = (kb & 1) == 0;
                const bool closes = (kb & 1) == 1 || kb == count - 1;
                const int buffer = partial & 1;
                if (opens && partial >= 2 &&
                    !mbarWait(consumed0 + 8 * buffer, ((partial >> 1) - 1) & 1, f.error_flag)) {
                    break;
                }
                if (!mbarWait(full0 + 8 * slot, (step / kFieldStages) & 1, f.error_flag)) break;
                if (step == pass1_step && !mbarWait(received_q, 0, f.error_flag)) break;
                if (step == pass2_step && !mbarWait(received_phi, 0, f.error_flag)) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t a_base = smemAddress(smem + slot * kFieldStageBytes);
                const uint32_t b_base = pass == 0 ? a_base + kATileBytes : gathered_s + static_cast<uint32_t>(kb * kBTile);
                const uint32_t main_acc = tmem + static_cast<uint32_t>(buffer * 2 * N);
                const uint32_t corr_acc = main_acc + N;
#pragma unroll
                for (int kk = 0; kk < kBlockK / 16; ++kk) {
                    // The B tile's planes are consecutive rows, [B_hi; B_lo], so one product of
                    // A_hi with both (2N columns) writes main and the first correction term
                    // (corr_acc follows main_acc); A_lo B_hi completes the correction.
                    const uint64_t a_hi = smemDescriptor(a_base + kk * 32);
                    const uint64_t a_lo = smemDescriptor(a_base + kAPlaneBytes + kk * 32);
                    const uint64_t b_both = smemDescriptor(b_base + kk * 32);
                    const uint32_t accumulate = kk > 0 || !opens ? 1u : 0u;
                    ummaF16(main_acc, a_hi, b_both, kPairDescriptor, accumulate);
                    ummaF16(corr_acc, a_lo, b_both, kDescriptor, 1u);
                }
                ummaCommit(empty0 + 8 * slot);
                if (closes) {
                    ummaCommit(partial0 + 8 * buffer);
                    ++partial;
                }
            }
        }
        __syncwarp();
    } else {
        asm volatile("bar.sync 2, 160;" ::: "memory");
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(tmem_slot);
        const uint32_t lane_base = tmem + (static_cast<uint32_t>(quarter * 32) << 16);
        const int et = static_cast<int>(threadIdx.x) - 64;
        const bool row_in = row < f.ny;
        const int exp_cx = f.exp_basis[0], exp_cy = f.exp_basis[1], exp_dy = f.exp_basis[2], exp_syw = f.exp_basis[5];
        const int exp_row = row_in ? f.row_exp[row] : 0;
        float top_phi = 0.0f;
        int exp_m1 = 0, exp_m2 = 0;
        if (!forward) {
            // The band's maximum |phi_hat| from the records the forward launch kept.
            const int* band_records = f.phi_records + static_cast<size_t>(band) * shares * row_blocks * 4;
            float band_top = 0.0f;
            for (int k = 0; k < shares * row_blocks; ++k) band_top = fmaxf(band_top, __int_as_float(band_records[k * 4 + 1]));
            exp_m1 = planeExponentOf(band_top * f.gain_dy);
            exp_m2 = planeExponentOf(band_top * f.gain_syw);
        }
        bool ok = true;
        int partial = 0;
#pragma unroll 1
        for (int pass = forward ? 0 : 2; pass < (gradient ? 4 : 2); ++pass) {
            double acc[N];
#pragma unroll
            for (int j = 0; j < N; ++j) acc[j] = 0.0;
            // The producers' exponents of the gathered operand (pass 1: Q, passes 2-3: phi_hat).
            if (pass == 1 || pass == 2) {
                // Waited for even after a failure, so that no peer's copy lands after this CTA exits.
                const uint32_t received = pass == 1 ? received_q : received_phi;
                const bool got = __all_sync(0xffffffffu, mbarWait(received, 0, f.error_flag) ? 1 : 0) != 0;
                ok = ok && got;
            }
            const int* exps = records + (pass == 1 ? 0 : kMaxRowBlocks * 4);
            const int pairs = ((pass == 0 ? s1 : s2) + 1) / 2;
            for (int pair = 0; pair < pairs; ++pair, ++partial) {
                if (!ok) continue;
                const int buffer = partial & 1;
                ok = __all_sync(0xffffffffu, mbarWait(partial0 + 8 * buffer, (partial >> 1) & 1, f.error_flag) ? 1 : 0) !=
                     0;
                if (!ok) continue;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const double k_scale = pass == 0 ? 1.0 : pow2(exps[pair * 4]);
#pragma unroll
                for (int c0 = 0; c0 < N; c0 += 16) {
                    uint32_t main_part[16], corr_part[16];
                    tmemLoad16(lane_base + static_cast<uint32_t>(buffer * 2 * N + c0), main_part);
                    tmemLoad16(lane_base + static_cast<uint32_t>(buffer * 2 * N + N + c0), corr_part);
                    tmemWait(main_part, corr_part);
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        // main + 2^-11 corr rounds once in FP32 (the product is exact), then
                        // joins the FP64 sum with the producer's scale (a power of two).
                        const float part = __fmaf_rn(__uint_as_float(corr_part[j]), 1.0f / kLoShift,
                                                     __uint_as_float(main_part[j]));
                        acc[c0 + j] = __fma_rn(static_cast<double>(part), k_scale, acc[c0 + j]);
                    }
                }
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                __syncwarp();
                if (lane == 0) mbarArrive(consumed0 + 8 * buffer);
            }

            if (pass == 0) {
                // Q = S Cx^T: split with this tile's exponent into the gathered Q^T.
                float v[N];
                float top = 0.0f;
                const double unscale = pow2(exp_row + exp_cx);
#pragma unroll
                for (int j = 0; j < N; ++j) {
                    v[j] = static_cast<float>(acc[j] * unscale);
                    top = fmaxf(top, fabsf(v[j]));
                }
                const int e = planeExponentOf(epilogueMax(top, reduce_f, quarter));
                writeGathered<N>(gathered, i, r, v, static_cast<float>(pow2(-e)));
                if (et == 0) records[i * 4] = e;
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                __syncwarp();
                if (lane == 0) mbarArrive(received_q);
                epilogueSync();
                if (et == 0 && row_blocks > 1) {
                    // This row block's K-blocks of Q^T and their exponent, to the other row blocks.
                    const uint32_t src = gathered_s + static_cast<uint32_t>(2 * i * kBTile);
                    for (int peer_block = 0; peer_block < row_blocks; ++peer_block) {
                        if (peer_block == i) continue;
                        const uint32_t peer = static_cast<uint32_t>(peer_block * shares + h);
                        const uint32_t bar = clusterAddress(received_q, peer);
                        bulkToPeer(clusterAddress(src, peer), src, push_bytes, bar);
                        bulkToPeer(clusterAddress(records_s + 16 * i, peer), records_s + 16 * i, 16, bar);
                    }
                    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
                }
            } else if (pass == 1) {
                // The copies of pass 0 have read this CTA's Q^T K-blocks long ago (their peers'
                // pass 1 needed them); phi_hat^T overwrites them below, after the energy
                // reduction's barrier orders every writer after this wait.
                if (et == 0) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
                // rho_hat = Cy Q; phi_hat = rho_hat .* scale (ElectrostaticField.cpp:212-221);
                // the Parseval energy sum_{ky,kx} w(ky) w(kx) phi_hat rho_hat.
                float phi[N];
                double energy = 0.0;
                const double unscale = pow2(exp_cy);
                const double wr = row == 0 ? 0.5 : 1.0;
#pragma unroll
                for (int j = 0; j < N; ++j) {
                    const float v = static_cast<float>(acc[j] * unscale);
                    phi[j] = v * scale[j];
                    if (row_in && kx0 + j < f.nx) {
                        energy += static_cast<double>(phi[j]) * static_cast<double>(v) * wr * (kx0 + j == 0 ? 0.5 : 1.0);
                    }
                    top_phi = fmaxf(top_phi, fabsf(phi[j]));
                }
#pragma unroll
                for (int offset = 16; offset > 0; offset >>= 1) energy += __shfl_xor_sync(0xffffffffu, energy, offset);
                if (lane == 0) reduce_d[quarter] = energy;
                epilogueSync();
                if (et == 0 && f.energy_partials != nullptr) {
                    f.energy_partials[local_block] = ((reduce_d[0] + reduce_d[1]) + reduce_d[2]) + reduce_d[3];
                }
                top_phi = epilogueMax(top_phi, reduce_f + 4, quarter);
                if (gradient) {
                    if (et == 0) {
                        // This tile's max |phi_hat| to every CTA of the cluster: the band's maximum
                        // bounds M1 and M2, whose planes share one exponent per band.
                        for (int peer = 0; peer < shape.cluster; ++peer) {
                            storeRemote(clusterAddress(smemAddress(phi_max + rank), static_cast<uint32_t>(peer)), top_phi);
                        }
                    }
                    // Every CTA's pass-1 operand reads are complete (its last partial is in):
                    // from now on the peers may overwrite its gathered operand.
                    clusterArrive();
                }
                // phi_hat^T into the gathered operand (its own K-blocks), and kept in global
                // memory with its exponent and maximum for a later inverse launch.
                const int e = planeExponentOf(top_phi);
                writeGathered<N>(gathered, i, r, phi, static_cast<float>(pow2(-e)));
                if (et == 0) {
                    records[kMaxRowBlocks * 4 + i * 4] = e;
                    records[kMaxRowBlocks * 4 + i * 4 + 1] = __float_as_int(top_phi);
                }
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                __syncwarp();
                if (gradient && lane == 0) mbarArrive(received_phi);
                epilogueSync();
                if (et == 0) {
                    const uint32_t own = gathered_s + static_cast<uint32_t>(2 * i * kBTile);
                    bulkToGlobal(store + static_cast<size_t>(2 * i) * kBTile, own, push_bytes);
                    bulkToGlobal(store_records + i * 4, records_s + static_cast<uint32_t>(16 * (kMaxRowBlocks + i)), 16);
                    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
                }
                if (gradient) {
                    clusterWait();
                    float band_top = 0.0f;
                    for (int peer = 0; peer < shape.cluster; ++peer) band_top = fmaxf(band_top, phi_max[peer]);
                    exp_m1 = planeExponentOf(band_top * f.gain_dy);
                    exp_m2 = planeExponentOf(band_top * f.gain_syw);
                    if (et == 0 && row_blocks > 1) {
                        const uint32_t src = gathered_s + static_cast<uint32_t>(2 * i * kBTile);
                        const uint32_t record = records_s + static_cast<uint32_t>(16 * (kMaxRowBlocks + i));
                        for (int peer_block = 0; peer_block < row_blocks; ++peer_block) {
                            if (peer_block == i) continue;
                            const uint32_t peer = static_cast<uint32_t>(peer_block * shares + h);
                            const uint32_t bar = clusterAddress(received_phi, peer);
                            bulkToPeer(clusterAddress(src, peer), src, push_bytes, bar);
                            bulkToPeer(clusterAddress(record, peer), record, 16, bar);
                        }
                        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
                    }
                }
            } else {
                // M1 = Dy phi_hat (pass 2) or M2 = Syw phi_hat (pass 3): planes with the band's exponent.
                const bool first = pass == 2;
                const int e = first ? exp_m1 : exp_m2;
                const double unscale = pow2(first ? exp_dy : exp_syw);
                const float inv_scale = static_cast<float>(pow2(-e));
                __half* hi = (first ? f.m1 : f.m2) + static_cast<size_t>(row) * f.m_ld + kx0;
                if (row_in) {
#pragma unroll
                    for (int j0 = 0; j0 < N; j0 += 8) {
                        float v[8];
#pragma unroll
                        for (int j = 0; j < 8; ++j) v[j] = static_cast<float>(acc[j0 + j] * unscale);
                        storeSplit8(v, inv_scale, hi + j0, hi + f.m_plane + j0);
                    }
                }
                if (rank == 0 && et == 0) (first ? f.m1_exp : f.m2_exp)[band] = e;
            }
        }
    }
    if (forward && gradient && warp < 2) clusterWait();
    // Every bulk copy this CTA issued has read its source and written its destination
    // (the kept phi_hat^T reaches global memory) before the grid completes.
    if (threadIdx.x == 64) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    if (local_block == 0 && threadIdx.x == 0 && f.clear != nullptr) *f.clear = 0u;
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 1) {
        const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(tmem_slot);
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemColumns));
    }
}

template <int N>
__global__ void __launch_bounds__(kFieldThreads, 1) fieldKernel(const __grid_constant__ FieldBand band, int mode) {
    releaseNext();
    const int cluster = band.shape.cluster;
    fieldBand<N>(band, static_cast<int>(blockIdx.x) / cluster, mode, static_cast<int>(blockIdx.x));
}

// Batched: cluster c computes band items[c].band of the grid items[c].field (a
// FieldBand in device memory, whose tensor maps the TMA reads there).
template <int N>
__global__ void __launch_bounds__(kFieldThreads, 1) fieldBatchKernel(const FieldItem* items, int cluster) {
    releaseNext();
    const FieldItem item = items[blockIdx.x / static_cast<unsigned>(cluster)];
    const FieldBand& band = *item.field;
    if (threadIdx.x == 0) {
        // The tensor maps live in global memory here (uploaded by a copy, possibly into
        // memory an earlier engine's maps used): make the TMA proxy see their current bytes.
        for (const CUtensorMap* map : {&band.map_s, &band.map_cx, &band.map_cy, &band.map_dy, &band.map_syw}) {
            asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(map) : "memory");
        }
    }
    fieldBand<N>(band, item.band, item.mode,
                 item.band * cluster + static_cast<int>(blockIdx.x % static_cast<unsigned>(cluster)));
}

template <int N>
void configureField() {
    constexpr int kMaxDevices = 64;
    static std::once_flag once[kMaxDevices];
    static cudaError_t attribute[kMaxDevices] = {};
    int device = 0;
    checkCuda(cudaGetDevice(&device), "Query the current device");
    require(device >= 0 && device < kMaxDevices, "Device index out of range.");
    std::call_once(once[device], [device] {
        attribute[device] =
            cudaFuncSetAttribute(fieldKernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, kFieldSmemBytes);
        if (attribute[device] == cudaSuccess) {
            attribute[device] =
                cudaFuncSetAttribute(fieldBatchKernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, kFieldSmemBytes);
        }
    });
    checkCuda(attribute[device], "Configure the banded field kernel");
}

cudaLaunchConfig_t fieldConfig(int blocks, int cluster, cudaStream_t stream, cudaLaunchAttribute* attribute) {
    cudaLaunchConfig_t config{};
    config.gridDim = dim3(static_cast<unsigned>(blocks));
    config.blockDim = dim3(kFieldThreads);
    config.dynamicSmemBytes = kFieldSmemBytes;
    config.stream = stream;
    attribute[0].id = cudaLaunchAttributeClusterDimension;
    attribute[0].val.clusterDim.x = static_cast<unsigned>(cluster);
    attribute[0].val.clusterDim.y = 1;
    attribute[0].val.clusterDim.z = 1;
    attribute[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attribute[1].val.programmaticStreamSerializationAllowed = 1;
    config.attrs = attribute;
    config.numAttrs = 2;
    return config;
}

void checkShape(const FieldShape& s) {
    require(s.cluster > 0 && s.cluster <= kMaxCluster && s.m_blocks <= kMaxRowBlocks && s.bands > 0 &&
                s.cluster == s.m_blocks * s.shares && s.share_n * s.shares == kBlockK,
            "The banded field solve does not take this grid.");
    require(s.share_n == 16 || s.share_n == 32, "The banded field solve takes shares of 16 or 32 columns.");
}

template <int N>
void launchFieldN(const FieldBand& band, int mode, cudaStream_t stream) {
    configureField<N>();
    cudaLaunchAttribute attribute[2] = {};
    const cudaLaunchConfig_t config = fieldConfig(band.shape.blocks(), band.shape.cluster, stream, attribute);
    checkCuda(cudaLaunchKernelEx(&config, fieldKernel<N>, band, mode), "Launch the banded field kernel");
}

template <int N>
void launchFieldBatchN(const FieldItem* items, int count, int cluster, cudaStream_t stream) {
    configureField<N>();
    cudaLaunchAttribute attribute[2] = {};
    const cudaLaunchConfig_t config = fieldConfig(count * cluster, cluster, stream, attribute);
    checkCuda(cudaLaunchKernelEx(&config, fieldBatchKernel<N>, items, cluster), "Launch the batched banded field kernel");
}

}  // namespace

FieldShape fieldShape(int nx, int ny) {
    FieldShape s;
    if (nx <= 0 || ny <= 0 || ny > kFieldMaxRows || nx > kFieldMaxColumns) return s;
    s.m_blocks = (ny + kTileM - 1) / kTileM;
    s.shares = s.m_blocks <= 2 ? 4 : 2;
    s.share_n = kBlockK / s.shares;
    s.cluster = s.m_blocks * s.shares;
    s.bands = (nx + kBlockK - 1) / kBlockK;
    return s;
}

size_t fieldStoreBytes(const FieldShape& shape) {
    // Per band and share: 2 m_blocks K-blocks of share_n x 64 halves, both planes.
    return static_cast<size_t>(shape.bands) * shape.shares * 2 * shape.m_blocks * kSplit * shape.share_n * kBlockK * 2;
}

size_t fieldRecordInts(const FieldShape& shape) {
    return static_cast<size_t>(shape.bands) * shape.shares * shape.m_blocks * 4;
}

void launchField(const FieldBand& band, FieldMode mode, cudaStream_t stream) {
    checkShape(band.shape);
    require(band.phi_store != nullptr && band.phi_records != nullptr, "The banded field solve needs its phi_hat store.");
    if (band.shape.share_n == 16) {
        launchFieldN<16>(band, mode, stream);
    } else {
        launchFieldN<32>(band, mode, stream);
    }
}

void launchFieldBatch(const FieldItem* items, int count, const FieldShape& shape, cudaStream_t stream) {
    if (count <= 0) return;
    checkShape(shape);
    if (shape.share_n == 16) {
        launchFieldBatchN<16>(items, count, shape.cluster, stream);
    } else {
        launchFieldBatchN<32>(items, count, shape.cluster, stream);
    }
}

}  // namespace mpgp
