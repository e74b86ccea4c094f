// Inline PTX shared by the tcgen05 contraction kernels (dct_tc.cu, field_tc.cu):
// shared-memory and cluster addressing, mbarriers with bounded waits, TMA and
// shared-to-shared bulk copies, UMMA descriptors and issue, TMEM loads, and the
// plane split of eight values.
#pragma once

#include <cuda.h>
#include <cuda_fp16.h>

#include <cstdint>

#include "dct_tc.cuh"
#include "split.cuh"

namespace mpgp {
namespace tc {

// Polls of a bounded mbarrier wait before it gives up and raises the error flag.
constexpr long kSpinLimit = 1L << 22;

__device__ __forceinline__ uint32_t smemAddress(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint32_t clusterRank() {
    uint32_t rank;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(rank));
    return rank;
}

// Address of the same shared-memory offset in cluster CTA `rank`.
__device__ __forceinline__ uint32_t clusterAddress(uint32_t address, uint32_t rank) {
    uint32_t out;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(out) : "r"(address), "r"(rank));
    return out;
}

__device__ __forceinline__ void clusterArrive() {
    asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
}

__device__ __forceinline__ void clusterWait() {
    asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
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

// Bulk copy of `bytes` from this CTA's shared memory into a peer's (cluster
// addresses for the destination and its mbarrier).
__device__ __forceinline__ void bulkToPeer(uint32_t dst, uint32_t src, uint32_t bytes, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.shared::cta.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(dst), "r"(src), "r"(bytes), "r"(bar)
        : "memory");
}

// Bulk copy of `bytes` from global memory into this CTA's shared memory (completion on `bar`).
__device__ __forceinline__ void bulkFromGlobal(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(dst), "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// Bulk copy of `bytes` from this CTA's shared memory to global memory (bulk async group).
__device__ __forceinline__ void bulkToGlobal(void* dst, uint32_t src, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(src), "r"(bytes)
                 : "memory");
}

// UMMA shared-memory descriptor: K-major, 128-byte swizzle, 8-row groups 1024 B apart.
__device__ __forceinline__ uint64_t smemDescriptor(uint32_t address) {
    return static_cast<uint64_t>((address >> 4) & 0x3FFFu) | (1ull << 16) | (64ull << 32) | (1ull << 46) |
           (2ull << 61);
}

// Instruction descriptor: F16 x F16 -> F32, both K-major, M = 128, N = n (a multiple of 16).
constexpr uint32_t instrDescriptor(int n) {
    return (1u << 4) | (static_cast<uint32_t>(n >> 3) << 17) | (static_cast<uint32_t>(kTileM >> 4) << 24);
}

__device__ __forceinline__ void ummaF16(uint32_t tmem, uint64_t a, uint64_t b, uint32_t descriptor,
                                        uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem), "l"(a), "l"(b), "r"(descriptor), "r"(accumulate));
}

__device__ __forceinline__ void ummaCommit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

// Issues a 16-column TMEM load into raw registers; they hold the values only
// after tmemWait, which takes them as operands so that no use moves above it.
__device__ __forceinline__ void tmemLoad16(uint32_t address, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(address));
}

__device__ __forceinline__ void tmemWait(uint32_t (&a)[16], uint32_t (&b)[16]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15]), "+r"(b[0]), "+r"(b[1]), "+r"(b[2]), "+r"(b[3]), "+r"(b[4]), "+r"(b[5]), "+r"(b[6]), "+r"(b[7]), "+r"(b[8]), "+r"(b[9]), "+r"(b[10]), "+r"(b[11]), "+r"(b[12]), "+r"(b[13]), "+r"(b[14]), "+r"(b[15])
                 :
                 : "memory");
}

// Plane exponent of an output bounded by ref_max * gain.
__device__ __forceinline__ int planeExponent(const unsigned* ref_max, float gain) {
    return min(120, max(-120, exponentOf(__uint_as_float(*ref_max) * gain) - kPlaneTop));
}

// Eight consecutive values as two 16-byte plane stores (dst 16-byte aligned).
__device__ __forceinline__ void storeSplit8(const float (&v)[8], float inv_scale, __half* hi_dst, __half* lo_dst) {
    __half hi[8], lo[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) splitScaled(v[i], inv_scale, hi[i], lo[i]);
    *reinterpret_cast<uint4*>(hi_dst) = make_uint4(packHalves(hi[0], hi[1]), packHalves(hi[2], hi[3]),
                                                   packHalves(hi[4], hi[5]), packHalves(hi[6], hi[7]));
    *reinterpret_cast<uint4*>(lo_dst) = make_uint4(packHalves(lo[0], lo[1]), packHalves(lo[2], lo[3]),
                                                   packHalves(lo[4], lo[5]), packHalves(lo[6], lo[7]));
}

__device__ __forceinline__ double2 loadShared2(uint32_t address) {
    double2 v;
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(address));
    return v;
}

__device__ __forceinline__ void storeShared(uint32_t address, float v) {
    asm volatile("st.shared.f32 [%0], %1;" ::"r"(address), "f"(v) : "memory");
}

__device__ __forceinline__ float loadShared(uint32_t address) {
    float v;
    asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(address) : "memory");
    return v;
}

// Parseval weight of a DCT-II index: 1/2 for the DC term, 1 otherwise.
__device__ __forceinline__ double parsevalWeight(int index) { return index == 0 ? 0.5 : 1.0; }

}  // namespace tc
}  // namespace mpgp
