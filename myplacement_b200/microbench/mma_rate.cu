// tcgen05.mma issue rate on one SM: cycles per 128 x N x 16 fp16 MMA for N = 64, 128, 256.
// Standalone measurement behind the tile-shape choice of dct_tc.cu (not part of libmpgp.so):
//   nvcc -gencode arch=compute_100a,code=sm_100a -O3 -o mma_rate myplacement_b200/microbench/mma_rate.cu && ./mma_rate
// One CTA per SM, zeroed operands, every mbarrier wait bounded.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdio>
#include <cstdint>

__device__ __forceinline__ uint32_t smemAddress(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }
__device__ __forceinline__ uint64_t desc(uint32_t address) {
    return static_cast<uint64_t>((address >> 4) & 0x3FFFu) | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}
__device__ __forceinline__ void mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\ttcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                 ::"r"(tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

template <int N>
__global__ void __launch_bounds__(128, 1) mmaKernel(int count, unsigned long long* cycles, int* error) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    __shared__ uint64_t bar;
    __shared__ uint32_t slot;
    // A: 128 rows x 64 halves (16 KB), B: N rows x 64 halves; zero them (values do not matter).
    for (int i = threadIdx.x; i < (128 + N) * 128 / 4; i += blockDim.x) reinterpret_cast<uint32_t*>(smem)[i] = 0u;
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smemAddress(&slot)), "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 32) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smemAddress(&bar)));
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = slot;
    if (threadIdx.x == 0) {
        const uint32_t idesc = (1u << 4) | (uint32_t(N >> 3) << 17) | (uint32_t(128 >> 4) << 24);
        const uint32_t a = smemAddress(smem), b = a + 128 * 128;
        const unsigned long long t0 = clock64();
        for (int i = 0; i < count; ++i) {
            const int kk = i & 3;
            mma(tmem, desc(a + kk * 32), desc(b + kk * 32), idesc, i > 0 ? 1u : 0u);
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smemAddress(&bar)) : "memory");
        bool done = false;
        for (long it = 0; it < (1L << 24) && !done; ++it) {
            uint32_t d;
            asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\tselp.b32 %0, 1, 0, p;\n\t}" : "=r"(d) : "r"(smemAddress(&bar)) : "memory");
            done = d != 0;
        }
        if (!done) atomicExch(error, 1);
        const unsigned long long t1 = clock64();
        cycles[blockIdx.x] = t1 - t0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (threadIdx.x < 32) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
}

template <int N>
void run(int ctas, int count) {
    unsigned long long* d; int* err;
    cudaMalloc(&d, ctas * 8); cudaMalloc(&err, 4); cudaMemset(err, 0, 4);
    const int smem = 120 * 1024;  // one CTA per SM
    cudaFuncSetAttribute(mmaKernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    for (int rep = 0; rep < 3; ++rep) mmaKernel<N><<<ctas, 128, smem>>>(count, d, err);
    cudaError_t e = cudaDeviceSynchronize();
    unsigned long long h[256]; int herr = 0;
    cudaMemcpy(h, d, ctas * 8, cudaMemcpyDeviceToHost); cudaMemcpy(&herr, err, 4, cudaMemcpyDeviceToHost);
    double avg = 0; for (int i = 0; i < ctas; ++i) avg += h[i]; avg /= ctas;
    const double macs = 128.0 * N * 16.0;
    printf("N=%3d ctas=%3d count=%4d: %8.1f clk total, %6.1f clk/mma, %6.0f MAC/clk/SM (err %d, %s)\n", N, ctas, count, avg,
           avg / count, macs * count / avg, herr, cudaGetErrorString(e));
    cudaFree(d); cudaFree(err);
}

int main() {
    for (int count : {12, 48, 192}) {
        run<64>(1, count); run<128>(1, count); run<256>(1, count);
    }
    run<64>(148, 192); run<128>(148, 192); run<256>(148, 192);
    return 0;
}
