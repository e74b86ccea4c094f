// Shared definitions of the B200 global-placement engine (device and host).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>

#include "mpgp.h"

namespace mpgp {

// Engine failure carrying the C-ABI status it maps to.
class Error : public std::runtime_error {
public:
    Error(int status, const std::string& message) : std::runtime_error(message), status_(status) {}
    [[nodiscard]] int status() const { return status_; }

private:
    int status_;
};

[[noreturn]] inline void fail(int status, const std::string& message) { throw Error(status, message); }

inline void checkCuda(cudaError_t status, const char* what) {
    if (status != cudaSuccess) {
        fail(MPGP_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(status));
    }
}

inline void require(bool condition, const std::string& message) {
    if (!condition) fail(MPGP_ERR_INVALID_ARGUMENT, message);
}

// The literal form builds no string unless the check fails (validation loops run per pin).
inline void require(bool condition, const char* message) {
    if (!condition) fail(MPGP_ERR_INVALID_ARGUMENT, message);
}

// The library's device-memory pool of `device` (created once per device): the
// engines' arrays and set-up scratch are sub-allocated from it with stream-ordered
// allocation, and memory a finished session frees stays in the pool for the next
// session, instead of a cudaMalloc and cudaFree per array (each about 0.15 ms).
cudaMemPool_t devicePool(int device);

constexpr double kEpsilon = 1e-9;  // Geometry.hpp:8
constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr int kThreads = 256;
constexpr float kFixedOne = 4294967296.0f;  // 2^32: one bin area in fixed-point density units
constexpr double kFixedUnit = 1.0 / 4294967296.0;

inline int ceilDiv(long long value, long long divisor) {
    return static_cast<int>((value + divisor - 1) / divisor);
}

// ---- device helpers -------------------------------------------------------------------

#ifdef __CUDACC__

// Programmatic dependent launch.  A kernel started with launchChained may begin
// while its predecessor on the stream is still running: it releases its own
// successor with releaseNext() at entry, does work that reads nothing the
// predecessor writes, and calls waitForPrior() before the first access to the
// predecessor's results (griddepcontrol.wait returns once the predecessor grid
// has completed and its memory is visible).
__device__ __forceinline__ void waitForPrior() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void releaseNext() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

__device__ __forceinline__ double warpSum(double value) {
#pragma unroll
    for (int offset = 16; offset > 0; offset >>= 1) value += __shfl_xor_sync(0xffffffffu, value, offset);
    return value;
}

__device__ __forceinline__ double warpMax(double value) {
#pragma unroll
    for (int offset = 16; offset > 0; offset >>= 1) value = fmax(value, __shfl_xor_sync(0xffffffffu, value, offset));
    return value;
}

// Deterministic block reduction of K doubles (sum, or max where `is_max[k]`);
// thread 0 returns the result in `values`.  blockDim.x must be a multiple of 32, <= 1024.
template <int K>
__device__ __forceinline__ void blockReduce(double (&values)[K], const bool (&is_max)[K]) {
    __shared__ double scratch[K][32];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int warps = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        values[k] = is_max[k] ? warpMax(values[k]) : warpSum(values[k]);
        if (lane == 0) scratch[k][warp] = values[k];
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double v = lane < warps ? scratch[k][lane] : (is_max[k] ? -1.0e308 : 0.0);
            values[k] = is_max[k] ? warpMax(v) : warpSum(v);
        }
    }
    __syncthreads();
}

// atomicAdd with acquire-release semantics at GPU scope: the caller's earlier
// writes are visible to whoever observes the new count, and a caller that sees
// the final count sees every earlier writer's data.
__device__ __forceinline__ unsigned int atomicAddAcqRel(unsigned int* address, unsigned int value) {
    unsigned int old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(address), "r"(value) : "memory");
    return old;
}

// Second level of a deterministic grid reduction, called by every block after
// thread 0 wrote the block's K partials at partials[k * grid + block]
// (column-major; block / grid are the block's index and the block count of its
// launch, or of its instance in a batched launch): the last block of each group
// of 32 consecutive blocks reduces the group's rows (in block order) into
// group_partials[k * groups + group].  counters holds 1 + groups
// zeros and is left zeroed.  Returns 0 in most blocks, 1 in a block that
// finished a group, 2 in the block that finished the last group (after which
// every group row is visible to it).  Thread 0 does every global write and
// counter update, so its release / acquire atomics order all of them.
template <int K>
__device__ int reduceGroups(const double* partials, double* group_partials, unsigned int* counters,
                            const bool (&is_max)[K], unsigned int block, unsigned int grid) {
    __shared__ int state;
    __shared__ double folded[K];
    const unsigned int group = block / 32U;
    const unsigned int groups = (grid + 31U) / 32U;
    const unsigned int first = group * 32U;
    const unsigned int size = min(32U, grid - first);
    if (threadIdx.x == 0) state = atomicAddAcqRel(counters + 1 + group, 1U) == size - 1U ? 1 : 0;
    __syncthreads();
    if (state == 0) return 0;
    const unsigned int lane = threadIdx.x & 31U;
    const int warp = static_cast<int>(threadIdx.x >> 5);
    const int warps = static_cast<int>(blockDim.x >> 5);
    for (int k = warp; k < K; k += warps) {
        double x = is_max[k] ? -1.0e308 : 0.0;
        if (lane < size) x = __ldcg(partials + static_cast<size_t>(k) * grid + first + lane);
        x = is_max[k] ? warpMax(x) : warpSum(x);
        if (lane == 0) folded[k] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) group_partials[static_cast<size_t>(k) * groups + group] = folded[k];
        counters[1 + group] = 0U;
        state = atomicAddAcqRel(counters, 1U) == groups - 1U ? 2 : 1;
        if (state == 2) counters[0] = 0U;
    }
    __syncthreads();
    return state;
}

// Batched launches: the blocks of `count` instances one after another, instance k
// owning blocks [offsets[k], offsets[k + 1]).  Returns (instance, block within the
// instance, block count of the instance) for block `block` of the launch.
__device__ __forceinline__ int3 batchSlot(const int* offsets, int count, int block) {
    int lo = 0, hi = count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(offsets + mid) <= block) {
            lo = mid;
        } else {
            hi = mid - 1;
        }
    }
    const int first = __ldg(offsets + lo);
    return make_int3(lo, block - first, __ldg(offsets + lo + 1) - first);
}

__device__ __forceinline__ long long warpSumI64(long long value) {
#pragma unroll
    for (int offset = 16; offset > 0; offset >>= 1) value += __shfl_xor_sync(0xffffffffu, value, offset);
    return value;
}

#endif

// Launch with programmatic stream serialisation (see waitForPrior / releaseNext).
template <typename... Params, typename... Args>
inline void launchChained(const char* what, void (*kernel)(Params...), dim3 grid, dim3 block, size_t smem,
                          cudaStream_t stream, Args&&... args) {
    cudaLaunchConfig_t config{};
    config.gridDim = grid;
    config.blockDim = block;
    config.dynamicSmemBytes = smem;
    config.stream = stream;
    cudaLaunchAttribute attribute[1];
    attribute[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attribute[0].val.programmaticStreamSerializationAllowed = 1;
    config.attrs = attribute;
    config.numAttrs = 1;
    checkCuda(cudaLaunchKernelEx(&config, kernel, std::forward<Args>(args)...), what);
}

}  // namespace mpgp
