// Two-plane fp16 operand split shared by the contraction kernels and the fused
// density-metrics pass: x * 2^-e = hi + 2^-11 lo with hi = fp16(x * 2^-e) and
// lo = fp16((x * 2^-e - hi) * 2^11).
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace mpgp {

// 2^e as a double (|e| < 1000), built from its exponent field.
__device__ __forceinline__ double pow2(int e) {
    return __longlong_as_double(static_cast<long long>(1023 + e) << 52);
}

// Smallest e with v <= 2^e for a positive finite v (0 otherwise).
__device__ __forceinline__ int exponentOf(float v) {
    if (!(v > 0.0f) || !isfinite(v)) return 0;
    int e = 0;
    const float m = frexpf(v, &e);  // v = m * 2^e, m in [0.5, 1)
    return m == 0.5f ? e - 1 : e;
}

constexpr float kLoShift = 2048.0f;  // 2^11: the lo plane's extra scale

// (hi, lo) planes of v * 2^-e.
__device__ __forceinline__ void splitScaled(float v, float inv_scale, __half& hi, __half& lo) {
    const float y = v * inv_scale;
    hi = __float2half_rn(y);
    lo = __float2half_rn((y - __half2float(hi)) * kLoShift);
}

__device__ __forceinline__ uint32_t packHalves(__half a, __half b) {
    return static_cast<uint32_t>(__half_as_ushort(a)) | (static_cast<uint32_t>(__half_as_ushort(b)) << 16);
}

}  // namespace mpgp
