#pragma once

// Test-oracle build shim.  Placed ahead of the reference include tree when the
// reference is compiled as the oracle, it replaces the reference's shared-server
// allow-list (include/myplacement/placement/CudaDevicePolicy.hpp:8-10, devices
// 1-4 and 7) so that the reference CUDA backend can run on a single-GPU host,
// where the only device is 0.
namespace myplacement {

constexpr bool isPermittedCudaDevice(int device) {
    return device >= 0;
}

}  // namespace myplacement
