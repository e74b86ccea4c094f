// Device-side design ingest (ingest.cu): the wirelength pass's bucketed net
// layout and the particle pin lists, built on the GPU from a Problem's pin CSR.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <functional>

#include "setup.hpp"

namespace mpgp {

// Device memory for the layout's lasting arrays (the engine's budgeted arena).
using DeviceAllocator = std::function<void*(std::size_t bytes, const char* what)>;
// Bytes the budget still allows (transient scratch counts against it while it lives).
using BudgetHeadroom = std::function<uint64_t()>;

struct NetLayout {
    int kept_nets = 0;            // nets with two or more pins, in bucket order
    int kept_pins = 0;
    int static_count = 0;
    int bucket_first[7] = {};     // first net of buckets 0..5; [6] = kept_nets
    int* net_start = nullptr;     // kept_nets + 1 pin offsets
    int* pin_particle = nullptr;  // particle, or -(static index) - 1
    float2* pin_offset = nullptr; // FP32 offset from the particle centre
    double2* static_pins = nullptr;
    float* net_weight = nullptr;  // FP32 (wirelength pass)
    double* net_weight64 = nullptr;  // FP64 (RUDY)
    int* particle_pin_start = nullptr;  // movable + 1
    int* pin_slot = nullptr;      // a pin's slot in its particle's range, -1 for static pins
};

NetLayout buildNetLayoutOnDevice(const Problem& problem, int movable, const DeviceAllocator& allocate,
                                 const BudgetHeadroom& headroom, cudaStream_t stream);

}  // namespace mpgp
