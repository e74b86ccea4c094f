// Device-side design ingest: the wirelength pass's net layout and the particle
// pin lists, built on the GPU from the flat pin CSR (buildHostLayout,
// CudaPlacementBackend.cu:784-839, produces the same CSR on the host).
//
//   1. every net's degree bucket (one thread per net): 2, <= 4, <= 8, <= 16,
//      <= 32, larger; nets with fewer than two pins are dropped;
//   2. a stable radix sort of the nets by bucket (CUB): nets keep their order
//      within a bucket, so the layout equals the host layout net for net;
//   3. an exclusive scan of the kept degrees gives the bucketed net offsets;
//      one thread per net copies its pins (particle, FP32 offset; static pins
//      keep their absolute FP64 position) and weights;
//   4. a scan of the static-pin flags numbers the static pins in layout order;
//   5. a stable radix sort of the pins by particle gives every movable pin its
//      gradient slot: a particle's pins own a contiguous range, in ascending
//      layout order, which the gather reads in a fixed order.
// Every step is deterministic (stable sorts, integer scans and counts).
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "ingest.cuh"

namespace mpgp {
namespace {

constexpr int kExcluded = 6;  // the bucket key of nets with fewer than two pins

__device__ __forceinline__ int bucketOf(long long degree) {
    if (degree < 2) return kExcluded;
    return degree <= 2 ? 0 : degree <= 4 ? 1 : degree <= 8 ? 2 : degree <= 16 ? 3 : degree <= 32 ? 4 : 5;
}

__global__ void netKeysKernel(const long long* net_pin_start, int nets, int* keys, int* values) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nets) return;
    keys[n] = bucketOf(net_pin_start[n + 1] - net_pin_start[n]);
    values[n] = n;
}

// Kept degree per sorted net and the first sorted position of every bucket.
__global__ void sortedNetsKernel(const long long* net_pin_start, const int* keys, const int* order, int nets,
                                 int* degree, int* bucket_first) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nets) return;
    const int key = keys[k];
    const int n = order[k];
    degree[k] = key == kExcluded ? 0 : static_cast<int>(net_pin_start[n + 1] - net_pin_start[n]);
    if (k == 0 || keys[k - 1] != key) bucket_first[key] = k;
}

__global__ void copyPinsKernel(const long long* net_pin_start, const int* order, const int* net_start, int kept,
                               const int* pin_particle, const double* pin_x, const double* pin_y,
                               const double* net_weight, int movable, int* out_particle, float2* out_offset,
                               double2* out_static, int* is_static, float* out_weight, double* out_weight64,
                               int* error) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= kept) return;
    const int n = order[k];
    const long long src = net_pin_start[n];
    const int dst = net_start[k];
    const int degree = net_start[k + 1] - dst;
    for (int j = 0; j < degree; ++j) {
        const int particle = pin_particle[src + j];
        if (particle >= movable) atomicExch(error, 1);
        const double x = pin_x[src + j];
        const double y = pin_y[src + j];
        out_particle[dst + j] = particle;
        out_offset[dst + j] = particle >= 0 ? make_float2(static_cast<float>(x), static_cast<float>(y))
                                            : make_float2(0.0f, 0.0f);
        out_static[dst + j] = make_double2(x, y);
        is_static[dst + j] = particle < 0 ? 1 : 0;
    }
    out_weight[k] = static_cast<float>(net_weight[n]);
    out_weight64[k] = net_weight[n];
}

// Static pins get their number in layout order; the particle sort keys are the
// particle (movable pins) or `movable` (static pins, sorted last).
__global__ void numberStaticKernel(int pins, const int* is_static, const int* static_index,
                                   const double2* staged_static, int movable, int* out_particle,
                                   double2* static_pins, int* particle_keys, int* pin_index, int* counts) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pins) return;
    if (is_static[i]) {
        const int s = static_index[i];
        out_particle[i] = -s - 1;
        static_pins[s] = staged_static[i];
        particle_keys[i] = movable;
    } else {
        const int particle = out_particle[i];
        particle_keys[i] = particle;
        atomicAdd(counts + particle, 1);
    }
    pin_index[i] = i;
}

__global__ void slotsKernel(int pins, const int* sorted_keys, const int* sorted_pins, int movable, int* slot) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pins) return;
    // The movable pins take slots 0 .. (movable pins - 1), in particle order.
    slot[sorted_pins[i]] = sorted_keys[i] < movable ? i : -1;
}

int blocksFor(long long count) { return std::max(1, ceilDiv(std::max(1LL, count), kThreads)); }

int bitsFor(int value) {
    int bits = 1;
    while (bits < 31 && (1LL << bits) <= value) ++bits;
    return bits;
}

// Stream-ordered scratch, released when the ingest returns.  While it lives it
// counts against the engine's device-memory budget like the lasting arrays.
class Scratch {
public:
    Scratch(cudaStream_t stream, const BudgetHeadroom& headroom) : stream_(stream), headroom_(headroom) {}
    ~Scratch() {
        for (void* p : blocks_) cudaFreeAsync(p, stream_);
    }
    // Fails unless `bytes` more fit in the budget beside the scratch held now.
    void check(std::size_t bytes) const {
        if (held_ + bytes > headroom_()) {
            fail(MPGP_ERR_BUDGET, "CUDA allocation budget exceeded while ingesting the design.");
        }
    }
    template <typename T>
    T* array(std::size_t count) {
        const std::size_t bytes = std::max<std::size_t>(1, count) * sizeof(T);
        check(bytes);
        void* p = nullptr;
        int device = 0;
        checkCuda(cudaGetDevice(&device), "Query the current device");
        checkCuda(cudaMallocFromPoolAsync(&p, bytes, devicePool(device), stream_), "ingest scratch");
        blocks_.push_back(p);
        held_ += bytes;
        return static_cast<T*>(p);
    }

private:
    cudaStream_t stream_;
    const BudgetHeadroom& headroom_;
    std::vector<void*> blocks_;
    uint64_t held_ = 0;
};

template <typename T>
void uploadVector(T* device, const std::vector<T>& host, cudaStream_t stream) {
    if (!host.empty()) {
        checkCuda(cudaMemcpyAsync(device, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice, stream),
                  "ingest upload");
    }
}

}  // namespace

NetLayout buildNetLayoutOnDevice(const Problem& p, int movable, const DeviceAllocator& lasting,
                                 const BudgetHeadroom& headroom, cudaStream_t stream) {
    const int nets = static_cast<int>(p.net_weight.size());
    const int pins_in = static_cast<int>(p.pin_particle.size());
    NetLayout out;
    Scratch scratch(stream, headroom);
    // The layout's lasting arrays, checked against the budget beside the scratch.
    const auto allocate = [&](std::size_t bytes, const char* what) {
        scratch.check(bytes);
        return lasting(bytes, what);
    };

    // The flat CSR on the device.
    long long* net_pin_start = scratch.array<long long>(static_cast<std::size_t>(nets) + 1);
    int* pin_particle = scratch.array<int>(static_cast<std::size_t>(pins_in));
    double* pin_x = scratch.array<double>(static_cast<std::size_t>(pins_in));
    double* pin_y = scratch.array<double>(static_cast<std::size_t>(pins_in));
    double* weight = scratch.array<double>(static_cast<std::size_t>(nets));
    static_assert(sizeof(long long) == sizeof(int64_t), "64-bit offsets");
    checkCuda(cudaMemcpyAsync(net_pin_start, p.net_pin_start.data(), (static_cast<std::size_t>(nets) + 1) * 8,
                              cudaMemcpyHostToDevice, stream),
              "ingest upload");
    uploadVector(pin_particle, p.pin_particle, stream);
    uploadVector(pin_x, p.pin_x, stream);
    uploadVector(pin_y, p.pin_y, stream);
    uploadVector(weight, p.net_weight, stream);

    // 1-2: buckets, stable sort of the nets.
    int* keys = scratch.array<int>(static_cast<std::size_t>(nets));
    int* values = scratch.array<int>(static_cast<std::size_t>(nets));
    int* sorted_keys = scratch.array<int>(static_cast<std::size_t>(nets));
    int* order = scratch.array<int>(static_cast<std::size_t>(nets));
    int* degree = scratch.array<int>(static_cast<std::size_t>(nets) + 1);
    int* bucket_first = scratch.array<int>(8);
    int* error = scratch.array<int>(1);
    checkCuda(cudaMemsetAsync(bucket_first, 0xff, 8 * sizeof(int), stream), "ingest");
    checkCuda(cudaMemsetAsync(error, 0, sizeof(int), stream), "ingest");
    if (nets > 0) {
        netKeysKernel<<<blocksFor(nets), kThreads, 0, stream>>>(net_pin_start, nets, keys, values);
        std::size_t bytes = 0;
        checkCuda(cub::DeviceRadixSort::SortPairs(nullptr, bytes, keys, sorted_keys, values, order, nets, 0, 3, stream),
                  "net sort size");
        void* temp = scratch.array<unsigned char>(bytes);
        checkCuda(cub::DeviceRadixSort::SortPairs(temp, bytes, keys, sorted_keys, values, order, nets, 0, 3, stream),
                  "net sort");
        sortedNetsKernel<<<blocksFor(nets), kThreads, 0, stream>>>(net_pin_start, sorted_keys, order, nets, degree,
                                                                   bucket_first);
        checkCuda(cudaGetLastError(), "Launch the net ordering");
    }
    checkCuda(cudaMemsetAsync(degree + nets, 0, sizeof(int), stream), "ingest");

    // 3: bucketed net offsets (prefix sums of the kept degrees).
    out.net_start = static_cast<int*>(allocate((static_cast<std::size_t>(nets) + 1) * sizeof(int), "net offsets"));
    {
        std::size_t bytes = 0;
        checkCuda(cub::DeviceScan::ExclusiveSum(nullptr, bytes, degree, out.net_start, nets + 1, stream), "scan size");
        void* temp = scratch.array<unsigned char>(bytes);
        checkCuda(cub::DeviceScan::ExclusiveSum(temp, bytes, degree, out.net_start, nets + 1, stream), "net scan");
    }
    int host_first[8];
    int host_total = 0;
    checkCuda(cudaMemcpyAsync(host_first, bucket_first, sizeof(host_first), cudaMemcpyDeviceToHost, stream), "ingest");
    checkCuda(cudaMemcpyAsync(&host_total, out.net_start + nets, sizeof(int), cudaMemcpyDeviceToHost, stream),
              "ingest");
    checkCuda(cudaStreamSynchronize(stream), "net layout");
    // Buckets that are empty start where the next non-empty one does.
    host_first[7] = nets;
    for (int b = kExcluded; b >= 0; --b) {
        if (host_first[b] < 0) host_first[b] = host_first[b + 1];
    }
    for (int b = 0; b <= kExcluded; ++b) out.bucket_first[b] = host_first[b];
    out.kept_nets = host_first[kExcluded];
    out.kept_pins = host_total;

    // 3 (cont.): the pins, weights and static positions in layout order.
    const std::size_t pins = static_cast<std::size_t>(std::max(1, out.kept_pins));
    out.pin_particle = static_cast<int*>(allocate(pins * sizeof(int), "pin particles"));
    out.pin_offset = static_cast<float2*>(allocate(pins * sizeof(float2), "pin offsets"));
    out.net_weight = static_cast<float*>(allocate(std::max<std::size_t>(1, out.kept_nets) * sizeof(float), "net weights"));
    out.net_weight64 =
        static_cast<double*>(allocate(std::max<std::size_t>(1, out.kept_nets) * sizeof(double), "net weights"));
    double2* staged_static = scratch.array<double2>(pins);
    int* is_static = scratch.array<int>(pins + 1);
    int* static_index = scratch.array<int>(pins + 1);
    checkCuda(cudaMemsetAsync(is_static + out.kept_pins, 0, sizeof(int), stream), "ingest");
    if (out.kept_nets > 0) {
        copyPinsKernel<<<blocksFor(out.kept_nets), kThreads, 0, stream>>>(
            net_pin_start, order, out.net_start, out.kept_nets, pin_particle, pin_x, pin_y, weight, movable,
            out.pin_particle, out.pin_offset, staged_static, is_static, out.net_weight, out.net_weight64, error);
        checkCuda(cudaGetLastError(), "Launch the pin copy");
    }

    // 4: number the static pins.
    {
        std::size_t bytes = 0;
        checkCuda(cub::DeviceScan::ExclusiveSum(nullptr, bytes, is_static, static_index, out.kept_pins + 1, stream),
                  "scan size");
        void* temp = scratch.array<unsigned char>(bytes);
        checkCuda(cub::DeviceScan::ExclusiveSum(temp, bytes, is_static, static_index, out.kept_pins + 1, stream),
                  "static scan");
    }
    int host_static = 0, host_error = 0;
    checkCuda(cudaMemcpyAsync(&host_static, static_index + out.kept_pins, sizeof(int), cudaMemcpyDeviceToHost, stream),
              "ingest");
    checkCuda(cudaMemcpyAsync(&host_error, error, sizeof(int), cudaMemcpyDeviceToHost, stream), "ingest");
    checkCuda(cudaStreamSynchronize(stream), "net layout");
    require(host_error == 0, "A pin refers to a non-movable particle.");
    out.static_count = host_static;
    out.static_pins = static_cast<double2*>(
        allocate(std::max<std::size_t>(1, static_cast<std::size_t>(host_static)) * sizeof(double2), "static pins"));

    // 5: gradient slots, a stable sort of the pins by particle.
    out.particle_pin_start =
        static_cast<int*>(allocate((static_cast<std::size_t>(movable) + 1) * sizeof(int), "particle pin offsets"));
    out.pin_slot = static_cast<int*>(allocate(pins * sizeof(int), "pin gradient slots"));
    int* particle_keys = scratch.array<int>(pins);
    int* pin_index = scratch.array<int>(pins);
    int* sorted_particles = scratch.array<int>(pins);
    int* sorted_pins = scratch.array<int>(pins);
    int* counts = scratch.array<int>(static_cast<std::size_t>(movable) + 1);
    checkCuda(cudaMemsetAsync(counts, 0, (static_cast<std::size_t>(movable) + 1) * sizeof(int), stream), "ingest");
    if (out.kept_pins > 0) {
        numberStaticKernel<<<blocksFor(out.kept_pins), kThreads, 0, stream>>>(
            out.kept_pins, is_static, static_index, staged_static, movable, out.pin_particle, out.static_pins,
            particle_keys, pin_index, counts);
        checkCuda(cudaGetLastError(), "Launch the static numbering");
        std::size_t bytes = 0;
        const int bits = bitsFor(movable);
        checkCuda(cub::DeviceRadixSort::SortPairs(nullptr, bytes, particle_keys, sorted_particles, pin_index,
                                                  sorted_pins, out.kept_pins, 0, bits, stream),
                  "pin sort size");
        void* temp = scratch.array<unsigned char>(bytes);
        checkCuda(cub::DeviceRadixSort::SortPairs(temp, bytes, particle_keys, sorted_particles, pin_index, sorted_pins,
                                                  out.kept_pins, 0, bits, stream),
                  "pin sort");
        slotsKernel<<<blocksFor(out.kept_pins), kThreads, 0, stream>>>(out.kept_pins, sorted_particles, sorted_pins,
                                                                       movable, out.pin_slot);
        checkCuda(cudaGetLastError(), "Launch the slot assignment");
    }
    {
        std::size_t bytes = 0;
        checkCuda(cub::DeviceScan::ExclusiveSum(nullptr, bytes, counts, out.particle_pin_start, movable + 1, stream),
                  "scan size");
        void* temp = scratch.array<unsigned char>(bytes);
        checkCuda(cub::DeviceScan::ExclusiveSum(temp, bytes, counts, out.particle_pin_start, movable + 1, stream),
                  "particle scan");
    }
    checkCuda(cudaStreamSynchronize(stream), "net layout");
    return out;
}

}  // namespace mpgp
