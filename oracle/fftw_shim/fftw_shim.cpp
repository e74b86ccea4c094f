// Test-oracle infrastructure: never linked into the product library.
//
// FP64 implementation of the FFTW3 subset declared in fftw3.h.  The 1-D
// real-to-real transforms use Makhoul's length-N complex-FFT mapping of the
// DCT (J. Makhoul, "A fast cosine transform in one and two dimensions",
// IEEE Trans. ASSP 28(1), 1980), so the CPU oracle stays O(N^2 log N) per 2-D
// transform.  Power-of-two lengths use an iterative radix-2 FFT; any other
// length falls back to a direct DFT with an exact twiddle table.
#include "fftw3.h"

#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <new>
#include <stdexcept>
#include <vector>

namespace {

using cd = std::complex<double>;
constexpr double kPi = 3.141592653589793238462643383279502884;

bool isPowerOfTwo(int n) { return n > 0 && (n & (n - 1)) == 0; }

// e^{sign * 2 pi i k / n}, with k reduced mod n so the angle stays small.
cd unitRoot(long long k, int n, int sign) {
    const long long r = ((k % n) + n) % n;
    const double angle = 2.0 * kPi * static_cast<double>(r) / static_cast<double>(n);
    return {std::cos(angle), sign * std::sin(angle)};
}

// In-place unnormalized DFT: X_k = sum_j x_j e^{sign 2 pi i jk/n}.
void dft(std::vector<cd>& data, int sign) {
    const int n = static_cast<int>(data.size());
    if (n <= 1) return;
    if (isPowerOfTwo(n)) {
        for (int i = 1, j = 0; i < n; ++i) {
            int bit = n >> 1;
            for (; j & bit; bit >>= 1) j ^= bit;
            j ^= bit;
            if (i < j) std::swap(data[i], data[j]);
        }
        for (int length = 2; length <= n; length <<= 1) {
            const int half = length / 2;
            for (int start = 0; start < n; start += length) {
                for (int k = 0; k < half; ++k) {
                    const cd w = unitRoot(static_cast<long long>(k) * (n / length), n, sign);
                    const cd u = data[start + k];
                    const cd v = data[start + k + half] * w;
                    data[start + k] = u + v;
                    data[start + k + half] = u - v;
                }
            }
        }
        return;
    }
    std::vector<cd> output(static_cast<std::size_t>(n));
    for (int k = 0; k < n; ++k) {
        cd sum = 0.0;
        for (int j = 0; j < n; ++j) sum += data[j] * unitRoot(static_cast<long long>(j) * k, n, sign);
        output[k] = sum;
    }
    data.swap(output);
}

// DCT-II with FFTW's factor 2 (REDFT10).
void redft10(const double* in, double* out, int n, std::vector<cd>& work) {
    work.assign(static_cast<std::size_t>(n), 0.0);
    for (int j = 0; 2 * j < n; ++j) work[j] = in[2 * j];
    for (int j = 0; 2 * j + 1 < n; ++j) work[n - 1 - j] = in[2 * j + 1];
    dft(work, -1);
    for (int k = 0; k < n; ++k) {
        const double angle = -kPi * static_cast<double>(k) / (2.0 * n);
        const cd twiddle{std::cos(angle), std::sin(angle)};
        out[k] = 2.0 * (twiddle * work[k]).real();
    }
}

// DCT-III (REDFT01): the inverse Makhoul mapping, unnormalized.
void redft01(const double* in, double* out, int n, std::vector<cd>& work) {
    work.assign(static_cast<std::size_t>(n), 0.0);
    for (int k = 0; k < n; ++k) {
        const double mirrored = k == 0 ? 0.0 : in[n - k];
        const double angle = kPi * static_cast<double>(k) / (2.0 * n);
        work[k] = cd{std::cos(angle), std::sin(angle)} * cd{in[k], -mirrored};
    }
    dft(work, +1);
    for (int j = 0; 2 * j < n; ++j) out[2 * j] = work[j].real();
    for (int j = 0; 2 * j + 1 < n; ++j) out[2 * j + 1] = work[n - 1 - j].real();
}

// DST-III (RODFT01) = (-1)^k * DCT-III of the reversed input.
void rodft01(const double* in, double* out, int n, std::vector<cd>& work, std::vector<double>& scratch) {
    scratch.resize(static_cast<std::size_t>(n));
    for (int j = 0; j < n; ++j) scratch[j] = in[n - 1 - j];
    redft01(scratch.data(), out, n, work);
    for (int k = 1; k < n; k += 2) out[k] = -out[k];
}

void transform1d(fftw_r2r_kind kind, const double* in, double* out, int n, std::vector<cd>& work,
                 std::vector<double>& scratch) {
    switch (kind) {
        case FFTW_REDFT10: redft10(in, out, n, work); return;
        case FFTW_REDFT01: redft01(in, out, n, work); return;
        case FFTW_RODFT01: rodft01(in, out, n, work, scratch); return;
        default: throw std::invalid_argument("fftw shim: unsupported r2r kind");
    }
}

}  // namespace

struct fftw_plan_s {
    enum Type { R2R, R2C, C2R } type;
    int n0 = 0;
    int n1 = 0;
    fftw_r2r_kind kind0 = FFTW_REDFT10;
    fftw_r2r_kind kind1 = FFTW_REDFT10;
    double* real_in = nullptr;
    double* real_out = nullptr;
    fftw_complex* complex_in = nullptr;
    fftw_complex* complex_out = nullptr;
};

extern "C" {

double* fftw_alloc_real(size_t n) {
    return static_cast<double*>(std::aligned_alloc(64, ((n * sizeof(double) + 63) / 64) * 64 + 64));
}

fftw_complex* fftw_alloc_complex(size_t n) {
    return static_cast<fftw_complex*>(
        std::aligned_alloc(64, ((n * sizeof(fftw_complex) + 63) / 64) * 64 + 64));
}

void fftw_free(void* p) { std::free(p); }

fftw_plan fftw_plan_r2r_2d(int n0, int n1, double* in, double* out, fftw_r2r_kind kind0,
                           fftw_r2r_kind kind1, unsigned) {
    if (n0 <= 0 || n1 <= 0) return nullptr;
    auto* plan = new (std::nothrow) fftw_plan_s{};
    if (plan == nullptr) return nullptr;
    plan->type = fftw_plan_s::R2R;
    plan->n0 = n0;
    plan->n1 = n1;
    plan->kind0 = kind0;
    plan->kind1 = kind1;
    plan->real_in = in;
    plan->real_out = out;
    return plan;
}

fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double* in, fftw_complex* out, unsigned) {
    if (n0 <= 0 || n1 <= 0) return nullptr;
    auto* plan = new (std::nothrow) fftw_plan_s{};
    if (plan == nullptr) return nullptr;
    plan->type = fftw_plan_s::R2C;
    plan->n0 = n0;
    plan->n1 = n1;
    plan->real_in = in;
    plan->complex_out = out;
    return plan;
}

fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex* in, double* out, unsigned) {
    if (n0 <= 0 || n1 <= 0) return nullptr;
    auto* plan = new (std::nothrow) fftw_plan_s{};
    if (plan == nullptr) return nullptr;
    plan->type = fftw_plan_s::C2R;
    plan->n0 = n0;
    plan->n1 = n1;
    plan->complex_in = in;
    plan->real_out = out;
    return plan;
}

void fftw_execute(const fftw_plan plan) {
    const int n0 = plan->n0;
    const int n1 = plan->n1;
    const std::size_t count = static_cast<std::size_t>(n0) * static_cast<std::size_t>(n1);
    std::vector<cd> work;
    std::vector<double> scratch;
    if (plan->type == fftw_plan_s::R2R) {
        std::vector<double> stage(count);
        std::vector<double> line_in;
        std::vector<double> line_out;
        for (int r = 0; r < n0; ++r) {
            transform1d(plan->kind1, plan->real_in + static_cast<std::size_t>(r) * n1,
                        stage.data() + static_cast<std::size_t>(r) * n1, n1, work, scratch);
        }
        line_in.resize(static_cast<std::size_t>(n0));
        line_out.resize(static_cast<std::size_t>(n0));
        for (int c = 0; c < n1; ++c) {
            for (int r = 0; r < n0; ++r) line_in[r] = stage[static_cast<std::size_t>(r) * n1 + c];
            transform1d(plan->kind0, line_in.data(), line_out.data(), n0, work, scratch);
            for (int r = 0; r < n0; ++r) plan->real_out[static_cast<std::size_t>(r) * n1 + c] = line_out[r];
        }
        return;
    }
    const int half = n1 / 2 + 1;
    std::vector<cd> grid(count);
    if (plan->type == fftw_plan_s::R2C) {
        for (std::size_t i = 0; i < count; ++i) grid[i] = plan->real_in[i];
    } else {
        for (int r = 0; r < n0; ++r) {
            for (int c = 0; c < n1; ++c) {
                cd value;
                if (c < half) {
                    const fftw_complex& v = plan->complex_in[static_cast<std::size_t>(r) * half + c];
                    value = {v[0], v[1]};
                } else {
                    const int rr = (n0 - r) % n0;
                    const fftw_complex& v = plan->complex_in[static_cast<std::size_t>(rr) * half + (n1 - c)];
                    value = {v[0], -v[1]};
                }
                grid[static_cast<std::size_t>(r) * n1 + c] = value;
            }
        }
    }
    const int sign = plan->type == fftw_plan_s::R2C ? -1 : +1;
    std::vector<cd> line;
    for (int r = 0; r < n0; ++r) {
        line.assign(grid.begin() + static_cast<std::ptrdiff_t>(r) * n1,
                    grid.begin() + static_cast<std::ptrdiff_t>(r + 1) * n1);
        dft(line, sign);
        std::copy(line.begin(), line.end(), grid.begin() + static_cast<std::ptrdiff_t>(r) * n1);
    }
    line.resize(static_cast<std::size_t>(n0));
    for (int c = 0; c < n1; ++c) {
        for (int r = 0; r < n0; ++r) line[r] = grid[static_cast<std::size_t>(r) * n1 + c];
        dft(line, sign);
        for (int r = 0; r < n0; ++r) grid[static_cast<std::size_t>(r) * n1 + c] = line[r];
    }
    if (plan->type == fftw_plan_s::R2C) {
        for (int r = 0; r < n0; ++r) {
            for (int c = 0; c < half; ++c) {
                const cd value = grid[static_cast<std::size_t>(r) * n1 + c];
                plan->complex_out[static_cast<std::size_t>(r) * half + c][0] = value.real();
                plan->complex_out[static_cast<std::size_t>(r) * half + c][1] = value.imag();
            }
        }
    } else {
        for (std::size_t i = 0; i < count; ++i) plan->real_out[i] = grid[i].real();
    }
}

void fftw_destroy_plan(fftw_plan plan) { delete plan; }

}  // extern "C"
