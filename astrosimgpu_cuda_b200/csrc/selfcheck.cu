// selfcheck.cu -- device arithmetic self-checks behind astrosim_selfcheck_division.

#include <cmath>
#include <vector>

#include "common.cuh"
#include "model.cuh"

namespace astrosim {

namespace {

// Dividend k of divisor d: even k draws a random |x| in [2^-40, 2^40) with a random
// sign; odd k builds x = RN(y * m) for m the midpoint between two neighbouring
// doubles, so that x / y lands within a few ulp of a rounding boundary.
__global__ void div_check_kernel(const double* __restrict__ y, const double* __restrict__ ry, u32 n_div,
                                 u64 samples, u64 seed, unsigned long long* mismatches) {
    const u64 total = 2 * samples * n_div;
    unsigned long long bad = 0;
    for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<u64>(gridDim.x) * blockDim.x) {
        const u32 d = static_cast<u32>(i % n_div);
        const u64 k = i / n_div;
        const u64 bits = rng_mix(seed + k * kStreamMul);
        const u64 mant = bits & ((1ull << 52) - 1);
        const int e = static_cast<int>((bits >> 52) % 80) - 40;
        const double sign = (bits >> 63) ? -1.0 : 1.0;
        double x = sign * ldexp(1.0 + static_cast<double>(mant) * 0x1p-52, e);
        if (k & 1) {
            const double lo = x, h = 0.5 * (nextafter(x, 2.0 * x) - x);  // half an ulp of x, exact
            x = fma(y[d], lo, y[d] * h);  // RN(y * (lo + h)), one rounding: y * h is exact
            if (x == 0.0 || !isfinite(x)) continue;
        }
        const double want = x / y[d];
        const double got = div_by(x, y[d], ry[d]);
        if (__double_as_longlong(want) != __double_as_longlong(got)) ++bad;
    }
    if (bad) atomicAdd(mismatches, bad);
}

}  // namespace

Status selfcheck_division(int device, const double* divisors, size_t n, u64 samples, u64 seed, u64* mismatches) {
    if (!divisors || n == 0 || !mismatches) return make_error(ASTROSIM_ERR_INVALID_ARG, "null or empty argument");
    if (n > (1u << 20)) return make_error(ASTROSIM_ERR_INVALID_ARG, "at most 2^20 divisors");
    if (samples == 0 || samples > (1ull << 36)) return make_error(ASTROSIM_ERR_INVALID_ARG, "samples out of range");
    std::vector<double> y(divisors, divisors + n), ry(n);
    for (size_t i = 0; i < n; ++i) {
        if (!std::isfinite(y[i]) || y[i] == 0.0) return make_error(ASTROSIM_ERR_INVALID_ARG, "divisor %zu is zero or not finite", i);
        ry[i] = 1.0 / y[i];  // as the model's constants are made
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return make_error(ASTROSIM_ERR_NO_DEVICE, "no CUDA device visible");
    }
    if (device < 0 || device >= ndev) return make_error(ASTROSIM_ERR_INVALID_ARG, "device out of range");
    AS_CUDA(cudaSetDevice(device));
    cudaStream_t st = nullptr;
    AS_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    Status s = [&]() -> Status {
        AllocStream scope(st);
        DevBuf<double> dy, dry;
        DevBuf<unsigned long long> cnt;
        AS_TRY(dy.alloc(n));
        AS_TRY(dry.alloc(n));
        AS_TRY(cnt.alloc_zero(1, st));
        AS_CUDA(cudaMemcpyAsync(dy.get(), y.data(), n * sizeof(double), cudaMemcpyHostToDevice, st));
        AS_CUDA(cudaMemcpyAsync(dry.get(), ry.data(), n * sizeof(double), cudaMemcpyHostToDevice, st));
        int sms = 0;
        AS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        div_check_kernel<<<sms * 8, 256, 0, st>>>(dy.get(), dry.get(), static_cast<u32>(n), samples, seed, cnt.get());
        AS_CUDA(cudaGetLastError());
        unsigned long long h = 0;
        AS_CUDA(cudaMemcpyAsync(&h, cnt.get(), sizeof(h), cudaMemcpyDeviceToHost, st));
        AS_CUDA(cudaStreamSynchronize(st));
        *mismatches = h;
        return Status::Ok();
    }();
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    return s;
}

}  // namespace astrosim
