// reduce.cu -- two-pass warp-shuffle reduction of the astrocyte summary.

#include "reduce.cuh"

namespace astrosim {

namespace {

__device__ __forceinline__ void warp_reduce(double& s, u32& a, u32& e) {
    for (int off = 16; off > 0; off >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, off);
        a += __shfl_down_sync(0xffffffffu, a, off);
        e += __shfl_down_sync(0xffffffffu, e, off);
    }
}

// Block b covers items [b * 2048, (b + 1) * 2048): each thread sums 8 strided items
// in order, warps reduce by shuffles, warp 0 combines the 8 warp results in order.
__global__ void __launch_bounds__(kReduceThreads) astro_partial_kernel(const double* __restrict__ ca,
                                                                       const unsigned char* __restrict__ engaged,
                                                                       u32 n, double sic_th, AstroPartial* part) {
    __shared__ double ws[kReduceThreads / 32];
    __shared__ u32 wa[kReduceThreads / 32], we[kReduceThreads / 32];
    const u32 base = blockIdx.x * kReduceItemsPerBlock;
    double s = 0.0;
    u32 a = 0, e = 0;
    for (u32 i = threadIdx.x; i < kReduceItemsPerBlock; i += kReduceThreads) {
        const u32 k = base + i;
        if (k < n) {
            const double v = ca[k];
            s += v;
            a += ((v - sic_th) * 1000.0 > 1.0) ? 1u : 0u;
            e += engaged[k] ? 1u : 0u;
        }
    }
    warp_reduce(s, a, e);
    const u32 warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        ws[warp] = s;
        wa[warp] = a;
        we[warp] = e;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ts = 0.0;
        u32 ta = 0, te = 0;
        for (u32 w = 0; w < kReduceThreads / 32; ++w) {
            ts += ws[w];
            ta += wa[w];
            te += we[w];
        }
        part[blockIdx.x] = AstroPartial{ts, ta, te};
    }
}

__global__ void __launch_bounds__(kReduceThreads) astro_final_kernel(const AstroPartial* __restrict__ part,
                                                                     u32 n_parts, u32 n, AstroTotals* out) {
    __shared__ double ws[kReduceThreads / 32];
    __shared__ u32 wa[kReduceThreads / 32], we[kReduceThreads / 32];
    double s = 0.0;
    u32 a = 0, e = 0;
    for (u32 i = threadIdx.x; i < n_parts; i += kReduceThreads) {
        s += part[i].sum_ca;
        a += part[i].active;
        e += part[i].engaged;
    }
    warp_reduce(s, a, e);
    const u32 warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        ws[warp] = s;
        wa[warp] = a;
        we[warp] = e;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ts = 0.0;
        u32 ta = 0, te = 0;
        for (u32 w = 0; w < kReduceThreads / 32; ++w) {
            ts += ws[w];
            ta += wa[w];
            te += we[w];
        }
        out->sum_ca = ts;
        out->mean_ca = ts / static_cast<double>(n > 0 ? n : 1u);  // src/astrosim_fused.cu:1119
        out->active = ta;
        out->engaged = te;
    }
}

}  // namespace

Status astro_totals(const double* ca, const unsigned char* engaged, u32 n, double sic_th, AstroPartial* partials,
                    AstroTotals* out, cudaStream_t st) {
    const u32 nb = reduce_blocks(n);
    astro_partial_kernel<<<nb, kReduceThreads, 0, st>>>(ca, engaged, n, sic_th, partials);
    AS_CUDA(cudaGetLastError());
    astro_final_kernel<<<1, kReduceThreads, 0, st>>>(partials, nb, n, out);
    AS_CUDA(cudaGetLastError());
    return Status::Ok();
}

}  // namespace astrosim
