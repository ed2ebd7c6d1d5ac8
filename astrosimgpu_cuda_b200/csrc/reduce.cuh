// reduce.cuh -- deterministic device reduction of the astrocyte summary
// (mean calcium, final-step threshold count, engaged count: src/astrosim_fused.cu:1111-1125).
#pragma once

#include "common.cuh"
#include "model.cuh"

namespace astrosim {

struct AstroPartial {
    double sum_ca;
    u32 active;
    u32 engaged;
};

struct AstroTotals {
    double sum_ca;
    double mean_ca;
    u32 active;
    u32 engaged;
};

constexpr u32 kReduceThreads = 256;
constexpr u32 kReduceItemsPerBlock = 2048;  // 8 per thread

inline u32 reduce_blocks(u32 n) { return n == 0 ? 1 : (n + kReduceItemsPerBlock - 1) / kReduceItemsPerBlock; }

// Enqueues the two reduction passes on `st`.  `partials` needs reduce_blocks(n)
// entries; `out` is device memory.  The summation order is fixed by n alone, so
// repeated calls give bit-identical results.
Status astro_totals(const double* ca, const unsigned char* engaged, u32 n, double sic_th, AstroPartial* partials,
                    AstroTotals* out, cudaStream_t st);

}  // namespace astrosim
