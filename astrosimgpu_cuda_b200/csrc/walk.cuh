// walk.cuh -- device pieces of the connectivity walk shared by the sequential and
// the chunked parallel builder: the geometric skip and the tie-break table for it.
#pragma once

#include "model.cuh"

namespace astrosim {

// The reference draws skips with the host C library's log1p
// (src/astrosim_fused.cu:617-624: floor(log1p(-u) / log1p(-p))).  The device
// evaluates the same formula with CUDA's log1p; the two can differ in the last
// bit, which moves the floor only when the quotient lies within a few ulps of an
// integer.  Such draws are "ambiguous": the device looks their tape position up
// in a small sorted table of host-computed values and, when the position is not
// there yet, logs it so the host can add it and the walk can be repeated.
struct SkipTable {
    const u64* pos = nullptr;     // sorted tape positions
    const double* val = nullptr;  // host floor value at each position
    int n = 0;
};

struct AmbiguityLog {
    u64* pos = nullptr;
    double* val = nullptr;  // the value the device used
    unsigned* count = nullptr;
    unsigned cap = 0;
};

// |q - rint(q)| below this many ulps of q marks a draw ambiguous.  CUDA's log1p and
// glibc's are each within 2 ulp of the true value, so two results differ by at most
// a handful of ulps; 64 ulps leaves a wide margin.
constexpr double kAmbiguityRel = 64.0 * 2.220446049250313e-16;

__device__ __forceinline__ double skip_value(u64 seed, double L, u64 t, const SkipTable& tab, const AmbiguityLog& amb) {
    double u = rng_uniform(seed, kSetupStream, t);
    if (u >= 1.0) u = nextafter(1.0, 0.0);
    const double q = log1p(-u) / L;
    double g = floor(q);
    const double r = rint(q);
    if (r != 0.0 && fabs(q - r) <= kAmbiguityRel * fabs(q)) {
        int lo = 0, hi = tab.n;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (tab.pos[mid] < t) lo = mid + 1; else hi = mid;
        }
        if (lo < tab.n && tab.pos[lo] == t) {
            g = tab.val[lo];
        } else if (amb.count) {
            const unsigned k = atomicAdd(amb.count, 1u);
            if (k < amb.cap) {
                amb.pos[k] = t;
                amb.val[k] = g;
            }
        }
    }
    return g;
}

// Host twin of the reference's formula, used to settle ambiguous draws.
inline double skip_value_host(u64 seed, double L, u64 t) {
    double u = rng_uniform(seed, kSetupStream, t);
    if (u >= 1.0) u = std::nextafter(1.0, 0.0);
    return std::floor(std::log1p(-u) / L);
}

}  // namespace astrosim
