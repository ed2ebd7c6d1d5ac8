// builder_internal.cuh -- pieces shared by the sequential and parallel builders.
#pragma once

#include "common.cuh"
#include "model.cuh"
#include "network.cuh"

namespace astrosim {

// Edge lists in the reference's emission order (src/astrosim_fused.cu:697-721).
struct EdgeLists {
    u32 *exc_src, *exc_dst;
    u32 *inh_src, *inh_dst;
    u32 *e2a_src, *e2a_dst;
    u32 *sic_src, *sic_dst;
    u64 cap_exc, cap_inh, cap_third;
    unsigned long long* counts;  // exc, inh, third-factor, end tape position
};

struct EdgeStorage {
    DevBuf<u32> exc_src, exc_dst, inh_src, inh_dst, e2a_src, e2a_dst, sic_src, sic_dst;
    DevBuf<unsigned long long> counts;
    u64 cap_exc = 0, cap_inh = 0, cap_third = 0;
    EdgeLists view();
};

Status alloc_edge_lists(const Sizes& sz, EdgeStorage& s, cudaStream_t st);
// Sorts the lists into the four CSRs.  counts: exc, inh, e2a, sic list lengths; the
// destinations are row indices of net.own (cell - lo), and the CSRs get the rows of
// the owned cells.  The source lists and the e2a and sic target lists are used as
// sort buffers (their contents are lost); the exc and inh target lists survive.
Status edge_lists_to_network(const EdgeLists& e, const u64 counts[4], Network& net, cudaStream_t st);
// Keeps rows [lo, hi) of a CSR (row r of the result is row lo + r of the input).
Status slice_csr(DeviceCSR& c, u32 lo, u32 hi, cudaStream_t st);

// Astrocyte pool of one postsynaptic neuron read from tape position c
// (src/astrosim_fused.cu:651-671); advances c past the draws it used.
__device__ __forceinline__ void pool_one(u64 seed, u32 n_astro, u64& c, u32* pl) {
    const u32 take = n_astro < kPoolSize ? n_astro : kPoolSize;
    if (take > 0 && static_cast<u64>(take) * 4 >= n_astro) {
        // exact partial shuffle (only reached when n_astro <= 20)
        u32 cand[20];
        for (u32 i = 0; i < n_astro; ++i) cand[i] = i;
        for (u32 k = 0; k < take; ++k) {
            const double u = rng_uniform(seed, kSetupStream, c++);
            const u64 pick = static_cast<u64>(u * static_cast<double>(n_astro - k)) + k;
            const u64 j = pick < n_astro - 1 ? pick : n_astro - 1;
            const u32 tmp = cand[k];
            cand[k] = cand[j];
            cand[j] = tmp;
            pl[k] = cand[k];
        }
    } else {
        u32 have = 0;
        while (have < take) {
            const u32 cnd =
                static_cast<u32>(rng_uniform(seed, kSetupStream, c++) * static_cast<double>(n_astro)) % n_astro;
            bool dup = false;
            for (u32 q = 0; q < have; ++q)
                if (pl[q] == cnd) dup = true;
            if (!dup) pl[have++] = cnd;
        }
    }
}

__device__ __forceinline__ void pools_sequential(u64 seed, u32 n_neurons, u32 n_astro, u64& c, u32* pool) {
    for (u32 post = 0; post < n_neurons; ++post) pool_one(seed, n_astro, c, pool + static_cast<u64>(post) * kPoolSize);
}

// Phase timing of the build, printed to stderr when ASTROSIM_TIMING is set.
struct PhaseClock {
    bool on;
    cudaStream_t st;
    double t0;
    explicit PhaseClock(cudaStream_t s);
    void mark(const char* what);
    // Prints the time since t (a PhaseClock::now() reading) under the same switch.
    void mark_since(const char* what, double t);
    static double now();
};

Status build_sequential(const Sizes& sz, u64 seed, u64 c0, Network& net, cudaStream_t st);
Status build_parallel(const Sizes& sz, u64 seed, u64 c0, Network& net, cudaStream_t st);
// The per-cell parameter buffers of net (on this thread's allocation stream), then
// their draws on stream st (src/astrosim_fused.cu:917-933).  The draws touch no other
// member of net.
Status alloc_cell_parameters(const Sizes& sz, Network& net);
Status draw_cell_parameters(const Sizes& sz, u64 seed, const Biology& bio, Network& net, cudaStream_t st);

}  // namespace astrosim
