// Host check of the pool-offset scan (astrosimgpu_cuda_b200/csrc/pool_offsets.h),
// compiled with g++ by test_pool_offsets.py.  The builder finds every tape position
// where an astrocyte pool started there would need redraws, then scans them to find
// which posts' pools redraw.  Here the pools are drawn on the host with the model's
// counter RNG and the pool rule (5 distinct picks of nA astrocytes, redrawing a
// duplicate; src/astrosim_fused.cu:651-671), and the scan's offsets are compared
// with a sequential walk of the same pools, over random sizes, seeds and starts.
// Test infrastructure.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <random>
#include <vector>

#include "../astrosimgpu_cuda_b200/csrc/model.cuh"
#include "../astrosimgpu_cuda_b200/csrc/pool_offsets.h"

using namespace astrosim;

// One pool from tape position c (the rule for nA > 20); returns the draws used.
static u64 pool_draws(u64 seed, u32 n_astro, u64 c) {
    const u64 c0 = c;
    u32 pl[kPoolSize];
    u32 have = 0;
    while (have < kPoolSize) {
        const u32 cnd = static_cast<u32>(rng_uniform(seed, kSetupStream, c++) * static_cast<double>(n_astro)) % n_astro;
        bool dup = false;
        for (u32 k = 0; k < have; ++k) dup |= pl[k] == cnd;
        if (!dup) pl[have++] = cnd;
    }
    return c - c0;
}

int main(int argc, char** argv) {
    const int trials = argc > 1 ? std::atoi(argv[1]) : 200;
    std::mt19937_64 rng(3);
    long bad = 0, redrawing = 0;
    for (int trial = 0; trial < trials; ++trial) {
        const u32 n_posts = 50 + static_cast<u32>(rng() % 6000), n_astro = 21 + static_cast<u32>(rng() % 3000);
        const u64 seed = rng(), c0 = rng() % 100000;
        std::vector<u64> truth(n_posts);  // redraws of the pools before each post
        u64 c = c0, acc = 0;
        for (u32 q = 0; q < n_posts; ++q) {
            truth[q] = acc;
            const u64 used = pool_draws(seed, n_astro, c);
            acc += used - kPoolSize;
            c += used;
        }
        // every position a pool can start at, with the builder's margin
        const u64 n = static_cast<u64>(kPoolSize) * n_posts + 4096 + static_cast<u64>(n_posts * 40.0 / n_astro);
        std::vector<PoolRedrawAt> redraws;
        for (u64 i = 0; i < n; ++i) {
            const u64 used = pool_draws(seed, n_astro, c0 + i);
            if (used > kPoolSize) redraws.push_back(PoolRedrawAt{c0 + i, static_cast<uint32_t>(used - kPoolSize)});
        }
        std::vector<uint32_t> q, extra;
        pools_with_redraws(redraws, c0, kPoolSize, n_posts, q, extra);
        redrawing += static_cast<long>(q.size());
        std::vector<u64> got(n_posts, 0);
        u64 run = 0;
        size_t k = 0;
        for (u32 p = 0; p < n_posts; ++p) {
            got[p] = run;
            if (k < q.size() && q[k] == p) run += extra[k++];
        }
        if (got != truth) ++bad;
    }
    std::printf("trials %d mismatches %ld redrawing_posts %ld\n", trials, bad, redrawing);
    return bad != 0;
}
