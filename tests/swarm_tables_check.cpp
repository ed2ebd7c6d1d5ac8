// Host check of the chunk-table bookkeeping of the warp swarms
// (astrosimgpu_cuda_b200/csrc/builder_parallel.cu: swarm_kernel, swarm_continue_kernel,
// swarm_resolve_kernel), compiled with g++ by test_swarm_tables.py.  A warp's 32 lanes
// are modelled in lockstep: each round every live walk claims its pre start in the
// chunk's table (or follows the walk that claimed it), idle lanes take the next
// candidates, and once every candidate has started and at most `handoff` walks are
// left they are walked to the chunk end without claims.  The resolved (exit, pres)
// of every candidate must equal a plain walk from it, for every merge order the
// rounds produce; the walks themselves are the builder's (walk_chunked.cuh, with host
// stand-ins for its two device intrinsics).  Test infrastructure: the GPU tests compare
// the device kernels with the one-CTA tables and the reference's connectivity.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

template <class T>
inline T __ldg(const T* p) { return *p; }
inline int atomicOr(int* p, int v) {
    const int o = *p;
    *p |= v;
    return o;
}

#include "../astrosimgpu_cuda_b200/csrc/walk_chunked.cuh"

using namespace astrosim;
using ull = unsigned long long;
constexpr ull kEmpty = ~0ull;
constexpr u32 kIdle = 0xFFFFFFFFu;
constexpr u32 kSlots = 4096;

struct Case {
    u32 posts;
    double landings;  // mean landings per pre
    int third;
    u32 chunk_len, delta, handoff;
};

// One chunk [T0, T0 + chunk_len): returns the number of candidates whose resolved
// table entry differs from the plain walk.
static long check_chunk(const Sec& s, const Case& k, u64 T0, std::mt19937_64& rng) {
    const u64 T1 = T0 + k.chunk_len;
    NoVisit nv;
    std::vector<ull> tab(kSlots, kEmpty);
    std::vector<int> par(k.delta, -7);
    std::vector<u32> mycnt(k.delta, 0), pcnt(k.delta, 0);
    std::vector<u64> ex(k.delta, 0);
    u32 w[32];
    u64 c[32];
    u32 cnt[32];
    bool claimed[32];
    for (u32 l = 0; l < 32; ++l) {
        w[l] = l < k.delta ? l : kIdle;
        c[l] = T0 + l;
        cnt[l] = 0;
    }
    u32 next = std::min(32u, k.delta);
    std::vector<u32> order(32);
    for (u32 l = 0; l < 32; ++l) order[l] = l;
    for (;;) {
        // claims, lanes in a random order each round (the atomics' order on the GPU)
        std::shuffle(order.begin(), order.end(), rng);
        for (u32 l : order) {
            claimed[l] = false;
            if (w[l] == kIdle) continue;
            if (c[l] >= T1) {
                par[w[l]] = -1;
                mycnt[w[l]] = cnt[l];
                ex[w[l]] = c[l];
                w[l] = kIdle;
                continue;
            }
            const u32 key = static_cast<u32>(c[l] - T0);
            u32 slot = (key * 2654435761u) & (kSlots - 1);
            const ull mine = (static_cast<ull>(key) << 32) | (static_cast<ull>(w[l]) << 22) | cnt[l];
            for (u32 probe = 0;; ++probe) {
                if (tab[slot] == kEmpty) {
                    tab[slot] = mine;
                    claimed[l] = true;
                    break;
                }
                if (static_cast<u32>(tab[slot] >> 32) == key) {
                    par[w[l]] = static_cast<int>((tab[slot] >> 22) & 0x3FFu);
                    pcnt[w[l]] = static_cast<u32>(tab[slot] & 0x3FFFFFu);
                    mycnt[w[l]] = cnt[l];
                    ex[w[l]] = c[l];
                    w[l] = kIdle;
                    break;
                }
                slot = (slot + 1) & (kSlots - 1);
                if (probe + 1 >= kSlots) {
                    std::printf("claim table full\n");
                    std::exit(2);
                }
            }
        }
        // refill
        u32 idle = 0, live = 0;
        for (u32 l = 0; l < 32; ++l)
            if (w[l] == kIdle) idle |= 1u << l;
        if (next < k.delta && idle) {
            for (u32 l = 0; l < 32; ++l) {
                const u32 rank = static_cast<u32>(__builtin_popcount(idle & ((1u << l) - 1u)));
                if (w[l] == kIdle && next + rank < k.delta) {
                    w[l] = next + rank;
                    c[l] = T0 + w[l];
                    cnt[l] = 0;
                }
            }
            next = std::min(k.delta, next + static_cast<u32>(__builtin_popcount(idle)));
        }
        for (u32 l = 0; l < 32; ++l)
            if (w[l] != kIdle) live |= 1u << l;
        if (live == 0) break;
        if (next >= k.delta && static_cast<u32>(__builtin_popcount(live)) <= k.handoff) {
            for (u32 l = 0; l < 32; ++l) {  // continuation: to the chunk end, no claims
                if (w[l] == kIdle) continue;
                u64 cc = c[l];
                u32 n = cnt[l];
                while (cc < T1) {
                    cc = walk_pre(s, cc, kNoSelf, nv);
                    ++n;
                }
                par[w[l]] = -1;
                mycnt[w[l]] = n;
                ex[w[l]] = cc;
            }
            break;
        }
        for (u32 l = 0; l < 32; ++l) {
            if (!claimed[l]) continue;
            c[l] = walk_pre(s, c[l], kNoSelf, nv);
            ++cnt[l];
        }
    }
    long bad = 0;
    for (u32 d = 0; d < k.delta; ++d) {  // resolve, then the plain walk
        u32 x = d;
        long long total = 0;
        for (u32 g = 0; par[x] >= 0; ++g) {
            if (g > k.delta) return k.delta;  // a cycle
            total += static_cast<long long>(mycnt[x]) - pcnt[x];
            x = static_cast<u32>(par[x]);
        }
        if (par[x] == -7) return k.delta;  // a candidate left unresolved
        total += mycnt[x];
        u64 cc = T0 + d;
        u32 n = 0;
        while (cc < T1) {
            cc = walk_pre(s, cc, kNoSelf, nv);
            ++n;
        }
        bad += (cc != ex[x] || n != static_cast<u32>(total));
    }
    return bad;
}

int main(int argc, char** argv) {
    const int chunks = argc > 1 ? std::atoi(argv[1]) : 6;
    // the three sections' shapes at N = 1e7 and at small N, with their hand-offs
    const Case cases[] = {
        {8000000, 64, 1, 32768, 384, 4}, {2000000, 16, 1, 4096, 192, 4}, {10000000, 80, 0, 8192, 192, 6},
        {1600, 64, 1, 2048, 384, 4},     {400, 16, 1, 2048, 192, 1},     {2000, 80, 0, 2048, 192, 8},
    };
    std::mt19937_64 rng(17);
    long walks = 0, bad = 0;
    for (const Case& k : cases) {
        const double p = k.landings / k.posts;
        const u64 len = 4ull * k.chunk_len;
        std::vector<u32> cache(len);
        std::vector<u32> pool(static_cast<size_t>(k.posts) * kPoolSize + 64, 3);
        for (int t = 0; t < chunks; ++t) {
            for (auto& v : cache) {
                const double u = static_cast<double>(rng() >> 11) * (1.0 / 9007199254740992.0);
                const double g = std::floor(std::log1p(-u) / std::log1p(-p));
                v = g >= 4294967295.0 ? 0xFFFFFFFFu : static_cast<u32>(g);
            }
            int err = 0;
            Sec s{};
            s.seed = rng();
            s.cache = cache.data();
            s.cache_base = 0;
            s.cache_len = len;
            s.err = &err;
            s.post_count = k.posts;
            s.post_off = 0;
            s.third = k.third;
            s.take = 5;
            s.pool = pool.data();
            bad += check_chunk(s, k, k.chunk_len, rng);
            walks += k.delta;
        }
    }
    std::printf("candidates %ld mismatches %ld\n", walks, bad);
    return bad != 0;
}
