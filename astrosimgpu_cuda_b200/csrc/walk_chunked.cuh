// walk_chunked.cuh -- one pre's walk over its postsynaptic block for the chunked
// parallel builder (builder_parallel.cu), on the precomputed skip cache.
//
// Device code, also compiled on the host by a CPU test (tests/walk_equivalence.cpp)
// that supplies __ldg and atomicOr, to show that the speculative end-position walk
// draws exactly what walk_pre draws.
#pragma once

#include "model.cuh"

namespace astrosim {

constexpr u32 kNoSelf = 0xFFFFFFFFu;  // no autapse rule for this walk

enum ErrBits : int {
    kErrCache = 1,     // a walk left the skip cache
    kErrHash = 2,      // claim table full
    kErrDelta = 4,     // an entry fell outside the candidate window
    kErrOrbit = 8      // materialised chunk did not meet its successor (internal)
};

struct Sec {
    u64 seed;
    const u32* cache;
    u64 cache_base, cache_len;
    int* err;
    u32 post_count, post_off;
    int third;
    u32 take;
    const u32* pool;
};

__device__ __forceinline__ u32 skip_at(const Sec& s, u64 t) {
    const u64 i = t - s.cache_base;
    if (i >= s.cache_len) {
        atomicOr(s.err, kErrCache);
        return 0xFFFFFFFFu;
    }
    return __ldg(s.cache + i);
}

// The skip at tape position t, loaded ahead of knowing whether the walk draws it
// (no error flag; the draw itself goes through skip_checked).
__device__ __forceinline__ u32 skip_peek(const Sec& s, u64 t) {
    const u64 i = t - s.cache_base;
    return i < s.cache_len ? __ldg(s.cache + i) : 0xFFFFFFFFu;
}

// Draws the skip at position t whose value was peeked: skip_at(s, t) without the load.
__device__ __forceinline__ u32 skip_checked(const Sec& s, u64 t, u32 peeked) {
    if (t - s.cache_base >= s.cache_len) {
        atomicOr(s.err, kErrCache);
        return 0xFFFFFFFFu;
    }
    return peeked;
}

// The third-factor test u < P_THIRD (src/astrosim_fused.cu:699) on the 53-bit integer m
// of u = m * 2^-53: u < P_THIRD exactly when m < kThirdLim = ceil(P_THIRD * 2^53)
// (the product is exact, a power-of-two scaling).
constexpr double kThirdScaled = kPThird * 9007199254740992.0;
constexpr u64 kThirdLim = static_cast<u64>(kThirdScaled) +
                          (static_cast<double>(static_cast<u64>(kThirdScaled)) < kThirdScaled ? 1u : 0u);

struct NoVisit {
    __device__ __forceinline__ void operator()(u32, bool, u32) const {}
};

// One pre's walk from tape position c (src/astrosim_fused.cu:688-707, 712-723).
// A landing on `self_post` is an autapse: no edge and no third-factor draws.
// Returns the tape position after the walk.  The draws and their order are the
// reference's; each post's next skip is loaded before its third-factor draws are
// hashed (both possible positions when the post has a third-factor test), so the
// cache load and the hash overlap instead of following each other.
template <class V>
__device__ __forceinline__ u64 walk_pre(const Sec& s, u64 c, u32 self_post, V& visit) {
    u32 pos = 0;
    const u32 n = s.post_count;
    if (n == 0) return c;
    u32 g = skip_at(s, c++);
    for (;;) {
        if (g >= n - pos) break;  // the skip reaches the end of the block
        pos += g;
        const u32 post = s.post_off + pos;
        ++pos;
        const bool more = pos < n;  // another skip is drawn after this post
        if (post == self_post) {
            if (!more) break;
            g = skip_at(s, c++);
            continue;
        }
        if (s.third) {
            const u32 g_miss = skip_peek(s, c + 1), g_hit = skip_peek(s, c + 2);
            const bool hit = (rng_bits(s.seed, kSetupStream, c++) >> 11) < kThirdLim;
            u32 astro = 0;
            if (hit) {
                const double u = rng_uniform(s.seed, kSetupStream, c++);
                astro = s.pool[static_cast<u64>(post) * kPoolSize +
                               static_cast<u32>(static_cast<u64>(u * static_cast<double>(s.take)) % s.take)];
            }
            visit(post, hit, astro);
            if (!more) break;
            g = skip_checked(s, c, hit ? g_hit : g_miss);
            ++c;
        } else {
            const u32 g_next = skip_peek(s, c);
            visit(post, false, 0u);
            if (!more) break;
            g = skip_checked(s, c, g_next);
            ++c;
        }
    }
    return c;
}

// The third-factor test at tape position t: u(t) < P_THIRD.
__device__ __forceinline__ bool third_hit(const Sec& s, u64 t) {
    return (rng_bits(s.seed, kSetupStream, t) >> 11) < kThirdLim;
}

// walk_pre for a walk that only needs the tape position it ends at, tuned for a
// single long walk per thread: while a post's third-factor test resolves, the tests
// of the next post at both positions it can take (one draw later if this test
// misses, two if it hits and a pool pick follows) are hashed too, so each post
// costs about the hashing throughput instead of a dependent hash latency.  It draws
// the same positions in the same order and returns walk_pre's result.
__device__ __forceinline__ u64 walk_pre_end(const Sec& s, u64 c, u32 self_post) {
    u32 pos = 0;
    const u32 n = s.post_count;
    if (n == 0) return c;
    u32 g = skip_at(s, c++);
    if (!s.third) {
        for (;;) {
            if (g >= n - pos) break;
            pos += g + 1;
            if (pos >= n) break;
            g = skip_at(s, c++);
        }
        return c;
    }
    bool hit_here = third_hit(s, c);  // c is the test position of the coming post
    for (;;) {
        if (g >= n - pos) break;  // the skip reaches the end of the block
        pos += g;
        const u32 post = s.post_off + pos;
        ++pos;
        const bool more = pos < n;
        if (post == self_post) {  // autapse: no draws; the next skip is at c
            if (!more) break;
            g = skip_at(s, c++);
            hit_here = third_hit(s, c);
            continue;
        }
        const u32 g_miss = skip_peek(s, c + 1), g_hit = skip_peek(s, c + 2);
        const bool next_miss = third_hit(s, c + 2), next_hit = third_hit(s, c + 3);
        const bool hit = hit_here;
        c += hit ? 2 : 1;  // the test, and the pool pick after a hit
        if (!more) break;
        g = skip_checked(s, c, hit ? g_hit : g_miss);
        ++c;
        hit_here = hit ? next_hit : next_miss;
    }
    return c;
}

}  // namespace astrosim
