// pool_offsets.h -- which posts' astrocyte pools need redraws, from the tape
// positions where a pool would need them (host code, no CUDA; also compiled by a CPU
// test, tests/pool_offsets_check.cpp).
//
// The pools of posts 0 .. n_posts - 1 lie end to end on the tape from c0: pool q
// takes `take` draws plus its redraws (src/astrosim_fused.cu:651-671), so it starts at
// c0 + take * q + (the redraws of the pools before it).  Given every position t at
// which a pool started there would need redraws, with their number, sorted by t,
// walking them in order with the running shift finds the posts whose pool redraws.
#pragma once

#include <cstdint>
#include <vector>

namespace astrosim {

struct PoolRedrawAt {
    uint64_t t;       // tape position a pool would start at
    uint32_t extra;   // its redraws
};

// Appends to q / extra the posts whose pool redraws and how many draws more, in post
// order; `redraws` sorted by t.  Positions past the ones listed are taken to need no
// redraws, so the list must cover every position a pool can start at.
inline void pools_with_redraws(const std::vector<PoolRedrawAt>& redraws, uint64_t c0, uint32_t take,
                               uint64_t n_posts, std::vector<uint32_t>& q, std::vector<uint32_t>& extra) {
    uint64_t next_start = c0, q_next = 0;  // the next pool's start and its post
    for (const PoolRedrawAt& b : redraws) {
        if (b.t < next_start || (b.t - next_start) % take) continue;  // not a pool start
        const uint64_t post = q_next + (b.t - next_start) / take;
        if (post >= n_posts) break;
        q.push_back(static_cast<uint32_t>(post));
        extra.push_back(b.extra);
        q_next = post + 1;
        next_start = b.t + take + b.extra;
    }
}

}  // namespace astrosim
