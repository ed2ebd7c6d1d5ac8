// builder_parallel.cu -- the chunked parallel connectivity builder.
//
// The reference builds connectivity from ONE sequential random stream
// (src/astrosim_fused.cu:631-723): after the pools, every presynaptic neuron
// ("pre") walks its postsynaptic block with geometric skips, and each landing may
// consume one or two more draws (the P_THIRD test and the pool pick).  The number
// of draws a pre consumes depends on the draws themselves, so the tape position
// where pre r starts is a prefix sum nobody knows in advance.  This file finds
// every pre's start exactly, in parallel, and then emits all edges in the
// reference's emission order:
//
//  1. Pools: each post's pool is 5 draws unless a duplicate forces a redraw;
//     offsets are found by a fixed-point iteration (each round fixes at least the
//     first misplaced post).
//  2. Skip cache: floor(log1p(-u) / log1p(-p)) for every tape position the walks
//     can reach, computed once; ambiguous values (quotient within a few ulps of an
//     integer) are settled with the host C library that the reference uses.
//  3. For each walk section (E block, I block, inhibitory pres), the section's
//     tape is cut into chunks.  For each chunk, walks start from EVERY candidate
//     entry position in [T, T + delta) -- the chunk's first pre start must be one
//     of them -- and merge when they land on the same pre start (a claim table):
//     one CTA per short chunk, all candidates at once; persistent warp swarms for
//     long chunks.  That gives an exact table: entry -> (exit, pres started).
//     Tables are composed (groups in parallel, then one thread over the groups),
//     which yields every chunk's true entry, and one thread per chunk then writes
//     every pre's start ("orbit").
//  4. The transfer tables ignore one index-dependent rule: in the E block a pre
//     that lands on its own index skips its P_THIRD draws (no autapses).  Such
//     landings are rare (about 80 per network) but shift the stream, so: every
//     pre whose walk lands within +-K of its own index is a hazard; for each hazard
//     a speculative exact walk from that point runs until it rejoins the table
//     orbit; the host then replays the hazards in order with the running index
//     shift and splices the true orbit.
//  5. Count and emit: one thread per pre walks its row again (exact rules,
//     including autapses), first counting, then writing edges at scanned offsets.
//     The lists are in emission order (the two excitatory blocks interleaved by pre,
//     which makes the excitatory list source-major); the stable radix sort of
//     builder.cu turns them into the target-keyed CSRs, and the exc and inh lists
//     are kept as the windowed engine's forward lists.
// Every step is exact; the outcome is bit-identical to the sequential walk.

#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <vector>

#include "builder_internal.cuh"
#include "pool_offsets.h"
#include "walk.cuh"
#include "walk_chunked.cuh"

namespace astrosim {

namespace {

constexpr u32 kHashSlots = 4096;  // per-CTA claim table (32 KB of shared memory)
constexpr unsigned long long kEmpty = ~0ull;
constexpr u32 kGroup = 64;  // chunks composed per group
constexpr u32 kMaxDelta = 512;  // candidate entries (walkers) per chunk
// A section with fewer than target_chunks() (8 per SM) chunks of its planned length
// runs with shorter chunks, down to kMinChunkLen (4 x kMaxDelta): the table and orbit
// passes walk one chunk per thread, position after position, so on small networks
// the chunk length, not the network, sets their time.  The chunking never changes
// the result, only how the walk is split.
inline u32 target_chunks() { return sm_count() * 8; }
constexpr u32 kMinChunkLen = 2048;

// ---------------------------------------------------------------- pools
__global__ void pool_pass_kernel(u64 seed, u32 n_neurons, u32 n_astro, u32 take, u64 base, const u64* prefix,
                                 u32* pool, u64* extra) {
    const u32 q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n_neurons) return;
    u64 c = base + static_cast<u64>(take) * q + prefix[q];
    const u64 c0 = c;
    pool_one(seed, n_astro, c, pool + static_cast<u64>(q) * kPoolSize);
    extra[q] = c - c0 - take;
}

// Tape positions where a pool started there needs redraws (a duplicate pick), with
// the number of extra draws: every t in [t0, t0 + n).
struct PoolRedraw {
    u64 t;
    u32 extra, pad_;
};

__global__ void pool_redraw_kernel(u64 seed, u32 n_astro, u32 take, u64 t0, u64 n, PoolRedraw* out, unsigned* count,
                                   unsigned cap) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    u32 pl[kPoolSize];
    for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        u64 c = t0 + i;
        pool_one(seed, n_astro, c, pl);
        const u64 extra = c - (t0 + i) - take;
        if (extra) {
            const unsigned k = atomicAdd(count, 1u);
            if (k < cap) out[k] = PoolRedraw{t0 + i, static_cast<u32>(extra), 0u};
        }
    }
}

__global__ void scatter_extra_kernel(const u32* q, const u32* e, u32 n, u64* extra) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) extra[q[i]] = e[i];
}

__global__ void diff_kernel(const u64* a, const u64* b, u64 n, int* flag) {
    const u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n && a[i] != b[i]) *flag = 1;
}

// ---------------------------------------------------------------- skip cache
__global__ void skip_cache_kernel(u64 seed, double L, u64 base, u64 n, u32* cache, AmbiguityLog amb) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    const SkipTable none{};
    for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double g = skip_value(seed, L, base + i, none, amb);
        cache[i] = g >= 4294967295.0 ? 0xFFFFFFFFu : static_cast<u32>(g);
    }
}

// ---------------------------------------------------------------- chunk tables
__global__ void table_kernel(Sec s, u64 sec_start, u32 chunk_len, u32 delta, u64* t_exit, u32* t_cnt) {
    __shared__ unsigned long long hash[kHashSlots];
    __shared__ int par[kMaxDelta];
    __shared__ u32 mycnt[kMaxDelta], pcnt[kMaxDelta];
    __shared__ unsigned long long ex[kMaxDelta];
    for (u32 i = threadIdx.x; i < kHashSlots; i += blockDim.x) hash[i] = kEmpty;
    __syncthreads();
    const u64 T0 = sec_start + static_cast<u64>(blockIdx.x) * chunk_len;
    const u64 T1 = T0 + chunk_len;
    const u32 w = threadIdx.x;
    if (w < delta) {
        u64 c = T0 + w;
        u32 cnt = 0, pc = 0;
        int p = -1;
        NoVisit nv;
        while (c < T1) {
            const u32 key = static_cast<u32>(c - T0);
            u32 slot = (key * 2654435761u) & (kHashSlots - 1);
            const unsigned long long mine =
                (static_cast<unsigned long long>(key) << 32) | (static_cast<unsigned long long>(w) << 22) | cnt;
            bool stop = false;
            for (u32 probe = 0;; ++probe) {
                const unsigned long long old = atomicCAS(&hash[slot], kEmpty, mine);
                if (old == kEmpty) break;  // claimed: this walk continues from here
                if (static_cast<u32>(old >> 32) == key) {  // another walk was here: follow it
                    p = static_cast<int>((old >> 22) & 0x3FFu);
                    pc = static_cast<u32>(old & 0x3FFFFFu);
                    stop = true;
                    break;
                }
                slot = (slot + 1) & (kHashSlots - 1);
                if (probe + 1 >= kHashSlots) {
                    atomicOr(s.err, kErrHash);
                    stop = true;
                    break;
                }
            }
            if (stop) break;
            c = walk_pre(s, c, kNoSelf, nv);
            ++cnt;
        }
        par[w] = p;
        mycnt[w] = cnt;
        pcnt[w] = pc;
        ex[w] = c;
    }
    __syncthreads();
    if (w < delta) {
        // pres from my candidate = sum over the merge chain of (mine before the merge - the
        // claimer's count at the merge point) + the root's full count
        long long total = 0;
        int x = static_cast<int>(w);
        for (u32 guard = 0; par[x] >= 0 && guard < kMaxDelta; ++guard) {
            total += static_cast<long long>(mycnt[x]) - static_cast<long long>(pcnt[x]);
            x = par[x];
        }
        total += mycnt[x];
        t_exit[static_cast<u64>(blockIdx.x) * delta + w] = ex[x];
        t_cnt[static_cast<u64>(blockIdx.x) * delta + w] = static_cast<u32>(total);
    }
}

// ---------------------------------------------------------------- chunk tables by warp swarms
// The same tables from persistent warps.  In the one-CTA-per-chunk form above, the
// walk that never merges holds its CTA (delta threads, 42 KB of shared memory) for
// the whole chunk, so an SM keeps only 5 chunks in flight and, late in each chunk,
// walks 5-10 chains.  Here a warp takes a chunk, its lanes take the candidates a few
// at a time (a lane whose walk merged or left the chunk takes the next candidate),
// claims go to a per-warp table in global memory, and once every candidate has
// started and at most `handoff` walks remain, the warp hands them to a
// one-thread-per-walk kernel and takes the next chunk.  A walk's exit and count are
// the same whoever it merges into, so the tables are identical.
constexpr u32 kSwarmSlots = 4096;  // claim slots per warp (32 KB of global memory)
constexpr u32 kSwarmIdle = 0xFFFFFFFFu;

struct SwarmRec {
    int* par;     // walk this one merged into, -1 for a walk that reached the chunk end
    u32* mycnt;   // pres walked before merging (or in all)
    u32* pcnt;    // the merged-into walk's count where they met
    u64* ex;      // where the walk stopped
};

struct SwarmCont {
    u32 chunk, w;
    u64 c;
    u32 cnt, pad_;
};

__global__ void __launch_bounds__(128) swarm_kernel(Sec s, u64 sec_start, u32 chunk_len, u32 delta, u32 n_chunks,
                                                    u32 handoff, unsigned* next_chunk, unsigned long long* tables,
                                                    SwarmRec rec, SwarmCont* cont, unsigned* n_cont,
                                                    unsigned cont_cap) {
    const u32 lane = threadIdx.x & 31u;
    const u64 warp = (static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    unsigned long long* tab = tables + warp * kSwarmSlots;
    NoVisit nv;
    for (;;) {
        u32 chunk = 0;
        if (lane == 0) chunk = atomicAdd(next_chunk, 1u);
        chunk = __shfl_sync(0xffffffffu, chunk, 0);
        if (chunk >= n_chunks) return;
        for (u32 i = lane; i < kSwarmSlots; i += 32) tab[i] = kEmpty;
        __threadfence();  // the cleared slots are in place before any lane's first claim
        __syncwarp();
        const u64 T0 = sec_start + static_cast<u64>(chunk) * chunk_len, T1 = T0 + chunk_len;
        const u64 rb = static_cast<u64>(chunk) * delta;
        u32 w = lane < delta ? lane : kSwarmIdle;
        u64 c = T0 + lane;
        u32 cnt = 0;
        u32 next = min(32u, delta);
        for (;;) {
            bool claimed = false;
            if (w != kSwarmIdle) {
                if (c >= T1) {  // reached the chunk end
                    rec.par[rb + w] = -1;
                    rec.mycnt[rb + w] = cnt;
                    rec.ex[rb + w] = c;
                    w = kSwarmIdle;
                } else {
                    const u32 key = static_cast<u32>(c - T0);
                    u32 slot = (key * 2654435761u) & (kSwarmSlots - 1);
                    const unsigned long long mine = (static_cast<unsigned long long>(key) << 32) |
                                                    (static_cast<unsigned long long>(w) << 22) | cnt;
                    for (u32 probe = 0;; ++probe) {
                        const unsigned long long old = atomicCAS(&tab[slot], kEmpty, mine);
                        if (old == kEmpty) {  // claimed: this walk continues from here
                            claimed = true;
                            break;
                        }
                        if (static_cast<u32>(old >> 32) == key) {  // another walk was here: follow it
                            rec.par[rb + w] = static_cast<int>((old >> 22) & 0x3FFu);
                            rec.pcnt[rb + w] = static_cast<u32>(old & 0x3FFFFFu);
                            rec.mycnt[rb + w] = cnt;
                            rec.ex[rb + w] = c;
                            w = kSwarmIdle;
                            break;
                        }
                        slot = (slot + 1) & (kSwarmSlots - 1);
                        if (probe + 1 >= kSwarmSlots) {  // table full: the host retries with shorter chunks
                            atomicOr(s.err, kErrHash);
                            rec.par[rb + w] = -1;
                            rec.mycnt[rb + w] = cnt;
                            rec.ex[rb + w] = c;
                            w = kSwarmIdle;
                            break;
                        }
                    }
                }
            }
            // idle lanes take the next candidates (they claim their start in the next round)
            const unsigned idle = __ballot_sync(0xffffffffu, w == kSwarmIdle);
            if (next < delta && idle) {
                const u32 rank = __popc(idle & ((1u << lane) - 1u));
                if (w == kSwarmIdle && next + rank < delta) {
                    w = next + rank;
                    c = T0 + w;
                    cnt = 0;
                }
                next = min(delta, next + static_cast<u32>(__popc(idle)));
            }
            const unsigned live = __ballot_sync(0xffffffffu, w != kSwarmIdle);
            if (live == 0) break;
            if (next >= delta && static_cast<u32>(__popc(live)) <= handoff) {
                if (w != kSwarmIdle) {
                    const unsigned k = atomicAdd(n_cont, 1u);
                    if (k < cont_cap) cont[k] = SwarmCont{chunk, w, c, cnt, 0u};
                    else atomicOr(s.err, kErrOrbit);
                }
                break;
            }
            if (claimed) {
                c = walk_pre(s, c, kNoSelf, nv);
                ++cnt;
            }
        }
        __syncwarp();
    }
}

// The walks a warp handed off, to the chunk end without claims.
__global__ void swarm_continue_kernel(Sec s, u64 sec_start, u32 chunk_len, u32 delta, const SwarmCont* cont,
                                      const unsigned* n_cont, unsigned cont_cap, SwarmRec rec) {
    const u32 k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= min(*n_cont, cont_cap)) return;
    const SwarmCont q = cont[k];
    const u64 T1 = sec_start + static_cast<u64>(q.chunk + 1) * chunk_len;
    u64 c = q.c;
    u32 cnt = q.cnt;
    NoVisit nv;
    while (c < T1) {
        c = walk_pre(s, c, kNoSelf, nv);
        ++cnt;
    }
    const u64 r = static_cast<u64>(q.chunk) * delta + q.w;
    rec.par[r] = -1;
    rec.mycnt[r] = cnt;
    rec.ex[r] = c;
}

// Exit and pre count of every candidate: along its merge chain, the sum of (pres
// before the merge - the merged-into walk's count there), plus the last walk's count.
__global__ void swarm_resolve_kernel(u32 delta, u64 n, SwarmRec rec, int* err, u64* t_exit, u32* t_cnt) {
    const u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const u64 base = i - i % delta;
    u64 x = i;
    long long total = 0;
    for (u32 guard = 0; rec.par[x] >= 0; ++guard) {
        if (guard >= delta) {  // merges point to earlier claims, so chains cannot cycle
            atomicOr(err, kErrOrbit);
            break;
        }
        total += static_cast<long long>(rec.mycnt[x]) - static_cast<long long>(rec.pcnt[x]);
        x = base + static_cast<u32>(rec.par[x]);
    }
    total += rec.mycnt[x];
    t_exit[i] = rec.ex[x];
    t_cnt[i] = static_cast<u32>(total);
}

// Composes the tables of kGroup consecutive chunks: thread d follows candidate d.
__global__ void group_compose_kernel(Sec s, u64 sec_start, u32 chunk_len, u32 delta, u32 n_chunks, const u64* t_exit,
                                     const u32* t_cnt, u64* g_exit, u64* g_cnt) {
    const u32 g = blockIdx.x, d = threadIdx.x;
    if (d >= delta) return;
    const u32 c0 = g * kGroup;
    const u32 c1 = min(c0 + kGroup, n_chunks);
    u64 x = d, cnt = 0, e = 0;
    for (u32 i = c0; i < c1; ++i) {
        if (x >= delta) {
            atomicOr(s.err, kErrDelta);
            break;
        }
        e = t_exit[static_cast<u64>(i) * delta + x];
        cnt += t_cnt[static_cast<u64>(i) * delta + x];
        x = e - (sec_start + static_cast<u64>(i + 1) * chunk_len);
    }
    g_exit[static_cast<u64>(g) * delta + d] = e;
    g_cnt[static_cast<u64>(g) * delta + d] = cnt;
}

// One thread over the groups: the true entry and pre index of every group, up to
// the group where `target` pres are reached.
__global__ void top_compose_kernel(Sec s, u64 sec_start, u32 chunk_len, u32 delta, u32 n_groups, const u64* g_exit,
                                   const u64* g_cnt, u64 target, u64* g_entry, u64* g_g0, u32* end_group) {
    u64 e = sec_start, cnt = 0;
    u32 g = 0;
    for (; g < n_groups; ++g) {
        g_entry[g] = e;
        g_g0[g] = cnt;
        const u64 d = e - (sec_start + static_cast<u64>(g) * kGroup * chunk_len);
        if (d >= delta) {
            atomicOr(s.err, kErrDelta);
            break;
        }
        cnt += g_cnt[static_cast<u64>(g) * delta + d];
        e = g_exit[static_cast<u64>(g) * delta + d];
        if (cnt >= target) break;
    }
    *end_group = g;
}

// Per group: the entry and first pre index of each of its chunks.
__global__ void chunk_entry_kernel(Sec s, u64 sec_start, u32 chunk_len, u32 delta, u32 n_chunks, u32 n_groups,
                                   const u64* t_exit, const u32* t_cnt, const u64* g_entry, const u64* g_g0,
                                   u64* c_entry, u64* c_g0) {
    const u32 g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_groups) return;
    u64 e = g_entry[g], cnt = g_g0[g];
    const u32 c0 = g * kGroup, c1 = min(c0 + kGroup, n_chunks);
    for (u32 i = c0; i < c1; ++i) {
        c_entry[i] = e;
        c_g0[i] = cnt;
        const u64 d = e - (sec_start + static_cast<u64>(i) * chunk_len);
        if (d >= delta) {
            atomicOr(s.err, kErrDelta);
            return;
        }
        cnt += t_cnt[static_cast<u64>(i) * delta + d];
        e = t_exit[static_cast<u64>(i) * delta + d];
    }
}

// One thread per chunk writes the start of every pre that begins in the chunk.
__global__ void materialize_kernel(Sec s, u64 sec_start, u32 chunk_len, u32 n_chunks, const u64* c_entry,
                                   const u64* c_g0, u64 limit, u64* orbit) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_chunks) return;
    u64 idx = c_g0[i];
    if (idx >= limit) return;
    const u64 T1 = sec_start + static_cast<u64>(i + 1) * chunk_len;
    u64 c = c_entry[i];
    NoVisit nv;
    while (c < T1 && idx < limit) {
        orbit[idx++] = c;
        c = walk_pre(s, c, kNoSelf, nv);
    }
    if (idx < limit && i + 1 < n_chunks && c != c_entry[i + 1]) atomicOr(s.err, kErrOrbit);
}

// ---------------------------------------------------------------- autapse hazards (E block)
struct Hazard {
    u32 r;    // index in the table orbit
    int d;    // landing post - r
};

struct HazardVisit {
    u32 r;
    int K;
    Hazard* out;
    unsigned* n;
    unsigned cap;
    __device__ __forceinline__ void operator()(u32 post, bool, u32) const {
        const long long d = static_cast<long long>(post) - static_cast<long long>(r);
        if (d >= -K && d <= K) {
            const unsigned k = atomicAdd(n, 1u);
            if (k < cap) out[k] = Hazard{r, static_cast<int>(d)};
        }
    }
};

__global__ void hazard_kernel(Sec s, const u64* orbit, u64 n, int K, Hazard* out, unsigned* count, unsigned cap) {
    const u64 r = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (r >= n) return;
    HazardVisit v{static_cast<u32>(r), K, out, count, cap};
    walk_pre(s, orbit[r], kNoSelf, v);
}

struct Remerge {
    long long k;       // table-orbit index where the exact walk rejoins (-1: section ended first)
    long long shift;   // true index - table index after rejoining
    u32 m;             // explicit pre starts recorded
    u32 ok;            // the walk rejoined or reached the section's end
    u64 end;           // section end when the walk reached the last pre
    // a walk that recorded its cap of starts first (ok == 0, capped == 1): the start
    // and true index of its next pre, from which it can be continued
    u64 c_next;
    long long r_next;
    u32 capped;
    u32 pad_;
};

// Index of c in the sorted orbit, or -1.  `from` is a lower bound of where c can be
// (the previous query's answer: a walk's queries only move forward); the search
// gallops from there, so a walk that keeps pace with the orbit costs one or two
// loads per query instead of a full binary search.  `from` becomes c's lower bound.
__device__ __forceinline__ long long find_in_orbit(const u64* orbit, u64 n, u64 c, u64& from) {
    u64 lo = from, hi = n;
    if (lo < n && orbit[lo] < c) {
        u64 step = 1;
        hi = lo + 1;
        while (hi < n && orbit[hi] < c) {
            lo = hi;
            step *= 2;
            hi = lo + step < n ? lo + step : n;
        }
        ++lo;  // orbit[lo - 1] < c
    } else {
        hi = lo;
    }
    while (lo < hi) {  // the first index in [lo, hi) with orbit[index] >= c
        const u64 mid = (lo + hi) >> 1;
        if (orbit[mid] < c) lo = mid + 1; else hi = mid;
    }
    from = lo;
    return (lo < n && orbit[lo] == c) ? static_cast<long long>(lo) : -1;
}

// The exact walk from pre start c with true index r, applying the autapse rule
// with true indices, until it lands on a start of the table orbit, the section's
// last pre ends, or it has recorded `cap` starts (then it stops where it stands and
// can be continued from there).
__device__ __forceinline__ void remerge_from(const Sec& s, u64 c, long long r, const u64* orbit, u64 n_orbit,
                                             u64 n_pres, u32 cap, u64* starts, Remerge& out) {
    out = Remerge{-1, 0, 0, 0, 0, 0, 0, 0, 0};
    starts[out.m++] = c;
    u64 from = 0;
    {
        u64 lo = 0, hi = n_orbit;  // c's lower bound in the orbit, once
        while (lo < hi) {
            const u64 mid = (lo + hi) >> 1;
            if (orbit[mid] < c) lo = mid + 1; else hi = mid;
        }
        from = lo;
    }
    for (;;) {
        c = walk_pre_end(s, c, static_cast<u32>(r));
        ++r;
        if (r >= static_cast<long long>(n_pres)) {
            out.end = c;
            out.ok = 1;
            return;
        }
        const long long k = find_in_orbit(orbit, n_orbit, c, from);
        if (k >= 0) {
            out.k = k;
            out.shift = r - k;
            out.ok = 1;
            return;
        }
        if (out.m >= cap) {
            out.capped = 1;
            out.c_next = c;
            out.r_next = r;
            return;
        }
        starts[out.m++] = c;
    }
}

// For each hazard, assume it is real (true index = r + d) and walk exactly from
// there (remerge_from) with at most max_explicit starts.  Most walks rejoin within a
// few pres; the host continues a capped walk only when its replay reaches it.
__global__ void remerge_kernel(Sec s, const Hazard* hz, u32 n_hz, const u64* orbit, u64 n_orbit, u64 n_pres,
                               u32 max_explicit, u64* expl, Remerge* res) {
    const u32 h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= n_hz) return;
    const long long r = static_cast<long long>(hz[h].r) + hz[h].d;
    if (r < 0 || r >= static_cast<long long>(n_pres)) {
        res[h] = Remerge{-1, 0, 0, 0, 0, 0, 0, 0, 0};
        return;
    }
    Remerge out;
    remerge_from(s, orbit[hz[h].r], r, orbit, n_orbit, n_pres, max_explicit, expl + static_cast<u64>(h) * max_explicit,
                 out);
    res[h] = out;
}

// One capped walk continued from where it stopped.
__global__ void remerge_continue_kernel(Sec s, u64 c, long long r, const u64* orbit, u64 n_orbit, u64 n_pres, u32 cap,
                                        u64* starts, Remerge* res) {
    Remerge out;
    remerge_from(s, c, r, orbit, n_orbit, n_pres, cap, starts, out);
    *res = out;
}

// The spliced orbit: piece p covers true indices [t_start[p], t_start[p] + len) and
// is read from src[p]; pieces are in index order and tile [0, n).
struct OrbitPiece {
    const u64* src;
    u64 t_start, len;
};

__global__ void splice_orbit_kernel(const OrbitPiece* pieces, u32 n_pieces, u64 n, u64* dst) {
    const u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    u32 lo = 0, hi = n_pieces;  // the last piece with t_start <= i
    while (hi - lo > 1) {
        const u32 mid = (lo + hi) >> 1;
        if (pieces[mid].t_start <= i) lo = mid; else hi = mid;
    }
    const OrbitPiece p = pieces[lo];
    dst[i] = p.src[i - p.t_start];
}

// ---------------------------------------------------------------- count and emit
// Owned targets of the build (CellRange): an exc/inh edge and an a2n (sic) edge are
// kept when their neuron target is owned, an e2a edge when its astrocyte is.
struct Owned {
    u32 n_lo, n_hi, a_lo, a_hi;
    __device__ __forceinline__ bool neuron(u32 post) const { return post >= n_lo && post < n_hi; }
    __device__ __forceinline__ bool astro(u32 a) const { return a >= a_lo && a < a_hi; }
};

// Per pre: kept primary edges, kept e2a edges, kept sic edges; and every edge for
// the whole network's totals.
struct CountVisit {
    Owned own;
    u64 ne = 0, na = 0, ns = 0;
    u32 te = 0, tt = 0;
    __device__ __forceinline__ void operator()(u32 post, bool hit, u32 astro) {
        const bool pn = own.neuron(post);
        ++te;
        ne += pn ? 1u : 0u;
        if (hit) {
            ++tt;
            na += own.astro(astro) ? 1u : 0u;
            ns += pn ? 1u : 0u;
        }
    }
};

__device__ __forceinline__ u32 self_post_of(int mode, u32 r, u32 self_off) {
    return mode == 0 ? kNoSelf : r + self_off;  // mode 1: autapse at post == r + self_off
}

// totals[0] += every primary edge, totals[1] += every third-factor edge (one atomic per warp).
__global__ void count_kernel(Sec s, const u64* orbit, u64 n, int self_mode, u32 self_off, Owned own, u64* ce,
                             u64* ca, u64* cs, unsigned long long* totals) {
    const u64 r = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x;
    CountVisit v{own};
    if (r < n) {
        walk_pre(s, orbit[r], self_post_of(self_mode, static_cast<u32>(r), self_off), v);
        ce[r] = v.ne;
        ca[r] = v.na;
        cs[r] = v.ns;
    }
    unsigned long long te = v.te, tt = v.tt;
    for (int off = 16; off > 0; off >>= 1) {
        te += __shfl_down_sync(0xffffffffu, te, off);
        tt += __shfl_down_sync(0xffffffffu, tt, off);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&totals[0], te);
        atomicAdd(&totals[1], tt);
    }
}

// One output stream of one emitting thread: values go to p[o], p[o + 1], ...  Whole
// 32-byte sectors leave as two 16-byte stores from an 8-value buffer in shared
// memory; only the partial sectors at the two ends of a pre's run get single
// stores.  With a single 4-byte store per value, L2 held partly written sectors
// and filled each from DRAM before writing it back: at N = 3e6 the E block's
// emission moved 32 GB of DRAM traffic for about 1.7 GB of edges.  The buffer is
// stream-major in shared memory (value k of thread t at buf[k * kEmitBlock]), so
// lanes at the same fill level hit different banks.
constexpr u32 kEmitBlock = 128;

struct SectorWriter {
    u32* p;
    u64 o;
    u32* buf;
    u32 k;
    __device__ __forceinline__ void put(u32 v) {
        if (k == 0 && (reinterpret_cast<unsigned long long>(p + o) & 31u)) {  // up to the next sector boundary
            p[o++] = v;
            return;
        }
        buf[k * kEmitBlock] = v;
        if (++k == 8) {
            const uint4 a = make_uint4(buf[0], buf[kEmitBlock], buf[2 * kEmitBlock], buf[3 * kEmitBlock]);
            const uint4 b = make_uint4(buf[4 * kEmitBlock], buf[5 * kEmitBlock], buf[6 * kEmitBlock],
                                       buf[7 * kEmitBlock]);
            *reinterpret_cast<uint4*>(p + o) = a;
            *reinterpret_cast<uint4*>(p + o + 4) = b;
            o += 8;
            k = 0;
        }
    }
    __device__ __forceinline__ void flush() {
        for (u32 i = 0; i < k; ++i) p[o + i] = buf[i * kEmitBlock];
        o += k;
        k = 0;
    }
};

// The edges of one pre.  The sources of the exc, inh and e2a lists are the pre
// itself and are filled in afterwards (fill_rows_kernel); the sic list's sources
// are astrocytes and are written here.
struct EmitVisit {
    Owned own;
    SectorWriter e_dst, t_dst, s_src, s_dst;
    __device__ __forceinline__ void operator()(u32 post, bool hit, u32 astro) {
        const bool pn = own.neuron(post);
        if (pn) e_dst.put(post - own.n_lo);
        if (hit) {
            if (own.astro(astro)) t_dst.put(astro - own.a_lo);
            if (pn) {
                s_src.put(astro);
                s_dst.put(post - own.n_lo);
            }
        }
    }
};

__global__ void __launch_bounds__(kEmitBlock) emit_kernel(Sec s, const u64* orbit, u64 n, int self_mode,
                                                          u32 self_off, Owned own, const u64* oe, const u64* oa,
                                                          const u64* os, u64 base_e, u64 base_a, u64 base_s,
                                                          u32* e_dst, u32* t_dst, u32* s_src, u32* s_dst) {
    __shared__ u32 sbuf[4 * 8 * kEmitBlock];
    const u64 r = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (r >= n) return;
    u32* b = sbuf + threadIdx.x;
    EmitVisit v{own,
                SectorWriter{e_dst, base_e + oe[r], b, 0u},
                SectorWriter{t_dst, base_a + oa[r], b + 8 * kEmitBlock, 0u},
                SectorWriter{s_src, base_s + os[r], b + 16 * kEmitBlock, 0u},
                SectorWriter{s_dst, base_s + os[r], b + 24 * kEmitBlock, 0u}};
    walk_pre(s, orbit[r], self_post_of(self_mode, static_cast<u32>(r), self_off), v);
    v.e_dst.flush();
    v.t_dst.flush();
    v.s_src.flush();
    v.s_dst.flush();
}

// out[i] = r for every i of row r, rows [base + o[r], base + o[r + 1]) (the last one
// ends at base + total): the source lists whose source is the row's pre.  One warp
// per row, so the writes are coalesced.
__global__ void fill_rows_kernel(const u64* o, u64 n, u64 base, u64 total, u32* out) {
    const u64 t = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x;
    const u64 r = t >> 5;
    if (r >= n) return;
    const u64 b = base + o[r], e = base + (r + 1 < n ? o[r + 1] : total);
    for (u64 i = b + (threadIdx.x & 31u); i < e; i += 32) out[i] = static_cast<u32>(r);
}

__global__ void section_end_kernel(Sec s, const u64* orbit, u64 last, int self_mode, u32 self_off, u64* end) {
    NoVisit nv;
    *end = walk_pre(s, orbit[last], self_post_of(self_mode, static_cast<u32>(last), self_off), nv);
}

// Excitatory edge layout, source-major: pre r's E-block edges (exc targets) then its
// I-block edges (inh targets) at fwd_rs[r] = oe_e[r] + oe_i[r] (the two blocks'
// exclusive scans over the same pres); o_e / o_i (the scans, in place) become each
// block's emission offsets.  fwd_rs[n] = total.
__global__ void exc_layout_kernel(u64 n, u64* o_e, u64* o_i, const u64* c_e, u64 total, u32* fwd_rs) {
    const u64 r = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (r < n) {
        const u64 base = o_e[r] + o_i[r];
        fwd_rs[r] = static_cast<u32>(base);
        o_e[r] = base;
        o_i[r] = base + c_e[r];
    }
    if (r == 0) fwd_rs[n] = static_cast<u32>(total);
}

// Row starts of a source-major list from its exclusive scan: rs[r] = o[r], rs[n] = total.
__global__ void rows_from_scan_kernel(u64 n, const u64* o, u64 total, u32* rs) {
    const u64 r = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (r < n) rs[r] = static_cast<u32>(o[r]);
    if (r == 0) rs[n] = static_cast<u32>(total);
}

__global__ void max_row_kernel(const u32* rs, u32 n, unsigned* mx) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) atomicMax(mx, rs[i + 1] - rs[i]);
}

// ---------------------------------------------------------------- host helpers
Status exclusive_scan_u64(const u64* in, u64* out, u64 n, cudaStream_t st) {
    size_t bytes = 0;
    AS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, st));
    DevBuf<unsigned char> tmp;
    AS_TRY(tmp.alloc(bytes));
    AS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), bytes, in, out, n, st));
    return Status::Ok();
}

template <typename T>
Status to_host(T* dst, const T* src, size_t n, cudaStream_t st) {
    AS_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyDeviceToHost, st));
    AS_CUDA(cudaStreamSynchronize(st));
    return Status::Ok();
}

Status read_err(const DevBuf<int>& err, int* out, cudaStream_t st) { return to_host(out, err.get(), 1, st); }

// A first guess of the pools' start offsets: prefix[q] = the extra draws of the
// pools before post q.  Pool q starts at c0 + take * q + prefix[q], and only the
// positions where a pool would need redraws matter -- about 250 of the 5 nN at any
// size (a duplicate among 5 picks from nA = N / 5 astrocytes).  They are found in
// one pass; walking them in order on the host with the running shift gives the
// offsets.  The fixed-point loop that follows checks the guess (one round when it
// is right, as it always is unless the list overflowed).
Status guess_pool_prefix(u64 seed, u32 nN, u32 nA, u32 take, u64 c0, u64* prefix, cudaStream_t st) {
    if (nN == 0 || take < kPoolSize || static_cast<u64>(take) * 4 >= nA) return Status::Ok();  // no redraws
    // the positions past the last pool's nominal start: about 4x the expected extra
    // draws (a pool redraws with probability about 10 / nA)
    const u64 margin = 4096 + static_cast<u64>(static_cast<double>(nN) * 40.0 / nA);
    const u64 n = static_cast<u64>(take) * nN + margin;
    const unsigned cap = 1u << 16;
    DevBuf<PoolRedraw> list;
    DevBuf<unsigned> count;
    AS_TRY(list.alloc(cap));
    AS_TRY(count.alloc_zero(1, st));
    pool_redraw_kernel<<<sm_count() * 8, 256, 0, st>>>(seed, nA, take, c0, n, list.get(), count.get(), cap);
    AS_CUDA(cudaGetLastError());
    unsigned m = 0;
    AS_TRY(to_host(&m, count.get(), 1, st));
    if (m > cap) return Status::Ok();  // leave the zero guess to the loop
    std::vector<PoolRedraw> h(m);
    if (m) AS_TRY(to_host(h.data(), list.get(), m, st));
    std::vector<PoolRedrawAt> sorted(m);
    for (unsigned i = 0; i < m; ++i) sorted[i] = PoolRedrawAt{h[i].t, h[i].extra};
    std::sort(sorted.begin(), sorted.end(), [](const PoolRedrawAt& a, const PoolRedrawAt& b) { return a.t < b.t; });
    std::vector<u32> bq, be;
    pools_with_redraws(sorted, c0, take, nN, bq, be);
    if (bq.empty()) return Status::Ok();
    DevBuf<u64> extra;
    DevBuf<u32> dq, de;
    AS_TRY(extra.alloc_zero(nN, st));
    AS_TRY(dq.alloc(bq.size()));
    AS_TRY(de.alloc(be.size()));
    AS_CUDA(cudaMemcpyAsync(dq.get(), bq.data(), bq.size() * sizeof(u32), cudaMemcpyHostToDevice, st));
    AS_CUDA(cudaMemcpyAsync(de.get(), be.data(), be.size() * sizeof(u32), cudaMemcpyHostToDevice, st));
    scatter_extra_kernel<<<ceil_div(bq.size(), 256), 256, 0, st>>>(dq.get(), de.get(), static_cast<u32>(bq.size()),
                                                                   extra.get());
    AS_CUDA(cudaGetLastError());
    AS_TRY(exclusive_scan_u64(extra.get(), prefix, nN, st));
    AS_CUDA(cudaStreamSynchronize(st));  // bq / be are host vectors
    return Status::Ok();
}

// Resident 128-thread blocks of swarm_kernel per SM, read once.
u32 swarm_blocks_per_sm() {
    static std::atomic<int> cached{0};
    int v = cached.load();
    if (v > 0) return static_cast<u32>(v);
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, swarm_kernel, 128, 0) != cudaSuccess || nb <= 0) {
        cudaGetLastError();
        nb = 8;
    }
    cached.store(nb);
    return static_cast<u32>(nb);
}

// The (exit, pres) table of every chunk candidate: t_exit/t_cnt[chunk * delta + d]
// for the walk from tape position sec_start + chunk * chunk_len + d.
// A section's chunks of swarm_min_chunk positions and more go to the warp swarms;
// shorter ones (the shortened chunks of small networks) to one CTA per chunk, which
// walks all candidates at once and measured faster there (N = 2e3-3e4: 0.3 vs 1.3
// ms per section; N = 1e7: 268 ms vs 33 ms for the E block the other way round).
Status chunk_tables(Sec s, u64 sec_start, u32 chunk_len, u32 delta, u32 n_chunks, u32 swarm_min_chunk, u32 handoff,
                    u64* t_exit, u32* t_cnt, cudaStream_t st) {
    // ASTROSIM_CHUNK_TABLES=cta|swarm forces one of the two (exact, equivalent) table
    // algorithms; the tests build the same networks both ways.
    bool cta = chunk_len < swarm_min_chunk;
    if (const char* env = std::getenv("ASTROSIM_CHUNK_TABLES")) {
        if (std::strcmp(env, "cta") == 0) cta = true;
        else if (std::strcmp(env, "swarm") == 0) cta = false;
    }
    if (cta) {
        table_kernel<<<n_chunks, delta, 0, st>>>(s, sec_start, chunk_len, delta, t_exit, t_cnt);
        AS_CUDA(cudaGetLastError());
        return Status::Ok();
    }
    const u64 n = static_cast<u64>(n_chunks) * delta;
    const u32 blocks = std::max<u32>(1, std::min<u32>(ceil_div(n_chunks, 4), sm_count() * swarm_blocks_per_sm()));
    const unsigned cont_cap = n_chunks * handoff;
    DevBuf<unsigned long long> tables;
    DevBuf<int> par;
    DevBuf<u32> mycnt, pcnt;
    DevBuf<u64> ex;
    DevBuf<SwarmCont> cont;
    DevBuf<unsigned> counters;  // next chunk, handed-off walks
    AS_TRY(tables.alloc(static_cast<u64>(blocks) * 4 * kSwarmSlots));
    AS_TRY(par.alloc(n));
    AS_TRY(mycnt.alloc(n));
    AS_TRY(pcnt.alloc(n));
    AS_TRY(ex.alloc(n));
    AS_TRY(cont.alloc(cont_cap));
    AS_TRY(counters.alloc_zero(2, st));
    const SwarmRec rec{par.get(), mycnt.get(), pcnt.get(), ex.get()};
    swarm_kernel<<<blocks, 128, 0, st>>>(s, sec_start, chunk_len, delta, n_chunks, handoff, counters.get(),
                                         tables.get(), rec, cont.get(), counters.get() + 1, cont_cap);
    AS_CUDA(cudaGetLastError());
    swarm_continue_kernel<<<ceil_div(cont_cap, 128), 128, 0, st>>>(s, sec_start, chunk_len, delta, cont.get(),
                                                                  counters.get() + 1, cont_cap, rec);
    AS_CUDA(cudaGetLastError());
    swarm_resolve_kernel<<<ceil_div(n, 256), 256, 0, st>>>(delta, n, rec, s.err, t_exit, t_cnt);
    AS_CUDA(cudaGetLastError());
    return Status::Ok();
}

struct SectionPlan {
    const char* name;
    u32 post_count, post_off;
    int third;
    u64 n_pres;
    double draws_per_pre;
    u32 chunk_len, delta;
    int self_mode;  // 0: no autapse possible; 1: autapse at post == r + self_off
    u32 self_off;
    bool autapse_shifts_stream;
    // Chunk tables by warp swarms from this chunk length up, handing off at most
    // `handoff` walks per chunk.  The continuation and orbit walks are one serial
    // walk per chunk, so their time follows the chunk length; the swarms' follows
    // the number of chunks.  Measured per section (N = 3e6, ncu): shortening the I
    // block's chunks (about 40 draws per pre) from 16384 to 4096 positions took its
    // tables and orbit from 10.8 to 3.8 ms, and the inhibitory section's (about 80
    // draws per pre, no third-factor draws) from 16384 to 8192 with hand-off at 6
    // from 17.5 to 9.6 ms; the E block (about 150 draws per pre) keeps 32768 and 4
    // (hand-off at 3: 16.9 instead of 14.4 ms).
    u32 swarm_min_chunk, handoff;
};

// Finds the start of every pre of one section (steps 3 and 4 of the file comment).
// On success `orbit` holds n_pres starts and *end the tape position after the section.
Status section_orbit(const SectionPlan& P, Sec s, u64 start, DevBuf<int>& err, DevBuf<u64>& orbit, u64* end,
                     cudaStream_t st) {
    u32 chunk_len = P.chunk_len, delta = P.delta;
    {
        const double draws = static_cast<double>(P.n_pres) * P.draws_per_pre;
        while (chunk_len > kMinChunkLen && draws / chunk_len < target_chunks()) chunk_len /= 2;
    }
    double slack = 1.04;
    int K = 32;
    // Explicit pre starts kept per speculative re-merge walk.  Walks rejoin after a
    // median of 2 pres (at most about 900 in every network measured, N = 2e3-1e6),
    // and the replay uses only the 50-90 on its chain of about 5,200; so every walk
    // stops at 64 starts and the replay continues, one at a time, the capped walks it
    // reaches.  The kernel then waits for 64 pres instead of the longest walk.
    const u32 max_explicit = 64;
    PhaseClock pc(st);
    for (int attempt = 0; attempt < 8; ++attempt) {
        AS_CUDA(cudaMemsetAsync(err.get(), 0, sizeof(int), st));
        const u64 margin = P.autapse_shifts_stream ? static_cast<u64>(K) + 16 : 0;
        const u64 target = P.n_pres + margin;
        const double est = static_cast<double>(target) * P.draws_per_pre * slack + 8.0 * chunk_len;
        const u32 n_chunks = std::max<u32>(1, static_cast<u32>(est / chunk_len) + 1);
        const u32 n_groups = ceil_div(n_chunks, kGroup);
        DevBuf<u64> t_exit, g_exit, g_cnt, g_entry, g_g0, c_entry, c_g0;
        DevBuf<u32> t_cnt, endg;
        AS_TRY(t_exit.alloc(static_cast<u64>(n_chunks) * delta));
        AS_TRY(t_cnt.alloc(static_cast<u64>(n_chunks) * delta));
        AS_TRY(g_exit.alloc(static_cast<u64>(n_groups) * delta));
        AS_TRY(g_cnt.alloc(static_cast<u64>(n_groups) * delta));
        AS_TRY(g_entry.alloc(n_groups));
        AS_TRY(g_g0.alloc(n_groups));
        AS_TRY(c_entry.alloc(n_chunks));
        AS_TRY(c_g0.alloc(n_chunks));
        AS_TRY(endg.alloc(1));
        AS_TRY(chunk_tables(s, start, chunk_len, delta, n_chunks, P.swarm_min_chunk, P.handoff, t_exit.get(),
                            t_cnt.get(), st));
        group_compose_kernel<<<n_groups, delta, 0, st>>>(s, start, chunk_len, delta, n_chunks, t_exit.get(),
                                                         t_cnt.get(), g_exit.get(), g_cnt.get());
        AS_CUDA(cudaGetLastError());
        top_compose_kernel<<<1, 1, 0, st>>>(s, start, chunk_len, delta, n_groups, g_exit.get(), g_cnt.get(), target,
                                            g_entry.get(), g_g0.get(), endg.get());
        AS_CUDA(cudaGetLastError());
        int herr = 0;
        u32 hend = 0;
        AS_TRY(read_err(err, &herr, st));
        AS_TRY(to_host(&hend, endg.get(), 1, st));
        pc.mark("  chunk tables + composition");
        if (herr & kErrHash) { chunk_len /= 2; continue; }
        if (herr & kErrDelta) {
            if (delta >= kMaxDelta) return make_error(ASTROSIM_ERR_UNSUPPORTED, "%s: a pre longer than %u draws", P.name, kMaxDelta);
            delta = std::min<u32>(kMaxDelta, delta * 2);
            continue;
        }
        if (herr & kErrCache) return make_error(ASTROSIM_ERR_UNSUPPORTED, "%s walk left the skip cache", P.name);
        if (hend >= n_groups) { slack *= 1.25; continue; }
        const u32 used_groups = hend + 1;
        const u32 used_chunks = std::min<u32>(n_chunks, used_groups * kGroup);
        // sentinel entries: a chunk left unset would start past every chunk end and write nothing
        AS_CUDA(cudaMemsetAsync(c_entry.get(), 0xFF, c_entry.bytes(), st));
        AS_CUDA(cudaMemsetAsync(c_g0.get(), 0xFF, c_g0.bytes(), st));
        chunk_entry_kernel<<<ceil_div(used_groups, 128), 128, 0, st>>>(s, start, chunk_len, delta, n_chunks,
                                                                       used_groups, t_exit.get(), t_cnt.get(),
                                                                       g_entry.get(), g_g0.get(), c_entry.get(),
                                                                       c_g0.get());
        AS_CUDA(cudaGetLastError());
        AS_TRY(read_err(err, &herr, st));
        if (herr & kErrDelta) {
            if (delta >= kMaxDelta) return make_error(ASTROSIM_ERR_UNSUPPORTED, "%s: a pre longer than %u draws", P.name, kMaxDelta);
            delta = std::min<u32>(kMaxDelta, delta * 2);
            continue;
        }
        DevBuf<u64> forbit;
        AS_TRY(forbit.alloc(target));
        materialize_kernel<<<ceil_div(used_chunks, 128), 128, 0, st>>>(s, start, chunk_len, used_chunks,
                                                                       c_entry.get(), c_g0.get(), target,
                                                                       forbit.get());
        AS_CUDA(cudaGetLastError());
        AS_TRY(read_err(err, &herr, st));
        if (herr & kErrDelta) {
            if (delta >= kMaxDelta) return make_error(ASTROSIM_ERR_UNSUPPORTED, "%s: a pre longer than %u draws", P.name, kMaxDelta);
            delta = std::min<u32>(kMaxDelta, delta * 2);
            continue;
        }
        if (herr) return make_error(ASTROSIM_ERR_CUDA, "%s orbit materialisation failed (flags %d)", P.name, herr);
        pc.mark("  chunk entries + orbit");

        if (!P.autapse_shifts_stream) {
            orbit = std::move(forbit);
            DevBuf<u64> e;
            AS_TRY(e.alloc(1));
            section_end_kernel<<<1, 1, 0, st>>>(s, orbit.get(), P.n_pres - 1, P.self_mode, P.self_off, e.get());
            AS_CUDA(cudaGetLastError());
            AS_TRY(to_host(end, e.get(), 1, st));
            return Status::Ok();
        }

        // ---- autapses of the E block (step 4)
        const unsigned hz_cap = static_cast<unsigned>(std::min<double>(4e6, 200.0 * (2 * K + 1) + 4096));
        DevBuf<Hazard> hz;
        DevBuf<unsigned> hz_n;
        AS_TRY(hz.alloc(hz_cap));
        AS_TRY(hz_n.alloc_zero(1, st));
        hazard_kernel<<<ceil_div(target, 128), 128, 0, st>>>(s, forbit.get(), target, K, hz.get(), hz_n.get(),
                                                             hz_cap);
        AS_CUDA(cudaGetLastError());
        unsigned n_hz = 0;
        AS_TRY(to_host(&n_hz, hz_n.get(), 1, st));
        if (n_hz > hz_cap)
            return make_error(ASTROSIM_ERR_UNSUPPORTED, "%s: %u autapse hazards exceed the buffer", P.name, n_hz);
        std::vector<Hazard> hh(n_hz);
        if (n_hz) AS_TRY(to_host(hh.data(), hz.get(), n_hz, st));
        std::sort(hh.begin(), hh.end(), [](const Hazard& a, const Hazard& b) {
            return a.r != b.r ? a.r < b.r : a.d < b.d;
        });
        pc.mark("  autapse hazards");
        // speculative exact walks from every hazard
        DevBuf<Hazard> hz_sorted;
        DevBuf<Remerge> rm;
        DevBuf<u64> expl;
        AS_TRY(hz_sorted.alloc(std::max<unsigned>(1, n_hz)));
        AS_TRY(rm.alloc(std::max<unsigned>(1, n_hz)));
        AS_TRY(expl.alloc(static_cast<u64>(std::max<unsigned>(1, n_hz)) * max_explicit));
        std::vector<Remerge> rr(n_hz);
        if (n_hz) {
            AS_CUDA(cudaMemcpyAsync(hz_sorted.get(), hh.data(), n_hz * sizeof(Hazard), cudaMemcpyHostToDevice, st));
            remerge_kernel<<<ceil_div(n_hz, 64), 64, 0, st>>>(s, hz_sorted.get(), n_hz, forbit.get(), target, P.n_pres,
                                                             max_explicit, expl.get(), rm.get());
            AS_CUDA(cudaGetLastError());
            AS_TRY(to_host(rr.data(), rm.get(), n_hz, st));
            AS_TRY(read_err(err, &herr, st));
            if (herr) return make_error(ASTROSIM_ERR_UNSUPPORTED, "%s: re-merge walks failed (flags %d)", P.name, herr);
        }
        pc.mark("  re-merge walks");
        // replay the hazards in order with the running shift (true index - table index)
        struct Piece { const u64* src; u64 t_start, len; };
        std::vector<Piece> pieces;
        std::vector<DevBuf<u64>> cont_starts;  // starts of the capped walks the replay continued
        DevBuf<Remerge> cont_res;
        AS_TRY(cont_res.alloc(1));
        long long d = 0;
        u64 cur_f = 0, cur_t = 0;
        bool ended = false;
        u64 end_pos = 0;
        bool shift_overflow = false;
        for (unsigned i = 0; i < n_hz && !ended; ++i) {
            const Hazard& h = hh[i];
            if (h.r < cur_f || h.d != d) continue;
            if (static_cast<long long>(h.r) + d >= static_cast<long long>(P.n_pres)) break;  // past the section
            Remerge m = rr[i];
            if (h.r > cur_f) pieces.push_back(Piece{forbit.get() + cur_f, cur_t, h.r - cur_f});
            const u64 t_autapse = static_cast<u64>(static_cast<long long>(h.r) + d);
            pieces.push_back(Piece{expl.get() + static_cast<u64>(i) * max_explicit, t_autapse, m.m});
            u64 walked = m.m;
            // This walk is on the chain: continue it from where it stopped (its tape
            // position and true index are all the state it has), in pieces of growing
            // size, until it rejoins the table orbit or the section ends.
            for (u32 cap = 4096; m.capped; cap = std::min<u32>(cap * 8, 1u << 24)) {
                DevBuf<u64> buf;
                AS_TRY(buf.alloc(cap));
                remerge_continue_kernel<<<1, 1, 0, st>>>(s, m.c_next, m.r_next, forbit.get(), target, P.n_pres, cap,
                                                         buf.get(), cont_res.get());
                AS_CUDA(cudaGetLastError());
                Remerge m2{};
                AS_TRY(to_host(&m2, cont_res.get(), 1, st));
                pieces.push_back(Piece{buf.get(), t_autapse + walked, m2.m});
                walked += m2.m;
                cont_starts.push_back(std::move(buf));
                m = m2;
            }
            if (!m.ok) return make_error(ASTROSIM_ERR_CUDA, "%s: re-merge walk incomplete", P.name);
            if (m.k < 0) {
                ended = true;
                end_pos = m.end;
                cur_t = t_autapse + walked;
                break;
            }
            cur_t = t_autapse + walked;
            cur_f = static_cast<u64>(m.k);
            d = m.shift;
            if (d < -K || d > K) { shift_overflow = true; break; }
        }
        if (shift_overflow) { K *= 4; continue; }
        if (!ended) {
            const u64 len = P.n_pres - cur_t;
            if (cur_f + len > target) { K *= 4; continue; }  // needed table orbit beyond the margin
            if (len) pieces.push_back(Piece{forbit.get() + cur_f, cur_t, len});
            cur_t += len;
        }
        if (cur_t != P.n_pres) return make_error(ASTROSIM_ERR_CUDA, "%s: spliced orbit has %llu of %llu pres", P.name,
                                                 static_cast<unsigned long long>(cur_t),
                                                 static_cast<unsigned long long>(P.n_pres));
        AS_TRY(orbit.alloc(P.n_pres));
        std::vector<OrbitPiece> table;
        for (const Piece& pc : pieces)
            if (pc.len) table.push_back(OrbitPiece{pc.src, pc.t_start, pc.len});
        if (!table.empty()) {
            DevBuf<OrbitPiece> dtab;
            AS_TRY(dtab.alloc(table.size()));
            AS_CUDA(cudaMemcpyAsync(dtab.get(), table.data(), table.size() * sizeof(OrbitPiece),
                                    cudaMemcpyHostToDevice, st));
            splice_orbit_kernel<<<ceil_div(P.n_pres, 256), 256, 0, st>>>(dtab.get(), static_cast<u32>(table.size()),
                                                                         P.n_pres, orbit.get());
            AS_CUDA(cudaGetLastError());
            AS_CUDA(cudaStreamSynchronize(st));  // the host table
        }
        if (ended) {
            *end = end_pos;
        } else {
            DevBuf<u64> e;
            AS_TRY(e.alloc(1));
            section_end_kernel<<<1, 1, 0, st>>>(s, orbit.get(), P.n_pres - 1, P.self_mode, P.self_off, e.get());
            AS_CUDA(cudaGetLastError());
            AS_TRY(to_host(end, e.get(), 1, st));
        }
        return Status::Ok();
    }
    return make_error(ASTROSIM_ERR_CUDA, "%s: chunked walk did not settle", P.name);
}

}  // namespace

Status build_parallel(const Sizes& sz, u64 seed, u64 c0, Network& net, cudaStream_t st) {
    if (sz.p >= 1.0 || sz.n_astro <= 20)
        return build_sequential(sz, seed, c0, net, st);  // all-to-all networks are tiny
    const u32 nN = sz.n_neurons, nA = sz.n_astro;
    const u32 take = nA < kPoolSize ? nA : kPoolSize;
    PhaseClock pc(st);
    DevBuf<int> err;
    AS_TRY(err.alloc_zero(1, st));

    // ---- 1. pools
    DevBuf<u32> pool;
    DevBuf<u64> extra, prefix, prefix_new;
    DevBuf<int> flag;
    AS_TRY(pool.alloc(static_cast<u64>(nN) * kPoolSize));
    AS_TRY(extra.alloc(nN));
    AS_TRY(prefix.alloc_zero(nN, st));
    AS_TRY(guess_pool_prefix(seed, nN, nA, take, c0, prefix.get(), st));
    AS_TRY(prefix_new.alloc(nN));
    AS_TRY(flag.alloc(1));
    u64 pools_end = 0;
    for (int it = 0;; ++it) {
        if (it > 100000) return make_error(ASTROSIM_ERR_CUDA, "pool offsets did not converge");
        pool_pass_kernel<<<ceil_div(nN, 256), 256, 0, st>>>(seed, nN, nA, take, c0, prefix.get(), pool.get(),
                                                            extra.get());
        AS_CUDA(cudaGetLastError());
        AS_TRY(exclusive_scan_u64(extra.get(), prefix_new.get(), nN, st));
        AS_CUDA(cudaMemsetAsync(flag.get(), 0, sizeof(int), st));
        diff_kernel<<<ceil_div(nN, 256), 256, 0, st>>>(prefix.get(), prefix_new.get(), nN, flag.get());
        AS_CUDA(cudaGetLastError());
        int changed = 0;
        AS_TRY(to_host(&changed, flag.get(), 1, st));
        if (!changed) {
            u64 last_prefix = 0, last_extra = 0;
            AS_TRY(to_host(&last_prefix, prefix.get() + (nN - 1), 1, st));
            AS_TRY(to_host(&last_extra, extra.get() + (nN - 1), 1, st));
            pools_end = c0 + static_cast<u64>(take) * nN + last_prefix + last_extra;
            break;
        }
        std::swap(prefix, prefix_new);
    }
    extra.release();
    prefix.release();
    prefix_new.release();
    pc.mark("pools");

    // ---- 2. skip cache over every tape position the three sections can reach
    const double ne = sz.n_exc, ni = sz.n_inh, nn = nN, p = sz.p;
    SectionPlan plans[3] = {
        {"E block", sz.n_exc, 0, 1, sz.n_exc, 1.0 + p * ne * (2.0 + kPThird), 32768, 384, 1, 0, true, 16384, 4},
        {"I block", sz.n_inh, sz.n_exc, 1, sz.n_exc, 1.0 + p * ni * (2.0 + kPThird), 4096, 192, 0, 0, false, 4096, 4},
        {"inhibitory", nN, 0, 0, sz.n_inh, 1.0 + p * nn, 8192, 192, 1, sz.n_exc, false, 8192, 6},
    };
    double est_total = 0.0;
    for (const auto& P : plans) est_total += static_cast<double>(P.n_pres) * P.draws_per_pre;
    const u64 cache_len = static_cast<u64>(est_total * 1.12) + 64ull * 65536 + 1000000;
    DevBuf<u32> cache;
    AS_TRY(cache.alloc(cache_len));
    const double L = std::log1p(-p);  // host value, as the reference computes it (src/astrosim_fused.cu:622)
    {
        DevBuf<u64> amb_pos;
        DevBuf<double> amb_val;
        DevBuf<unsigned> amb_n;
        const unsigned amb_cap = 1u << 16;
        AS_TRY(amb_pos.alloc(amb_cap));
        AS_TRY(amb_val.alloc(amb_cap));
        AS_TRY(amb_n.alloc_zero(1, st));
        AmbiguityLog amb{amb_pos.get(), amb_val.get(), amb_n.get(), amb_cap};
        skip_cache_kernel<<<sm_count() * 16, 256, 0, st>>>(seed, L, pools_end, cache_len, cache.get(), amb);
        AS_CUDA(cudaGetLastError());
        unsigned n_amb = 0;
        AS_TRY(to_host(&n_amb, amb_n.get(), 1, st));
        if (n_amb > amb_cap) return make_error(ASTROSIM_ERR_UNSUPPORTED, "too many ambiguous skip draws");
        std::vector<u64> pos(n_amb);
        if (n_amb) AS_TRY(to_host(pos.data(), amb_pos.get(), n_amb, st));
        for (u64 t : pos) {  // settle with the host formula
            const double g = skip_value_host(seed, L, t);
            const u32 v = g >= 4294967295.0 ? 0xFFFFFFFFu : static_cast<u32>(g);
            AS_CUDA(cudaMemcpyAsync(cache.get() + (t - pools_end), &v, sizeof(u32), cudaMemcpyHostToDevice, st));
            AS_CUDA(cudaStreamSynchronize(st));
        }
    }

    pc.mark("skip cache");
    // ---- 3-4. every pre's start, section by section
    Sec s{};
    s.seed = seed;
    s.cache = cache.get();
    s.cache_base = pools_end;
    s.cache_len = cache_len;
    s.err = err.get();
    s.take = take;
    s.pool = pool.get();
    DevBuf<u64> orbits[3];
    u64 start = pools_end;
    for (int k = 0; k < 3; ++k) {
        s.post_count = plans[k].post_count;
        s.post_off = plans[k].post_off;
        s.third = plans[k].third;
        u64 end = 0;
        AS_TRY(section_orbit(plans[k], s, start, err, orbits[k], &end, st));
        start = end;
        pc.mark(plans[k].name);
    }

    // ---- 5. count, scan, emit (only the edges whose target this network owns)
    const Owned own{net.own.n_lo, net.own.n_hi, net.own.a_lo, net.own.a_hi};
    DevBuf<u64> oe[3], oa[3], os[3];
    DevBuf<unsigned long long> totals;
    AS_TRY(totals.alloc_zero(6, st));
    u64 tot_e[3] = {0, 0, 0}, tot_a[3] = {0, 0, 0}, tot_s[3] = {0, 0, 0};
    DevBuf<u64> ce_block0;  // the E block's per-pre primary counts (the exc layout needs them)
    for (int k = 0; k < 3; ++k) {
        const SectionPlan& P = plans[k];
        s.post_count = P.post_count;
        s.post_off = P.post_off;
        s.third = P.third;
        DevBuf<u64> ce, ca, cs;
        AS_TRY(ce.alloc(P.n_pres));
        AS_TRY(ca.alloc(P.n_pres));
        AS_TRY(cs.alloc(P.n_pres));
        AS_TRY(oe[k].alloc(P.n_pres));
        AS_TRY(oa[k].alloc(P.n_pres));
        AS_TRY(os[k].alloc(P.n_pres));
        count_kernel<<<ceil_div(P.n_pres, 128), 128, 0, st>>>(s, orbits[k].get(), P.n_pres, P.self_mode, P.self_off,
                                                             own, ce.get(), ca.get(), cs.get(),
                                                             totals.get() + 2 * k);
        AS_CUDA(cudaGetLastError());
        AS_TRY(exclusive_scan_u64(ce.get(), oe[k].get(), P.n_pres, st));
        AS_TRY(exclusive_scan_u64(ca.get(), oa[k].get(), P.n_pres, st));
        AS_TRY(exclusive_scan_u64(cs.get(), os[k].get(), P.n_pres, st));
        u64 h[6] = {0, 0, 0, 0, 0, 0};
        AS_TRY(to_host(&h[0], oe[k].get() + (P.n_pres - 1), 1, st));
        AS_TRY(to_host(&h[1], ce.get() + (P.n_pres - 1), 1, st));
        AS_TRY(to_host(&h[2], oa[k].get() + (P.n_pres - 1), 1, st));
        AS_TRY(to_host(&h[3], ca.get() + (P.n_pres - 1), 1, st));
        AS_TRY(to_host(&h[4], os[k].get() + (P.n_pres - 1), 1, st));
        AS_TRY(to_host(&h[5], cs.get() + (P.n_pres - 1), 1, st));
        tot_e[k] = h[0] + h[1];
        tot_a[k] = h[2] + h[3];
        tot_s[k] = h[4] + h[5];
        if (k == 0) ce_block0 = std::move(ce);
    }
    // Both excitatory blocks walk the same pres (the exc neurons), so their edges can
    // be laid out source-major: the list is then the forward exc list itself, and the
    // target CSR (a stable sort by target) is unchanged, since each target row's
    // sources all come from one block, in ascending pre order either way.  The
    // inhibitory section's emission order is already source-major.
    if (plans[0].n_pres != plans[1].n_pres)
        return make_error(ASTROSIM_ERR_CUDA, "excitatory blocks over different pres (%llu, %llu)",
                          static_cast<unsigned long long>(plans[0].n_pres),
                          static_cast<unsigned long long>(plans[1].n_pres));
    if (tot_e[0] + tot_e[1] >= (1ull << 32) || tot_e[2] >= (1ull << 32))
        return make_error(ASTROSIM_ERR_UNSUPPORTED, "more than 2^32 - 1 primary edges in one CSR");
    DevBuf<u32> fwd_exc_rs, fwd_inh_rs;
    AS_TRY(fwd_exc_rs.alloc(plans[0].n_pres + 1));
    AS_TRY(fwd_inh_rs.alloc(plans[2].n_pres + 1));
    exc_layout_kernel<<<ceil_div(std::max<u64>(1, plans[0].n_pres), 256), 256, 0, st>>>(
        plans[0].n_pres, oe[0].get(), oe[1].get(), ce_block0.get(), tot_e[0] + tot_e[1], fwd_exc_rs.get());
    AS_CUDA(cudaGetLastError());
    rows_from_scan_kernel<<<ceil_div(std::max<u64>(1, plans[2].n_pres), 256), 256, 0, st>>>(
        plans[2].n_pres, oe[2].get(), tot_e[2], fwd_inh_rs.get());
    AS_CUDA(cudaGetLastError());
    ce_block0.release();
    {
        unsigned long long t[6];
        AS_TRY(to_host(t, totals.get(), 6, st));
        net.total_edges[0] = t[0] + t[2];  // excitatory primary edges: sections 0 and 1
        net.total_edges[1] = t[4];         // inhibitory: section 2
        net.total_edges[2] = t[1] + t[3];  // third-factor pairs: one e2a and one sic edge each
        net.total_edges[3] = t[1] + t[3];
    }
    EdgeStorage es;
    es.cap_exc = tot_e[0] + tot_e[1];
    es.cap_inh = tot_e[2];
    const u64 cap_e2a = tot_a[0] + tot_a[1], cap_sic = tot_s[0] + tot_s[1];
    AS_TRY(es.exc_src.alloc(es.cap_exc));
    AS_TRY(es.exc_dst.alloc(es.cap_exc));
    AS_TRY(es.inh_src.alloc(es.cap_inh));
    AS_TRY(es.inh_dst.alloc(es.cap_inh));
    AS_TRY(es.e2a_src.alloc(cap_e2a));
    AS_TRY(es.e2a_dst.alloc(cap_e2a));
    AS_TRY(es.sic_src.alloc(cap_sic));
    AS_TRY(es.sic_dst.alloc(cap_sic));
    AS_TRY(es.counts.alloc_zero(4, st));
    for (int k = 0; k < 3; ++k) {
        const SectionPlan& P = plans[k];
        s.post_count = P.post_count;
        s.post_off = P.post_off;
        s.third = P.third;
        const u64 base_e = 0, base_a = k == 1 ? tot_a[0] : 0, base_s = k == 1 ? tot_s[0] : 0;
        u32* e_dst = k == 2 ? es.inh_dst.get() : es.exc_dst.get();
        emit_kernel<<<ceil_div(P.n_pres, kEmitBlock), kEmitBlock, 0, st>>>(
            s, orbits[k].get(), P.n_pres, P.self_mode, P.self_off, own, oe[k].get(), oa[k].get(), os[k].get(),
            base_e, base_a, base_s, e_dst, es.e2a_dst.get(), es.sic_src.get(), es.sic_dst.get());
        AS_CUDA(cudaGetLastError());
    }
    // the pre-index sources: exc (both blocks, source-major), inh, and e2a (E block, then I block)
    const auto fill = [&](const DevBuf<u64>& o, u64 n, u64 base, u64 total, u32* out) -> Status {
        if (n == 0 || total == 0) return Status::Ok();
        fill_rows_kernel<<<ceil_div(n * 32, 256), 256, 0, st>>>(o.get(), n, base, total, out);
        AS_CUDA(cudaGetLastError());
        return Status::Ok();
    };
    AS_TRY(fill(oe[0], plans[0].n_pres, 0, tot_e[0] + tot_e[1], es.exc_src.get()));
    AS_TRY(fill(oe[2], plans[2].n_pres, 0, tot_e[2], es.inh_src.get()));
    AS_TRY(fill(oa[0], plans[0].n_pres, 0, tot_a[0], es.e2a_src.get()));
    AS_TRY(fill(oa[1], plans[1].n_pres, tot_a[0], tot_a[1], es.e2a_src.get()));
    int herr = 0;
    AS_TRY(read_err(err, &herr, st));
    if (herr) return make_error(ASTROSIM_ERR_CUDA, "edge emission failed (flags %d)", herr);
    for (int k = 0; k < 3; ++k) {
        orbits[k].release();
        oe[k].release();
        oa[k].release();
        os[k].release();
    }
    cache.release();
    pool.release();
    pc.mark("count + emit");
    const u64 counts[4] = {es.cap_exc, es.cap_inh, cap_e2a, cap_sic};
    AS_TRY(edge_lists_to_network(es.view(), counts, net, st));
    net.fwd_exc_rs = std::move(fwd_exc_rs);
    net.fwd_exc_dst = std::move(es.exc_dst);
    net.fwd_inh_rs = std::move(fwd_inh_rs);
    net.fwd_inh_dst = std::move(es.inh_dst);
    net.has_fwd = true;
    pc.mark("CSR sort");

    // The astrocyte out-degree cap (src/astrosim_fused.cu:702) drops a third-factor
    // edge only once an astrocyte already has 10000; with at most 10000 candidates
    // per astrocyte it never fires and the lists above are exact.
    DevBuf<unsigned> mx;
    AS_TRY(mx.alloc_zero(1, st));
    const u32 own_astro = net.own.a_hi - net.own.a_lo;  // each rank checks its own astrocytes
    if (own_astro)
        max_row_kernel<<<ceil_div(own_astro, 256), 256, 0, st>>>(net.e2a.row_start.get(), own_astro, mx.get());
    AS_CUDA(cudaGetLastError());
    unsigned hmx = 0;
    AS_TRY(to_host(&hmx, mx.get(), 1, st));
    if (hmx > kMaxAstroOutDegree)
        return make_error(ASTROSIM_ERR_UNSUPPORTED,
                          "an astrocyte has %u third-factor candidates; the out-degree cap of %u would bind", hmx,
                          kMaxAstroOutDegree);
    return Status::Ok();
}

}  // namespace astrosim
