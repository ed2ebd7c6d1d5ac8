// Host check of the chunked builder's walks (astrosimgpu_cuda_b200/csrc/walk_chunked.cuh),
// compiled with g++ by test_walk_equivalence.py: over random skip caches, sections
// and autapse positions, walk_pre_end (the re-merge walk, which hashes the next
// post's tests ahead) ends at the same tape position and raises the same error
// flags as walk_pre (the walk every other pass of the builder uses, and which the
// device tests pin to the reference's connectivity).  Test infrastructure.
#include <cmath>
#include <cstdint>
#include <cstdio>
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

int main(int argc, char** argv) {
    const int trials = argc > 1 ? std::atoi(argv[1]) : 2000;
    std::mt19937_64 rng(7);
    long checks = 0, bad = 0, errs = 0;
    for (int trial = 0; trial < trials; ++trial) {
        const u64 len = 2000 + rng() % 20000;
        std::vector<u32> cache(len);
        const double p = 0.02 + static_cast<double>(rng() % 1000) / 1000.0 * 0.5;  // connection probability
        for (auto& v : cache) {
            const double u = static_cast<double>(rng() >> 11) * (1.0 / 9007199254740992.0);
            v = static_cast<u32>(std::floor(std::log1p(-u) / std::log1p(-p)));
        }
        Sec s{};
        s.seed = rng();
        s.cache = cache.data();
        s.cache_base = 1000 + rng() % 1000;
        s.cache_len = len;
        s.post_count = 1 + static_cast<u32>(rng() % 300);
        s.post_off = static_cast<u32>(rng() % 5000);
        s.third = static_cast<int>(rng() % 4 != 0);
        s.take = 5;
        std::vector<u32> pool((static_cast<size_t>(s.post_off) + s.post_count + 10) * kPoolSize, 3);
        s.pool = pool.data();
        for (int w = 0; w < 40; ++w) {
            const u64 c0 = s.cache_base + rng() % (len - 10);  // late starts run off the cache
            u32 self = kNoSelf;
            if (rng() % 2) self = s.post_off + static_cast<u32>(rng() % s.post_count);
            int err1 = 0, err2 = 0;
            NoVisit nv;
            s.err = &err1;
            const u64 e1 = walk_pre(s, c0, self, nv);
            s.err = &err2;
            const u64 e2 = walk_pre_end(s, c0, self);
            ++checks;
            errs += err1 != 0;
            if (e1 != e2 || err1 != err2) {
                ++bad;
                if (bad <= 5)
                    std::printf("mismatch: start %llu, walk_pre %llu (err %d), walk_pre_end %llu (err %d)\n",
                                static_cast<unsigned long long>(c0), static_cast<unsigned long long>(e1), err1,
                                static_cast<unsigned long long>(e2), err2);
            }
        }
    }
    std::printf("walks %ld mismatches %ld cache_overruns %ld\n", checks, bad, errs);
    return bad != 0;
}
