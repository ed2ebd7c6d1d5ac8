// builder.cu -- builds the network on the device: the setup-stream prologue, the
// astrocyte pools, the three presynaptic walk sections, the target-keyed CSRs and
// the per-cell parameters.  The reference does all of this serially on the host
// (src/astrosim_fused.cu:631-735 and 917-933); the device reproduces the same
// sequential random stream exactly.
//
// Two connectivity paths produce identical results:
//   - a one-thread walk (this file) for small networks, where launching the
//     chunked machinery costs more than walking the stream;
//   - the chunked parallel builder (builder_parallel.cu) for everything else.

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <thread>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>

#include "builder_internal.cuh"
#include "network.cuh"
#include "walk.cuh"

namespace astrosim {

// ------------------------------------------------------------------ setup-stream prologue
// The reference first steps over 4 normals per astrocyte and 2 per neuron
// (src/astrosim_fused.cu:644-645).  Normals come in Box-Muller pairs, so that is
// 2 * n_pairs uniforms unless a pair's first uniform is exactly zero (probability
// 2^-53 per draw), which makes the reference redraw it.  This kernel looks for such a draw.
__global__ void zero_draw_scan_kernel(u64 seed, u64 first, u64 n, unsigned* found) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        if (rng_uniform_is_zero(seed, kSetupStream, first + i)) atomicAdd(found, 1u);
    }
}

Status prologue_end(const Sizes& sz, u64 seed, cudaStream_t st, u64* c_out, unsigned* scratch) {
    const u64 n_pairs = 2ull * sz.n_astro + sz.n_neurons;
    const u64 n = 2ull * n_pairs;
    AS_CUDA(cudaMemsetAsync(scratch, 0, sizeof(unsigned), st));
    zero_draw_scan_kernel<<<1184, 256, 0, st>>>(seed, 0, n, scratch);
    AS_CUDA(cudaGetLastError());
    unsigned found = 0;
    AS_CUDA(cudaMemcpyAsync(&found, scratch, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    AS_CUDA(cudaStreamSynchronize(st));
    if (found)
        return make_error(ASTROSIM_ERR_UNSUPPORTED,
                          "seed %llu: a 53-bit zero draw occurs in the parameter-skip prologue "
                          "(probability 2^-53 per draw); this stream is not supported",
                          static_cast<unsigned long long>(seed));
    *c_out = n;
    return Status::Ok();
}

// ------------------------------------------------------------------ sequential walk
struct SeqConnArgs {
    u64 seed;
    u32 n_exc, n_inh, n_astro;
    double p, L;
    u64 c0;
    u32* pool;
    u32* astro_deg;
    EdgeLists e;
    SkipTable tab;
    AmbiguityLog amb;
    int* error;
};

__device__ __forceinline__ u32 seq_skip(const SeqConnArgs& a, u64& c, u32 remaining) {
    // src/astrosim_fused.cu:617-624
    if (remaining == 0 || a.p >= 1.0) return 0;
    if (a.p <= 0.0) return remaining;
    const double g = skip_value(a.seed, a.L, c++, a.tab, a.amb);
    return g >= static_cast<double>(remaining) ? remaining : static_cast<u32>(g);
}

// One thread walks the whole connectivity stream in the reference's order
// (src/astrosim_fused.cu:651-723).
__global__ void seq_connect_kernel(SeqConnArgs a) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const u64 seed = a.seed;
    const u32 n_exc = a.n_exc, n_inh = a.n_inh, n_astro = a.n_astro;
    const u32 n_neurons = n_exc + n_inh;
    u64 c = a.c0;
    const u32 take = n_astro < kPoolSize ? n_astro : kPoolSize;
    pools_sequential(seed, n_neurons, n_astro, c, a.pool);

    unsigned long long ne = 0, ni = 0, nt = 0;
    for (int block = 0; block < 2; ++block) {  // E block then I block (src/astrosim_fused.cu:709-710)
        const u32 off = block == 0 ? 0u : n_exc;
        const u32 cnt = block == 0 ? n_exc : n_inh;
        for (u32 pre = 0; pre < n_exc; ++pre) {
            u32 pos = 0;
            while (pos < cnt) {
                pos += seq_skip(a, c, cnt - pos);
                if (pos >= cnt) break;
                const u32 post = off + pos;
                ++pos;
                if (pre == post) continue;  // no autapses
                if (ne >= a.e.cap_exc) { *a.error = 1; return; }
                a.e.exc_src[ne] = pre;
                a.e.exc_dst[ne] = post;
                ++ne;
                if (n_astro == 0 || rng_uniform(seed, kSetupStream, c++) >= kPThird) continue;
                const u32* pl = a.pool + static_cast<u64>(post) * kPoolSize;
                const u32 astro =
                    pl[static_cast<u64>(rng_uniform(seed, kSetupStream, c++) * static_cast<double>(take)) % take];
                if (a.astro_deg[astro] >= kMaxAstroOutDegree) continue;
                if (nt >= a.e.cap_third) { *a.error = 1; return; }
                a.e.e2a_src[nt] = pre;
                a.e.e2a_dst[nt] = astro;
                a.e.sic_src[nt] = astro;
                a.e.sic_dst[nt] = post;
                ++a.astro_deg[astro];
                ++nt;
            }
        }
    }
    for (u32 pre = 0; pre < n_inh; ++pre) {  // src/astrosim_fused.cu:712-723
        const u32 pre_global = n_exc + pre;
        u32 pos = 0;
        while (pos < n_neurons) {
            pos += seq_skip(a, c, n_neurons - pos);
            if (pos >= n_neurons) break;
            const u32 post = pos;
            ++pos;
            if (pre_global == post) continue;
            if (ni >= a.e.cap_inh) { *a.error = 1; return; }
            a.e.inh_src[ni] = pre;  // local inhibitory index, as the reference stores it
            a.e.inh_dst[ni] = post;
            ++ni;
        }
    }
    a.e.counts[0] = ne;
    a.e.counts[1] = ni;
    a.e.counts[2] = nt;
    a.e.counts[3] = c;
}

// ------------------------------------------------------------------ edge lists -> CSR
__global__ void row_start_kernel(const u32* sorted_dst, u64 n, u32 n_targets, u32* row_start) {
    const u64 t = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t > n_targets) return;
    // first index with sorted_dst[i] >= t
    u64 lo = 0, hi = n;
    while (lo < hi) {
        const u64 mid = (lo + hi) >> 1;
        if (sorted_dst[mid] < t) lo = mid + 1; else hi = mid;
    }
    row_start[t] = static_cast<u32>(lo);
}

static int bits_for(u32 n) {
    int b = 1;
    while (b < 32 && (1ull << b) < static_cast<u64>(n) + 1) ++b;
    return b;
}

// Scratch of the four sorts of one network: two key buffers and CUB's temporary
// storage, allocated once for the largest list (the per-sort alternate buffers of
// the plain SortPairs came to about 20 GB of allocations at N = 1e7).
struct SortScratch {
    DevBuf<u32> ka, kb;
    DevBuf<unsigned char> temp;
};

// Stable counting sort by target (src/astrosim_fused.cu:307-314).  The input lists
// are in emission order; an LSD radix sort is stable, so each row keeps that order.
// The source list is consumed (it is one of the sort's two value buffers).  With
// keep_dst the target list is copied into the scratch first and survives (the exc
// and inh lists are kept as forward lists); otherwise it is sorted in place.
Status edges_to_csr(u32* src, u32* dst, u64 n, u32 n_targets, bool keep_dst, SortScratch& sc, DeviceCSR& out,
                    cudaStream_t st) {
    out.n_targets = n_targets;
    out.n_edges = n;
    AS_TRY(out.row_start.alloc(static_cast<size_t>(n_targets) + 1));
    AS_TRY(out.src.alloc(n));
    if (n == 0) {
        AS_CUDA(cudaMemsetAsync(out.row_start.get(), 0, (static_cast<size_t>(n_targets) + 1) * sizeof(u32), st));
        return Status::Ok();
    }
    u32* k_cur = dst;
    u32* k_alt = sc.ka.get();
    if (keep_dst) {
        AS_CUDA(cudaMemcpyAsync(sc.ka.get(), dst, n * sizeof(u32), cudaMemcpyDeviceToDevice, st));
        k_cur = sc.ka.get();
        k_alt = sc.kb.get();
    }
    cub::DoubleBuffer<u32> keys(k_cur, k_alt), vals(src, out.src.get());
    const int end_bit = bits_for(n_targets);
    size_t temp_bytes = sc.temp.bytes();
    AS_CUDA(cub::DeviceRadixSort::SortPairs(sc.temp.get(), temp_bytes, keys, vals, n, 0, end_bit, st));
    if (vals.Current() != out.src.get())
        AS_CUDA(cudaMemcpyAsync(out.src.get(), vals.Current(), n * sizeof(u32), cudaMemcpyDeviceToDevice, st));
    row_start_kernel<<<ceil_div(static_cast<u64>(n_targets) + 1, 256), 256, 0, st>>>(keys.Current(), n, n_targets,
                                                                                   out.row_start.get());
    AS_CUDA(cudaGetLastError());
    AS_CUDA(cudaStreamSynchronize(st));
    return Status::Ok();
}

Status edge_lists_to_network(const EdgeLists& e, const u64 counts[4], Network& net, cudaStream_t st) {
    const u32 nn = net.own.n_hi - net.own.n_lo, na = net.own.a_hi - net.own.a_lo;
    const u32 n_targets[4] = {nn, nn, na, nn};
    const u64 n_max = std::max(std::max(counts[0], counts[1]), std::max(counts[2], counts[3]));
    SortScratch sc;
    AS_TRY(sc.ka.alloc(n_max));
    AS_TRY(sc.kb.alloc(std::max(counts[0], counts[1])));
    size_t temp_bytes = 1;
    for (int k = 0; k < 4; ++k) {
        if (counts[k] == 0) continue;
        size_t b = 0;
        cub::DoubleBuffer<u32> keys(sc.ka.get(), sc.kb.get()), vals(sc.ka.get(), sc.kb.get());
        AS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, b, keys, vals, counts[k], 0, bits_for(n_targets[k]), st));
        temp_bytes = std::max(temp_bytes, b);
    }
    AS_TRY(sc.temp.alloc(temp_bytes));
    AS_TRY(edges_to_csr(e.exc_src, e.exc_dst, counts[0], nn, true, sc, net.exc, st));
    AS_TRY(edges_to_csr(e.inh_src, e.inh_dst, counts[1], nn, true, sc, net.inh, st));
    AS_TRY(edges_to_csr(e.e2a_src, e.e2a_dst, counts[2], na, false, sc, net.e2a, st));
    AS_TRY(edges_to_csr(e.sic_src, e.sic_dst, counts[3], nn, false, sc, net.sic, st));
    return Status::Ok();
}

__global__ void slice_rows_kernel(const u32* rs, u32 lo, u32 n_rows, u32* out) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i <= n_rows) out[i] = rs[lo + i] - rs[lo];
}

Status slice_csr(DeviceCSR& c, u32 lo, u32 hi, cudaStream_t st) {
    if (lo == 0 && hi == c.n_targets) return Status::Ok();
    std::vector<u32> ends(2);
    AS_CUDA(cudaMemcpyAsync(&ends[0], c.row_start.get() + lo, sizeof(u32), cudaMemcpyDeviceToHost, st));
    AS_CUDA(cudaMemcpyAsync(&ends[1], c.row_start.get() + hi, sizeof(u32), cudaMemcpyDeviceToHost, st));
    AS_CUDA(cudaStreamSynchronize(st));
    DeviceCSR out;
    out.n_targets = hi - lo;
    out.n_edges = ends[1] - ends[0];
    AS_TRY(out.row_start.alloc(static_cast<size_t>(out.n_targets) + 1));
    AS_TRY(out.src.alloc(out.n_edges));
    slice_rows_kernel<<<ceil_div(static_cast<u64>(out.n_targets) + 1, 256), 256, 0, st>>>(c.row_start.get(), lo,
                                                                                        out.n_targets,
                                                                                        out.row_start.get());
    AS_CUDA(cudaGetLastError());
    if (out.n_edges)
        AS_CUDA(cudaMemcpyAsync(out.src.get(), c.src.get() + ends[0], out.n_edges * sizeof(u32),
                                cudaMemcpyDeviceToDevice, st));
    AS_CUDA(cudaStreamSynchronize(st));
    c = std::move(out);
    return Status::Ok();
}

// ------------------------------------------------------------------ ambiguity settling
Status settle_ambiguities(u64 seed, double L, const DevBuf<u64>& amb_pos, const DevBuf<double>& amb_val,
                          const DevBuf<unsigned>& amb_count, std::map<u64, double>& table, bool* rerun,
                          cudaStream_t st) {
    unsigned n = 0;
    AS_CUDA(cudaMemcpyAsync(&n, amb_count.get(), sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    AS_CUDA(cudaStreamSynchronize(st));
    *rerun = false;
    if (n == 0) return Status::Ok();
    const unsigned m = std::min<unsigned>(n, static_cast<unsigned>(amb_pos.size()));
    std::vector<u64> pos(m);
    std::vector<double> val(m);
    AS_CUDA(cudaMemcpyAsync(pos.data(), amb_pos.get(), m * sizeof(u64), cudaMemcpyDeviceToHost, st));
    AS_CUDA(cudaMemcpyAsync(val.data(), amb_val.get(), m * sizeof(double), cudaMemcpyDeviceToHost, st));
    AS_CUDA(cudaStreamSynchronize(st));
    if (n > m) *rerun = true;  // log overflowed: record what we have and walk again
    for (unsigned i = 0; i < m; ++i) {
        const double host = skip_value_host(seed, L, pos[i]);
        if (host != val[i]) *rerun = true;
        table[pos[i]] = host;
    }
    return Status::Ok();
}

Status upload_table(const std::map<u64, double>& table, DevBuf<u64>& pos, DevBuf<double>& val, SkipTable& tab,
                    cudaStream_t st) {
    std::vector<u64> p;
    std::vector<double> v;
    for (const auto& kv : table) {
        p.push_back(kv.first);
        v.push_back(kv.second);
    }
    AS_TRY(pos.alloc(p.size()));
    AS_TRY(val.alloc(v.size()));
    if (!p.empty()) {
        AS_CUDA(cudaMemcpyAsync(pos.get(), p.data(), p.size() * sizeof(u64), cudaMemcpyHostToDevice, st));
        AS_CUDA(cudaMemcpyAsync(val.get(), v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice, st));
        AS_CUDA(cudaStreamSynchronize(st));
    }
    tab.pos = pos.get();
    tab.val = val.get();
    tab.n = static_cast<int>(p.size());
    return Status::Ok();
}

// ------------------------------------------------------------------ capacities
static u64 edge_cap(double n_pairs, double p) {
    const double mean = n_pairs * p;
    const double cap = std::min(n_pairs, mean * 1.25 + 12.0 * std::sqrt(mean + 1.0) + 1024.0);
    return static_cast<u64>(cap) + 16;
}

Status alloc_edge_lists(const Sizes& sz, EdgeStorage& s, cudaStream_t st) {
    const double nn = sz.n_neurons;
    s.cap_exc = edge_cap(static_cast<double>(sz.n_exc) * nn, sz.p);
    s.cap_inh = edge_cap(static_cast<double>(sz.n_inh) * nn, sz.p);
    s.cap_third = std::min<u64>(s.cap_exc, edge_cap(static_cast<double>(sz.n_exc) * nn, sz.p * kPThird));
    AS_TRY(s.exc_src.alloc(s.cap_exc));
    AS_TRY(s.exc_dst.alloc(s.cap_exc));
    AS_TRY(s.inh_src.alloc(s.cap_inh));
    AS_TRY(s.inh_dst.alloc(s.cap_inh));
    AS_TRY(s.e2a_src.alloc(s.cap_third));
    AS_TRY(s.e2a_dst.alloc(s.cap_third));
    AS_TRY(s.sic_src.alloc(s.cap_third));
    AS_TRY(s.sic_dst.alloc(s.cap_third));
    AS_TRY(s.counts.alloc_zero(4, st));
    return Status::Ok();
}

EdgeLists EdgeStorage::view() {
    EdgeLists e;
    e.exc_src = exc_src.get(); e.exc_dst = exc_dst.get();
    e.inh_src = inh_src.get(); e.inh_dst = inh_dst.get();
    e.e2a_src = e2a_src.get(); e.e2a_dst = e2a_dst.get();
    e.sic_src = sic_src.get(); e.sic_dst = sic_dst.get();
    e.cap_exc = cap_exc; e.cap_inh = cap_inh; e.cap_third = cap_third;
    e.counts = counts.get();
    return e;
}

double estimated_walk_draws(const Sizes& sz) {
    const double ne = sz.n_exc, ni = sz.n_inh, nn = sz.n_neurons, p = sz.p;
    const double skips = p >= 1.0 ? 0.0 : 1.0;
    const double e_edges = ne * nn * p;
    return 5.0 * nn + ne * 2.0 * skips + e_edges * (skips + 1.0 + kPThird) + ni * (nn * p * skips + skips);
}

Status build_sequential(const Sizes& sz, u64 seed, u64 c0, Network& net, cudaStream_t st) {
    EdgeStorage s;
    AS_TRY(alloc_edge_lists(sz, s, st));
    DevBuf<u32> pool, deg;
    AS_TRY(pool.alloc(static_cast<size_t>(sz.n_neurons) * kPoolSize));
    AS_TRY(deg.alloc(sz.n_astro));
    DevBuf<int> err;
    AS_TRY(err.alloc(1));
    DevBuf<u64> amb_pos, tab_pos;
    DevBuf<double> amb_val, tab_val;
    DevBuf<unsigned> amb_count;
    AS_TRY(amb_pos.alloc(4096));
    AS_TRY(amb_val.alloc(4096));
    AS_TRY(amb_count.alloc(1));
    std::map<u64, double> table;
    const double L = std::log1p(-sz.p);  // the reference's host value (src/astrosim_fused.cu:622)

    for (int attempt = 0; attempt < 6; ++attempt) {
        SeqConnArgs a{};
        a.seed = seed;
        a.n_exc = sz.n_exc;
        a.n_inh = sz.n_inh;
        a.n_astro = sz.n_astro;
        a.p = sz.p;
        a.L = L;
        a.c0 = c0;
        a.pool = pool.get();
        a.astro_deg = deg.get();
        a.e = s.view();
        AS_TRY(upload_table(table, tab_pos, tab_val, a.tab, st));
        a.amb.pos = amb_pos.get();
        a.amb.val = amb_val.get();
        a.amb.count = amb_count.get();
        a.amb.cap = 4096;
        a.error = err.get();
        AS_CUDA(cudaMemsetAsync(deg.get(), 0, deg.bytes(), st));
        AS_CUDA(cudaMemsetAsync(err.get(), 0, sizeof(int), st));
        AS_CUDA(cudaMemsetAsync(amb_count.get(), 0, sizeof(unsigned), st));
        seq_connect_kernel<<<1, 32, 0, st>>>(a);
        AS_CUDA(cudaGetLastError());
        int herr = 0;
        AS_CUDA(cudaMemcpyAsync(&herr, err.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
        AS_CUDA(cudaStreamSynchronize(st));
        if (herr) return make_error(ASTROSIM_ERR_INVALID_ARG, "edge list capacity exceeded in the sequential builder");
        bool rerun = false;
        AS_TRY(settle_ambiguities(seed, L, amb_pos, amb_val, amb_count, table, &rerun, st));
        if (rerun) continue;
        unsigned long long counts[4];
        AS_CUDA(cudaMemcpyAsync(counts, s.counts.get(), sizeof(counts), cudaMemcpyDeviceToHost, st));
        AS_CUDA(cudaStreamSynchronize(st));
        const u64 c3[4] = {counts[0], counts[1], counts[2], counts[2]};
        return edge_lists_to_network(s.view(), c3, net, st);
    }
    return make_error(ASTROSIM_ERR_CUDA, "skip tie-break table did not settle");
}

static double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

PhaseClock::PhaseClock(cudaStream_t s) : on(std::getenv("ASTROSIM_TIMING") != nullptr), st(s), t0(now_s()) {}

void PhaseClock::mark(const char* what) {
    if (!on) return;
    cudaStreamSynchronize(st);
    const double t = now_s();
    std::fprintf(stderr, "[astrosim build] %-28s %8.3f ms\n", what, (t - t0) * 1e3);
    t0 = t;
}

double PhaseClock::now() { return now_s(); }

void PhaseClock::mark_since(const char* what, double t) {
    if (!on) return;
    cudaStreamSynchronize(st);
    std::fprintf(stderr, "[astrosim build] %-28s %8.3f ms\n", what, (now_s() - t) * 1e3);
}

namespace {

// A host thread running one stream-ordered job on a pooled stream of its own; every
// path out joins it and returns the stream.
class ParamThread {
public:
    template <class F>
    Status start(F job) {
        AS_CUDA(cudaGetDevice(&dev_));
        AS_CUDA(take_stream(dev_, &st_));
        th_ = std::thread([this, job] {
            cudaSetDevice(dev_);
            AllocStream scope(st_);
            result_ = job(st_);
            if (result_.ok()) {
                const cudaError_t e = cudaStreamSynchronize(st_);
                if (e != cudaSuccess) result_ = make_error(ASTROSIM_ERR_CUDA, "parameter draws: %s", cudaGetErrorString(e));
            }
        });
        return Status::Ok();
    }
    Status finish() {
        stop();
        return result_;
    }
    ~ParamThread() { stop(); }

private:
    void stop() {
        if (th_.joinable()) th_.join();
        if (st_) {
            give_stream(dev_, st_);
            st_ = nullptr;
        }
    }
    int dev_ = 0;
    cudaStream_t st_ = nullptr;
    std::thread th_;
    Status result_;
};

}  // namespace

Status build_network(const Sizes& sz, u64 seed, const Biology& bio, const BuildOptions& opt, Network& net,
                     cudaStream_t st) {
    PhaseClock pc(st);
    const auto t0 = std::chrono::steady_clock::now();
    net.sz = sz;
    net.seed = seed;
    DevBuf<unsigned> scratch;
    AS_TRY(scratch.alloc(1));
    u64 c0 = 0;
    AS_TRY(prologue_end(sz, seed, st, &c0, scratch.get()));
    pc.mark("prologue");
    const double est = estimated_walk_draws(sz);
    // ASTROSIM_BUILDER=sequential|parallel forces one connectivity path (used by the
    // tests to run both paths on the same networks).
    u64 threshold = opt.sequential_max_draws;
    if (const char* env = std::getenv("ASTROSIM_BUILDER")) {
        if (std::strcmp(env, "sequential") == 0) threshold = ~0ull;
        else if (std::strcmp(env, "parallel") == 0) threshold = 0;
    }
    net.own = opt.own.clamped(sz);
    // The cell parameters come from counter 0 of their own sequence of draws, so they
    // do not depend on the connectivity walk: a second host thread draws them on a
    // second stream while the walk runs (the walk's phases wait on the host between
    // small kernels, which leaves the GPU room).  Their buffers are allocated here, on
    // this thread's allocation stream, like the rest of the network.
    AS_TRY(alloc_cell_parameters(sz, net));
    ParamThread params;
    AS_TRY(params.start([&](cudaStream_t ps) { return draw_cell_parameters(sz, seed, bio, net, ps); }));
    if (est <= static_cast<double>(threshold)) {
        // a small network: the one-thread walk builds every row, then the owned rows are kept
        net.builder_path = 0;
        const CellRange own = net.own;
        net.own = CellRange{}.clamped(sz);
        AS_TRY(build_sequential(sz, seed, c0, net, st));
        net.total_edges[0] = net.exc.n_edges;
        net.total_edges[1] = net.inh.n_edges;
        net.total_edges[2] = net.e2a.n_edges;
        net.total_edges[3] = net.sic.n_edges;
        net.own = own;
        AS_TRY(slice_csr(net.exc, own.n_lo, own.n_hi, st));
        AS_TRY(slice_csr(net.inh, own.n_lo, own.n_hi, st));
        AS_TRY(slice_csr(net.sic, own.n_lo, own.n_hi, st));
        AS_TRY(slice_csr(net.e2a, own.a_lo, own.a_hi, st));
    } else {
        // the chunked walk emits only the owned rows' edges (and counts every edge)
        net.builder_path = 1;
        AS_TRY(build_parallel(sz, seed, c0, net, st));
    }
    pc.mark("connectivity");
    AS_TRY(params.finish());
    pc.mark("parameters (wait after the walk)");
    AS_CUDA(cudaStreamSynchronize(st));
    net.build_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return Status::Ok();
}

Status download_csr(const DeviceCSR& c, std::vector<u32>& row_start, std::vector<u32>& src, cudaStream_t st) {
    row_start.resize(static_cast<size_t>(c.n_targets) + 1);
    src.resize(c.n_edges);
    AS_CUDA(cudaMemcpyAsync(row_start.data(), c.row_start.get(), row_start.size() * sizeof(u32),
                            cudaMemcpyDeviceToHost, st));
    if (c.n_edges)
        AS_CUDA(cudaMemcpyAsync(src.data(), c.src.get(), src.size() * sizeof(u32), cudaMemcpyDeviceToHost, st));
    AS_CUDA(cudaStreamSynchronize(st));
    return Status::Ok();
}

}  // namespace astrosim
