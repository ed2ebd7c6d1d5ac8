// shard.cu -- one network split across ranks by cell ranges (see shard.cuh).

#include <dlfcn.h>
#include <nccl.h>

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <thread>

#include "shard.cuh"
#include "window_kernels.cuh"

namespace astrosim {

ShardPlan shard_plan(u32 n_neurons, u32 n_astro, int rank, int world) {
    auto cut = [&](u32 n, int r) -> u32 {
        const u64 blocks = (static_cast<u64>(n) + 127) / 128;
        const u64 b = blocks * static_cast<u64>(r) / static_cast<u64>(world);
        return static_cast<u32>(std::min<u64>(n, b * 128));
    };
    return ShardPlan{cut(n_neurons, rank), cut(n_neurons, rank + 1), cut(n_astro, rank), cut(n_astro, rank + 1)};
}

namespace {

// One window of this rank's cells: astrocyte blocks [a_blk0, a_blk0 + a_nblk), then
// neuron blocks from n_blk0.
template <typename R, int MB>
__global__ void __launch_bounds__(128, MB) shard_window_kernel(RunConsts rc, StepPtrs<R> p, WinPtrs<R> w,
                                                               i64 win_start, int buf, i64 mark, u32 a_blk0,
                                                               u32 a_nblk, u32 n_blk0) {
    const bool astro = blockIdx.x < a_nblk;
    window_cells<R>(rc, net_scalars(rc), p, w, win_start, 0, w.W, buf, mark, astro ? a_blk0 + blockIdx.x : n_blk0 + (blockIdx.x - a_nblk),
                    astro);
}

template <typename R>
__global__ void shard_push_kernel(WinPtrs<R> w, u32 n_exc, u32 n_inh, u64 n_neurons, u64 n_astro, int buf, u32 t_lo,
                                  u32 t_hi, u32 a_lo, u32 a_hi) {
    push_cells<R>(w, n_exc, n_inh, n_neurons, n_astro, buf, blockIdx.x, gridDim.x, t_lo, t_hi, a_lo, a_hi);
}

// Every spike of this rank's neurons in the window: key neuron << 5 | step, and its value.
template <typename R>
__global__ void pack_spikes_kernel(const u32* __restrict__ word, const R* __restrict__ val, u64 nN, u32 n_lo,
                                   u32 n_hi, u32* keys, R* vals, u32* cnt) {
    const u32 j = n_lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n_hi) return;
    u32 wd = word[j];
    while (wd) {
        const u32 st = static_cast<u32>(__ffs(wd) - 1);
        wd &= wd - 1;
        const u32 i = atomicAdd(cnt, 1u);  // at most one spike per neuron and step: i < (n_hi - n_lo) * W
        keys[i] = (j << 5) | st;
        vals[i] = val[static_cast<u64>(st) * nN + j];
    }
}

// Every active astrocyte of this rank: its id and its W factors.
template <typename R>
__global__ void pack_astro_kernel(const u32* __restrict__ act, const R* __restrict__ sic, u32 a_lo, u32 a_hi, int W,
                                  u32* ids, R* facs, u32* cnt) {
    const u32 a = a_lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= a_hi || !((act[a >> 5] >> (a & 31)) & 1u)) return;
    const u32 i = atomicAdd(cnt, 1u);
    ids[i] = a;
    for (int s = 0; s < W; ++s) facs[static_cast<u64>(i) * W + s] = sic[static_cast<u64>(a) * W + s];
}

// Another rank's spikes into this rank's window buffers, spike list and counts.
template <typename R>
__global__ void import_spikes_kernel(const u32* __restrict__ keys, const R* __restrict__ vals, u32 n, WinPtrs<R> w,
                                     u64 nN, int buf, i64 win_start, u32* counts, u32* raster, i64 raster_steps,
                                     u32 words) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const u32 key = keys[i];
    const u32 j = key >> 5, st = key & 31u;
    w.spk_val[(static_cast<u64>(buf) * w.W + st) * nN + j] = vals[i];
    atomicOr(&w.spk_word[static_cast<u64>(buf) * nN + j], 1u << st);
    const u32 slot = atomicAdd(&w.spk_count[buf], 1u);
    if (slot < w.cap) w.spk_list[static_cast<u64>(buf) * w.cap + slot] = key;
    const i64 t = win_start + st;
    atomicAdd(&counts[t], 1u);
    if (t < raster_steps) atomicOr(&raster[static_cast<u64>(t) * words + (j >> 5)], 1u << (j & 31));
}

// Another rank's active astrocytes into the active mask and the factor table.
template <typename R>
__global__ void import_astro_kernel(const u32* __restrict__ ids, const R* __restrict__ facs, u32 n, WinPtrs<R> w,
                                    u64 nA, int buf) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const u32 a = ids[i];
    atomicOr(&w.astro_active[static_cast<u64>(buf) * w.astro_words + (a >> 5)], 1u << (a & 31));
    R* dst = w.sic_win + (static_cast<u64>(buf) * nA + a) * w.W;
    for (int s = 0; s < w.W; ++s) dst[s] = facs[static_cast<u64>(i) * w.W + s];
}

template <typename R>
Status window_phase(ShardSim& s, i64 k) {
    Simulation& sim = s.sim;
    const RunConsts& rc = sim.consts();
    WindowState& ws = *sim.window_state();
    StepPtrs<R> p = make_ptrs<R>(sim.state_buffers(), sim.network(), rc, sim.raster_steps());
    WinPtrs<R> w = win_ptrs<R>(ws, rc);
    const u32 a_blk0 = s.plan.a_lo / 128, a_nblk = ceil_div(s.plan.a_hi - s.plan.a_lo, 128);
    const u32 n_blk0 = s.plan.n_lo / 128, n_nblk = ceil_div(s.plan.n_hi - s.plan.n_lo, 128);
    const u32 grid = a_nblk + n_nblk;
    const i64 mark = sim.pre_steps() == 0 ? 0 : sim.pre_steps() - 1;
    if (grid == 0) return Status::Ok();
    constexpr int MB = std::is_same<R, float>::value ? 6 : 4;
    shard_window_kernel<R, MB><<<grid, 128, 0, sim.stream()>>>(rc, p, w, k * ws.W, static_cast<int>(k & 1), mark,
                                                               a_blk0, a_nblk, n_blk0);
    AS_CUDA(cudaGetLastError());
    return Status::Ok();
}

template <typename R>
Status pack_phase(ShardSim& s, i64 k) {
    Simulation& sim = s.sim;
    const RunConsts& rc = sim.consts();
    WindowState& ws = *sim.window_state();
    WinPtrs<R> w = win_ptrs<R>(ws, rc);
    const int buf = static_cast<int>(k & 1);
    const u64 nN = rc.n_neurons, nA = rc.n_astro;
    cudaStream_t st = sim.stream();
    AS_CUDA(cudaMemsetAsync(s.x_cnt.get(), 0, 2 * sizeof(u32), st));
    const u32 nl = s.plan.n_hi - s.plan.n_lo, al = s.plan.a_hi - s.plan.a_lo;
    if (nl)
        pack_spikes_kernel<R><<<ceil_div(nl, 256), 256, 0, st>>>(
            w.spk_word + buf * nN, w.spk_val + static_cast<u64>(buf) * ws.W * nN, nN, s.plan.n_lo, s.plan.n_hi,
            s.x_keys.get(), reinterpret_cast<R*>(s.x_vals.get()), s.x_cnt.get());
    if (al)
        pack_astro_kernel<R><<<ceil_div(al, 256), 256, 0, st>>>(
            w.astro_active + static_cast<u64>(buf) * w.astro_words, w.sic_win + static_cast<u64>(buf) * nA * ws.W,
            s.plan.a_lo, s.plan.a_hi, ws.W, s.x_ids.get(), reinterpret_cast<R*>(s.x_facs.get()), s.x_cnt.get() + 1);
    AS_CUDA(cudaGetLastError());
    return Status::Ok();
}

template <typename R>
Status import_phase(ShardSim& s, i64 k, const u32* counts, u64 stride_spk, u64 stride_ast) {
    Simulation& sim = s.sim;
    const RunConsts& rc = sim.consts();
    WindowState& ws = *sim.window_state();
    WinPtrs<R> w = win_ptrs<R>(ws, rc);
    StepPtrs<R> p = make_ptrs<R>(sim.state_buffers(), sim.network(), rc, sim.raster_steps());
    const int buf = static_cast<int>(k & 1);
    const u64 nN = rc.n_neurons, nA = rc.n_astro;
    cudaStream_t st = sim.stream();
    // other ranks' parts of this window's buffers start empty
    u32* words = w.spk_word + buf * nN;
    if (s.plan.n_lo) AS_CUDA(cudaMemsetAsync(words, 0, s.plan.n_lo * sizeof(u32), st));
    if (s.plan.n_hi < nN) AS_CUDA(cudaMemsetAsync(words + s.plan.n_hi, 0, (nN - s.plan.n_hi) * sizeof(u32), st));
    u32* act = w.astro_active + static_cast<u64>(buf) * w.astro_words;
    const u32 w_lo = s.plan.a_lo / 32, w_hi = s.plan.a_hi == rc.n_astro ? w.astro_words : s.plan.a_hi / 32;
    if (w_lo) AS_CUDA(cudaMemsetAsync(act, 0, w_lo * sizeof(u32), st));
    if (w_hi < w.astro_words) AS_CUDA(cudaMemsetAsync(act + w_hi, 0, (w.astro_words - w_hi) * sizeof(u32), st));
    const size_t rb = sizeof(R);
    for (int r = 0; r < s.world; ++r) {
        if (r == s.rank) continue;
        const u32 ns = counts[2 * r], na = counts[2 * r + 1];
        if (ns)
            import_spikes_kernel<R><<<ceil_div(ns, 256), 256, 0, st>>>(
                s.r_keys.get() + r * stride_spk, reinterpret_cast<const R*>(s.r_vals.get() + r * stride_spk * rb), ns,
                w, nN, buf, k * ws.W, p.counts, p.raster, p.raster_steps, rc.words);
        if (na)
            import_astro_kernel<R><<<ceil_div(na, 256), 256, 0, st>>>(
                s.r_ids.get() + r * stride_ast,
                reinterpret_cast<const R*>(s.r_facs.get() + r * stride_ast * ws.W * rb), na, w, nA, buf);
    }
    AS_CUDA(cudaGetLastError());
    return Status::Ok();
}

template <typename R>
Status push_phase(ShardSim& s, i64 k) {
    Simulation& sim = s.sim;
    const RunConsts& rc = sim.consts();
    WindowState& ws = *sim.window_state();
    WinPtrs<R> w = win_ptrs<R>(ws, rc);
    const u32 blocks = std::max<u32>(1, std::min<u32>(sm_count() * 8, ceil_div(ws.push_limit, 8)));
    shard_push_kernel<R><<<blocks, 256, 0, sim.stream()>>>(w, rc.n_exc, sim.network().sz.n_inh, rc.n_neurons,
                                                           rc.n_astro, static_cast<int>(k & 1), s.plan.n_lo,
                                                           s.plan.n_hi, s.plan.a_lo, s.plan.a_hi);
    AS_CUDA(cudaGetLastError());
    return Status::Ok();
}

}  // namespace

// ---------------------------------------------------------------- bounded waits
double default_shard_timeout() {
    if (const char* env = std::getenv("ASTROSIM_SHARD_TIMEOUT_S")) {
        const double v = std::atof(env);
        if (v > 0.0) return v;
    }
    return 120.0;
}

Status bounded_wait(ShardComm* comm, const std::function<int()>& query, double timeout_s, const char* what) {
    using clock = std::chrono::steady_clock;
    const auto start = clock::now();
    const auto deadline = start + std::chrono::duration_cast<clock::duration>(std::chrono::duration<double>(timeout_s));
    auto next_poll = start;
    for (u64 it = 0;; ++it) {
        const int q = query();
        if (q == 0) return Status::Ok();
        if (q < 0) {
            if (comm) comm->abort();
            return make_error(ASTROSIM_ERR_CUDA, "%s: the device work failed", what);
        }
        const auto now = clock::now();
        if (comm && now >= next_poll) {  // the communicator's view of its peers, every 10 ms
            bool pending = false;
            Status st = comm->async_state(&pending);
            if (!st.ok()) {
                comm->abort();
                return make_error(ASTROSIM_ERR_PEER, "%s: %s", what, st.msg.c_str());
            }
            next_poll = now + std::chrono::milliseconds(10);
        }
        if (now >= deadline) {
            if (comm) comm->abort();
            return make_error(ASTROSIM_ERR_TIMEOUT,
                              "%s: no progress within %.3g s (a rank failed or left); the communicator is aborted",
                              what, timeout_s);
        }
        // spin for the first ~2 ms (an exchange usually completes within that), then back off
        if (now - start > std::chrono::milliseconds(2)) std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

Status bounded_stream_wait(ShardComm* comm, cudaStream_t st, double timeout_s, const char* what) {
    return bounded_wait(
        comm,
        [st]() {
            const cudaError_t e = cudaStreamQuery(st);
            if (e == cudaSuccess) return 0;
            if (e == cudaErrorNotReady) return 1;
            cudaGetLastError();
            return -1;
        },
        timeout_s, what);
}

namespace {

// A communicator whose peers behave as one failure scenario prescribes (no device).
class StandInComm : public ShardComm {
public:
    explicit StandInComm(int scenario) : scenario_(scenario) {}
    Status all_gather(const void*, void*, size_t, cudaStream_t) override { return Status::Ok(); }
    Status async_state(bool* pending) override {
        *pending = false;
        if (scenario_ == 2 && ++polls_ >= 3) return make_error(ASTROSIM_ERR_PEER, "a peer reported a failure");
        return Status::Ok();
    }
    void abort() override { aborted = true; }
    bool aborted = false;

private:
    int scenario_;
    int polls_ = 0;
};

}  // namespace

Status selftest_bounded_wait(int scenario, double timeout_s, int* windows_done, int* aborted, double* waited_s) {
    if (scenario < 0 || scenario > 3) return make_error(ASTROSIM_ERR_INVALID_ARG, "scenario must be 0-3");
    if (!(timeout_s > 0.0)) return make_error(ASTROSIM_ERR_INVALID_ARG, "timeout_s must be > 0");
    StandInComm comm(scenario);
    const auto t0 = std::chrono::steady_clock::now();
    int done = 0;
    Status st;
    for (int k = 0; k < 4 && st.ok(); ++k) {
        // window k's exchange: complete after a few polls, or never (a rank that left)
        const bool never = scenario == 1 || scenario == 2 || (scenario == 3 && k >= 2);
        int polls = 0;
        st = bounded_wait(&comm, [&]() { return (!never && ++polls > 3) ? 0 : 1; }, timeout_s, "window exchange");
        if (st.ok()) ++done;
    }
    if (windows_done) *windows_done = done;
    if (aborted) *aborted = comm.aborted ? 1 : 0;
    if (waited_s) *waited_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return st;
}

namespace {

// ---------------------------------------------------------------- NCCL, loaded at run time
struct NcclApi {
    void* lib = nullptr;
    ncclResult_t (*get_unique_id)(ncclUniqueId*) = nullptr;
    ncclResult_t (*comm_init_rank_config)(ncclComm_t*, int, ncclUniqueId, int, ncclConfig_t*) = nullptr;
    ncclResult_t (*all_gather)(const void*, void*, size_t, ncclDataType_t, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*group_start)() = nullptr;
    ncclResult_t (*group_end)() = nullptr;
    ncclResult_t (*comm_destroy)(ncclComm_t) = nullptr;
    ncclResult_t (*comm_abort)(ncclComm_t) = nullptr;
    ncclResult_t (*get_async_error)(ncclComm_t, ncclResult_t*) = nullptr;
    const char* (*error_string)(ncclResult_t) = nullptr;
};

Status nccl_api(NcclApi** out) {
    static NcclApi api;
    static bool tried = false;
    static Status status;
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    if (!tried) {
        tried = true;
        api.lib = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
        if (!api.lib) {
            status = make_error(ASTROSIM_ERR_UNSUPPORTED, "cannot load libnccl.so.2: %s", dlerror());
        } else {
            auto sym = [&](const char* name) { return dlsym(api.lib, name); };
            api.get_unique_id = reinterpret_cast<decltype(api.get_unique_id)>(sym("ncclGetUniqueId"));
            api.comm_init_rank_config =
                reinterpret_cast<decltype(api.comm_init_rank_config)>(sym("ncclCommInitRankConfig"));
            api.all_gather = reinterpret_cast<decltype(api.all_gather)>(sym("ncclAllGather"));
            api.group_start = reinterpret_cast<decltype(api.group_start)>(sym("ncclGroupStart"));
            api.group_end = reinterpret_cast<decltype(api.group_end)>(sym("ncclGroupEnd"));
            api.comm_destroy = reinterpret_cast<decltype(api.comm_destroy)>(sym("ncclCommDestroy"));
            api.comm_abort = reinterpret_cast<decltype(api.comm_abort)>(sym("ncclCommAbort"));
            api.get_async_error = reinterpret_cast<decltype(api.get_async_error)>(sym("ncclCommGetAsyncError"));
            api.error_string = reinterpret_cast<decltype(api.error_string)>(sym("ncclGetErrorString"));
            if (!api.get_unique_id || !api.comm_init_rank_config || !api.all_gather || !api.group_start ||
                !api.group_end || !api.comm_destroy || !api.comm_abort || !api.get_async_error || !api.error_string)
                status = make_error(ASTROSIM_ERR_UNSUPPORTED, "libnccl.so.2 lacks an entry point");
        }
    }
    *out = &api;
    return status;
}

// A non-blocking communicator: set-up and every enqueue may return ncclInProgress,
// and ncclCommGetAsyncError then reports when it has finished, so each wait has a
// deadline and a communicator whose peer vanished is aborted instead of hanging.
class NcclComm : public ShardComm {
public:
    ~NcclComm() override {
        if (comm_) api_->comm_destroy(comm_);
    }
    Status init(const unsigned char id[128], int rank, int world, int device, double timeout_s) {
        AS_TRY(nccl_api(&api_));
        AS_CUDA(cudaSetDevice(device));
        timeout_s_ = timeout_s;
        ncclUniqueId uid;
        static_assert(sizeof(uid) == 128, "ncclUniqueId is 128 bytes");
        std::memcpy(&uid, id, sizeof(uid));
        ncclConfig_t config = NCCL_CONFIG_INITIALIZER;
        config.blocking = 0;
        AS_TRY(settle(api_->comm_init_rank_config(&comm_, world, uid, rank, &config), "ncclCommInitRankConfig"));
        return Status::Ok();
    }
    Status all_gather(const void* send, void* recv, size_t bytes, cudaStream_t st) override {
        if (bytes == 0) return Status::Ok();
        return settle(api_->all_gather(send, recv, bytes, ncclUint8, comm_, st), "ncclAllGather");
    }
    Status group_begin() override { return settle(api_->group_start(), "ncclGroupStart"); }
    Status group_end() override { return settle(api_->group_end(), "ncclGroupEnd"); }
    Status async_state(bool* pending) override {
        *pending = false;
        if (!comm_) return make_error(ASTROSIM_ERR_PEER, "the communicator was aborted");
        ncclResult_t state = ncclSuccess;
        const ncclResult_t r = api_->get_async_error(comm_, &state);
        if (r != ncclSuccess) return make_error(ASTROSIM_ERR_PEER, "ncclCommGetAsyncError: %s", api_->error_string(r));
        if (state == ncclInProgress) {
            *pending = true;
            return Status::Ok();
        }
        if (state != ncclSuccess) return make_error(ASTROSIM_ERR_PEER, "NCCL: %s", api_->error_string(state));
        return Status::Ok();
    }
    void abort() override {
        if (comm_) api_->comm_abort(comm_);
        comm_ = nullptr;
    }

private:
    // A call's result once it has settled: ncclInProgress is polled to completion
    // under the deadline.
    Status settle(ncclResult_t r, const char* what) {
        if (r == ncclSuccess) return Status::Ok();
        if (r != ncclInProgress) {
            abort();
            return make_error(ASTROSIM_ERR_PEER, "%s failed: %s", what, api_->error_string(r));
        }
        Status st;
        return bounded_wait(
            this,
            [&]() {
                bool pending = false;
                st = async_state(&pending);
                return !st.ok() ? -1 : (pending ? 1 : 0);
            },
            timeout_s_, what);
    }
    NcclApi* api_ = nullptr;
    ncclComm_t comm_ = nullptr;
    double timeout_s_ = 120.0;
};

}  // namespace

Status nccl_unique_id(unsigned char id[128]) {
    NcclApi* api = nullptr;
    AS_TRY(nccl_api(&api));
    ncclUniqueId uid;
    const ncclResult_t r = api->get_unique_id(&uid);
    if (r != ncclSuccess) return make_error(ASTROSIM_ERR_CUDA, "ncclGetUniqueId failed: %s", api->error_string(r));
    std::memcpy(id, &uid, 128);
    return Status::Ok();
}

Status make_nccl_comm(const unsigned char id[128], int rank, int world, int device, double timeout_s,
                      std::unique_ptr<ShardComm>& out) {
    auto c = std::make_unique<NcclComm>();
    AS_TRY(c->init(id, rank, world, device, timeout_s));
    out = std::move(c);
    return Status::Ok();
}

// ---------------------------------------------------------------- ShardSim
ShardSim::~ShardSim() {
    if (h_cnt_) cudaFreeHost(h_cnt_);
}

Status ShardSim::create(const astrosim_config& cfg, const char* biology_json, int r, int n) {
    if (n < 1 || r < 0 || r >= n) return make_error(ASTROSIM_ERR_INVALID_ARG, "rank %d of %d", r, n);
    rank = r;
    world = n;
    {
        // this rank keeps the connectivity rows of its own cells only (about 1 / world of it)
        const Sizes sz = scaling_law(cfg.n_total);
        const ShardPlan pl = shard_plan(sz.n_neurons, sz.n_astro, r, n);
        CellRange own;
        own.n_lo = pl.n_lo;
        own.n_hi = pl.n_hi;
        own.a_lo = pl.a_lo;
        own.a_hi = pl.a_hi;
        AS_TRY(sim.create(cfg, biology_json, &own));
    }
    if (!sim.windowed())
        return make_error(ASTROSIM_ERR_UNSUPPORTED,
                          "a sharded network needs the windowed engine (equal delays of 2-16 steps)");
    const RunConsts& rc = sim.consts();
    W_ = sim.window_state()->W;
    plan = shard_plan(rc.n_neurons, rc.n_astro, rank, world);
    u64 max_n = 0, max_a = 0;
    for (int q = 0; q < world; ++q) {
        const ShardPlan pq = shard_plan(rc.n_neurons, rc.n_astro, q, world);
        max_n = std::max<u64>(max_n, pq.n_hi - pq.n_lo);
        max_a = std::max<u64>(max_a, pq.a_hi - pq.a_lo);
    }
    cap_spk = max_n * W_;  // a neuron spikes at most once per step
    cap_ast = max_a;
    const size_t rb = real_bytes();
    AS_CUDA(cudaSetDevice(device()));
    AllocStream scope(sim.stream());
    AS_TRY(x_keys.alloc(cap_spk));
    AS_TRY(x_vals.alloc(cap_spk * rb));
    AS_TRY(x_ids.alloc(cap_ast));
    AS_TRY(x_facs.alloc(cap_ast * W_ * rb));
    AS_TRY(x_cnt.alloc_zero(2, sim.stream()));
    AS_TRY(r_keys.alloc(cap_spk * world));
    AS_TRY(r_vals.alloc(cap_spk * world * rb));
    AS_TRY(r_ids.alloc(cap_ast * world));
    AS_TRY(r_facs.alloc(cap_ast * world * W_ * rb));
    AS_TRY(r_cnt.alloc_zero(2 * world, sim.stream()));
    AS_CUDA(cudaMallocHost(&h_cnt_, 2 * world * sizeof(u32)));
    std::memset(h_cnt_, 0, 2 * world * sizeof(u32));
    AS_CUDA(cudaStreamSynchronize(sim.stream()));
    return Status::Ok();
}

Status ShardSim::run_window(i64 k) {
    AS_CUDA(cudaSetDevice(device()));
    return sim.fp32() ? window_phase<float>(*this, k) : window_phase<double>(*this, k);
}

Status ShardSim::pack(i64 k) {
    AS_CUDA(cudaSetDevice(device()));
    AS_TRY(sim.fp32() ? pack_phase<float>(*this, k) : pack_phase<double>(*this, k));
    AS_CUDA(cudaMemcpyAsync(h_cnt_ + 2 * rank, x_cnt.get(), 2 * sizeof(u32), cudaMemcpyDeviceToHost, stream()));
    return Status::Ok();
}

Status ShardSim::import(i64 k, const u32* counts, u64 stride_spk, u64 stride_ast) {
    AS_CUDA(cudaSetDevice(device()));
    return sim.fp32() ? import_phase<float>(*this, k, counts, stride_spk, stride_ast)
                      : import_phase<double>(*this, k, counts, stride_spk, stride_ast);
}

Status ShardSim::push(i64 k) {
    AS_CUDA(cudaSetDevice(device()));
    return sim.fp32() ? push_phase<float>(*this, k) : push_phase<double>(*this, k);
}

void ShardSim::note_window(double seconds) { sim.note_external_steps(W_, seconds); }

namespace {

Status check_whole_windows(Simulation& sim, int W, i64 n) {
    if (n < 0) return make_error(ASTROSIM_ERR_INVALID_ARG, "n_steps must be >= 0");
    if (n % W != 0 || sim.steps_done() % W != 0)
        return make_error(ASTROSIM_ERR_INVALID_ARG, "a sharded network steps in whole windows of %d steps", W);
    return sim.reserve_steps(sim.steps_done() + n);
}

// Offsets of rank r's slice of a state array.
void slice_of(const ShardPlan& p, bool astro, u64* lo, u64* len) {
    *lo = astro ? p.a_lo : p.n_lo;
    *len = astro ? p.a_hi - p.a_lo : p.n_hi - p.n_lo;
}

}  // namespace

// ---------------------------------------------------------------- ShardRank (NCCL)
Status ShardRank::create(const astrosim_config& cfg, const char* biology_json, int rank, int world) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return make_error(ASTROSIM_ERR_NO_DEVICE, "no CUDA device visible");
    }
    s_ = std::make_unique<ShardSim>();
    return s_->create(cfg, biology_json, rank, world);
}

Status ShardRank::connect(const unsigned char id[128]) {
    if (!s_) return make_error(ASTROSIM_ERR_STATE, "create the shard first");
    if (s_->world == 1) return Status::Ok();
    Status st = make_nccl_comm(id, s_->rank, s_->world, s_->device(), timeout_s_, comm_);
    if (!st.ok()) failed_ = true;
    return st;
}

Status ShardRank::usable() const {
    if (!s_) return make_error(ASTROSIM_ERR_STATE, "create the shard first");
    if (failed_)
        return make_error(ASTROSIM_ERR_STATE,
                          "an earlier wait on the other ranks failed; the communicator is aborted and the "
                          "network is mid-window: destroy this rank");
    if (!comm_ && s_->world > 1) return make_error(ASTROSIM_ERR_STATE, "connect the ranks first");
    return Status::Ok();
}

Status ShardRank::wait(const char* what) {
    Status st = bounded_stream_wait(comm_.get(), s_->stream(), timeout_s_, what);
    if (!st.ok()) failed_ = true;
    return st;
}

Status ShardRank::step(i64 n) {
    AS_TRY(usable());
    ShardSim& s = *s_;
    const int W = s.window();
    AS_TRY(check_whole_windows(s.sim, W, n));
    AS_CUDA(cudaSetDevice(s.device()));
    cudaStream_t st = s.stream();
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    AS_CUDA(cudaEventCreate(&e0));
    AS_CUDA(cudaEventCreate(&e1));
    AS_CUDA(cudaEventRecord(e0, st));
    const size_t rb = s.real_bytes();
    Status status;
    for (i64 k = s.sim.steps_done() / W, end = (s.sim.steps_done() + n) / W; k < end && status.ok(); ++k) {
        const auto t0 = std::chrono::steady_clock::now();
        status = [&]() -> Status {
            AS_TRY(s.run_window(k));
            if (s.world == 1) return s.push(k);  // nothing to exchange
            AS_TRY(s.pack(k));
            AS_TRY(comm_->all_gather(s.x_cnt.get(), s.r_cnt.get(), 2 * sizeof(u32), st));
            // pinned destination: a copy into pageable memory would block until the
            // all-gather ends, outside the deadline
            u32* hc = s.host_counts_buffer();
            AS_CUDA(cudaMemcpyAsync(hc, s.r_cnt.get(), 2 * s.world * sizeof(u32), cudaMemcpyDeviceToHost, st));
            AS_TRY(wait("window count exchange"));
            const std::vector<u32> c(hc, hc + 2 * s.world);
            u64 ms = 0, ma = 0;
            for (int r = 0; r < s.world; ++r) {
                ms = std::max<u64>(ms, c[2 * r]);
                ma = std::max<u64>(ma, c[2 * r + 1]);
            }
            AS_TRY(comm_->group_begin());
            AS_TRY(comm_->all_gather(s.x_keys.get(), s.r_keys.get(), ms * sizeof(u32), st));
            AS_TRY(comm_->all_gather(s.x_vals.get(), s.r_vals.get(), ms * rb, st));
            AS_TRY(comm_->all_gather(s.x_ids.get(), s.r_ids.get(), ma * sizeof(u32), st));
            AS_TRY(comm_->all_gather(s.x_facs.get(), s.r_facs.get(), ma * W * rb, st));
            AS_TRY(comm_->group_end());
            AS_TRY(s.import(k, c.data(), ms, ma));
            AS_TRY(s.push(k));
            return Status::Ok();
        }();
        s.note_window(std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
    }
    if (!status.ok()) failed_ = true;  // a window stopped part-way
    AS_CUDA(cudaEventRecord(e1, st));
    if (status.ok()) status = wait("window exchange");
    if (!status.ok()) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return status;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    last_ms_ = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return status;
}

Status ShardRank::gather(int which) {
    if (s_->world == 1) return Status::Ok();
    AS_TRY(usable());
    ShardSim& s = *s_;
    void* base = nullptr;
    size_t elem = 0;
    u64 n = 0;
    bool astro = false;
    AS_TRY(s.sim.state_location(which, &base, &elem, &n, &astro));
    u64 max_len = 0;
    std::vector<ShardPlan> plans(s.world);
    for (int r = 0; r < s.world; ++r) {
        plans[r] = shard_plan(s.sim.consts().n_neurons, s.sim.consts().n_astro, r, s.world);
        u64 lo, len;
        slice_of(plans[r], astro, &lo, &len);
        max_len = std::max(max_len, len);
    }
    if (max_len == 0) return Status::Ok();
    cudaStream_t st = s.stream();
    AS_CUDA(cudaSetDevice(s.device()));
    AllocStream scope(st);
    DevBuf<unsigned char> send, recv;
    AS_TRY(send.alloc(max_len * elem));
    AS_TRY(recv.alloc(max_len * elem * s.world));
    u64 lo, len;
    slice_of(s.plan, astro, &lo, &len);
    unsigned char* b = static_cast<unsigned char*>(base);
    if (len) AS_CUDA(cudaMemcpyAsync(send.get(), b + lo * elem, len * elem, cudaMemcpyDeviceToDevice, st));
    AS_TRY(comm_->all_gather(send.get(), recv.get(), max_len * elem, st));
    for (int r = 0; r < s.world; ++r) {
        if (r == s.rank) continue;
        slice_of(plans[r], astro, &lo, &len);
        if (len)
            AS_CUDA(cudaMemcpyAsync(b + lo * elem, recv.get() + r * max_len * elem, len * elem,
                                    cudaMemcpyDeviceToDevice, st));
    }
    return wait("state gather");
}

Status ShardRank::summary(astrosim_summary_t& out) {
    AS_TRY(usable());
    AS_TRY(gather(ASTROSIM_STATE_CA));
    // the engaged flags sit beside the state arrays; gather them as bytes
    if (s_->world > 1) {
        ShardSim& s = *s_;
        u64 max_len = 0;
        std::vector<ShardPlan> plans(s.world);
        for (int r = 0; r < s.world; ++r) {
            plans[r] = shard_plan(s.sim.consts().n_neurons, s.sim.consts().n_astro, r, s.world);
            max_len = std::max<u64>(max_len, plans[r].a_hi - plans[r].a_lo);
        }
        cudaStream_t st = s.stream();
        AllocStream scope(st);
        DevBuf<unsigned char> send, recv;
        AS_TRY(send.alloc(max_len));
        AS_TRY(recv.alloc(max_len * s.world));
        unsigned char* ev = s.sim.state_buffers().ever_active.get();
        const u64 len = s.plan.a_hi - s.plan.a_lo;
        if (len) AS_CUDA(cudaMemcpyAsync(send.get(), ev + s.plan.a_lo, len, cudaMemcpyDeviceToDevice, st));
        AS_TRY(comm_->all_gather(send.get(), recv.get(), max_len, st));
        for (int r = 0; r < s.world; ++r) {
            const u64 l = plans[r].a_hi - plans[r].a_lo;
            if (r != s.rank && l)
                AS_CUDA(cudaMemcpyAsync(ev + plans[r].a_lo, recv.get() + r * max_len, l, cudaMemcpyDeviceToDevice, st));
        }
        AS_TRY(wait("engaged-flag gather"));
    }
    return s_->sim.summary(out);
}

Status ShardRank::get_state(int which, double* dst, size_t count) {
    AS_TRY(usable());
    AS_TRY(gather(which));
    return s_->sim.get_state(which, dst, count);
}

// ---------------------------------------------------------------- ShardGroup (one process)
Status ShardGroup::create(const astrosim_config& cfg, const char* biology_json, int world, const int* devices) {
    if (world < 1) return make_error(ASTROSIM_ERR_INVALID_ARG, "world must be >= 1");
    for (int r = 0; r < world; ++r) {
        astrosim_config c = cfg;
        c.device = devices ? devices[r] : cfg.device;
        auto s = std::make_unique<ShardSim>();
        AS_TRY(s->create(c, biology_json, r, world));
        shards_.push_back(std::move(s));
    }
    counts_.assign(2 * world, 0);
    return Status::Ok();
}

namespace {

// Copies `bytes` from shard src's device memory to shard dst's on dst's stream.
Status copy_between(ShardSim& dst, void* to, ShardSim& src, const void* from, size_t bytes) {
    if (bytes == 0) return Status::Ok();
    if (dst.device() == src.device())
        AS_CUDA(cudaMemcpyAsync(to, from, bytes, cudaMemcpyDeviceToDevice, dst.stream()));
    else
        AS_CUDA(cudaMemcpyPeerAsync(to, dst.device(), from, src.device(), bytes, dst.stream()));
    return Status::Ok();
}

Status sync_all(std::vector<std::unique_ptr<ShardSim>>& shards) {
    for (auto& s : shards) {
        AS_CUDA(cudaSetDevice(s->device()));
        AS_CUDA(cudaStreamSynchronize(s->stream()));
    }
    return Status::Ok();
}

}  // namespace

Status ShardGroup::step(i64 n) {
    const int world = this->world();
    ShardSim& s0 = *shards_[0];
    const int W = s0.window();
    for (auto& s : shards_) AS_TRY(check_whole_windows(s->sim, W, n));
    const auto t_start = std::chrono::steady_clock::now();
    const size_t rb = s0.real_bytes();
    for (i64 k = s0.sim.steps_done() / W, end = (s0.sim.steps_done() + n) / W; k < end; ++k) {
        const auto t0 = std::chrono::steady_clock::now();
        for (auto& s : shards_) {
            AS_TRY(s->run_window(k));
            AS_TRY(s->pack(k));
        }
        AS_TRY(sync_all(shards_));
        u64 ms = 0, ma = 0;
        for (int r = 0; r < world; ++r) {
            counts_[2 * r] = shards_[r]->host_counts()[2 * r];
            counts_[2 * r + 1] = shards_[r]->host_counts()[2 * r + 1];
            ms = std::max<u64>(ms, counts_[2 * r]);
            ma = std::max<u64>(ma, counts_[2 * r + 1]);
        }
        // the all-gather, rank by rank: rank r's lists land at r * stride in every receive buffer
        for (int d = 0; d < world; ++d) {
            ShardSim& D = *shards_[d];
            AS_CUDA(cudaSetDevice(D.device()));
            for (int r = 0; r < world; ++r) {
                if (r == d) continue;
                ShardSim& S = *shards_[r];
                const u64 ns = counts_[2 * r], na = counts_[2 * r + 1];
                AS_TRY(copy_between(D, D.r_keys.get() + r * ms, S, S.x_keys.get(), ns * sizeof(u32)));
                AS_TRY(copy_between(D, D.r_vals.get() + r * ms * rb, S, S.x_vals.get(), ns * rb));
                AS_TRY(copy_between(D, D.r_ids.get() + r * ma, S, S.x_ids.get(), na * sizeof(u32)));
                AS_TRY(copy_between(D, D.r_facs.get() + r * ma * W * rb, S, S.x_facs.get(), na * W * rb));
            }
            AS_TRY(D.import(k, counts_.data(), ms, ma));
            AS_TRY(D.push(k));
        }
        AS_TRY(sync_all(shards_));  // every export is consumed before the next window overwrites it
        const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        for (auto& s : shards_) s->note_window(secs);
    }
    last_ms_ = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    return Status::Ok();
}

Status ShardGroup::gather(int which) {
    const int world = this->world();
    for (int d = 0; d < world; ++d) {
        ShardSim& D = *shards_[d];
        void* base_d = nullptr;
        size_t elem = 0;
        u64 n = 0;
        bool astro = false;
        AS_TRY(D.sim.state_location(which, &base_d, &elem, &n, &astro));
        AS_CUDA(cudaSetDevice(D.device()));
        for (int r = 0; r < world; ++r) {
            if (r == d) continue;
            ShardSim& S = *shards_[r];
            void* base_s = nullptr;
            AS_TRY(S.sim.state_location(which, &base_s, &elem, &n, &astro));
            u64 lo, len;
            slice_of(S.plan, astro, &lo, &len);
            AS_TRY(copy_between(D, static_cast<unsigned char*>(base_d) + lo * elem, S,
                                static_cast<unsigned char*>(base_s) + lo * elem, len * elem));
        }
    }
    return sync_all(shards_);
}

Status ShardGroup::summary(astrosim_summary_t& out) {
    AS_TRY(gather(ASTROSIM_STATE_CA));
    const int world = this->world();
    for (int d = 0; d < world; ++d) {
        ShardSim& D = *shards_[d];
        AS_CUDA(cudaSetDevice(D.device()));
        for (int r = 0; r < world; ++r) {
            if (r == d) continue;
            ShardSim& S = *shards_[r];
            const u64 len = S.plan.a_hi - S.plan.a_lo;
            AS_TRY(copy_between(D, D.sim.state_buffers().ever_active.get() + S.plan.a_lo, S,
                                S.sim.state_buffers().ever_active.get() + S.plan.a_lo, len));
        }
    }
    AS_TRY(sync_all(shards_));
    return shards_[0]->sim.summary(out);
}

Status ShardGroup::get_state(int which, double* dst, size_t count) {
    AS_TRY(gather(which));
    return shards_[0]->sim.get_state(which, dst, count);
}

}  // namespace astrosim
