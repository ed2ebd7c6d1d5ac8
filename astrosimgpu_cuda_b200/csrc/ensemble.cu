// ensemble.cu -- batched stepping of many independent networks (see ensemble.cuh).

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <type_traits>

#include "ensemble.cuh"
#include "window_kernels.cuh"

namespace astrosim {

namespace {

template <typename R>
struct alignas(16) NetDesc {
    NetScalars ns;  // the constants that differ between networks
    StepPtrs<R> p;
    WinPtrs<R> w;
    i64 mark;  // last step of the pre-run (src/astrosim_fused.cu:1066)
};

// Variants the autotuner chooses from: (tile size = block size, minimum resident
// blocks per SM).  A tile is `tile` consecutive cells of one population of one
// network; each block stages its network's descriptor once, so larger tiles stage
// less per cell and smaller tiles balance networks of very different sizes better.
struct EnsVariant {
    int tile, min_blocks;
};
constexpr EnsVariant kEnsVariantsF32[] = {{128, 6}, {128, 8}, {128, 4}, {64, 12}, {64, 16}, {64, 8},
                                          {256, 3}, {256, 4}, {256, 2}};
constexpr EnsVariant kEnsVariantsF64[] = {{128, 4}, {128, 5}, {128, 3}, {64, 8}, {64, 10}, {64, 6},
                                          {256, 2}, {256, 3}, {256, 1}};
constexpr int kEnsNumVariants = 9;
constexpr int kTileSizes[kNumTileSizes] = {64, 128, 256};
int tile_index(int tile) { return tile == 64 ? 0 : (tile == 256 ? 2 : 1); }
constexpr int kEnsTuneRounds = 2;
constexpr int kGraphWindows = 10;
constexpr u32 kPushBlocksPerNet = 4;

// One window of one tile of blockDim.x cells.  UNI: every network shares the constants
// outside NetScalars, which then come from the kernel parameters (`common`); otherwise
// each block also stages its network's full constants (`rcs`) into shared memory.
template <typename R, int TILE, int MB, bool UNI>
__global__ void __launch_bounds__(TILE, MB) ens_window_kernel(RunConsts common, const RunConsts* __restrict__ rcs,
                                                             const NetDesc<R>* __restrict__ descs,
                                                             const u32* __restrict__ tile_net,
                                                             const u32* __restrict__ tile_blk,
                                                             const i64* __restrict__ win,
                                                             const i64* __restrict__ stop, int W) {
    constexpr u32 kDescBytes = sizeof(NetDesc<R>);
    constexpr u32 kConstBytes = UNI ? 0 : sizeof(RunConsts);
    static_assert(kDescBytes % 16 == 0 && sizeof(RunConsts) % 16 == 0, "16-byte staging");
    __shared__ __align__(16) unsigned char smem[kDescBytes + kConstBytes];
    const u32 net = tile_net[blockIdx.x];
    const i64 k = win[net];
    const i64 start = k * W;
    const i64 end = stop[net];
    if (start >= end) return;  // finished or retired network: the whole block leaves
    {
        const uint4* src = reinterpret_cast<const uint4*>(descs + net);
        uint4* dst = reinterpret_cast<uint4*>(smem);
        for (u32 i = threadIdx.x; i < kDescBytes / 16; i += blockDim.x) dst[i] = src[i];
        if constexpr (!UNI) {
            const uint4* rsrc = reinterpret_cast<const uint4*>(rcs + net);
            uint4* rdst = reinterpret_cast<uint4*>(smem + kDescBytes);
            for (u32 i = threadIdx.x; i < kConstBytes / 16; i += blockDim.x) rdst[i] = rsrc[i];
        }
    }
    __syncthreads();
    const NetDesc<R>& d = *reinterpret_cast<const NetDesc<R>*>(smem);
    const int s_end = static_cast<int>(end - start < W ? end - start : W);
    const u32 tb = tile_blk[blockIdx.x];
    if constexpr (UNI) {
        window_cells<R>(common, d.ns, d.p, d.w, start, 0, s_end, static_cast<int>(k & 1), d.mark, tb & 0x7FFFFFFFu,
                        (tb >> 31) != 0);
    } else {
        const RunConsts& rc = *reinterpret_cast<const RunConsts*>(smem + kDescBytes);
        window_cells<R>(rc, d.ns, d.p, d.w, start, 0, s_end, static_cast<int>(k & 1), d.mark, tb & 0x7FFFFFFFu,
                        (tb >> 31) != 0);
    }
}

template <typename R>
__global__ void ens_push_kernel(const NetDesc<R>* __restrict__ descs, const i64* __restrict__ win,
                                const i64* __restrict__ stop, int W) {
    const u32 net = blockIdx.y;
    const i64 k = win[net];
    if (k * W + W > stop[net]) return;  // the window did not complete: no window follows it
    const NetDesc<R>& d = descs[net];
    push_cells<R>(d.w, d.ns.n_exc, d.ns.n_neurons - d.ns.n_exc, d.ns.n_neurons, d.ns.n_astro,
                  static_cast<int>(k & 1), blockIdx.x, gridDim.x);
}

__global__ void ens_advance_kernel(i64* win, const i64* stop, u32 n, int W) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && win[i] * W < stop[i]) win[i] += 1;
}

template <typename R, bool UNI>
void launch_ens_window_v(int v, u32 grid, cudaStream_t st, const RunConsts& common, const RunConsts* rcs,
                         const NetDesc<R>* d, const u32* tn, const u32* tb, const i64* win, const i64* stop, int W) {
    constexpr bool f32 = std::is_same<R, float>::value;
    const EnsVariant x = f32 ? kEnsVariantsF32[v] : kEnsVariantsF64[v];
#define AS_ENS(T, M) ens_window_kernel<R, T, M, UNI><<<grid, T, 0, st>>>(common, rcs, d, tn, tb, win, stop, W)
    if constexpr (f32) {
        switch (x.tile * 100 + x.min_blocks) {
            case 12808: AS_ENS(128, 8); break;
            case 12804: AS_ENS(128, 4); break;
            case 6412: AS_ENS(64, 12); break;
            case 6416: AS_ENS(64, 16); break;
            case 6408: AS_ENS(64, 8); break;
            case 25603: AS_ENS(256, 3); break;
            case 25604: AS_ENS(256, 4); break;
            case 25602: AS_ENS(256, 2); break;
            default: AS_ENS(128, 6); break;
        }
    } else {
        switch (x.tile * 100 + x.min_blocks) {
            case 12805: AS_ENS(128, 5); break;
            case 12803: AS_ENS(128, 3); break;
            case 6408: AS_ENS(64, 8); break;
            case 6410: AS_ENS(64, 10); break;
            case 6406: AS_ENS(64, 6); break;
            case 25602: AS_ENS(256, 2); break;
            case 25603: AS_ENS(256, 3); break;
            case 25601: AS_ENS(256, 1); break;
            default: AS_ENS(128, 4); break;
        }
    }
#undef AS_ENS
}

int variant_tile(bool fp32, int v) { return fp32 ? kEnsVariantsF32[v].tile : kEnsVariantsF64[v].tile; }

// One window and its push for every network.
template <typename R>
void launch_ens_window(int v, bool uniform, u32 grid, u32 n, cudaStream_t st, const RunConsts& common,
                       const void* rcs, const void* descs, const u32* tn, const u32* tb, const i64* win,
                       const i64* stop, int W) {
    const RunConsts* r = static_cast<const RunConsts*>(rcs);
    const NetDesc<R>* d = static_cast<const NetDesc<R>*>(descs);
    if (uniform) launch_ens_window_v<R, true>(v, grid, st, common, r, d, tn, tb, win, stop, W);
    else launch_ens_window_v<R, false>(v, grid, st, common, r, d, tn, tb, win, stop, W);
    ens_push_kernel<R><<<dim3(kPushBlocksPerNet, n), 256, 0, st>>>(d, win, stop, W);
}

// `rc` with the NetScalars fields cleared.  RunConsts has no implicit padding, so
// equal constants compare equal bytewise; a signed zero that differs only sends a
// batch to the staged-constants kernel, never the reverse.
RunConsts common_part(const RunConsts& rc) {
    RunConsts m;
    std::memcpy(static_cast<void*>(&m), &rc, sizeof(RunConsts));
    m.seed = 0;
    m.n_exc = m.n_neurons = m.n_astro = m.words = 0;
    m.lambda_astro = m.limit_astro = m.lambda_exc = m.limit_exc = m.lambda_inh = m.limit_inh = 0.0;
    m.lim53_astro = m.lim53_exc = m.lim53_inh = 0;
    m.w_a2n = 0.0;
    m.f_w_a2n = 0.0f;
    return m;
}

template <typename R>
Status build_descs(std::vector<std::unique_ptr<Simulation>>& nets, DevBuf<unsigned char>& descs,
                   DevBuf<unsigned char>& rcs, RunConsts& common, bool& uniform, cudaStream_t st) {
    std::vector<NetDesc<R>> h(nets.size());
    std::vector<RunConsts> hr(nets.size());
    std::memset(static_cast<void*>(h.data()), 0, h.size() * sizeof(NetDesc<R>));
    std::memset(static_cast<void*>(hr.data()), 0, hr.size() * sizeof(RunConsts));
    bool first = true;
    uniform = true;
    std::memset(static_cast<void*>(&common), 0, sizeof(RunConsts));
    for (size_t i = 0; i < nets.size(); ++i) {
        Simulation* s = nets[i].get();
        if (!s) continue;
        const RunConsts& rc = s->consts();
        std::memcpy(static_cast<void*>(&hr[i]), &rc, sizeof(RunConsts));
        const RunConsts c = common_part(rc);
        if (first) {
            std::memcpy(static_cast<void*>(&common), &c, sizeof(RunConsts));
            first = false;
        } else if (std::memcmp(&common, &c, sizeof(RunConsts)) != 0) {
            uniform = false;
        }
        h[i].ns = net_scalars(rc);
        h[i].p = make_ptrs<R>(s->state_buffers(), s->network(), rc, s->raster_steps());
        h[i].w = win_ptrs<R>(*s->window_state(), rc);
        h[i].mark = s->pre_steps() == 0 ? 0 : s->pre_steps() - 1;
    }
    AS_TRY(descs.alloc(std::max<size_t>(1, h.size()) * sizeof(NetDesc<R>)));
    AS_TRY(rcs.alloc(std::max<size_t>(1, hr.size()) * sizeof(RunConsts)));
    if (!h.empty()) {
        AS_CUDA(cudaMemcpyAsync(descs.get(), h.data(), h.size() * sizeof(NetDesc<R>), cudaMemcpyHostToDevice, st));
        AS_CUDA(cudaMemcpyAsync(rcs.get(), hr.data(), hr.size() * sizeof(RunConsts), cudaMemcpyHostToDevice, st));
    }
    AS_CUDA(cudaStreamSynchronize(st));
    return Status::Ok();
}

}  // namespace

Ensemble::~Ensemble() {
    if (stream_) cudaStreamSynchronize(stream_);
    if (graph_) cudaGraphExecDestroy(graph_);
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
    nets_.clear();
    for (cudaStream_t s : build_streams_)
        if (s) {
            cudaSetDevice(build_device_);
            if (cudaStreamSynchronize(s) == cudaSuccess) give_stream(build_device_, s);
            else cudaStreamDestroy(s);
        }
    build_streams_.clear();
    descs_.release();
    rcs_.release();
    for (int ti = 0; ti < kNumTileSizes; ++ti) {
        tile_net_[ti].release();
        tile_blk_[ti].release();
    }
    win_.release();
    stop_.release();
    if (stream_) {
        cudaStreamSynchronize(stream_);
        cudaStreamDestroy(stream_);
    }
}

Status Ensemble::init_empty(bool fp32, int window, int device) {
    fp32_ = fp32;
    W_ = window;
    device_ = device;
    AS_CUDA(cudaSetDevice(device_));
    AS_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    AS_CUDA(cudaEventCreate(&ev0_));
    AS_CUDA(cudaEventCreate(&ev1_));
    dirty_ = true;
    return Status::Ok();
}

Status Ensemble::create(const astrosim_config* cfgs, u32 n, const char* const* biology_json) {
    if (!cfgs || n == 0) return make_error(ASTROSIM_ERR_INVALID_ARG, "an ensemble needs at least one network");
    for (u32 i = 1; i < n; ++i) {
        if (cfgs[i].dt != cfgs[0].dt || cfgs[i].substeps != cfgs[0].substeps ||
            cfgs[i].precision != cfgs[0].precision || cfgs[i].device != cfgs[0].device)
            return make_error(ASTROSIM_ERR_INVALID_ARG,
                              "ensemble networks must share dt, substeps, precision and device (network %u differs)", i);
    }
    const auto t0 = std::chrono::steady_clock::now();
    nets_.resize(n);
    std::vector<Status> st(n);
    std::atomic<u32> next{0};
    // Builds overlap on the GPU but each waits on the host between its kernels, so
    // the threads contend for CPU past about three quarters of the host cores
    // (measured on a 16-core host: 12 threads build 62-71 networks/s at N = 2e3-2e4,
    // 8 threads 59-76, 16 threads 51-80).
    const u32 workers =
        std::min<u32>(n, std::max(1u, std::min(12u, std::thread::hardware_concurrency() * 3 / 4)));
    // Each worker lends one stream to every network it builds.  A stream per network
    // cost more than the builds in a fresh process: creating and first synchronising
    // 256 new streams from 12 threads took 8.7 s of thread time (2.3 s of a 2.3 s
    // build; 0.85 s once the streams existed).  The ensemble keeps the streams until
    // its networks are gone.
    AS_CUDA(cudaSetDevice(cfgs[0].device));
    build_device_ = cfgs[0].device;
    build_streams_.assign(workers, nullptr);
    for (u32 t = 0; t < workers; ++t) AS_CUDA(take_stream(build_device_, &build_streams_[t]));
    // per worker: first start, busy time, last end (ms from t0), printed under ASTROSIM_TIMING
    std::vector<double> w_first(workers, -1.0), w_busy(workers, 0.0), w_last(workers, 0.0);
    const auto ms_since = [&](std::chrono::steady_clock::time_point a) {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - a).count();
    };
    auto work = [&](u32 t) {
        for (u32 i = next++; i < n; i = next++) {
            const double a = ms_since(t0);
            if (w_first[t] < 0) w_first[t] = a;
            auto s = std::make_unique<Simulation>();
            s->lend_stream(build_streams_[t]);
            st[i] = s->create(cfgs[i], biology_json ? biology_json[i] : nullptr);
            nets_[i] = std::move(s);
            w_last[t] = ms_since(t0);
            w_busy[t] += w_last[t] - a;
        }
    };
    // networks are built concurrently, one worker stream each
    std::vector<std::thread> pool;
    for (u32 t = 1; t < workers; ++t) pool.emplace_back(work, t);
    work(0);
    for (auto& th : pool) th.join();
    const auto t_built = std::chrono::steady_clock::now();
    for (u32 i = 0; i < n; ++i)
        if (!st[i].ok()) return make_error(st[i].code, "network %u: %s", i, st[i].msg.c_str());
    for (u32 i = 0; i < n; ++i)
        if (!nets_[i]->windowed() || nets_[i]->consts().d_e != nets_[0]->consts().d_e)
            return make_error(ASTROSIM_ERR_UNSUPPORTED, "ensemble networks need the windowed engine with one window");
    AS_TRY(init_empty(cfgs[0].precision == ASTROSIM_PRECISION_FP32, nets_[0]->consts().d_e, cfgs[0].device));
    AllocStream alloc_scope(stream_);
    win_host_.assign(n, 0);
    AS_TRY(win_.alloc_zero(n, stream_));
    std::vector<i64> stops(n);
    for (u32 i = 0; i < n; ++i) stops[i] = nets_[i]->total_steps();
    AS_TRY(stop_.alloc(n));
    AS_CUDA(cudaMemcpyAsync(stop_.get(), stops.data(), n * sizeof(i64), cudaMemcpyHostToDevice, stream_));
    AS_TRY(rebuild());
    const auto t_end = std::chrono::steady_clock::now();
    build_seconds_ = std::chrono::duration<double>(t_end - t0).count();
    if (std::getenv("ASTROSIM_TIMING")) {
        std::fprintf(stderr, "[astrosim ensemble] %u networks on %u threads %.3f ms, descriptors and tiles %.3f ms\n", n,
                     workers, std::chrono::duration<double, std::milli>(t_built - t0).count(),
                     std::chrono::duration<double, std::milli>(t_end - t_built).count());
        for (u32 t = 0; t < workers; ++t)
            std::fprintf(stderr, "[astrosim ensemble] worker %u: first start %.1f ms, busy %.1f ms, last end %.1f ms\n", t,
                         w_first[t], w_busy[t], w_last[t]);
    }
    return Status::Ok();
}

Status Ensemble::rebuild() {
    AS_CUDA(cudaSetDevice(device_));
    AllocStream alloc_scope(stream_);
    if (fp32_) AS_TRY(build_descs<float>(nets_, descs_, rcs_, common_, uniform_, stream_));
    else AS_TRY(build_descs<double>(nets_, descs_, rcs_, common_, uniform_, stream_));
    // one tile table per tile size: tile b of a population covers its cells [b * tile, (b + 1) * tile)
    for (int ti = 0; ti < kNumTileSizes; ++ti) {
        const u32 tile = static_cast<u32>(kTileSizes[ti]);
        std::vector<u32> tn, tb;
        for (u32 i = 0; i < nets_.size(); ++i) {
            if (!nets_[i]) continue;
            const RunConsts& rc = nets_[i]->consts();
            for (u32 b = 0; b < ceil_div(rc.n_astro, tile); ++b) {
                tn.push_back(i);
                tb.push_back(b | 0x80000000u);
            }
            for (u32 b = 0; b < ceil_div(rc.n_neurons, tile); ++b) {
                tn.push_back(i);
                tb.push_back(b);
            }
        }
        n_tiles_[ti] = static_cast<u32>(tn.size());
        AS_TRY(tile_net_[ti].alloc(std::max<size_t>(1, tn.size())));
        AS_TRY(tile_blk_[ti].alloc(std::max<size_t>(1, tb.size())));
        if (!tn.empty()) {
            AS_CUDA(cudaMemcpyAsync(tile_net_[ti].get(), tn.data(), tn.size() * sizeof(u32), cudaMemcpyHostToDevice,
                                    stream_));
            AS_CUDA(cudaMemcpyAsync(tile_blk_[ti].get(), tb.data(), tb.size() * sizeof(u32), cudaMemcpyHostToDevice,
                                    stream_));
        }
        AS_CUDA(cudaStreamSynchronize(stream_));  // the host vectors die at the end of this iteration
    }
    if (graph_) {
        cudaGraphExecDestroy(graph_);
        graph_ = nullptr;
    }
    dirty_ = false;
    return Status::Ok();
}

void Ensemble::launch_window(int v) {
    const u32 n = static_cast<u32>(nets_.size());
    const int ti = tile_index(variant_tile(fp32_, v));
    if (fp32_)
        launch_ens_window<float>(v, uniform_, n_tiles_[ti], n, stream_, common_, rcs_.get(), descs_.get(),
                                 tile_net_[ti].get(), tile_blk_[ti].get(), win_.get(), stop_.get(), W_);
    else
        launch_ens_window<double>(v, uniform_, n_tiles_[ti], n, stream_, common_, rcs_.get(), descs_.get(),
                                  tile_net_[ti].get(), tile_blk_[ti].get(), win_.get(), stop_.get(), W_);
}

Status Ensemble::capture_graph() {
    if (graph_) return Status::Ok();
    const u32 n = static_cast<u32>(nets_.size());
    cudaGraph_t g = nullptr;
    AS_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < kGraphWindows; ++k) {
        launch_window(variant_);
        ens_advance_kernel<<<ceil_div(n, 256), 256, 0, stream_>>>(win_.get(), stop_.get(), n, W_);
    }
    const cudaError_t e = cudaStreamEndCapture(stream_, &g);
    if (e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return cuda_status(e, "cudaStreamEndCapture", __FILE__, __LINE__);
    }
    const cudaError_t e2 = cudaGraphInstantiate(&graph_, g, 0);
    cudaGraphDestroy(g);
    if (e2 != cudaSuccess) {
        graph_ = nullptr;
        return cuda_status(e2, "cudaGraphInstantiate", __FILE__, __LINE__);
    }
    graph_windows_ = kGraphWindows;
    return Status::Ok();
}

Status Ensemble::advance_windows(i64 windows) {
    AS_CUDA(cudaSetDevice(device_));
    if (dirty_) AS_TRY(rebuild());
    const u32 n = static_cast<u32>(nets_.size());
    if (n == 0 || n_tiles_[1] == 0 || windows <= 0) return Status::Ok();
    const auto t0 = std::chrono::steady_clock::now();
    AS_CUDA(cudaEventRecord(ev0_, stream_));
    i64 done = 0;
    auto one_window = [&](int v) -> Status {
        launch_window(v);
        ens_advance_kernel<<<ceil_div(n, 256), 256, 0, stream_>>>(win_.get(), stop_.get(), n, W_);
        AS_CUDA(cudaGetLastError());
        return Status::Ok();
    };
    // autotune the (tile size, launch bounds) variant on the first windows (results do not
    // depend on it); ASTROSIM_ENSEMBLE_VARIANT fixes it (the tests run every variant)
    if (variant_ < 0) {
        if (const char* env = std::getenv("ASTROSIM_ENSEMBLE_VARIANT"))
            variant_ = std::min(kEnsNumVariants - 1, std::max(0, std::atoi(env)));
    }
    while (variant_ < 0 && done < windows) {
        const int v = tune_step_ % kEnsNumVariants;
        cudaEvent_t a = nullptr, b = nullptr;
        AS_CUDA(cudaEventCreate(&a));
        AS_CUDA(cudaEventCreate(&b));
        AS_CUDA(cudaEventRecord(a, stream_));
        Status s = one_window(v);
        AS_CUDA(cudaEventRecord(b, stream_));
        AS_CUDA(cudaEventSynchronize(b));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        AS_TRY(s);
        tune_ms_[v] = std::min(tune_ms_[v], ms);
        ++done;
        if (++tune_step_ == kEnsNumVariants * kEnsTuneRounds) {
            int best = 0;
            for (int i = 1; i < kEnsNumVariants; ++i)
                if (tune_ms_[i] < tune_ms_[best]) best = i;
            variant_ = best;
        }
    }
    if (done < windows) {
        AS_TRY(capture_graph());
        while (windows - done >= graph_windows_) {
            AS_CUDA(cudaGraphLaunch(graph_, stream_));
            done += graph_windows_;
        }
        while (done < windows) {
            AS_TRY(one_window(variant_));
            ++done;
        }
    }
    AS_CUDA(cudaEventRecord(ev1_, stream_));
    have_events_ = true;
    AS_CUDA(cudaStreamSynchronize(stream_));
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    // every unfinished network advanced one window per window launched
    for (u32 i = 0; i < n; ++i) {
        if (!nets_[i]) continue;
        const i64 before = nets_[i]->steps_done();
        const i64 after = std::min<i64>(nets_[i]->total_steps(), (win_host_[i] + windows) * W_);
        win_host_[i] = std::min<i64>(win_host_[i] + windows, (nets_[i]->total_steps() + W_ - 1) / W_);
        if (after > before) nets_[i]->note_external_steps(after - before, secs);
    }
    return Status::Ok();
}

Status Ensemble::step(i64 n_steps) {
    if (n_steps < 0) return make_error(ASTROSIM_ERR_INVALID_ARG, "n_steps must be >= 0");
    if (n_steps % W_ != 0)
        return make_error(ASTROSIM_ERR_INVALID_ARG, "ensemble steps come in whole windows of %d steps", W_);
    AS_TRY(advance_windows(n_steps / W_));
    steps_done_ += n_steps;
    return Status::Ok();
}

i64 Ensemble::net_steps_done(u32 i) const { return nets_[i] ? nets_[i]->steps_done() : 0; }

Status Ensemble::summary(u32 i, astrosim_summary_t& out) {
    if (!active(i)) return make_error(ASTROSIM_ERR_INVALID_ARG, "no network %u", i);
    AS_CUDA(cudaSetDevice(device_));
    AS_CUDA(cudaStreamSynchronize(stream_));
    return nets_[i]->summary(out);
}

Status Ensemble::get_state(u32 i, int which, double* dst, size_t count) {
    if (!active(i)) return make_error(ASTROSIM_ERR_INVALID_ARG, "no network %u", i);
    AS_CUDA(cudaStreamSynchronize(stream_));
    return nets_[i]->get_state(which, dst, count);
}

Status Ensemble::spike_counts(u32 i, i64 first, i64 n, u32* dst) {
    if (!active(i)) return make_error(ASTROSIM_ERR_INVALID_ARG, "no network %u", i);
    AS_CUDA(cudaStreamSynchronize(stream_));
    return nets_[i]->spike_counts(first, n, dst);
}

Status Ensemble::last_step_ms(double* ms) {
    if (!have_events_) return make_error(ASTROSIM_ERR_STATE, "no step has run yet");
    AS_CUDA(cudaEventSynchronize(ev1_));
    float f = 0.f;
    AS_CUDA(cudaEventElapsedTime(&f, ev0_, ev1_));
    *ms = f;
    return Status::Ok();
}

Status Ensemble::add(std::unique_ptr<Simulation> sim) {
    if (!sim || !sim->windowed() || sim->consts().d_e != W_ || sim->fp32() != fp32_)
        return make_error(ASTROSIM_ERR_INVALID_ARG, "network does not match the ensemble's window or precision");
    AS_CUDA(cudaSetDevice(device_));
    AS_CUDA(cudaStreamSynchronize(stream_));
    AS_CUDA(cudaStreamSynchronize(sim->stream()));
    // reuse a retired slot when one is free
    u32 slot = static_cast<u32>(nets_.size());
    for (u32 i = 0; i < nets_.size(); ++i)
        if (!nets_[i]) {
            slot = i;
            break;
        }
    const i64 stop = sim->total_steps();
    AllocStream alloc_scope(stream_);
    if (slot == nets_.size()) {
        nets_.push_back(std::move(sim));
        win_host_.push_back(0);
        DevBuf<i64> nw, ns;
        AS_TRY(nw.alloc(nets_.size()));
        AS_TRY(ns.alloc(nets_.size()));
        if (slot > 0) {
            AS_CUDA(cudaMemcpyAsync(nw.get(), win_.get(), slot * sizeof(i64), cudaMemcpyDeviceToDevice, stream_));
            AS_CUDA(cudaMemcpyAsync(ns.get(), stop_.get(), slot * sizeof(i64), cudaMemcpyDeviceToDevice, stream_));
        }
        win_ = std::move(nw);
        stop_ = std::move(ns);
    } else {
        nets_[slot] = std::move(sim);
        win_host_[slot] = 0;
    }
    const i64 zero = 0;
    AS_CUDA(cudaMemcpyAsync(win_.get() + slot, &zero, sizeof(i64), cudaMemcpyHostToDevice, stream_));
    AS_CUDA(cudaMemcpyAsync(stop_.get() + slot, &stop, sizeof(i64), cudaMemcpyHostToDevice, stream_));
    AS_CUDA(cudaStreamSynchronize(stream_));
    dirty_ = true;
    return Status::Ok();
}

Status Ensemble::retire(u32 i) {
    if (!active(i)) return make_error(ASTROSIM_ERR_INVALID_ARG, "no network %u", i);
    AS_CUDA(cudaSetDevice(device_));
    AS_CUDA(cudaStreamSynchronize(stream_));
    const i64 zero = 0;
    AS_CUDA(cudaMemcpyAsync(stop_.get() + i, &zero, sizeof(i64), cudaMemcpyHostToDevice, stream_));
    AS_CUDA(cudaStreamSynchronize(stream_));
    nets_[i].reset();
    dirty_ = true;
    return Status::Ok();
}

}  // namespace astrosim
