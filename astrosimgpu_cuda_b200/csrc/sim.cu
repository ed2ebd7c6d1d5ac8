// sim.cu -- device-resident simulation of one network: state set-up, the time
// loop (src/astrosim_fused.cu:1020-1102) and the summary (src/astrosim_fused.cu:1103-1141).

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <vector>

#include "biology.cuh"
#include "sim.cuh"
#include "step_kernels.cuh"
#include "window.cuh"
#include "builder_internal.cuh"
#include "reduce.cuh"

namespace astrosim {

namespace {


// One launch = one time step for every cell: the first `astro_blocks` blocks update
// astrocytes, the rest update neurons.  The two populations of one step read only
// rings written at least one step earlier (every delay is >= 1 step), so they may
// run concurrently; this replaces the reference's two launches per step
// (src/astrosim_fused.cu:1054-1064).
template <typename R>
__global__ void fused_step_kernel(RunConsts rc, StepPtrs<R> p, i64 step, u32 astro_blocks,
                                                         int sic_refresh, u64 noise_idx) {
    const NetScalars ns = net_scalars(rc);
    if (blockIdx.x < astro_blocks) {
        const u32 a = blockIdx.x * blockDim.x + threadIdx.x;
        if (a < rc.n_astro) astro_cell_step<R>(rc, ns, p, a, step);
        return;
    }
    const u32 j = (blockIdx.x - astro_blocks) * blockDim.x + threadIdx.x;
    R out = static_cast<R>(0.0);
    bool spiked = false;
    if (j < rc.n_neurons) spiked = neuron_cell_step<R>(rc, ns, p, j, step, sic_refresh != 0, noise_idx, out);
    // pack this warp's 32 spike bits into one word of the ring (warps cover aligned 32-neuron groups)
    const unsigned ballot = __ballot_sync(0xffffffffu, spiked);
    const int S = rc.slots;
    const u64 slot = static_cast<u64>(step % S);
    if ((threadIdx.x & 31) == 0 && j < rc.n_neurons) {
        const u32 word = j >> 5;
        p.bits[slot * rc.words + word] = ballot;
        if (ballot) atomicAdd(&p.counts[step], static_cast<u32>(__popc(ballot)));
        if (step < p.raster_steps) p.raster[static_cast<u64>(step) * rc.words + word] = ballot;
    }
    if (spiked) p.val[slot * rc.n_neurons + j] = out;
}

// exp(-lambda) of the Poisson drives and the constant synaptic decays are evaluated
// on the device, where the reference evaluates them (src/astrosim_fused.cu:167, 515-516).
__global__ void device_constants_kernel(double la, double le, double li, double* out) {
    out[0] = exp(-la);
    out[1] = exp(-le);
    out[2] = exp(-li);
}

template <typename R>
__global__ void init_state_kernel(StepPtrs<R> p, RunConsts rc, double V_e, double V_i, double Ca0, double IP30,
                                  double h0, double U) {
    const u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x;
    // src/astrosim_fused.cu:981-1005
    if (i < rc.n_neurons) {
        p.V[i] = i < rc.n_exc ? V_e : V_i;
        p.w[i] = 0.0;
        p.g_ex[i] = p.dg_ex[i] = p.g_in[i] = p.dg_in[i] = p.I_sic[i] = static_cast<R>(0.0);
        p.refr[i] = 0;
        p.stp_x[i] = static_cast<R>(1.0);
        p.stp_u[i] = static_cast<R>(U);
        p.stp_t[i] = -1e12;
    }
    if (i < rc.n_astro) {
        p.Ca[i] = Ca0;
        p.IP3[i] = IP30;
        p.h[i] = static_cast<R>(h0);
        p.ever_active[i] = 0;
        p.sic_last[i] = static_cast<R>(0.0);
    }
}

Biology biology_for(const astrosim_config& cfg, Biology b) {
    if (b.noise_dt <= 0.0) b.noise_dt = 10.0 * cfg.dt;  // src/astrosim_fused.cu:848
    if (!std::isnan(cfg.w_n2a)) b.w_n2a = cfg.w_n2a;
    if (!std::isnan(cfg.w_a2n)) b.w_a2n = cfg.w_a2n;
    if (!cfg.stp_enabled) b.stp_enabled = false;
    b.exc_poiss_rate = b.exc_poiss_rate * cfg.neuron_drive_scale;
    b.inh_poiss_rate = b.inh_poiss_rate * cfg.neuron_drive_scale;
    return b;
}

}  // namespace

void fill_stage_constants(RunConsts& rc) {
    rc.h6 = rc.h_step / 6.0;
    rc.f_h_step = static_cast<float>(rc.h_step);
    rc.f_h6 = rc.f_h_step / 6.0f;
    rc.f_w_e = static_cast<float>(rc.w_e);
    rc.f_neg_w_i = static_cast<float>(-rc.w_i);
    rc.f_w_n2a = static_cast<float>(rc.w_n2a);
    rc.f_w_a2n = static_cast<float>(rc.w_a2n);
    rc.f_weight_astro = static_cast<float>(rc.weight_astro);
    rc.f_weight_exc = static_cast<float>(rc.weight_exc);
    rc.f_weight_inh = static_cast<float>(rc.weight_inh);
    rc.f_noise_astro = static_cast<float>(rc.noise_astro);
    rc.pe.ref_steps = static_cast<int>(rc.pe.t_ref / rc.h_step + 0.5);
    rc.pi.ref_steps = static_cast<int>(rc.pi.t_ref / rc.h_step + 0.5);
}

Simulation::~Simulation() {
    // buffers are freed on stream_ (stream-ordered), so release them before the stream goes
    if (stream_) cudaStreamSynchronize(stream_);
    delete win_;
    win_ = nullptr;
    st_ = StateBuffers();
    net_ = Network();
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
    if (stream_ && stream_owned_) {
        if (cudaStreamSynchronize(stream_) == cudaSuccess) give_stream(device_, stream_);
        else cudaStreamDestroy(stream_);
    }
}

Status Simulation::create(const astrosim_config& cfg, const char* biology_json, const CellRange* own) {
    if (cfg.n_total == 0) return make_error(ASTROSIM_ERR_INVALID_ARG, "n_total must be >= 1");
    if (!(cfg.dt > 0.0) || !std::isfinite(cfg.dt)) return make_error(ASTROSIM_ERR_INVALID_ARG, "dt must be > 0");
    if (cfg.substeps < 1) return make_error(ASTROSIM_ERR_INVALID_ARG, "substeps must be >= 1");
    if (!(cfg.pre_ms >= 0.0) || !(cfg.sim_ms >= 0.0))
        return make_error(ASTROSIM_ERR_INVALID_ARG, "pre_ms and sim_ms must be >= 0");
    if (cfg.block != 0 && (cfg.block < 32 || cfg.block > 1024 || cfg.block % 32 != 0))
        return make_error(ASTROSIM_ERR_INVALID_ARG, "block must be 0 or a multiple of 32 in [32, 1024]");
    if (cfg.precision != ASTROSIM_PRECISION_FP64 && cfg.precision != ASTROSIM_PRECISION_FP32)
        return make_error(ASTROSIM_ERR_INVALID_ARG, "unknown precision %d", cfg.precision);
    if (cfg.raster_steps < 0) return make_error(ASTROSIM_ERR_INVALID_ARG, "raster_steps must be >= 0");
    cfg_ = cfg;
    fp32_ = cfg.precision == ASTROSIM_PRECISION_FP32;
    block_ = cfg.block == 0 ? 128 : cfg.block;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return make_error(ASTROSIM_ERR_NO_DEVICE, "no CUDA device visible");
    }
    if (cfg.device < 0 || cfg.device >= ndev)
        return make_error(ASTROSIM_ERR_INVALID_ARG, "device %d out of range (%d visible)", cfg.device, ndev);
    device_ = cfg.device;
    const double t_create = PhaseClock::now();
    AS_CUDA(cudaSetDevice(device_));
    if (!stream_) AS_CUDA(take_stream(device_, &stream_));
    keep_pool_memory(device_, 8ull << 30);
    AllocStream alloc_scope(stream_);
    PhaseClock(stream_).mark_since("stream", t_create);

    {
        Biology base;  // the reference's constants, then the JSON overrides, then cfg's fields
        AS_TRY(apply_biology_json(biology_json, base));
        bio_ = biology_for(cfg, base);
    }
    const Sizes sz = scaling_law(cfg.n_total);
    BuildOptions bo;
    if (own) bo.own = *own;
    AS_TRY(build_network(sz, cfg.seed, bio_, bo, net_, stream_));

    // run constants (src/astrosim_fused.cu:935-957, 1021-1024)
    RunConsts& rc = rc_;
    rc.ak = astro_constants(bio_);
    rc.pe = neuron_constants(bio_, true);
    rc.pi = neuron_constants(bio_, false);
    rc.dt = cfg.dt;
    rc.substeps = cfg.substeps;
    rc.h_step = cfg.dt / static_cast<double>(cfg.substeps);
    rc.d_e = delay_to_steps(bio_.d_e, cfg.dt);
    rc.d_i = delay_to_steps(bio_.d_i, cfg.dt);
    rc.d_a2n = delay_to_steps(bio_.d_a2n, cfg.dt);
    rc.slots = std::max({rc.d_e, rc.d_i, rc.d_a2n}) + 1;
    rc.steps_per_noise = std::max(1, static_cast<int>(std::llround(bio_.noise_dt / cfg.dt)));
    rc.sic_interval = bio_.sic_interval;
    rc.w_e = bio_.w_e;
    rc.w_i = bio_.w_i;
    rc.w_n2a = bio_.w_n2a;
    rc.w_a2n = bio_.w_a2n;
    rc.lambda_astro = bio_.astro_poiss_rate > 0.0 ? bio_.astro_poiss_rate * cfg.dt * 1e-3 : 0.0;
    rc.lambda_exc = bio_.exc_poiss_rate > 0.0 ? bio_.exc_poiss_rate * cfg.dt * 1e-3 : 0.0;
    rc.lambda_inh = bio_.inh_poiss_rate > 0.0 ? bio_.inh_poiss_rate * cfg.dt * 1e-3 : 0.0;
    rc.weight_astro = bio_.astro_poiss_weight;
    rc.weight_exc = bio_.exc_poiss_weight;
    rc.weight_inh = bio_.inh_poiss_weight;
    rc.noise_astro = bio_.astro_noise_std;
    rc.noise_exc = bio_.exc_noise_std;
    rc.noise_inh = bio_.inh_noise_std;
    rc.independent_noise = bio_.independent_noise;
    rc.stp_enabled = bio_.stp_enabled;
    rc.stp_U = bio_.stp_U;
    rc.stp_tau_rec = bio_.stp_tau_rec;
    rc.stp_tau_fac = bio_.stp_tau_fac;
    rc.SIC_th = bio_.SIC_th;
    rc.seed = cfg.seed;
    rc.n_exc = sz.n_exc;
    rc.n_neurons = sz.n_neurons;
    rc.n_astro = sz.n_astro;
    rc.words = (sz.n_neurons + 31) / 32;
    fill_stage_constants(rc);
    {
        DevBuf<double> lim;
        AS_TRY(lim.alloc(3));
        device_constants_kernel<<<1, 1, 0, stream_>>>(rc.lambda_astro, rc.lambda_exc, rc.lambda_inh, lim.get());
        AS_CUDA(cudaGetLastError());
        double h[3];
        AS_CUDA(cudaMemcpyAsync(h, lim.get(), sizeof(h), cudaMemcpyDeviceToHost, stream_));
        AS_CUDA(cudaStreamSynchronize(stream_));
        rc.limit_astro = h[0];
        rc.limit_exc = h[1];
        rc.limit_inh = h[2];
        rc.lim53_astro = static_cast<u64>(std::floor(h[0] * 9007199254740992.0));
        rc.lim53_exc = static_cast<u64>(std::floor(h[1] * 9007199254740992.0));
        rc.lim53_inh = static_cast<u64>(std::floor(h[2] * 9007199254740992.0));
    }

    pre_steps_ = static_cast<i64>(cfg.pre_ms / cfg.dt + 0.5);
    sim_steps_ = static_cast<i64>(cfg.sim_ms / cfg.dt + 0.5);
    total_steps_ = pre_steps_ + sim_steps_;

    // state
    const u64 nN = sz.n_neurons, nA = sz.n_astro;
    const size_t rbytes = fp32_ ? sizeof(float) : sizeof(double);
    AS_TRY(st_.V.alloc(nN));
    AS_TRY(st_.w.alloc(nN));
    AS_TRY(st_.Ca.alloc(nA));
    AS_TRY(st_.IP3.alloc(nA));
    AS_TRY(st_.g_raw.alloc((7 * nN + nA) * rbytes));
    AS_TRY(st_.stp_t.alloc(nN));
    AS_TRY(st_.refr.alloc(nN));
    AS_TRY(st_.ever_active.alloc(nA));
    // The windowed engine runs whenever every delay is the same D in [2, 16] steps,
    // which holds for the model's 1 ms delays at every dt from 0.0625 to 0.5 ms;
    // ASTROSIM_STEPPER=plain keeps the per-step path (used to cross-check the two).
    const char* stepper = std::getenv("ASTROSIM_STEPPER");
    windowed_ = rc.d_e == rc.d_i && rc.d_i == rc.d_a2n && rc.d_e >= 2 && rc.d_e <= kMaxWindow &&
                rc.n_neurons < (1u << 27) &&  // spike-list entries pack the neuron id in 27 bits
                !(stepper && std::strcmp(stepper, "plain") == 0);
    if (!windowed_) {
        net_.drop_forward();  // the per-step path reads only the target CSRs
        AS_TRY(st_.spike_bits.alloc_zero(static_cast<u64>(rc.slots) * rc.words, stream_));
        AS_TRY(st_.spike_val_raw.alloc_zero(static_cast<u64>(rc.slots) * nN * rbytes, stream_));
        AS_TRY(st_.sic_ring_raw.alloc_zero(static_cast<u64>(rc.slots) * nA * rbytes, stream_));
    } else {
        win_ = new WindowState();
        PhaseClock pc(stream_);
        AS_TRY(window_setup(rc, net_, fp32_, *win_, stream_));
        pc.mark("window set-up (forward CSRs)");
    }
    AS_TRY(st_.sic_last_raw.alloc(nA * rbytes));
    AS_TRY(st_.raster.alloc_zero(static_cast<u64>(cfg.raster_steps) * rc.words, stream_));
    AS_TRY(ensure_counts(std::max<i64>(total_steps_, 1)));
    AS_TRY(st_.reduce_raw.alloc(reduce_blocks(sz.n_astro) * sizeof(AstroPartial) + sizeof(AstroTotals)));
    const unsigned grid = ceil_div(std::max<u64>(nN, nA), 256);
    if (fp32_) {
        auto p = make_ptrs<float>(st_, net_, rc, cfg.raster_steps);
        init_state_kernel<float><<<grid, 256, 0, stream_>>>(p, rc, bio_.e_V_m, bio_.i_V_m, bio_.Ca_init,
                                                             bio_.IP3_init, bio_.h_init, bio_.stp_U);
    } else {
        auto p = make_ptrs<double>(st_, net_, rc, cfg.raster_steps);
        init_state_kernel<double><<<grid, 256, 0, stream_>>>(p, rc, bio_.e_V_m, bio_.i_V_m, bio_.Ca_init,
                                                              bio_.IP3_init, bio_.h_init, bio_.stp_U);
    }
    AS_CUDA(cudaGetLastError());
    AS_CUDA(cudaStreamSynchronize(stream_));
    PhaseClock(stream_).mark_since("simulation set-up (total)", t_create);
    return Status::Ok();
}

Status Simulation::ensure_counts(i64 steps) {
    if (steps <= counts_cap_) return Status::Ok();
    AllocStream alloc_scope(stream_);
    i64 cap = std::max<i64>(steps, counts_cap_ * 2);
    DevBuf<u32> nb;
    AS_TRY(nb.alloc_zero(static_cast<size_t>(cap), stream_));
    if (counts_cap_ > 0)
        AS_CUDA(cudaMemcpyAsync(nb.get(), st_.counts.get(), counts_cap_ * sizeof(u32), cudaMemcpyDeviceToDevice,
                                stream_));
    st_.counts = std::move(nb);
    counts_cap_ = cap;
    return Status::Ok();
}

Status Simulation::launch_steps(i64 first, i64 count) {
    if (windowed_) {
        const i64 mark = pre_steps_ == 0 ? 0 : pre_steps_ - 1;
        return window_launch(rc_, st_, net_, fp32_, *win_, cfg_.raster_steps, mark, first, count, stream_, cfg_.block);
    }
    const u32 astro_blocks = ceil_div(rc_.n_astro, block_);
    const u32 neuron_blocks = ceil_div(rc_.n_neurons, block_);
    for (i64 s = first; s < first + count; ++s) {
        // per-step scalars of the reference loop (src/astrosim_fused.cu:1043-1046)
        const u64 noise_idx = static_cast<u64>(s / rc_.steps_per_noise);
        const bool refresh = (s - rc_.d_a2n >= 0) && ((s - rc_.d_a2n) % rc_.sic_interval == 0);
        if (fp32_) {
            auto p = make_ptrs<float>(st_, net_, rc_, cfg_.raster_steps);
            fused_step_kernel<float><<<astro_blocks + neuron_blocks, block_, 0, stream_>>>(
                rc_, p, s, astro_blocks, refresh ? 1 : 0, noise_idx);
        } else {
            auto p = make_ptrs<double>(st_, net_, rc_, cfg_.raster_steps);
            fused_step_kernel<double><<<astro_blocks + neuron_blocks, block_, 0, stream_>>>(
                rc_, p, s, astro_blocks, refresh ? 1 : 0, noise_idx);
        }
        AS_CUDA(cudaGetLastError());
        // end of the pre-run: forget threshold crossings of the transient (src/astrosim_fused.cu:1066-1076)
        if (s == pre_steps_ - 1 || (pre_steps_ == 0 && s == 0))
            AS_CUDA(cudaMemsetAsync(st_.ever_active.get(), 0, rc_.n_astro, stream_));
    }
    return Status::Ok();
}

Status Simulation::step(i64 n) {
    if (n < 0) return make_error(ASTROSIM_ERR_INVALID_ARG, "n_steps must be >= 0");
    if (n == 0) return Status::Ok();
    AS_CUDA(cudaSetDevice(device_));
    AS_TRY(ensure_counts(steps_done_ + n));
    const auto t0 = std::chrono::steady_clock::now();
    // timing events are made on the first step: networks stepped by a batch never need them
    if (!ev0_) AS_CUDA(cudaEventCreate(&ev0_));
    if (!ev1_) AS_CUDA(cudaEventCreate(&ev1_));
    AS_CUDA(cudaEventRecord(ev0_, stream_));
    AS_TRY(launch_steps(steps_done_, n));
    AS_CUDA(cudaEventRecord(ev1_, stream_));
    have_step_events_ = true;
    steps_done_ += n;
    AS_CUDA(cudaStreamSynchronize(stream_));
    run_seconds_ += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return Status::Ok();
}

Status Simulation::record_calcium(i64 every, u32 first, u32 n, i64 max_samples) {
    if (every < 1) return make_error(ASTROSIM_ERR_INVALID_ARG, "every_steps must be >= 1");
    if (n == 0 || first >= rc_.n_astro || n > rc_.n_astro - first)
        return make_error(ASTROSIM_ERR_INVALID_ARG, "astrocytes [%u, %u + %u) not in [0, %u)", first, first, n,
                          rc_.n_astro);
    if (max_samples < 1) return make_error(ASTROSIM_ERR_INVALID_ARG, "max_samples must be >= 1");
    AS_CUDA(cudaSetDevice(device_));
    AS_CUDA(cudaStreamSynchronize(stream_));
    AllocStream alloc_scope(stream_);
    DevBuf<double> buf;
    AS_TRY(buf.alloc(static_cast<size_t>(max_samples) * n));
    st_.ca_rec = std::move(buf);
    st_.rec_every = every;
    st_.rec_k0 = (steps_done_ + every) / every;  // first sample ends the first interval after steps_done_
    st_.rec_cap = max_samples;
    st_.rec_first = first;
    st_.rec_n = n;
    return Status::Ok();
}

Status Simulation::calcium_samples(i64* n_samples, i64* first_step) {
    if (!st_.rec_n) return make_error(ASTROSIM_ERR_STATE, "calcium recording is off");
    const i64 last = steps_done_ / st_.rec_every;  // last interval completed
    i64 k = last - st_.rec_k0 + 1;
    k = k < 0 ? 0 : (k > st_.rec_cap ? st_.rec_cap : k);
    if (n_samples) *n_samples = k;
    if (first_step) *first_step = st_.rec_k0 * st_.rec_every - 1;
    return Status::Ok();
}

Status Simulation::copy_calcium(i64 first, i64 n, double* dst, bool wait) {
    i64 have = 0;
    AS_TRY(calcium_samples(&have, nullptr));
    if (first < 0 || n < 0 || first + n > have)
        return make_error(ASTROSIM_ERR_INVALID_ARG, "samples [%lld, %lld) not recorded (have %lld)",
                          static_cast<long long>(first), static_cast<long long>(first + n),
                          static_cast<long long>(have));
    if (n == 0) return Status::Ok();
    if (!dst) return make_error(ASTROSIM_ERR_INVALID_ARG, "null destination");
    AS_CUDA(cudaSetDevice(device_));
    AS_CUDA(cudaMemcpyAsync(dst, st_.ca_rec.get() + static_cast<u64>(first) * st_.rec_n,
                            static_cast<size_t>(n) * st_.rec_n * sizeof(double), cudaMemcpyDeviceToHost, stream_));
    if (wait) AS_CUDA(cudaStreamSynchronize(stream_));
    return Status::Ok();
}

Status Simulation::sync() {
    AS_CUDA(cudaSetDevice(device_));
    AS_CUDA(cudaStreamSynchronize(stream_));
    return Status::Ok();
}

Status Simulation::last_step_ms(double* ms) {
    if (!have_step_events_) return make_error(ASTROSIM_ERR_STATE, "no step has run yet");
    AS_CUDA(cudaEventSynchronize(ev1_));
    float f = 0.f;
    AS_CUDA(cudaEventElapsedTime(&f, ev0_, ev1_));
    *ms = f;
    return Status::Ok();
}

Status Simulation::spike_counts(i64 first, i64 n, u32* dst) {
    if (first < 0 || n < 0 || first + n > steps_done_)
        return make_error(ASTROSIM_ERR_INVALID_ARG, "steps [%lld, %lld) not done (done: %lld)",
                          static_cast<long long>(first), static_cast<long long>(first + n),
                          static_cast<long long>(steps_done_));
    if (n == 0) return Status::Ok();
    if (!dst) return make_error(ASTROSIM_ERR_INVALID_ARG, "null counts pointer");
    AS_CUDA(cudaMemcpyAsync(dst, st_.counts.get() + first, n * sizeof(u32), cudaMemcpyDeviceToHost, stream_));
    AS_CUDA(cudaStreamSynchronize(stream_));
    return Status::Ok();
}

Status Simulation::raster(u32* dst, size_t words) {
    const size_t need = static_cast<size_t>(cfg_.raster_steps) * rc_.words;
    if (!dst || words < need) return make_error(ASTROSIM_ERR_INVALID_ARG, "raster buffer needs %zu words", need);
    if (need) AS_CUDA(cudaMemcpyAsync(dst, st_.raster.get(), need * sizeof(u32), cudaMemcpyDeviceToHost, stream_));
    AS_CUDA(cudaStreamSynchronize(stream_));
    return Status::Ok();
}

Status Simulation::summary(astrosim_summary_t& out) {
    AS_CUDA(cudaSetDevice(device_));
    AS_CUDA(cudaStreamSynchronize(stream_));
    std::memset(&out, 0, sizeof(out));
    const Sizes& sz = net_.sz;
    out.n_total = sz.n_total;
    out.n_exc = sz.n_exc;
    out.n_inh = sz.n_inh;
    out.n_astro = sz.n_astro;
    out.p_primary = sz.p;
    out.n_exc_edges = net_.total_edges[0];  // the whole network's, also on a rank that keeps part of it
    out.n_inh_edges = net_.total_edges[1];
    out.n_e2a_edges = net_.total_edges[2];
    out.n_sic_edges = net_.total_edges[3];
    out.pre_steps = pre_steps_;
    out.sim_steps = sim_steps_;
    out.total_steps = total_steps_;
    out.steps_done = steps_done_;
    std::vector<u32> c(static_cast<size_t>(steps_done_));
    if (steps_done_) AS_TRY(spike_counts(0, steps_done_, c.data()));
    uint64_t tot = 0, before = 0;
    const i64 mark = pre_steps_ == 0 ? 0 : pre_steps_ - 1;  // last step counted as pre-run
    for (i64 s = 0; s < steps_done_; ++s) {
        tot += c[s];
        if (s <= mark) before += c[s];
    }
    if (steps_done_ <= mark) before = 0;  // the reference reads its counter only once the mark step is done
    out.spikes_total = tot;
    out.spikes_measured = tot - before;
    out.mean_rate_hz = static_cast<double>(out.spikes_measured) /
                       (static_cast<double>(sz.n_neurons) * (cfg_.sim_ms * 1e-3));
    // mean calcium, final-step threshold count and engaged count (src/astrosim_fused.cu:1111-1125),
    // reduced on the device
    AstroPartial* parts = reinterpret_cast<AstroPartial*>(st_.reduce_raw.get());
    AstroTotals* dtot = reinterpret_cast<AstroTotals*>(parts + reduce_blocks(sz.n_astro));
    AS_TRY(astro_totals(st_.Ca.get(), st_.ever_active.get(), sz.n_astro, bio_.SIC_th, parts, dtot, stream_));
    AstroTotals at{};
    AS_CUDA(cudaMemcpyAsync(&at, dtot, sizeof(at), cudaMemcpyDeviceToHost, stream_));
    AS_CUDA(cudaStreamSynchronize(stream_));
    out.mean_ca = at.mean_ca;
    out.active_astro = at.active;
    out.engaged_astro = at.engaged;
    out.sic_th = bio_.SIC_th;
    out.build_seconds = net_.build_seconds;
    out.run_seconds = run_seconds_;
    return Status::Ok();
}

namespace {
template <typename R>
__global__ void to_double_kernel(const R* src, double* dst, u64 n) {
    const u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = static_cast<double>(src[i]);
}
}  // namespace

Status Simulation::state_location(int which, void** ptr, size_t* elem, u64* count, bool* per_astro) {
    const u64 nN = rc_.n_neurons, nA = rc_.n_astro;
    const size_t rb = fp32_ ? sizeof(float) : sizeof(double);
    unsigned char* g = st_.g_raw.get();
    void* p = nullptr;
    size_t e = sizeof(double);
    bool astro = false;
    switch (which) {
        case ASTROSIM_STATE_CA: p = st_.Ca.get(); astro = true; break;
        case ASTROSIM_STATE_IP3: p = st_.IP3.get(); astro = true; break;
        case ASTROSIM_STATE_H: p = g + 7 * nN * rb; e = rb; astro = true; break;
        case ASTROSIM_STATE_V: p = st_.V.get(); break;
        case ASTROSIM_STATE_W: p = st_.w.get(); break;
        case ASTROSIM_STATE_G_EX: p = g; e = rb; break;
        case ASTROSIM_STATE_DG_EX: p = g + 1 * nN * rb; e = rb; break;
        case ASTROSIM_STATE_G_IN: p = g + 2 * nN * rb; e = rb; break;
        case ASTROSIM_STATE_DG_IN: p = g + 3 * nN * rb; e = rb; break;
        case ASTROSIM_STATE_I_SIC: p = g + 4 * nN * rb; e = rb; break;
        case ASTROSIM_STATE_STP_X: p = g + 5 * nN * rb; e = rb; break;
        case ASTROSIM_STATE_STP_U: p = g + 6 * nN * rb; e = rb; break;
        case ASTROSIM_STATE_STP_T_LAST: p = st_.stp_t.get(); break;
        case ASTROSIM_STATE_CA_TOT: p = net_.Ca_tot.get(); astro = true; break;
        case ASTROSIM_STATE_IP3_0: p = net_.IP3_0.get(); astro = true; break;
        case ASTROSIM_STATE_TAU_IP3: p = net_.tau_IP3.get(); astro = true; break;
        case ASTROSIM_STATE_DELTA_IP3: p = net_.delta_IP3.get(); astro = true; break;
        case ASTROSIM_STATE_V_RESET: p = net_.V_reset.get(); break;
        case ASTROSIM_STATE_B: p = net_.b.get(); break;
        case ASTROSIM_STATE_SIC_FACTOR: p = st_.sic_last_raw.get(); e = rb; astro = true; break;
        default: return make_error(ASTROSIM_ERR_INVALID_ARG, "unknown state array %d", which);
    }
    *ptr = p;
    *elem = e;
    *count = astro ? nA : nN;
    if (per_astro) *per_astro = astro;
    return Status::Ok();
}

Status Simulation::get_state(int which, double* dst, size_t count) {
    if (!dst) return make_error(ASTROSIM_ERR_INVALID_ARG, "null destination");
    void* src = nullptr;
    size_t elem = 0;
    u64 n = 0;
    AS_TRY(state_location(which, &src, &elem, &n, nullptr));
    if (count < n) return make_error(ASTROSIM_ERR_INVALID_ARG, "state array needs %llu elements",
                                     static_cast<unsigned long long>(n));
    AS_CUDA(cudaSetDevice(device_));
    if (elem == sizeof(double)) {  // double arrays, and `real` arrays of the FP64 path
        AS_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToHost, stream_));
    } else {
        AllocStream alloc_scope(stream_);
        DevBuf<double> tmp;
        AS_TRY(tmp.alloc(n));
        to_double_kernel<float><<<ceil_div(n, 256), 256, 0, stream_>>>(reinterpret_cast<const float*>(src),
                                                                      tmp.get(), n);
        AS_CUDA(cudaGetLastError());
        AS_CUDA(cudaMemcpyAsync(dst, tmp.get(), n * sizeof(double), cudaMemcpyDeviceToHost, stream_));
        AS_CUDA(cudaStreamSynchronize(stream_));
    }
    AS_CUDA(cudaStreamSynchronize(stream_));
    return Status::Ok();
}

Status Simulation::get_csr(int which, u32* rs, size_t rs_cap, u32* src, size_t src_cap, u32* n_targets,
                           u64* n_edges) {
    const DeviceCSR* c = nullptr;
    switch (which) {
        case ASTROSIM_CSR_EXC: c = &net_.exc; break;
        case ASTROSIM_CSR_INH: c = &net_.inh; break;
        case ASTROSIM_CSR_SIC: c = &net_.sic; break;
        case ASTROSIM_CSR_E2A: c = &net_.e2a; break;
        default: return make_error(ASTROSIM_ERR_INVALID_ARG, "unknown CSR %d", which);
    }
    if (n_targets) *n_targets = c->n_targets;
    if (n_edges) *n_edges = c->n_edges;
    AS_CUDA(cudaSetDevice(device_));
    if (rs) {
        if (rs_cap < static_cast<size_t>(c->n_targets) + 1)
            return make_error(ASTROSIM_ERR_INVALID_ARG, "row_start needs %u entries", c->n_targets + 1);
        AS_CUDA(cudaMemcpyAsync(rs, c->row_start.get(), (static_cast<size_t>(c->n_targets) + 1) * sizeof(u32),
                                cudaMemcpyDeviceToHost, stream_));
    }
    if (src) {
        if (src_cap < c->n_edges) return make_error(ASTROSIM_ERR_INVALID_ARG, "src needs %llu entries",
                                                    static_cast<unsigned long long>(c->n_edges));
        if (c->n_edges)
            AS_CUDA(cudaMemcpyAsync(src, c->src.get(), c->n_edges * sizeof(u32), cudaMemcpyDeviceToHost, stream_));
    }
    AS_CUDA(cudaStreamSynchronize(stream_));
    return Status::Ok();
}

// src/astrosim_fused.cu:873-902: one "type,source,target" row per edge, rows in CSR
// order, inhibitory sources offset by n_exc, astrocyte ids prefixed with 'A'.
Status Simulation::dump_edges(const char* path) {
    if (!path) return make_error(ASTROSIM_ERR_INVALID_ARG, "null path");
    std::ofstream out(path);
    if (!out) return make_error(ASTROSIM_ERR_IO, "cannot open %s for --dump-edges", path);
    out << "type,source,target\n";
    // rows are the owned cells' (all of them unless this is a rank of a sharded network)
    struct Item { const DeviceCSR* c; const char* type; long long off; const char* sp; const char* tp; u32 row0; };
    const Item items[4] = {{&net_.exc, "exc_primary", 0, "", "", net_.own.n_lo},
                           {&net_.inh, "inh_primary", static_cast<long long>(net_.sz.n_exc), "", "", net_.own.n_lo},
                           {&net_.e2a, "n2a", 0, "", "A", net_.own.a_lo},
                           {&net_.sic, "a2n", 0, "A", "", net_.own.n_lo}};
    std::vector<u32> rs, src;
    std::string buf;
    for (const Item& it : items) {
        AS_TRY(download_csr(*it.c, rs, src, stream_));
        for (size_t t = 0; t + 1 < rs.size(); ++t) {
            for (u32 k = rs[t]; k < rs[t + 1]; ++k) {
                buf += it.type;
                buf += ',';
                buf += it.sp;
                buf += std::to_string(static_cast<long long>(src[k]) + it.off);
                buf += ',';
                buf += it.tp;
                buf += std::to_string(t + it.row0);
                buf += '\n';
            }
            if (buf.size() > (1u << 22)) {
                out << buf;
                buf.clear();
            }
        }
    }
    out << buf;
    if (!out) return make_error(ASTROSIM_ERR_IO, "write to %s failed", path);
    return Status::Ok();
}

}  // namespace astrosim
