// sim.cuh -- one simulated network resident on the device and its time stepping.
#pragma once

#include <vector>

#include "common.cuh"
#include "model.cuh"
#include "network.cuh"

namespace astrosim { struct WindowState; }

namespace astrosim {

// Everything the step kernels read that does not change between steps.
struct RunConsts {
    AstroK ak;
    NeuronK pe, pi;
    double dt, h_step;
    int substeps;
    int d_e, d_i, d_a2n, slots;
    int steps_per_noise;
    int sic_interval;
    int pad0_;  // explicit padding, zero (see the size check below)
    double w_e, w_i, w_n2a, w_a2n;
    double lambda_astro, limit_astro, weight_astro, noise_astro;
    double lambda_exc, limit_exc, weight_exc, noise_exc;
    double lambda_inh, limit_inh, weight_inh, noise_inh;
    u64 lim53_astro, lim53_exc, lim53_inh;  // floor(exp(-lambda) * 2^53) for the integer first test
    bool independent_noise;
    bool stp_enabled;
    bool pad1_[6];
    double stp_U, stp_tau_rec, stp_tau_fac;
    double SIC_th;
    u64 seed;
    u32 n_exc, n_neurons, n_astro, words;  // words = ceil(n_neurons / 32)
    // Stage-type copies, converted once on the host (see fill_stage_constants):
    // h_step / 6 for the RK4 weights, and float copies of the weights and noise.
    double h6;
    float f_h_step, f_h6, f_w_e, f_neg_w_i, f_w_n2a, f_w_a2n;
    float f_weight_astro, f_weight_exc, f_weight_inh, f_noise_astro;
};
// Every byte of RunConsts is a member (the padding is explicit and zero), so two
// copies built from the same values compare equal bytewise; the batched engine
// relies on that to find networks that share their constants.
static_assert(sizeof(RunConsts) == sizeof(AstroK) + 2 * sizeof(NeuronK) + 2 * 8 + 8 * 4 + 16 * 8 + 3 * 8 + 8 +
                                       5 * 8 + 4 * 4 + 8 + 10 * 4,
              "RunConsts has no implicit padding");

// The run constants that differ between the networks of a batch (seed, sizes,
// drive rates, astrocyte-to-neuron weight).  Everything else in RunConsts is the
// same for networks built with the same biology, so a batched launch can read it
// from its kernel parameters and only these from each network's descriptor.
struct NetScalars {
    u64 seed;
    u32 n_exc, n_neurons, n_astro, words;
    double lambda_astro, limit_astro, lambda_exc, limit_exc, lambda_inh, limit_inh;
    u64 lim53_astro, lim53_exc, lim53_inh;
    double w_a2n;
    float f_w_a2n;
};

__host__ __device__ __forceinline__ NetScalars net_scalars(const RunConsts& rc) {
    NetScalars n{};
    n.seed = rc.seed;
    n.n_exc = rc.n_exc;
    n.n_neurons = rc.n_neurons;
    n.n_astro = rc.n_astro;
    n.words = rc.words;
    n.lambda_astro = rc.lambda_astro;
    n.limit_astro = rc.limit_astro;
    n.lambda_exc = rc.lambda_exc;
    n.limit_exc = rc.limit_exc;
    n.lambda_inh = rc.lambda_inh;
    n.limit_inh = rc.limit_inh;
    n.lim53_astro = rc.lim53_astro;
    n.lim53_exc = rc.lim53_exc;
    n.lim53_inh = rc.lim53_inh;
    n.w_a2n = rc.w_a2n;
    n.f_w_a2n = rc.f_w_a2n;
    return n;
}

// Derives the stage-type copies in `rc` from its double fields.  Every value equals
// what the device would compute from the double (host and device division and
// double-to-float conversion are both IEEE round-to-nearest).
void fill_stage_constants(RunConsts& rc);

// Device state arrays.  V, w, Ca and IP3 are double in every precision; the
// remaining state and the rings are `real` (double or float).
struct StateBuffers {
    StateBuffers() = default;
    StateBuffers(StateBuffers&&) = default;
    StateBuffers& operator=(StateBuffers&&) = default;
    DevBuf<double> V, w, Ca, IP3;
    DevBuf<unsigned char> g_raw;  // g_ex, dg_ex, g_in, dg_in, I_sic, h, stp_x, stp_u as `real` (8 arrays)
    DevBuf<double> stp_t;
    DevBuf<int> refr;
    DevBuf<unsigned char> ever_active;
    DevBuf<u32> spike_bits;        // [slots][words]
    DevBuf<unsigned char> spike_val_raw;  // [slots][n_neurons] real, written only by spiking neurons
    DevBuf<unsigned char> sic_ring_raw;   // [slots][n_astro] real
    DevBuf<unsigned char> sic_last_raw;   // [n_astro] real
    DevBuf<u32> counts;            // spikes per step
    DevBuf<u32> raster;            // [raster_steps][words]
    DevBuf<unsigned char> reduce_raw;  // summary reduction partials + totals
    // Calcium recording: sample k (0-based) is the Ca of astrocytes [rec_first,
    // rec_first + rec_n) after step t = (rec_k0 + k) * rec_every - 1; [rec_cap][rec_n].
    DevBuf<double> ca_rec;
    i64 rec_every = 0, rec_k0 = 0, rec_cap = 0;
    u32 rec_first = 0, rec_n = 0;
};

class Simulation {
public:
    // biology_json: optional overrides of the biology constants (see apply_biology_json).
    // own: the cells whose connectivity rows this network keeps (a rank of a sharded
    // network); null keeps the whole network.  Only the owned cells may be stepped.
    Status create(const astrosim_config& cfg, const char* biology_json = nullptr, const CellRange* own = nullptr);
    // Before create: run on stream s, which the caller owns and keeps alive for as
    // long as this simulation exists (other simulations may share it), instead of a
    // stream of this simulation's own.
    void lend_stream(cudaStream_t s) {
        stream_ = s;
        stream_owned_ = false;
    }
    Status step(i64 n);
    Status summary(astrosim_summary_t& out);
    Status spike_counts(i64 first, i64 n, u32* dst);
    Status raster(u32* dst, size_t words);
    Status get_state(int which, double* dst, size_t count);
    // Device location of a STATE_* array: base, element size (8, or 4 for `real` arrays
    // in the FP32 form), length, and whether it has one entry per astrocyte.
    Status state_location(int which, void** ptr, size_t* elem, u64* count, bool* per_astro);
    Status get_csr(int which, u32* rs, size_t rs_cap, u32* src, size_t src_cap, u32* n_targets, u64* n_edges);
    Status dump_edges(const char* path);
    Status last_step_ms(double* ms);
    Status record_calcium(i64 every, u32 first, u32 n, i64 max_samples);
    Status calcium_samples(i64* n_samples, i64* first_step);
    Status copy_calcium(i64 first, i64 n, double* dst, bool wait);
    Status sync();
    ~Simulation();

    const Sizes& sizes() const { return net_.sz; }
    i64 steps_done() const { return steps_done_; }

    // Access for the batched engine (ensemble.cu), which steps many simulations'
    // windowed state with shared launches.
    const RunConsts& consts() const { return rc_; }
    StateBuffers& state_buffers() { return st_; }
    Network& network() { return net_; }
    WindowState* window_state() { return win_; }
    bool fp32() const { return fp32_; }
    bool windowed() const { return windowed_; }
    i64 pre_steps() const { return pre_steps_; }
    i64 total_steps() const { return total_steps_; }
    i64 raster_steps() const { return cfg_.raster_steps; }
    cudaStream_t stream() const { return stream_; }
    const astrosim_config& config() const { return cfg_; }
    Status reserve_steps(i64 n) { return ensure_counts(n); }
    void note_external_steps(i64 n, double seconds) {
        steps_done_ += n;
        run_seconds_ += seconds;
    }

private:
    Status launch_steps(i64 first, i64 count);
    Status ensure_counts(i64 steps);

    astrosim_config cfg_{};
    Biology bio_;
    Network net_;
    RunConsts rc_{};
    StateBuffers st_;
    cudaStream_t stream_ = nullptr;
    bool stream_owned_ = true;
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    bool have_step_events_ = false;
    int device_ = 0;
    int block_ = 128;
    bool fp32_ = false;
    i64 pre_steps_ = 0, sim_steps_ = 0, total_steps_ = 0, steps_done_ = 0;
    i64 counts_cap_ = 0;
    double run_seconds_ = 0.0;
    bool windowed_ = false;
    WindowState* win_ = nullptr;  // owned; set when the windowed engine runs this network
};

}  // namespace astrosim
