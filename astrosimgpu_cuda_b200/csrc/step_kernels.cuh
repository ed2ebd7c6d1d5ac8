// step_kernels.cuh -- per-cell update rules of one time step, shared by the
// step kernels.  `R` is the stage type (double, or float in the FP32 form);
// V, w, Ca and IP3 always accumulate in double.
#pragma once

#include "model.cuh"
#include "sim.cuh"

namespace astrosim {

template <typename R>
struct StepPtrs {
    double *V, *w, *Ca, *IP3;
    R *g_ex, *dg_ex, *g_in, *dg_in, *I_sic, *h, *stp_x, *stp_u;
    double* stp_t;
    int* refr;
    unsigned char* ever_active;
    u32* bits;     // [slots][words] spike bits
    R* val;        // [slots][n_neurons] STP multiplier of each spike
    R* sic_ring;   // [slots][n_astro]
    R* sic_last;   // [n_astro]
    u32* counts;   // spikes per step
    u32* raster;   // [raster_steps][words]
    i64 raster_steps;
    const double *Ca_tot, *IP3_0, *tau_IP3, *delta_IP3, *V_reset, *b;
    const u32 *exc_rs, *exc_src, *inh_rs, *inh_src, *sic_rs, *sic_src, *e2a_rs, *e2a_src;
};

// Sum of the delayed spike values of one CSR row, in row order, reading the packed
// bit ring first and the value ring only for sources that spiked.  Skipped terms are
// +0.0 in the reference's dense ring, so the sum is bit-identical.
template <typename R>
__device__ __forceinline__ R gather_spikes(const u32* __restrict__ rs, const u32* __restrict__ src, u32 row,
                                           const u32* __restrict__ bits_slot, const R* __restrict__ val_slot) {
    R sum = static_cast<R>(0.0);
    const u32 k1 = rs[row + 1];
    for (u32 k = rs[row]; k < k1; ++k) {
        const u32 s = src[k];
        if ((bits_slot[s >> 5] >> (s & 31)) & 1u) sum += val_slot[s];
    }
    return sum;
}

// Li-Rinzel RK4 with clamps (src/astrosim_fused.cu:255-278); noise held over the stages.
template <typename R>
__device__ __forceinline__ void astro_advance(const AstroK& c, double Ca_tot, double IP3_0, double tau_IP3,
                                              double delta_IP3, R ip3_input, R noise, double h_step, int substeps,
                                              double& Ca, double& IP3, R& h) {
    if (ip3_input != static_cast<R>(0.0)) IP3 += delta_IP3 * static_cast<double>(ip3_input);
    const R hs = static_cast<R>(h_step);
    const R Ct = static_cast<R>(Ca_tot), I0 = static_cast<R>(IP3_0), tI = static_cast<R>(tau_IP3);
    for (int s = 0; s < substeps; ++s) {
        const R ca = static_cast<R>(Ca), ip = static_cast<R>(IP3);
        R k1c, k1i, k1h, k2c, k2i, k2h, k3c, k3i, k3h, k4c, k4i, k4h;
        astro_rhs<R>(c, Ct, I0, tI, ca, ip, h, noise, k1c, k1i, k1h);
        astro_rhs<R>(c, Ct, I0, tI, ca + static_cast<R>(0.5) * hs * k1c, ip + static_cast<R>(0.5) * hs * k1i,
                     h + static_cast<R>(0.5) * hs * k1h, noise, k2c, k2i, k2h);
        astro_rhs<R>(c, Ct, I0, tI, ca + static_cast<R>(0.5) * hs * k2c, ip + static_cast<R>(0.5) * hs * k2i,
                     h + static_cast<R>(0.5) * hs * k2h, noise, k3c, k3i, k3h);
        astro_rhs<R>(c, Ct, I0, tI, ca + hs * k3c, ip + hs * k3i, h + hs * k3h, noise, k4c, k4i, k4h);
        Ca += static_cast<double>((hs / static_cast<R>(6.0)) *
                                  (k1c + static_cast<R>(2.0) * k2c + static_cast<R>(2.0) * k3c + k4c));
        IP3 += static_cast<double>((hs / static_cast<R>(6.0)) *
                                   (k1i + static_cast<R>(2.0) * k2i + static_cast<R>(2.0) * k3i + k4i));
        h += (hs / static_cast<R>(6.0)) * (k1h + static_cast<R>(2.0) * k2h + static_cast<R>(2.0) * k3h + k4h);
        Ca = Ca < 0.0 ? 0.0 : (Ca > Ca_tot ? Ca_tot : Ca);
        h = h < static_cast<R>(0.0) ? static_cast<R>(0.0) : (h > static_cast<R>(1.0) ? static_cast<R>(1.0) : h);
        IP3 = IP3 < 0.0 ? 0.0 : IP3;
    }
}

__device__ __forceinline__ double log_r(double x) { return log(x); }
__device__ __forceinline__ float log_r(float x) { return logf(x); }

// One astrocyte for step `step` (src/astrosim_fused.cu:374-427).
template <typename R>
__device__ __forceinline__ void astro_cell_step(const RunConsts& rc, const StepPtrs<R>& p, u32 a, i64 step) {
    const int S = rc.slots;
    const int read_slot = static_cast<int>((step + S - rc.d_e) % S);  // the e2a delay is d_e (384)
    const R gathered = gather_spikes<R>(p.e2a_rs, p.e2a_src, a, p.bits + static_cast<u64>(read_slot) * rc.words,
                                        p.val + static_cast<u64>(read_slot) * rc.n_neurons);
    R ip3_input = static_cast<R>(rc.w_n2a) * gathered;
    if (rc.lambda_astro > 0.0) {
        const int ev = rng_poisson_knuth(rc.seed ^ kAstroPoissonKey, static_cast<u64>(step) * kCellStride + a,
                                         rc.lambda_astro, rc.limit_astro);
        if (ev > 0) ip3_input += static_cast<R>(rc.weight_astro) * static_cast<R>(ev);
    }
    R noise = static_cast<R>(0.0);
    if (rc.noise_astro > 0.0) {
        if (rc.independent_noise)
            noise = static_cast<R>(rc.noise_astro *
                                   rng_normal(rc.seed ^ kAstroNoiseKey, static_cast<u64>(step) * kCellStride + a));
        else
            noise = static_cast<R>(rc.noise_astro * rng_normal(rc.seed ^ kAstroNoiseKey,
                                                               static_cast<u64>(step / rc.steps_per_noise)));
    }
    double Ca = p.Ca[a], IP3 = p.IP3[a];
    R h = p.h[a];
    astro_advance<R>(rc.ak, p.Ca_tot[a], p.IP3_0[a], p.tau_IP3[a], p.delta_IP3[a], ip3_input, noise, rc.h_step,
                     rc.substeps, Ca, IP3, h);
    p.Ca[a] = Ca;
    p.IP3[a] = IP3;
    p.h[a] = h;
    // SIC factor (416-417); the threshold test runs on the double Ca in every precision
    const double y = (Ca - rc.ak.SIC_th) * 1000.0;
    R factor = static_cast<R>(0.0);
    if (!(y <= 1.0)) factor = static_cast<R>(rc.ak.SIC_scale) * log_r(static_cast<R>(y));
    if (factor > static_cast<R>(0.0)) p.ever_active[a] = 1;
    p.sic_ring[static_cast<u64>(step % S) * rc.n_astro + a] = factor;
    p.sic_last[a] = factor;
}

// One neuron for step `step` (src/astrosim_fused.cu:433-587).  Returns whether it
// spiked and the value its ring entry carries.
template <typename R>
__device__ __forceinline__ bool neuron_cell_step(const RunConsts& rc, const StepPtrs<R>& p, u32 j, i64 step,
                                                 bool sic_refresh, u64 noise_idx, R& out_value) {
    const int S = rc.slots;
    const bool excitatory = j < rc.n_exc;
    const NeuronK& pk = excitatory ? rc.pe : rc.pi;
    const int slot_ex = static_cast<int>((step + S - rc.d_e) % S);
    const int slot_in = static_cast<int>((step + S - rc.d_i) % S);
    const R exc_sum = gather_spikes<R>(p.exc_rs, p.exc_src, j, p.bits + static_cast<u64>(slot_ex) * rc.words,
                                       p.val + static_cast<u64>(slot_ex) * rc.n_neurons);
    // inh sources are local inhibitory indices that index the ring by global id (458-463)
    const R inh_sum = gather_spikes<R>(p.inh_rs, p.inh_src, j, p.bits + static_cast<u64>(slot_in) * rc.words,
                                       p.val + static_cast<u64>(slot_in) * rc.n_neurons);
    R exc_input = static_cast<R>(rc.w_e) * exc_sum;
    const R inh_input = static_cast<R>(-rc.w_i) * inh_sum;
    const double lambda = excitatory ? rc.lambda_exc : rc.lambda_inh;
    if (lambda > 0.0) {
        const int ev = rng_poisson_knuth(rc.seed ^ kNeuronPoissonKey, static_cast<u64>(step) * kCellStride + j, lambda,
                                         excitatory ? rc.limit_exc : rc.limit_inh);
        if (ev > 0) exc_input += static_cast<R>(excitatory ? rc.weight_exc : rc.weight_inh) * static_cast<R>(ev);
    }
    if (sic_refresh) {
        const int slot_sic = static_cast<int>((step + S - rc.d_a2n) % S);
        const R* row = p.sic_ring + static_cast<u64>(slot_sic) * rc.n_astro;
        R sic_sum = static_cast<R>(0.0);
        const u32 k1 = p.sic_rs[j + 1];
        for (u32 k = p.sic_rs[j]; k < k1; ++k) sic_sum += row[p.sic_src[k]];
        p.I_sic[j] = static_cast<R>(rc.w_a2n) * sic_sum;
    }
    R I_ext = p.I_sic[j];
    const double nstd = excitatory ? rc.noise_exc : rc.noise_inh;
    if (nstd > 0.0 && rc.independent_noise)
        I_ext += static_cast<R>(nstd * rng_normal(rc.seed ^ kNeuronNoiseKey, noise_idx * kNoiseStride + j));

    double V = p.V[j], w = p.w[j];
    R g_ex = p.g_ex[j], dg_ex = p.dg_ex[j] + exc_input * static_cast<R>(pk.psc_init_ex);
    R g_in = p.g_in[j], dg_in = p.dg_in[j] + inh_input * static_cast<R>(pk.psc_init_in);
    int refractory = p.refr[j];
    bool spiked = false;
    const R hs = static_cast<R>(rc.h_step);
    const R ex_decay = exp_r(-hs / static_cast<R>(pk.tau_syn_ex));
    const R in_decay = exp_r(-hs / static_cast<R>(pk.tau_syn_in));
    for (int sub = 0; sub < rc.substeps; ++sub) {
        const R g_ex_next = ex_decay * (g_ex + hs * dg_ex);
        const R dg_ex_next = ex_decay * dg_ex;
        const R g_in_next = in_decay * (g_in + hs * dg_in);
        const R dg_in_next = in_decay * dg_in;
        if (refractory > 0) {
            V = p.V_reset[j];
            R dV, dw;
            neuron_rhs<R>(pk, static_cast<R>(V), static_cast<R>(w), g_ex, g_in, I_ext, dV, dw);
            w += static_cast<double>(hs * dw);
        } else {
            const R g_ex_mid = static_cast<R>(0.5) * (g_ex + g_ex_next);
            const R g_in_mid = static_cast<R>(0.5) * (g_in + g_in_next);
            const R v = static_cast<R>(V), ww = static_cast<R>(w);
            R k1V, k1w, k2V, k2w, k3V, k3w, k4V, k4w;
            neuron_rhs<R>(pk, v, ww, g_ex, g_in, I_ext, k1V, k1w);
            neuron_rhs<R>(pk, v + static_cast<R>(0.5) * hs * k1V, ww + static_cast<R>(0.5) * hs * k1w, g_ex_mid,
                          g_in_mid, I_ext, k2V, k2w);
            neuron_rhs<R>(pk, v + static_cast<R>(0.5) * hs * k2V, ww + static_cast<R>(0.5) * hs * k2w, g_ex_mid,
                          g_in_mid, I_ext, k3V, k3w);
            neuron_rhs<R>(pk, v + hs * k3V, ww + hs * k3w, g_ex_next, g_in_next, I_ext, k4V, k4w);
            V += static_cast<double>((hs / static_cast<R>(6.0)) *
                                     (k1V + static_cast<R>(2.0) * k2V + static_cast<R>(2.0) * k3V + k4V));
            w += static_cast<double>((hs / static_cast<R>(6.0)) *
                                     (k1w + static_cast<R>(2.0) * k2w + static_cast<R>(2.0) * k3w + k4w));
        }
        g_ex = g_ex_next;
        dg_ex = dg_ex_next;
        g_in = g_in_next;
        dg_in = dg_in_next;
        if (refractory > 0) {
            --refractory;
        } else if (V >= pk.V_peak) {  // threshold test in double
            V = p.V_reset[j];
            w += p.b[j];
            refractory = static_cast<int>(pk.t_ref / rc.h_step + 0.5);
            spiked = true;
        }
    }
    p.V[j] = V;
    p.w[j] = w;
    p.g_ex[j] = g_ex;
    p.dg_ex[j] = dg_ex;
    p.g_in[j] = g_in;
    p.dg_in[j] = dg_in;
    p.refr[j] = refractory;

    out_value = static_cast<R>(0.0);
    if (spiked) {  // Tsodyks-Markram update of this presynaptic neuron (564-579)
        if (rc.stp_enabled) {
            double x = static_cast<double>(p.stp_x[j]), u = static_cast<double>(p.stp_u[j]);
            const double t_now = static_cast<double>(step) * rc.dt;
            const double elapsed = t_now - p.stp_t[j];
            const double x_decay = exp(-elapsed / rc.stp_tau_rec);
            const double u_decay = rc.stp_tau_fac < 1e-10 ? 0.0 : exp(-elapsed / rc.stp_tau_fac);
            x = 1.0 + (x - x * u - 1.0) * x_decay;
            u = rc.stp_U + u * (1.0 - rc.stp_U) * u_decay;
            p.stp_x[j] = static_cast<R>(x);
            p.stp_u[j] = static_cast<R>(u);
            p.stp_t[j] = t_now;
            out_value = static_cast<R>(x * u);
        } else {
            out_value = static_cast<R>(1.0);
        }
    }
    return spiked;
}

}  // namespace astrosim
