// step_kernels.cuh -- per-cell update rules of one time step, shared by the
// step kernels.  `R` is the stage type (double, or float in the FP32 form);
// V, w, Ca and IP3 always accumulate in double.
#pragma once

#include <type_traits>

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
    double* ca_rec;  // calcium recording (null = off): [rec_cap][rec_n]
    i64 rec_every, rec_k0, rec_cap;
    u32 rec_first, rec_n;
};

// Stores astrocyte a's calcium as sample (t + 1) / rec_every - rec_k0 when step t
// ends a recording interval and the sample fits.  `due` = ((t + 1) % rec_every == 0).
template <typename R>
__device__ __forceinline__ void record_ca(const StepPtrs<R>& p, u32 a, i64 t, bool due, double ca) {
    const u32 i = a - p.rec_first;
    if (!due || i >= p.rec_n) return;
    const i64 k = (t + 1) / p.rec_every - p.rec_k0;
    if (k >= 0 && k < p.rec_cap) p.ca_rec[static_cast<u64>(k) * p.rec_n + i] = ca;
}

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
__device__ __forceinline__ void astro_stage(const AstroK& c, R Ct, R I0, R tI, R inv_tI, R Ca, R IP3, R h, R noise,
                                            R& dCa, R& dIP3, R& dh) {
    if constexpr (std::is_same<R, float>::value) {
        astro_rhs_fast(c, Ct, I0, tI, inv_tI, Ca, IP3, h, noise, dCa, dIP3, dh);
    } else {
        astro_rhs(c, Ct, I0, tI, inv_tI, Ca, IP3, h, noise, dCa, dIP3, dh);
    }
}

__device__ __forceinline__ double log_r(double x) { return log(x); }
__device__ __forceinline__ float log_r(float x) { return log_fast(x); }

// Register-resident state of one astrocyte.  The parameters are kept in double
// (the accumulator updates and clamps use them) and in the stage type, converted
// once per load rather than once per step.
template <typename R>
struct AstroRegs {
    double Ca, IP3;
    R h;
    double Ca_tot, IP3_0, tau_IP3, delta_IP3;
    R Ct, I0, tI, inv_tI;  // stage copies of Ca_tot, IP3_0, tau_IP3 and RN(1 / tau_IP3)
};

template <typename R>
__device__ __forceinline__ AstroRegs<R> load_astro(double Ca, double IP3, R h, double Ca_tot, double IP3_0,
                                                   double tau_IP3, double delta_IP3) {
    AstroRegs<R> s;
    s.Ca = Ca;
    s.IP3 = IP3;
    s.h = h;
    s.Ca_tot = Ca_tot;
    s.IP3_0 = IP3_0;
    s.tau_IP3 = tau_IP3;
    s.delta_IP3 = delta_IP3;
    s.Ct = static_cast<R>(Ca_tot);
    s.I0 = static_cast<R>(IP3_0);
    s.tI = static_cast<R>(tau_IP3);
    s.inv_tI = static_cast<R>(1.0) / s.tI;
    return s;
}

// One step of the astrocyte ODEs: the IP3 kick, then Li-Rinzel RK4 with clamps
// (src/astrosim_fused.cu:255-278); noise held over the stages.  hs is the substep,
// h6 = hs / 6.
template <typename R>
__device__ __forceinline__ void astro_advance(const AstroK& c, AstroRegs<R>& s, R ip3_input, R noise, R hs, R h6,
                                              int substeps) {
    if (ip3_input != static_cast<R>(0.0)) s.IP3 += s.delta_IP3 * static_cast<double>(ip3_input);
    for (int k = 0; k < substeps; ++k) {
        const R ca = static_cast<R>(s.Ca), ip = static_cast<R>(s.IP3), h = s.h;
        R k1c, k1i, k1h, k2c, k2i, k2h, k3c, k3i, k3h, k4c, k4i, k4h;
        astro_stage<R>(c, s.Ct, s.I0, s.tI, s.inv_tI, ca, ip, h, noise, k1c, k1i, k1h);
        astro_stage<R>(c, s.Ct, s.I0, s.tI, s.inv_tI, ca + static_cast<R>(0.5) * hs * k1c,
                       ip + static_cast<R>(0.5) * hs * k1i, h + static_cast<R>(0.5) * hs * k1h, noise, k2c, k2i, k2h);
        astro_stage<R>(c, s.Ct, s.I0, s.tI, s.inv_tI, ca + static_cast<R>(0.5) * hs * k2c,
                       ip + static_cast<R>(0.5) * hs * k2i, h + static_cast<R>(0.5) * hs * k2h, noise, k3c, k3i, k3h);
        astro_stage<R>(c, s.Ct, s.I0, s.tI, s.inv_tI, ca + hs * k3c, ip + hs * k3i, h + hs * k3h, noise, k4c, k4i,
                       k4h);
        s.Ca += static_cast<double>(h6 * (k1c + static_cast<R>(2.0) * k2c + static_cast<R>(2.0) * k3c + k4c));
        s.IP3 += static_cast<double>(h6 * (k1i + static_cast<R>(2.0) * k2i + static_cast<R>(2.0) * k3i + k4i));
        R hn = h + h6 * (k1h + static_cast<R>(2.0) * k2h + static_cast<R>(2.0) * k3h + k4h);
        s.Ca = s.Ca < 0.0 ? 0.0 : (s.Ca > s.Ca_tot ? s.Ca_tot : s.Ca);
        s.h = hn < static_cast<R>(0.0) ? static_cast<R>(0.0) : (hn > static_cast<R>(1.0) ? static_cast<R>(1.0) : hn);
        s.IP3 = s.IP3 < 0.0 ? 0.0 : s.IP3;
    }
}

// Everything astrocyte `a` does in step `step` once its delayed spike sum is known
// (src/astrosim_fused.cu:390-417): Poisson IP3 drive, noise, RK4, SIC factor.
template <typename R>
__device__ __forceinline__ R astro_advance_step(const RunConsts& rc, const NetScalars& ns, AstroRegs<R>& s, R gathered, u32 a, i64 step,
                                                u64 poisson_base, u64 noise_base) {
    R ip3_input = as_r<R>(rc.w_n2a, rc.f_w_n2a) * gathered;
    if (ns.lambda_astro > 0.0) {
        const int ev = rng_poisson_at(poisson_base, ns.lambda_astro, ns.limit_astro, ns.lim53_astro);
        if (ev > 0) ip3_input += as_r<R>(rc.weight_astro, rc.f_weight_astro) * static_cast<R>(ev);
    }
    R noise = static_cast<R>(0.0);
    if (rc.noise_astro > 0.0) {
        u64 base = noise_base;
        if (!rc.independent_noise)
            base = rng_base(ns.seed ^ kAstroNoiseKey, static_cast<u64>(step / rc.steps_per_noise));
        if constexpr (std::is_same<R, float>::value) {
            noise = rc.f_noise_astro * normal_fast(base);
        } else {
            double u1 = rng_uniform_at(base, 0);  // rng_normal (src/astrosim_fused.cu:143-149)
            if (u1 <= 1e-300) u1 = 1e-300;
            const double u2 = rng_uniform_at(base, 1);
            noise = rc.noise_astro * (sqrt(-2.0 * log(u1)) * cos(kTwoPi * u2));
        }
    }
    astro_advance<R>(rc.ak, s, ip3_input, noise, as_r<R>(rc.h_step, rc.f_h_step), as_r<R>(rc.h6, rc.f_h6),
                     rc.substeps);
    // SIC factor (416-417); the threshold test runs on the double Ca in every precision
    const double y = (s.Ca - rc.ak.SIC_th) * 1000.0;
    R factor = static_cast<R>(0.0);
    if (!(y <= 1.0)) factor = as_r<R>(rc.ak.SIC_scale, rc.ak.f_SIC_scale) * log_r(static_cast<R>(y));
    return factor;
}

// Stream bases of a cell's per-step draws (stream = step * 1000003 + cell); the next
// step's base is this one plus kStepAdvance.
constexpr u64 kStepAdvance = kCellStride * kStreamMul;
__device__ __forceinline__ u64 step_base(u64 seed, u64 key, i64 step, u32 cell) {
    return rng_base(seed ^ key, static_cast<u64>(step) * kCellStride + cell);
}

// One astrocyte for step `step` on the per-step rings (src/astrosim_fused.cu:374-427).
template <typename R>
__device__ __forceinline__ void astro_cell_step(const RunConsts& rc, const NetScalars& ns, const StepPtrs<R>& p, u32 a,
                                                i64 step) {
    const int S = rc.slots;
    const int read_slot = static_cast<int>((step + S - rc.d_e) % S);  // the e2a delay is d_e (384)
    const R gathered = gather_spikes<R>(p.e2a_rs, p.e2a_src, a, p.bits + static_cast<u64>(read_slot) * ns.words,
                                        p.val + static_cast<u64>(read_slot) * ns.n_neurons);
    AstroRegs<R> s = load_astro<R>(p.Ca[a], p.IP3[a], p.h[a], p.Ca_tot[a], p.IP3_0[a], p.tau_IP3[a], p.delta_IP3[a]);
    const R factor = astro_advance_step<R>(rc, ns, s, gathered, a, step, step_base(ns.seed, kAstroPoissonKey, step, a),
                                           step_base(ns.seed, kAstroNoiseKey, step, a));
    p.Ca[a] = s.Ca;
    p.IP3[a] = s.IP3;
    p.h[a] = s.h;
    if (p.ca_rec) record_ca<R>(p, a, step, (step + 1) % p.rec_every == 0, s.Ca);
    if (factor > static_cast<R>(0.0)) p.ever_active[a] = 1;
    p.sic_ring[static_cast<u64>(step % S) * ns.n_astro + a] = factor;
    p.sic_last[a] = factor;
}

// The AdEx right-hand side at one set of conductances (each RK4 step uses three:
// the step's start, its midpoint and its end).  FP64: the reference's term-by-term
// formula (neuron_rhs, src/astrosim_fused.cu:281-290).  FP32 form: the refolded
// formula (adex_rhs_folded), its conductance terms computed once per set.
template <typename R>
struct AdexStage {
    const NeuronK& p;
    R g_ex, g_in, I_ext;
    __device__ __forceinline__ AdexStage(const NeuronK& pk, R gex, R gin, R iext)
        : p(pk), g_ex(gex), g_in(gin), I_ext(iext) {}
    __device__ __forceinline__ void operator()(R V, R w, R& dV, R& dw) const {
        neuron_rhs(p, V, w, g_ex, g_in, I_ext, dV, dw);
    }
};
#ifndef ASTROSIM_FP32_IEEE
template <>
struct AdexStage<float> {
    const NeuronK& p;
    AdexCoef c;
    __device__ __forceinline__ AdexStage(const NeuronK& pk, float gex, float gin, float iext)
        : p(pk), c(adex_coef(pk, gex, gin, fmaf(iext, pk.f_inv_Cm, pk.f_C0))) {}
    __device__ __forceinline__ void operator()(float V, float w, float& dV, float& dw) const {
        adex_rhs_folded(p, c, V, w, dV, dw);
    }
};
#endif

// Register-resident state of one neuron.
template <typename R>
struct NeuronRegs {
    double V, w, V_reset, b;
    R g_ex, dg_ex, g_in, dg_in, I_sic;
    int refr;
};

// Everything neuron j does in step `step` once its delayed sums are known
// (src/astrosim_fused.cu:465-558): synaptic inputs, Poisson drive, SIC refresh,
// noise, the alpha-cascade closed form and AdEx RK4 (or the refractory Euler step),
// the spike test.  `noise` is noise_std * N(0,1) for this step when `has_noise`.
template <typename R>
__device__ __forceinline__ bool neuron_advance_step(const RunConsts& rc, const NetScalars& ns, const NeuronK& pk,
                                                    bool excitatory,
                                                    NeuronRegs<R>& n, R exc_sum, R inh_sum, bool sic_refresh,
                                                    R sic_sum, bool has_noise, double noise, u64 poisson_base,
                                                    R ex_decay, R in_decay) {
    R exc_input = as_r<R>(rc.w_e, rc.f_w_e) * exc_sum;
    const R inh_input = as_r<R>(-rc.w_i, rc.f_neg_w_i) * inh_sum;
    const double lambda = excitatory ? ns.lambda_exc : ns.lambda_inh;
    if (lambda > 0.0) {
        const int ev = rng_poisson_at(poisson_base, lambda, excitatory ? ns.limit_exc : ns.limit_inh,
                                      excitatory ? ns.lim53_exc : ns.lim53_inh);
        if (ev > 0)
            exc_input += (excitatory ? as_r<R>(rc.weight_exc, rc.f_weight_exc) : as_r<R>(rc.weight_inh, rc.f_weight_inh)) *
                         static_cast<R>(ev);
    }
    if (sic_refresh) n.I_sic = as_r<R>(ns.w_a2n, ns.f_w_a2n) * sic_sum;
    R I_ext = n.I_sic;
    if (has_noise) I_ext += static_cast<R>(noise);

    double V = n.V, w = n.w;
    R g_ex = n.g_ex, dg_ex = n.dg_ex + exc_input * as_r<R>(pk.psc_init_ex, pk.f_psc_init_ex);
    R g_in = n.g_in, dg_in = n.dg_in + inh_input * as_r<R>(pk.psc_init_in, pk.f_psc_init_in);
    int refractory = n.refr;
    bool spiked = false;
    const R hs = as_r<R>(rc.h_step, rc.f_h_step);
    const R h6 = as_r<R>(rc.h6, rc.f_h6);
    for (int sub = 0; sub < rc.substeps; ++sub) {
        const R g_ex_next = ex_decay * (g_ex + hs * dg_ex);
        const R dg_ex_next = ex_decay * dg_ex;
        const R g_in_next = in_decay * (g_in + hs * dg_in);
        const R dg_in_next = in_decay * dg_in;
        if (refractory > 0) {
            V = n.V_reset;
            R dV, dw;
            const AdexStage<R> r0(pk, g_ex, g_in, I_ext);
            r0(static_cast<R>(V), static_cast<R>(w), dV, dw);
            w += static_cast<double>(hs * dw);
        } else {
            const R g_ex_mid = static_cast<R>(0.5) * (g_ex + g_ex_next);
            const R g_in_mid = static_cast<R>(0.5) * (g_in + g_in_next);
            const R v = static_cast<R>(V), ww = static_cast<R>(w);
            R k1V, k1w, k2V, k2w, k3V, k3w, k4V, k4w;
            const AdexStage<R> r1(pk, g_ex, g_in, I_ext);
            r1(v, ww, k1V, k1w);
            const AdexStage<R> rm(pk, g_ex_mid, g_in_mid, I_ext);
            rm(v + static_cast<R>(0.5) * hs * k1V, ww + static_cast<R>(0.5) * hs * k1w, k2V, k2w);
            rm(v + static_cast<R>(0.5) * hs * k2V, ww + static_cast<R>(0.5) * hs * k2w, k3V, k3w);
            const AdexStage<R> r4(pk, g_ex_next, g_in_next, I_ext);
            r4(v + hs * k3V, ww + hs * k3w, k4V, k4w);
            V += static_cast<double>(h6 * (k1V + static_cast<R>(2.0) * k2V + static_cast<R>(2.0) * k3V + k4V));
            w += static_cast<double>(h6 * (k1w + static_cast<R>(2.0) * k2w + static_cast<R>(2.0) * k3w + k4w));
        }
        g_ex = g_ex_next;
        dg_ex = dg_ex_next;
        g_in = g_in_next;
        dg_in = dg_in_next;
        if (refractory > 0) {
            --refractory;
        } else if (V >= pk.V_peak) {  // threshold test in double
            V = n.V_reset;
            w += n.b;
            refractory = pk.ref_steps;  // static_cast<int>(t_ref / h_step + 0.5)
            spiked = true;
        }
    }
    n.V = V;
    n.w = w;
    n.g_ex = g_ex;
    n.dg_ex = dg_ex;
    n.g_in = g_in;
    n.dg_in = dg_in;
    n.refr = refractory;
    return spiked;
}

// Tsodyks-Markram update of a presynaptic neuron at its spike (src/astrosim_fused.cu:564-579);
// returns the multiplier its outgoing synapses carry.  Every operation's rounding is
// written out, because the compiler's choice of which multiply-adds to fuse here
// varied between launch-bounds instantiations of the window kernel (one fused
// step * dt - t_last; measured on every spike of a run with facilitation): these are
// the roundings the per-step kernel computes, so every engine and variant gives
// the same bits.  x = 1 + (x - x u - 1) x_decay with x - x u and the last
// multiply-add fused; u = U + (u (1 - U)) u_decay with the last one fused.
template <typename R>
__device__ __forceinline__ R stp_on_spike(const RunConsts& rc, R& sx, R& su, double& st, i64 step) {
    if (!rc.stp_enabled) return static_cast<R>(1.0);
    double x = static_cast<double>(sx), u = static_cast<double>(su);
    const double t_now = __dmul_rn(static_cast<double>(step), rc.dt);
    const double elapsed = __dsub_rn(t_now, st);
    const double x_decay = exp(__ddiv_rn(-elapsed, rc.stp_tau_rec));
    const double u_decay = rc.stp_tau_fac < 1e-10 ? 0.0 : exp(__ddiv_rn(-elapsed, rc.stp_tau_fac));
    x = __fma_rn(__dsub_rn(__fma_rn(-x, u, x), 1.0), x_decay, 1.0);
    u = __fma_rn(__dmul_rn(u, __dsub_rn(1.0, rc.stp_U)), u_decay, rc.stp_U);
    sx = static_cast<R>(x);
    su = static_cast<R>(u);
    st = t_now;
    return static_cast<R>(__dmul_rn(x, u));
}

// noise_std * N(0,1) of neuron j for noise index idx (src/astrosim_fused.cu:494-504).
template <typename R>
__device__ __forceinline__ double neuron_noise(const NetScalars& ns, double nstd, u64 idx, u32 j) {
    const u64 base = rng_base(ns.seed ^ kNeuronNoiseKey, idx * kNoiseStride + j);
    if constexpr (std::is_same<R, float>::value) {
        return static_cast<double>(static_cast<float>(nstd) * normal_fast(base));
    } else {
        double u1 = rng_uniform_at(base, 0);
        if (u1 <= 1e-300) u1 = 1e-300;
        const double u2 = rng_uniform_at(base, 1);
        return nstd * (sqrt(-2.0 * log(u1)) * cos(kTwoPi * u2));
    }
}

// One neuron for step `step` on the per-step rings (src/astrosim_fused.cu:433-587).
// Returns whether it spiked and the value its ring entry carries.
template <typename R>
__device__ __forceinline__ bool neuron_cell_step(const RunConsts& rc, const NetScalars& ns, const StepPtrs<R>& p, u32 j,
                                                 i64 step,
                                                 bool sic_refresh, u64 noise_idx, R& out_value) {
    const int S = rc.slots;
    const bool excitatory = j < ns.n_exc;
    const NeuronK& pk = excitatory ? rc.pe : rc.pi;
    const int slot_ex = static_cast<int>((step + S - rc.d_e) % S);
    const int slot_in = static_cast<int>((step + S - rc.d_i) % S);
    const R exc_sum = gather_spikes<R>(p.exc_rs, p.exc_src, j, p.bits + static_cast<u64>(slot_ex) * ns.words,
                                       p.val + static_cast<u64>(slot_ex) * ns.n_neurons);
    // inh sources are local inhibitory indices that index the ring by global id (458-463)
    const R inh_sum = gather_spikes<R>(p.inh_rs, p.inh_src, j, p.bits + static_cast<u64>(slot_in) * ns.words,
                                       p.val + static_cast<u64>(slot_in) * ns.n_neurons);
    R sic_sum = static_cast<R>(0.0);
    if (sic_refresh) {
        const int slot_sic = static_cast<int>((step + S - rc.d_a2n) % S);
        const R* row = p.sic_ring + static_cast<u64>(slot_sic) * ns.n_astro;
        const u32 k1 = p.sic_rs[j + 1];
        for (u32 k = p.sic_rs[j]; k < k1; ++k) sic_sum += row[p.sic_src[k]];
    }
    const double nstd = excitatory ? rc.noise_exc : rc.noise_inh;
    const bool has_noise = nstd > 0.0 && rc.independent_noise;
    const double noise = has_noise ? neuron_noise<R>(ns, nstd, noise_idx, j) : 0.0;
    NeuronRegs<R> n{p.V[j], p.w[j], p.V_reset[j], p.b[j], p.g_ex[j], p.dg_ex[j], p.g_in[j], p.dg_in[j], p.I_sic[j],
                    p.refr[j]};
    const R hs = as_r<R>(rc.h_step, rc.f_h_step);
    const R ex_decay = exp_r(-hs / static_cast<R>(pk.tau_syn_ex));
    const R in_decay = exp_r(-hs / static_cast<R>(pk.tau_syn_in));
    const bool spiked = neuron_advance_step<R>(rc, ns, pk, excitatory, n, exc_sum, inh_sum, sic_refresh, sic_sum,
                                               has_noise, noise, step_base(ns.seed, kNeuronPoissonKey, step, j),
                                               ex_decay, in_decay);
    p.V[j] = n.V;
    p.w[j] = n.w;
    p.g_ex[j] = n.g_ex;
    p.dg_ex[j] = n.dg_ex;
    p.g_in[j] = n.g_in;
    p.dg_in[j] = n.dg_in;
    p.refr[j] = n.refr;
    if (sic_refresh) p.I_sic[j] = n.I_sic;
    out_value = static_cast<R>(0.0);
    if (spiked) out_value = stp_on_spike<R>(rc, p.stp_x[j], p.stp_u[j], p.stp_t[j], step);
    return spiked;
}

// Device pointers of a simulation's state and network (host side).
template <typename R>
inline StepPtrs<R> make_ptrs(StateBuffers& s, Network& n, const RunConsts& rc, i64 raster_steps) {
    StepPtrs<R> p{};
    p.V = s.V.get();
    p.w = s.w.get();
    p.Ca = s.Ca.get();
    p.IP3 = s.IP3.get();
    R* base = reinterpret_cast<R*>(s.g_raw.get());
    const u64 nN = rc.n_neurons;
    p.g_ex = base;
    p.dg_ex = base + nN;
    p.g_in = base + 2 * nN;
    p.dg_in = base + 3 * nN;
    p.I_sic = base + 4 * nN;
    p.stp_x = base + 5 * nN;
    p.stp_u = base + 6 * nN;
    p.h = base + 7 * nN;  // n_astro entries
    p.stp_t = s.stp_t.get();
    p.refr = s.refr.get();
    p.ever_active = s.ever_active.get();
    p.bits = s.spike_bits.get();
    p.val = reinterpret_cast<R*>(s.spike_val_raw.get());
    p.sic_ring = reinterpret_cast<R*>(s.sic_ring_raw.get());
    p.sic_last = reinterpret_cast<R*>(s.sic_last_raw.get());
    p.counts = s.counts.get();
    p.raster = s.raster.get();
    p.raster_steps = raster_steps;
    p.Ca_tot = n.Ca_tot.get();
    p.IP3_0 = n.IP3_0.get();
    p.tau_IP3 = n.tau_IP3.get();
    p.delta_IP3 = n.delta_IP3.get();
    p.V_reset = n.V_reset.get();
    p.b = n.b.get();
    // The kernels index rows by cell id.  A network that keeps only the rows of its
    // owned cells (a rank of a sharded network) stores row r for cell lo + r, so its
    // row pointers are shifted back by lo; only owned cells are ever stepped, so only
    // rows inside the arrays are read.  The shift is plain 64-bit address arithmetic.
    p.exc_rs = n.exc.row_start.get() - n.own.n_lo;
    p.exc_src = n.exc.src.get();
    p.inh_rs = n.inh.row_start.get() - n.own.n_lo;
    p.inh_src = n.inh.src.get();
    p.sic_rs = n.sic.row_start.get() - n.own.n_lo;
    p.sic_src = n.sic.src.get();
    p.e2a_rs = n.e2a.row_start.get() - n.own.a_lo;
    p.e2a_src = n.e2a.src.get();
    p.ca_rec = s.rec_n ? s.ca_rec.get() : nullptr;
    p.rec_every = s.rec_every;
    p.rec_k0 = s.rec_k0;
    p.rec_cap = s.rec_cap;
    p.rec_first = s.rec_first;
    p.rec_n = s.rec_n;
    return p;
}

}  // namespace astrosim
