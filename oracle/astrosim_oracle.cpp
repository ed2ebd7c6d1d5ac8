// astrosim_oracle.cpp -- TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.
//
// FP64 CPU restatement of the reference program src/astrosim_fused.cu
// (praveen-dedigamage/astrosimgpu_cuda), written plainly so that it can serve
// as the checker for the CUDA implementation:
//   - counter RNG and the sequential stream           (src/astrosim_fused.cu:127-216)
//   - scaling law, biology constants, delays          (src/astrosim_fused.cu:595-615, 742-786)
//   - serial connectivity builder + CSR inversion     (src/astrosim_fused.cu:296-315, 617-735)
//   - per-cell parameter draws and initial state      (src/astrosim_fused.cu:917-1018)
//   - the two per-step kernels, one cell at a time    (src/astrosim_fused.cu:236-290, 374-587)
//   - the host time loop's per-step scalars + summary (src/astrosim_fused.cu:1042-1141)
// Every expression keeps the reference's operand order; the file is compiled
// with -ffp-contract=off so each operation is rounded separately, like the
// reference's host code on x86-64.  Transcendental functions come from the host
// C library (the reference's host code uses the same ones; its device code uses
// CUDA's, which may differ in the last bit).
//
// Only tests/, the smoke check and bench.py's CPU-baseline leg use this file.

#include "astrosim_oracle.h"

#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <utility>
#include <vector>

namespace {

using u32 = std::uint32_t;
using u64 = std::uint64_t;

// ---------------------------------------------------------------- RNG
// src/astrosim_fused.cu:127-135
u64 bits(u64 seed, u64 stream, u64 counter) {
    u64 z = seed + stream * 0x9E3779B97F4A7C15ULL + counter * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
// src/astrosim_fused.cu:137-141
double uniform(u64 seed, u64 stream, u64 counter) {
    return static_cast<double>(bits(seed, stream, counter) >> 11) * (1.0 / 9007199254740992.0);
}
const double kTwoPi = 6.283185307179586476925286766559;
// src/astrosim_fused.cu:143-149
double normal(u64 seed, u64 stream) {
    double u1 = uniform(seed, stream, 0);
    if (u1 <= 1e-300) u1 = 1e-300;
    const double u2 = uniform(seed, stream, 1);
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(kTwoPi * u2);
}
// src/astrosim_fused.cu:154-175 (Knuth, normal approximation above lambda 30)
int poisson(u64 seed, u64 stream, double lambda) {
    if (lambda <= 0.0) return 0;
    if (lambda > 30.0) {
        double u1 = uniform(seed, stream, 0);
        if (u1 <= 1e-300) u1 = 1e-300;
        const double u2 = uniform(seed, stream, 1);
        const double z = std::sqrt(-2.0 * std::log(u1)) * std::cos(kTwoPi * u2);
        const double v = lambda + std::sqrt(lambda) * z;
        return v < 0.0 ? 0 : static_cast<int>(v + 0.5);
    }
    const double limit = std::exp(-lambda);
    u64 c = 0;
    double prod = uniform(seed, stream, c++);
    int k = 0;
    while (prod > limit) {
        ++k;
        prod *= uniform(seed, stream, c++);
    }
    return k;
}

// src/astrosim_fused.cu:180-208: one counter stream read in order, Box-Muller
// pairs with the sine half kept as a spare.
struct SeqStream {
    u64 seed, stream, counter = 0;
    bool have_spare = false;
    double spare = 0.0;
    SeqStream(u64 s, u64 st) : seed(s), stream(st) {}
    double next_uniform() { return uniform(seed, stream, counter++); }
    double next_normal() {
        if (have_spare) {
            have_spare = false;
            return spare;
        }
        double u1;
        do {
            u1 = next_uniform();
        } while (u1 <= 1e-300);
        const double u2 = next_uniform();
        const double r = std::sqrt(-2.0 * std::log(u1));
        const double th = kTwoPi * u2;
        spare = r * std::sin(th);
        have_spare = true;
        return r * std::cos(th);
    }
    // src/astrosim_fused.cu:196-202 (truncated normal by redraw, 1000 tries)
    double truncated(double mean, double sd, double lo, double hi) {
        for (int i = 0; i < 1000; ++i) {
            const double v = mean + sd * next_normal();
            if (v >= lo && v <= hi) return v;
        }
        return std::min(std::max(mean, lo), hi);
    }
};

// src/astrosim_fused.cu:210-216
double draw_scaled(double mean, bool on, double lower, double upper, double var, SeqStream& rs) {
    if (!on || var <= 0.0) return mean;
    const double lo = mean < 0.0 ? mean * upper : mean * lower;
    const double hi = mean < 0.0 ? mean * lower : mean * upper;
    return rs.truncated(mean, var * std::abs(mean), lo, hi);
}

// ---------------------------------------------------------------- constants
// src/astrosim_fused.cu:742-781 (compiled-in biology)
struct Bio {
    double Ca_tot = 1.8958264782990153, IP3_0 = 0.010925583871830699;
    double tau_IP3 = 1058.7589568400845, delta_IP3 = 0.04911592657233997;
    double SIC_scale = 1.0, Kd_IP3_1 = 0.13, Kd_IP3_2 = 0.9434, Kd_act = 0.08234, Kd_inh = 1.049;
    double Km_SERCA = 0.1, SIC_th = 0.19669, k_IP3R = 0.0002, rate_IP3R = 0.006, rate_L = 0.00011;
    double rate_SERCA = 0.0009, ratio_ER_cyt = 0.185, Ca_init = 0.073, h_init = 0.793,
           IP3_init = 0.010925583871830699;
    bool randomize_astro = true;
    double ra_lower = 0.9, ra_upper = 1.05, ra_var = 0.1;
    double e_Delta_T = 2.0, e_a = 4.0, e_tau_w = 450.0, e_V_reset = -50.0, e_b = 300.0, e_V_m = -50.0;
    double e_C_m = 130.0, e_g_L = 18.0, e_E_L = -58.0, e_V_th = -50.0, e_V_peak = 0.0, e_t_ref = 0.0;
    double e_E_ex = 0.0, e_E_in = -85.0, e_tau_syn_ex = 0.2, e_tau_syn_in = 2.0;
    double i_Delta_T = 2.0, i_a = -0.8, i_tau_w = 264.0, i_V_reset = -60.0, i_b = 130.0, i_V_m = -60.0;
    double i_C_m = 104.0, i_g_L = 4.3, i_E_L = -65.0, i_V_th = -52.0, i_V_peak = 0.0, i_t_ref = 0.0;
    double i_E_ex = 0.0, i_E_in = -85.0, i_tau_syn_ex = 0.2, i_tau_syn_in = 2.0;
    bool randomize_neuron = true;
    double rn_lower = 0.9, rn_upper = 1.1, rn_var = 0.05;
    double w_e = 5.0, w_i = -5.0, w_n2a = 0.2, w_a2n = 1.0;
    double d_e = 1.0, d_i = 1.0, d_a2n = 1.0;
    bool stp_enabled = true;
    double stp_U = 0.5, stp_tau_rec = 800.0, stp_tau_fac = 0.0;
    int sic_interval = 1;
    double astro_poiss_rate = 3.029715502945856, astro_poiss_weight = 1.0, astro_noise_std = 0.0003;
    double exc_poiss_rate = 2700.0, exc_poiss_weight = 1.0, exc_noise_std = 100.0;
    double inh_poiss_rate = 2500.0, inh_poiss_weight = 1.0, inh_noise_std = 100.0;
    bool independent_noise = true;
    double noise_dt = 0.0;
};

struct NeuronP {  // src/astrosim_fused.cu:228-232
    double C_m, g_L, E_L, V_th, Delta_T, a, tau_w, V_peak, t_ref, E_ex, E_in, tau_syn_ex, tau_syn_in,
        I_e, psc_ex, psc_in;
    // Test knob (oracle_set_exp_perturbation): the fraction of the AdEx exponential's
    // arguments whose result is moved by one ulp; 0 evaluates the plain formula.
    double exp_perturb = 0.0;
    // Test knob (oracle_set_contraction): evaluate the AdEx right-hand side and the
    // neuron's RK4 updates with fused multiply-adds, as a GPU compiler contracts them.
    bool contract = false;
};

// exp(x), moved one ulp up or down for a fraction `rate` of the arguments (chosen by a
// hash of x's bits, so the same argument always gets the same result): a stand-in for
// another correctly working math library that disagrees with this one in the last bit.
inline double exp_maybe_perturbed(double x, double rate) {
    const double r = std::exp(x);
    if (rate <= 0.0) return r;
    u64 z = 0;
    std::memcpy(&z, &x, sizeof z);
    z = (z ^ (z >> 33)) * 0xFF51AFD7ED558CCDULL;
    z = (z ^ (z >> 33)) * 0xC4CEB9FE1A85EC53ULL;
    z ^= z >> 33;
    if (static_cast<double>(z >> 11) * (1.0 / 9007199254740992.0) >= rate) return r;
    return std::nextafter(r, (z & 1) ? HUGE_VAL : -HUGE_VAL);
}
NeuronP make_neuron(bool exc, const Bio& b) {  // src/astrosim_fused.cu:940-951
    NeuronP p{};
    p.C_m = exc ? b.e_C_m : b.i_C_m;
    p.g_L = exc ? b.e_g_L : b.i_g_L;
    p.E_L = exc ? b.e_E_L : b.i_E_L;
    p.V_th = exc ? b.e_V_th : b.i_V_th;
    p.Delta_T = exc ? b.e_Delta_T : b.i_Delta_T;
    p.a = exc ? b.e_a : b.i_a;
    p.tau_w = exc ? b.e_tau_w : b.i_tau_w;
    p.V_peak = exc ? b.e_V_peak : b.i_V_peak;
    p.t_ref = exc ? b.e_t_ref : b.i_t_ref;
    p.E_ex = exc ? b.e_E_ex : b.i_E_ex;
    p.E_in = exc ? b.e_E_in : b.i_E_in;
    p.tau_syn_ex = exc ? b.e_tau_syn_ex : b.i_tau_syn_ex;
    p.tau_syn_in = exc ? b.e_tau_syn_in : b.i_tau_syn_in;
    p.I_e = 0.0;
    p.psc_ex = 2.7182818284590452353602874713527 / p.tau_syn_ex;
    p.psc_in = 2.7182818284590452353602874713527 / p.tau_syn_in;
    return p;
}

int delay_steps(double delay_ms, double dt) {  // src/astrosim_fused.cu:783-786
    const int s = static_cast<int>(delay_ms / dt + 0.5);
    return s < 1 ? 1 : s;
}

// ---------------------------------------------------------------- connectivity
struct CSR {  // src/astrosim_fused.cu:296-315: counting sort by target, stable
    std::vector<u32> rs, src;
    void build(u32 n_targets, const std::vector<std::pair<u32, u32>>& edges) {
        rs.assign(static_cast<size_t>(n_targets) + 1, 0);
        for (const auto& e : edges) rs[e.second + 1]++;
        for (u32 i = 0; i < n_targets; ++i) rs[i + 1] += rs[i];
        src.assign(edges.size(), 0);
        std::vector<u32> cur(rs.begin(), rs.end() - 1);
        for (const auto& e : edges) src[cur[e.second]++] = e.first;
    }
};

struct Sizes {  // src/astrosim_fused.cu:595-615
    u32 n_total = 0, n_exc = 0, n_inh = 0, n_astro = 0;
    double p = 0.0;
};
Sizes scaling(u32 n_total) {
    Sizes s;
    s.n_total = n_total;
    s.n_exc = std::max<u32>(1, static_cast<u32>(std::lround(n_total * 0.8)));
    s.n_inh = std::max<u32>(1, n_total - s.n_exc);
    s.n_astro = std::max<u32>(1, static_cast<u32>(std::lround(n_total / 5.0)));
    s.p = std::min<double>(1.0, 80.0 / static_cast<double>(s.n_exc));
    return s;
}

// src/astrosim_fused.cu:617-624
u32 skip_draw(double p, u32 remaining, SeqStream& rs) {
    if (remaining == 0 || p >= 1.0) return 0;
    if (p <= 0.0) return remaining;
    double u = rs.next_uniform();
    if (u >= 1.0) u = std::nextafter(1.0, 0.0);
    const double g = std::floor(std::log1p(-u) / std::log1p(-p));
    return g >= static_cast<double>(remaining) ? remaining : static_cast<u32>(g);
}

struct Net {
    CSR exc, inh, sic, e2a;
};

// src/astrosim_fused.cu:631-735
Net build_network(const Sizes& sz, u64 seed) {
    const u32 n_exc = sz.n_exc, n_inh = sz.n_inh, n_astro = sz.n_astro;
    const u32 n_neurons = n_exc + n_inh;
    SeqStream rs(seed, 0x5EEDULL);
    // 644-645: step over the per-cell parameter draws (4 normals per astrocyte, 2 per neuron)
    for (u32 i = 0; i < n_astro; ++i)
        for (int k = 0; k < 4; ++k) rs.next_normal();
    for (u32 i = 0; i < n_neurons; ++i)
        for (int k = 0; k < 2; ++k) rs.next_normal();

    // 651-671: astrocyte pool of up to 5 distinct astrocytes per postsynaptic neuron
    const int take = std::min<int>(5, static_cast<int>(n_astro));
    std::vector<u32> pool(static_cast<size_t>(n_neurons) * 5, 0);
    for (u32 post = 0; post < n_neurons; ++post) {
        u32* pl = &pool[static_cast<size_t>(post) * 5];
        if (take > 0 && static_cast<int64_t>(take) * 4 >= static_cast<int64_t>(n_astro)) {
            std::vector<u32> cand(n_astro);
            for (u32 i = 0; i < n_astro; ++i) cand[i] = i;
            for (int k = 0; k < take; ++k) {
                const size_t pick = static_cast<size_t>(rs.next_uniform() * (cand.size() - k)) + k;
                std::swap(cand[k], cand[std::min(pick, cand.size() - 1)]);
                pl[k] = cand[k];
            }
        } else {
            int have = 0;
            while (have < take) {
                const u32 c = static_cast<u32>(rs.next_uniform() * static_cast<double>(n_astro)) % n_astro;
                bool dup = false;
                for (int q = 0; q < have; ++q)
                    if (pl[q] == c) dup = true;
                if (!dup) pl[have++] = c;
            }
        }
    }

    std::vector<u32> astro_deg(n_astro, 0);
    std::vector<std::pair<u32, u32>> e_exc, e_inh, e_e2a, e_sic;  // (source, target)
    const size_t est = static_cast<size_t>(80.0 * n_neurons * 1.05) + 64;
    e_exc.reserve(est);
    e_inh.reserve(est / 4 + 64);
    e_e2a.reserve(est / 5 + 64);
    e_sic.reserve(est / 5 + 64);

    // 688-710: excitatory presynaptic walks, first over the E block then over the I block
    auto walk_exc = [&](u32 post_off, u32 post_n) {
        for (u32 pre = 0; pre < n_exc; ++pre) {
            u32 pos = 0;
            while (pos < post_n) {
                pos += skip_draw(sz.p, post_n - pos, rs);
                if (pos >= post_n) break;
                const u32 post = post_off + pos;
                ++pos;
                if (pre == post) continue;  // no autapses
                e_exc.emplace_back(pre, post);
                if (n_astro == 0 || rs.next_uniform() >= 0.2) continue;  // P_THIRD
                const u32* pl = &pool[static_cast<size_t>(post) * 5];
                const u32 astro = pl[static_cast<size_t>(rs.next_uniform() * take) % take];
                if (astro_deg[astro] >= 10000) continue;  // MAX_ASTRO_OUT_DEGREE
                e_e2a.emplace_back(pre, astro);
                e_sic.emplace_back(astro, post);
                ++astro_deg[astro];
            }
        }
    };
    walk_exc(0, n_exc);
    walk_exc(n_exc, n_inh);

    // 712-723: inhibitory presynaptic walks over every neuron; sources stored as LOCAL
    // inhibitory indices (the reference's quirk, kept for parity).
    for (u32 pre = 0; pre < n_inh; ++pre) {
        const u32 pre_global = n_exc + pre;
        u32 pos = 0;
        while (pos < n_neurons) {
            pos += skip_draw(sz.p, n_neurons - pos, rs);
            if (pos >= n_neurons) break;
            const u32 post = pos;
            ++pos;
            if (pre_global == post) continue;
            e_inh.emplace_back(pre, post);
        }
    }

    Net net;
    net.exc.build(n_neurons, e_exc);
    net.inh.build(n_neurons, e_inh);
    net.sic.build(n_neurons, e_sic);
    net.e2a.build(n_astro, e_e2a);
    return net;
}

}  // namespace

// ---------------------------------------------------------------- simulation
struct oracle_sim {
    astrosim_config cfg{};
    Sizes sz;
    Bio bio;
    Net net;
    NeuronP pe{}, pi{};
    u32 n_neurons = 0;
    int d_e = 0, d_i = 0, d_a2n = 0, slots = 0, steps_per_noise = 1;
    int64_t pre_steps = 0, sim_steps = 0, total_steps = 0, step = 0;
    double h_step = 0.0, build_s = 0.0;
    int threads = 1;
    // astrocyte state + per-cell parameters
    std::vector<double> Ca, IP3, h, Ca_tot, IP3_0, tau_IP3, delta_IP3, sic_last;
    std::vector<unsigned char> ever_active;
    // neuron state + per-cell parameters
    std::vector<double> V, w, g_ex, dg_ex, g_in, dg_in, I_sic, V_reset, b, stp_x, stp_u, stp_t;
    std::vector<int> refr;
    std::vector<double> ring_n, ring_s;  // [slot][cell]
    std::vector<unsigned char> spiked;
    std::vector<uint32_t> counts;        // spikes per completed step
    std::vector<uint32_t> raster;        // first cfg.raster_steps steps
    uint64_t spikes_before = 0;
    bool pre_mark_done = false;
};

namespace {

void init_state(oracle_sim* s) {
    Bio& bio = s->bio;
    const astrosim_config& cfg = s->cfg;
    // 846-851: flag overrides
    if (bio.noise_dt <= 0.0) bio.noise_dt = 10.0 * cfg.dt;
    if (!std::isnan(cfg.w_n2a)) bio.w_n2a = cfg.w_n2a;
    if (!std::isnan(cfg.w_a2n)) bio.w_a2n = cfg.w_a2n;
    if (!cfg.stp_enabled) bio.stp_enabled = false;
    bio.exc_poiss_rate = bio.exc_poiss_rate * cfg.neuron_drive_scale;
    bio.inh_poiss_rate = bio.inh_poiss_rate * cfg.neuron_drive_scale;

    const u32 nA = s->sz.n_astro;
    const u32 nN = s->sz.n_exc + s->sz.n_inh;
    s->n_neurons = nN;
    // 917-933: per-cell parameters from a fresh stream (seed, 0x5EED)
    SeqStream rs(cfg.seed, 0x5EEDULL);
    s->Ca_tot.resize(nA);
    s->IP3_0.resize(nA);
    s->tau_IP3.resize(nA);
    s->delta_IP3.resize(nA);
    for (u32 i = 0; i < nA; ++i) {
        s->Ca_tot[i] = draw_scaled(bio.Ca_tot, bio.randomize_astro, bio.ra_lower, bio.ra_upper, bio.ra_var, rs);
        s->IP3_0[i] = draw_scaled(bio.IP3_0, bio.randomize_astro, bio.ra_lower, bio.ra_upper, bio.ra_var, rs);
        s->tau_IP3[i] = draw_scaled(bio.tau_IP3, bio.randomize_astro, bio.ra_lower, bio.ra_upper, bio.ra_var, rs);
        s->delta_IP3[i] = draw_scaled(bio.delta_IP3, bio.randomize_astro, bio.ra_lower, bio.ra_upper, bio.ra_var, rs);
    }
    s->V_reset.resize(nN);
    s->b.resize(nN);
    for (u32 i = 0; i < nN; ++i) {
        const bool exc = i < s->sz.n_exc;
        s->V_reset[i] = draw_scaled(exc ? bio.e_V_reset : bio.i_V_reset, bio.randomize_neuron, bio.rn_lower,
                                    bio.rn_upper, bio.rn_var, rs);
        s->b[i] = draw_scaled(exc ? bio.e_b : bio.i_b, bio.randomize_neuron, bio.rn_lower, bio.rn_upper,
                              bio.rn_var, rs);
    }
    s->pe = make_neuron(true, bio);
    s->pi = make_neuron(false, bio);
    // 954-957
    s->d_e = delay_steps(bio.d_e, cfg.dt);
    s->d_i = delay_steps(bio.d_i, cfg.dt);
    s->d_a2n = delay_steps(bio.d_a2n, cfg.dt);
    s->slots = std::max({s->d_e, s->d_i, s->d_a2n}) + 1;
    // 981-1018: initial state
    s->Ca.assign(nA, bio.Ca_init);
    s->IP3.assign(nA, bio.IP3_init);
    s->h.assign(nA, bio.h_init);
    s->sic_last.assign(nA, 0.0);
    s->ever_active.assign(nA, 0);
    s->V.resize(nN);
    for (u32 i = 0; i < nN; ++i) s->V[i] = i < s->sz.n_exc ? bio.e_V_m : bio.i_V_m;
    s->w.assign(nN, 0.0);
    s->g_ex.assign(nN, 0.0);
    s->dg_ex.assign(nN, 0.0);
    s->g_in.assign(nN, 0.0);
    s->dg_in.assign(nN, 0.0);
    s->I_sic.assign(nN, 0.0);
    s->refr.assign(nN, 0);
    s->stp_x.assign(nN, 1.0);
    s->stp_u.assign(nN, bio.stp_U);
    s->stp_t.assign(nN, -1e12);
    s->ring_n.assign(static_cast<size_t>(s->slots) * nN, 0.0);
    s->ring_s.assign(static_cast<size_t>(s->slots) * nA, 0.0);
    s->spiked.assign(nN, 0);
    // 1021-1024
    s->pre_steps = static_cast<int64_t>(cfg.pre_ms / cfg.dt + 0.5);
    s->sim_steps = static_cast<int64_t>(cfg.sim_ms / cfg.dt + 0.5);
    s->total_steps = s->pre_steps + s->sim_steps;
    s->h_step = cfg.dt / static_cast<double>(cfg.substeps);
    s->steps_per_noise = std::max(1, static_cast<int>(std::llround(bio.noise_dt / cfg.dt)));
    if (cfg.raster_steps > 0) {
        const size_t words = (static_cast<size_t>(nN) + 31) / 32;
        s->raster.assign(words * static_cast<size_t>(cfg.raster_steps), 0u);
    }
}

// src/astrosim_fused.cu:236-253
inline void astro_rhs(const Bio& c, double Ca_tot, double IP3_0, double tau_IP3, double Ca, double IP3,
                      double h, double noise, double& dCa, double& dIP3, double& dh) {
    const double Ca_ER = (Ca_tot - Ca) / c.ratio_ER_cyt;
    const double m_inf = IP3 / (IP3 + c.Kd_IP3_1);
    const double n_inf = Ca / (Ca + c.Kd_act);
    const double m3 = m_inf * m_inf * m_inf;
    const double n3 = n_inf * n_inf * n_inf;
    const double h3 = h * h * h;
    const double J_channel = c.ratio_ER_cyt * c.rate_IP3R * m3 * n3 * h3 * (Ca_ER - Ca);
    const double J_pump = c.rate_SERCA * Ca * Ca / (c.Km_SERCA * c.Km_SERCA + Ca * Ca);
    const double J_leak = c.ratio_ER_cyt * c.rate_L * (Ca_ER - Ca);
    const double alpha_h = c.k_IP3R * c.Kd_inh * (IP3 + c.Kd_IP3_1) / (IP3 + c.Kd_IP3_2);
    const double beta_h = c.k_IP3R * Ca;
    dCa = J_channel - J_pump + J_leak + noise;
    dIP3 = (IP3_0 - IP3) / tau_IP3;
    dh = alpha_h * (1.0 - h) - beta_h * h;
}

// src/astrosim_fused.cu:281-290
inline void neuron_rhs(const NeuronP& p, double V, double w, double g_ex, double g_in, double I_ext,
                       double& dV, double& dw) {
    const double Vc = V < p.V_peak ? V : p.V_peak;
    const double I_spike = p.g_L * p.Delta_T * exp_maybe_perturbed((Vc - p.V_th) / p.Delta_T, p.exp_perturb);
    if (p.contract) {  // the same expression with each product fused into the sum that uses it
        double t = std::fma(-p.g_L, Vc - p.E_L, I_spike);
        t = std::fma(-g_ex, Vc - p.E_ex, t);
        t = std::fma(-g_in, Vc - p.E_in, t);
        dV = (t - w + p.I_e + I_ext) / p.C_m;
        dw = std::fma(p.a, Vc - p.E_L, -w) / p.tau_w;
        return;
    }
    const double I_syn_ex = g_ex * (Vc - p.E_ex);
    const double I_syn_in = g_in * (Vc - p.E_in);
    dV = (-p.g_L * (Vc - p.E_L) + I_spike - I_syn_ex - I_syn_in - w + p.I_e + I_ext) / p.C_m;
    dw = (p.a * (Vc - p.E_L) - w) / p.tau_w;
}

// src/astrosim_fused.cu:374-427 for one astrocyte
void astro_cell(oracle_sim* s, u32 a, int64_t step) {
    const Bio& bio = s->bio;
    const u64 seed = s->cfg.seed;
    const int S = s->slots;
    const int read_slot = static_cast<int>((step + S - s->d_e) % S);  // e2a delay uses d_e (384)
    const double* row = s->ring_n.data() + static_cast<size_t>(read_slot) * s->n_neurons;
    double gathered = 0.0;
    for (u32 k = s->net.e2a.rs[a]; k < s->net.e2a.rs[a + 1]; ++k) gathered += row[s->net.e2a.src[k]];
    double ip3_input = bio.w_n2a * gathered;
    if (bio.astro_poiss_rate > 0.0) {
        const double lambda = bio.astro_poiss_rate * s->cfg.dt * 1e-3;
        const int ev = poisson(seed ^ 0xC2B2AE3D27D4EB4FULL, static_cast<u64>(step) * 1000003ULL + a, lambda);
        if (ev > 0) ip3_input += bio.astro_poiss_weight * static_cast<double>(ev);
    }
    double noise = 0.0;
    if (bio.astro_noise_std > 0.0 && bio.independent_noise)
        noise = bio.astro_noise_std * normal(seed ^ 0x9E3779B97F4A7C15ULL, static_cast<u64>(step) * 1000003ULL + a);
    else if (bio.astro_noise_std > 0.0)
        noise = bio.astro_noise_std *
                normal(seed ^ 0x9E3779B97F4A7C15ULL,
                       static_cast<u64>(step / s->steps_per_noise));  // shared draw, 1048-1051
    // 255-278: astro_advance
    double Ca = s->Ca[a], IP3 = s->IP3[a], h = s->h[a];
    const double Ct = s->Ca_tot[a], I0 = s->IP3_0[a], tI = s->tau_IP3[a], dI = s->delta_IP3[a];
    const double hs = s->h_step;
    if (ip3_input != 0.0) IP3 += dI * ip3_input;
    for (int sub = 0; sub < s->cfg.substeps; ++sub) {
        double k1c, k1i, k1h, k2c, k2i, k2h, k3c, k3i, k3h, k4c, k4i, k4h;
        astro_rhs(bio, Ct, I0, tI, Ca, IP3, h, noise, k1c, k1i, k1h);
        astro_rhs(bio, Ct, I0, tI, Ca + 0.5 * hs * k1c, IP3 + 0.5 * hs * k1i, h + 0.5 * hs * k1h, noise, k2c,
                  k2i, k2h);
        astro_rhs(bio, Ct, I0, tI, Ca + 0.5 * hs * k2c, IP3 + 0.5 * hs * k2i, h + 0.5 * hs * k2h, noise, k3c,
                  k3i, k3h);
        astro_rhs(bio, Ct, I0, tI, Ca + hs * k3c, IP3 + hs * k3i, h + hs * k3h, noise, k4c, k4i, k4h);
        Ca += (hs / 6.0) * (k1c + 2.0 * k2c + 2.0 * k3c + k4c);
        IP3 += (hs / 6.0) * (k1i + 2.0 * k2i + 2.0 * k3i + k4i);
        h += (hs / 6.0) * (k1h + 2.0 * k2h + 2.0 * k3h + k4h);
        Ca = Ca < 0.0 ? 0.0 : (Ca > Ct ? Ct : Ca);
        h = h < 0.0 ? 0.0 : (h > 1.0 ? 1.0 : h);
        IP3 = IP3 < 0.0 ? 0.0 : IP3;
    }
    s->Ca[a] = Ca;
    s->IP3[a] = IP3;
    s->h[a] = h;
    // 416-426: SIC factor, engaged flag, own ring slot
    const double y = (Ca - bio.SIC_th) * 1000.0;
    const double factor = (y <= 1.0) ? 0.0 : bio.SIC_scale * std::log(y);
    if (factor > 0.0) s->ever_active[a] = 1;
    s->sic_last[a] = factor;
    s->ring_s[static_cast<size_t>(step % S) * s->sz.n_astro + a] = factor;
}

// src/astrosim_fused.cu:433-587 for one neuron; returns 1 if it spiked
int neuron_cell(oracle_sim* s, u32 j, int64_t step, bool sic_refresh, u64 noise_idx) {
    const Bio& bio = s->bio;
    const u64 seed = s->cfg.seed;
    const int S = s->slots;
    const bool exc = j < s->sz.n_exc;
    const NeuronP& p = exc ? s->pe : s->pi;
    const u32 nN = s->n_neurons;

    const double* row_ex = s->ring_n.data() + static_cast<size_t>((step + S - s->d_e) % S) * nN;
    double exc_sum = 0.0;
    for (u32 k = s->net.exc.rs[j]; k < s->net.exc.rs[j + 1]; ++k) exc_sum += row_ex[s->net.exc.src[k]];
    const double* row_in = s->ring_n.data() + static_cast<size_t>((step + S - s->d_i) % S) * nN;
    double inh_sum = 0.0;
    for (u32 k = s->net.inh.rs[j]; k < s->net.inh.rs[j + 1]; ++k) inh_sum += row_in[s->net.inh.src[k]];
    double exc_input = bio.w_e * exc_sum;
    const double inh_input = (-bio.w_i) * inh_sum;

    const double rate = exc ? bio.exc_poiss_rate : bio.inh_poiss_rate;
    const double weight = exc ? bio.exc_poiss_weight : bio.inh_poiss_weight;
    if (rate > 0.0) {
        const double lambda = rate * s->cfg.dt * 1e-3;
        const int ev = poisson(seed ^ 0x2545F4914F6CDD1DULL, static_cast<u64>(step) * 1000003ULL + j, lambda);
        if (ev > 0) exc_input += weight * static_cast<double>(ev);
    }
    if (sic_refresh) {
        const double* row_s =
            s->ring_s.data() + static_cast<size_t>((step + S - s->d_a2n) % S) * s->sz.n_astro;
        double sic_sum = 0.0;
        for (u32 k = s->net.sic.rs[j]; k < s->net.sic.rs[j + 1]; ++k) sic_sum += row_s[s->net.sic.src[k]];
        s->I_sic[j] = bio.w_a2n * sic_sum;
    }
    double I_ext = s->I_sic[j];
    const double nstd = exc ? bio.exc_noise_std : bio.inh_noise_std;
    if (nstd > 0.0) {
        if (bio.independent_noise)
            I_ext += nstd * normal(seed ^ 0x9E3779B185EBCA87ULL, noise_idx * 1000033ULL + static_cast<u64>(j));
        // shared exc/inh noise is 0 in the reference loop (1052)
    }

    double V = s->V[j], w = s->w[j];
    double g_ex = s->g_ex[j], dg_ex = s->dg_ex[j] + exc_input * p.psc_ex;
    double g_in = s->g_in[j], dg_in = s->dg_in[j] + inh_input * p.psc_in;
    int refr = s->refr[j];
    bool spiked = false;
    const double hs = s->h_step;
    for (int sub = 0; sub < s->cfg.substeps; ++sub) {
        const double ex_decay = std::exp(-hs / p.tau_syn_ex);
        const double in_decay = std::exp(-hs / p.tau_syn_in);
        const double g_ex_next = ex_decay * (g_ex + hs * dg_ex);
        const double dg_ex_next = ex_decay * dg_ex;
        const double g_in_next = in_decay * (g_in + hs * dg_in);
        const double dg_in_next = in_decay * dg_in;
        if (refr > 0) {
            V = s->V_reset[j];
            double dV, dw;
            neuron_rhs(p, V, w, g_ex, g_in, I_ext, dV, dw);
            w += hs * dw;
        } else {
            const double g_ex_mid = 0.5 * (g_ex + g_ex_next);
            const double g_in_mid = 0.5 * (g_in + g_in_next);
            double k1V, k1w, k2V, k2w, k3V, k3w, k4V, k4w;
            if (p.contract) {  // stage arguments and the weighted sum with fused multiply-adds
                const double hh = 0.5 * hs;
                neuron_rhs(p, V, w, g_ex, g_in, I_ext, k1V, k1w);
                neuron_rhs(p, std::fma(hh, k1V, V), std::fma(hh, k1w, w), g_ex_mid, g_in_mid, I_ext, k2V, k2w);
                neuron_rhs(p, std::fma(hh, k2V, V), std::fma(hh, k2w, w), g_ex_mid, g_in_mid, I_ext, k3V, k3w);
                neuron_rhs(p, std::fma(hs, k3V, V), std::fma(hs, k3w, w), g_ex_next, g_in_next, I_ext, k4V, k4w);
                V = std::fma(hs / 6.0, std::fma(2.0, k3V, std::fma(2.0, k2V, k1V)) + k4V, V);
                w = std::fma(hs / 6.0, std::fma(2.0, k3w, std::fma(2.0, k2w, k1w)) + k4w, w);
            } else {
                neuron_rhs(p, V, w, g_ex, g_in, I_ext, k1V, k1w);
                neuron_rhs(p, V + 0.5 * hs * k1V, w + 0.5 * hs * k1w, g_ex_mid, g_in_mid, I_ext, k2V, k2w);
                neuron_rhs(p, V + 0.5 * hs * k2V, w + 0.5 * hs * k2w, g_ex_mid, g_in_mid, I_ext, k3V, k3w);
                neuron_rhs(p, V + hs * k3V, w + hs * k3w, g_ex_next, g_in_next, I_ext, k4V, k4w);
                V += (hs / 6.0) * (k1V + 2.0 * k2V + 2.0 * k3V + k4V);
                w += (hs / 6.0) * (k1w + 2.0 * k2w + 2.0 * k3w + k4w);
            }
        }
        g_ex = g_ex_next;
        dg_ex = dg_ex_next;
        g_in = g_in_next;
        dg_in = dg_in_next;
        if (refr > 0) {
            --refr;
        } else if (V >= p.V_peak) {
            V = s->V_reset[j];
            w += s->b[j];
            refr = static_cast<int>(p.t_ref / hs + 0.5);
            spiked = true;
        }
    }
    s->V[j] = V;
    s->w[j] = w;
    s->g_ex[j] = g_ex;
    s->dg_ex[j] = dg_ex;
    s->g_in[j] = g_in;
    s->dg_in[j] = dg_in;
    s->refr[j] = refr;

    double out = 0.0;
    if (spiked) {  // 564-579: per-presynaptic Tsodyks-Markram update
        double x = s->stp_x[j], u = s->stp_u[j];
        if (bio.stp_enabled) {
            const double t_now = static_cast<double>(step) * s->cfg.dt;
            const double elapsed = t_now - s->stp_t[j];
            const double x_decay = std::exp(-elapsed / bio.stp_tau_rec);
            const double u_decay = bio.stp_tau_fac < 1e-10 ? 0.0 : std::exp(-elapsed / bio.stp_tau_fac);
            x = 1.0 + (x - x * u - 1.0) * x_decay;
            u = bio.stp_U + u * (1.0 - bio.stp_U) * u_decay;
            s->stp_x[j] = x;
            s->stp_u[j] = u;
            s->stp_t[j] = t_now;
            out = x * u;
        } else {
            out = 1.0;
        }
    }
    s->ring_n[static_cast<size_t>(step % S) * nN + j] = out;
    return spiked ? 1 : 0;
}

void one_step(oracle_sim* s) {
    const int64_t step = s->step;
    // 1043-1046: loop scalars
    const u64 noise_idx = static_cast<u64>(step / s->steps_per_noise);
    const bool sic_refresh = (step - s->d_a2n >= 0) && ((step - s->d_a2n) % s->bio.sic_interval == 0);
    const int nA = static_cast<int>(s->sz.n_astro);
    const int nN = static_cast<int>(s->n_neurons);
#pragma omp parallel for schedule(static) num_threads(s->threads)
    for (int a = 0; a < nA; ++a) astro_cell(s, static_cast<u32>(a), step);
    uint64_t count = 0;
#pragma omp parallel for schedule(static) num_threads(s->threads) reduction(+ : count)
    for (int j = 0; j < nN; ++j) {
        const int sp = neuron_cell(s, static_cast<u32>(j), step, sic_refresh, noise_idx);
        s->spiked[j] = static_cast<unsigned char>(sp);
        count += static_cast<uint64_t>(sp);
    }
    s->counts.push_back(static_cast<uint32_t>(count));
    if (step < s->cfg.raster_steps) {
        const size_t words = (static_cast<size_t>(nN) + 31) / 32;
        uint32_t* r = s->raster.data() + static_cast<size_t>(step) * words;
        for (int j = 0; j < nN; ++j)
            if (s->spiked[j]) r[j / 32] |= 1u << (j % 32);
    }
    // 1066-1076: at the end of the pre-run, note the spike total and clear the engaged flags
    if (step == s->pre_steps - 1 || (s->pre_steps == 0 && step == 0)) {
        uint64_t tot = 0;
        for (uint32_t c : s->counts) tot += c;
        s->spikes_before = tot;
        std::fill(s->ever_active.begin(), s->ever_active.end(), 0);
        s->pre_mark_done = true;
    }
    s->step = step + 1;
}

oracle_sim* make_sim(const astrosim_config* cfg, int n_threads) {
    if (!cfg || cfg->n_total == 0 || !(cfg->dt > 0.0) || cfg->substeps < 1) return nullptr;
    auto* s = new oracle_sim();
    s->cfg = *cfg;
    s->threads = n_threads > 0 ? n_threads : omp_get_max_threads();
    s->sz = scaling(cfg->n_total);
    return s;
}

}  // namespace

extern "C" {

uint64_t oracle_rng_bits(uint64_t seed, uint64_t stream, uint64_t counter) { return bits(seed, stream, counter); }
double oracle_rng_uniform(uint64_t seed, uint64_t stream, uint64_t counter) {
    return uniform(seed, stream, counter);
}
double oracle_rng_normal(uint64_t seed, uint64_t stream) { return normal(seed, stream); }
int oracle_rng_poisson(uint64_t seed, uint64_t stream, double lambda) { return poisson(seed, stream, lambda); }

void oracle_seq_normals(uint64_t seed, uint64_t stream, size_t n, double* out) {
    SeqStream rs(seed, stream);
    for (size_t i = 0; i < n; ++i) out[i] = rs.next_normal();
}

// Sets Bio fields by name (the same names as the reference's Biology struct,
// src/astrosim_fused.cu:742-781): numbers for reals and sic_interval, 0/1 for flags.
static bool set_bio(Bio& b, const char* name, double v) {
#define R_(f) if (std::strcmp(name, #f) == 0) { b.f = v; return true; }
#define F_(f) if (std::strcmp(name, #f) == 0) { b.f = v != 0.0; return true; }
    R_(Ca_tot) R_(IP3_0) R_(tau_IP3) R_(delta_IP3) R_(SIC_scale) R_(Kd_IP3_1) R_(Kd_IP3_2) R_(Kd_act) R_(Kd_inh)
    R_(Km_SERCA) R_(SIC_th) R_(k_IP3R) R_(rate_IP3R) R_(rate_L) R_(rate_SERCA) R_(ratio_ER_cyt) R_(Ca_init)
    R_(h_init) R_(IP3_init) F_(randomize_astro) R_(ra_lower) R_(ra_upper) R_(ra_var)
    R_(e_Delta_T) R_(e_a) R_(e_tau_w) R_(e_V_reset) R_(e_b) R_(e_V_m) R_(e_C_m) R_(e_g_L) R_(e_E_L) R_(e_V_th)
    R_(e_V_peak) R_(e_t_ref) R_(e_E_ex) R_(e_E_in) R_(e_tau_syn_ex) R_(e_tau_syn_in)
    R_(i_Delta_T) R_(i_a) R_(i_tau_w) R_(i_V_reset) R_(i_b) R_(i_V_m) R_(i_C_m) R_(i_g_L) R_(i_E_L) R_(i_V_th)
    R_(i_V_peak) R_(i_t_ref) R_(i_E_ex) R_(i_E_in) R_(i_tau_syn_ex) R_(i_tau_syn_in)
    F_(randomize_neuron) R_(rn_lower) R_(rn_upper) R_(rn_var) R_(w_e) R_(w_i) R_(w_n2a) R_(w_a2n)
    R_(d_e) R_(d_i) R_(d_a2n) F_(stp_enabled) R_(stp_U) R_(stp_tau_rec) R_(stp_tau_fac)
    R_(astro_poiss_rate) R_(astro_poiss_weight) R_(astro_noise_std) R_(exc_poiss_rate) R_(exc_poiss_weight)
    R_(exc_noise_std) R_(inh_poiss_rate) R_(inh_poiss_weight) R_(inh_noise_std) F_(independent_noise) R_(noise_dt)
#undef R_
#undef F_
    if (std::strcmp(name, "sic_interval") == 0) { b.sic_interval = static_cast<int>(v); return true; }
    return false;
}

oracle_sim* oracle_create_with_biology(const astrosim_config* cfg, int n_threads, const char* const* names,
                                       const double* values, size_t n) {
    oracle_sim* s = make_sim(cfg, n_threads);
    if (!s) return nullptr;
    for (size_t i = 0; i < n; ++i) {
        if (!set_bio(s->bio, names[i], values[i])) {
            delete s;
            return nullptr;
        }
    }
    const auto t0 = std::chrono::steady_clock::now();
    s->net = build_network(s->sz, cfg->seed);
    s->build_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    init_state(s);
    return s;
}

oracle_sim* oracle_create(const astrosim_config* cfg, int n_threads) {
    oracle_sim* s = make_sim(cfg, n_threads);
    if (!s) return nullptr;
    const auto t0 = std::chrono::steady_clock::now();
    s->net = build_network(s->sz, cfg->seed);
    s->build_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    init_state(s);
    return s;
}

oracle_sim* oracle_create_with_csr(const astrosim_config* cfg, int n_threads, const uint32_t* exc_rs,
                                   const uint32_t* exc_src, const uint32_t* inh_rs, const uint32_t* inh_src,
                                   const uint32_t* sic_rs, const uint32_t* sic_src, const uint32_t* e2a_rs,
                                   const uint32_t* e2a_src) {
    oracle_sim* s = make_sim(cfg, n_threads);
    if (!s) return nullptr;
    const u32 nN = s->sz.n_exc + s->sz.n_inh, nA = s->sz.n_astro;
    auto load = [](CSR& c, u32 n, const uint32_t* rs, const uint32_t* src) {
        c.rs.assign(rs, rs + n + 1);
        c.src.assign(src, src + rs[n]);
    };
    load(s->net.exc, nN, exc_rs, exc_src);
    load(s->net.inh, nN, inh_rs, inh_src);
    load(s->net.sic, nN, sic_rs, sic_src);
    load(s->net.e2a, nA, e2a_rs, e2a_src);
    init_state(s);
    return s;
}

void oracle_destroy(oracle_sim* s) { delete s; }

void oracle_step(oracle_sim* s, int64_t n_steps) {
    for (int64_t i = 0; i < n_steps; ++i) one_step(s);
}

void oracle_summary(oracle_sim* s, astrosim_summary_t* out) {
    std::memset(out, 0, sizeof(*out));
    out->n_total = s->sz.n_total;
    out->n_exc = s->sz.n_exc;
    out->n_inh = s->sz.n_inh;
    out->n_astro = s->sz.n_astro;
    out->p_primary = s->sz.p;
    out->n_exc_edges = s->net.exc.src.size();
    out->n_inh_edges = s->net.inh.src.size();
    out->n_e2a_edges = s->net.e2a.src.size();
    out->n_sic_edges = s->net.sic.src.size();
    out->pre_steps = s->pre_steps;
    out->sim_steps = s->sim_steps;
    out->total_steps = s->total_steps;
    out->steps_done = s->step;
    uint64_t tot = 0;
    for (uint32_t c : s->counts) tot += c;
    out->spikes_total = tot;
    out->spikes_measured = tot - s->spikes_before;
    out->mean_rate_hz = static_cast<double>(out->spikes_measured) /
                        (static_cast<double>(s->n_neurons) * (s->cfg.sim_ms * 1e-3));
    // 1111-1125: mean calcium, final-step threshold count, engaged count
    double mean_ca = 0.0;
    uint32_t active = 0;
    for (double ca : s->Ca) {
        mean_ca += ca;
        if ((ca - s->bio.SIC_th) * 1000.0 > 1.0) ++active;
    }
    mean_ca /= std::max<u32>(1, s->sz.n_astro);
    uint32_t engaged = 0;
    for (unsigned char v : s->ever_active) engaged += v;
    out->mean_ca = mean_ca;
    out->active_astro = active;
    out->engaged_astro = engaged;
    out->sic_th = s->bio.SIC_th;
    out->build_seconds = s->build_s;
}

int64_t oracle_get_state(oracle_sim* s, int which, double* dst, size_t cap) {
    const std::vector<double>* v = nullptr;
    switch (which) {
        case ASTROSIM_STATE_CA: v = &s->Ca; break;
        case ASTROSIM_STATE_IP3: v = &s->IP3; break;
        case ASTROSIM_STATE_H: v = &s->h; break;
        case ASTROSIM_STATE_V: v = &s->V; break;
        case ASTROSIM_STATE_W: v = &s->w; break;
        case ASTROSIM_STATE_G_EX: v = &s->g_ex; break;
        case ASTROSIM_STATE_DG_EX: v = &s->dg_ex; break;
        case ASTROSIM_STATE_G_IN: v = &s->g_in; break;
        case ASTROSIM_STATE_DG_IN: v = &s->dg_in; break;
        case ASTROSIM_STATE_I_SIC: v = &s->I_sic; break;
        case ASTROSIM_STATE_STP_X: v = &s->stp_x; break;
        case ASTROSIM_STATE_STP_U: v = &s->stp_u; break;
        case ASTROSIM_STATE_STP_T_LAST: v = &s->stp_t; break;
        case ASTROSIM_STATE_CA_TOT: v = &s->Ca_tot; break;
        case ASTROSIM_STATE_IP3_0: v = &s->IP3_0; break;
        case ASTROSIM_STATE_TAU_IP3: v = &s->tau_IP3; break;
        case ASTROSIM_STATE_DELTA_IP3: v = &s->delta_IP3; break;
        case ASTROSIM_STATE_V_RESET: v = &s->V_reset; break;
        case ASTROSIM_STATE_B: v = &s->b; break;
        case ASTROSIM_STATE_SIC_FACTOR: v = &s->sic_last; break;
        default: return -1;
    }
    if (dst) {
        if (cap < v->size()) return -1;
        std::copy(v->begin(), v->end(), dst);
    }
    return static_cast<int64_t>(v->size());
}

int oracle_get_csr(oracle_sim* s, int which, uint32_t* row_start, uint32_t* src, uint32_t* n_targets,
                   uint64_t* n_edges) {
    const CSR* c = nullptr;
    switch (which) {
        case ASTROSIM_CSR_EXC: c = &s->net.exc; break;
        case ASTROSIM_CSR_INH: c = &s->net.inh; break;
        case ASTROSIM_CSR_SIC: c = &s->net.sic; break;
        case ASTROSIM_CSR_E2A: c = &s->net.e2a; break;
        default: return -1;
    }
    if (n_targets) *n_targets = static_cast<uint32_t>(c->rs.size() - 1);
    if (n_edges) *n_edges = c->src.size();
    if (row_start) std::copy(c->rs.begin(), c->rs.end(), row_start);
    if (src) std::copy(c->src.begin(), c->src.end(), src);
    return 0;
}

int oracle_spike_counts(oracle_sim* s, int64_t first, int64_t n, uint32_t* counts) {
    if (first < 0 || n < 0 || first + n > static_cast<int64_t>(s->counts.size())) return -1;
    std::copy(s->counts.begin() + first, s->counts.begin() + first + n, counts);
    return 0;
}

int oracle_raster(oracle_sim* s, uint32_t* bits_out, size_t words) {
    if (words < s->raster.size()) return -1;
    std::copy(s->raster.begin(), s->raster.end(), bits_out);
    return 0;
}

double oracle_build_seconds(oracle_sim* s) { return s->build_s; }

void oracle_set_exp_perturbation(oracle_sim* s, double rate) {
    if (!s) return;
    s->pe.exp_perturb = rate;
    s->pi.exp_perturb = rate;
}

void oracle_set_contraction(oracle_sim* s, int on) {
    if (!s) return;
    s->pe.contract = on != 0;
    s->pi.contract = on != 0;
}

}  // extern "C"
