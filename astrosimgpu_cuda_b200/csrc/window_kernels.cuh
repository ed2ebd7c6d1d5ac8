// window_kernels.cuh -- device bodies of the windowed engine, shared by the
// single-network kernels (window.cu) and the batched ensemble kernels (ensemble.cu).
#pragma once

#include "step_kernels.cuh"
#include "window.cuh"

namespace astrosim {

template <typename R>
struct WinPtrs {
    u32 *nin_cnt, *ain_cnt;          // [2][n]
    Deposit<R> *nin_ent, *ain_ent;   // [2][n][kInboxSlots]
    u32* spk_word;                   // [2][n_neurons]
    R* spk_val;                      // [2][W][n_neurons]
    u32* spk_list;                   // [2][cap]
    u32* spk_count;                  // [2]
    R* sic_win;                      // [2][n_astro][W]
    u32* astro_active;               // [2][astro_words]
    u32* sic_flag;                   // [2][neuron_words]
    int* mode;                       // [2]
    const u32 *fe_rs, *fe_dst, *fi_rs, *fi_dst, *fa_rs, *fa_astro, *fa_pos, *fs_rs, *fs_dst;
    u32 cap, push_limit, astro_words, neuron_words;
    int W;
};

template <typename R>
inline WinPtrs<R> win_ptrs(WindowState& ws, const RunConsts& rc) {
    WinPtrs<R> w{};
    w.nin_cnt = ws.nin_cnt.get();
    w.ain_cnt = ws.ain_cnt.get();
    w.nin_ent = reinterpret_cast<Deposit<R>*>(ws.nin_ent.get());
    w.ain_ent = reinterpret_cast<Deposit<R>*>(ws.ain_ent.get());
    w.spk_word = ws.spk_word.get();
    w.spk_val = reinterpret_cast<R*>(ws.spk_val.get());
    w.spk_list = ws.spk_list.get();
    w.spk_count = ws.spk_count.get();
    w.sic_win = reinterpret_cast<R*>(ws.sic_win.get());
    w.astro_active = ws.astro_active.get();
    w.sic_flag = ws.sic_flag.get();
    w.mode = ws.mode.get();
    w.fe_rs = ws.fwd.exc_rs.get();
    w.fe_dst = ws.fwd.exc_dst.get();
    w.fi_rs = ws.fwd.inh_rs.get();
    w.fi_dst = ws.fwd.inh_dst.get();
    w.fa_rs = ws.fwd.e2a_rs.get();
    w.fa_astro = ws.fwd.e2a_astro.get();
    w.fa_pos = ws.fwd.e2a_pos.get();
    w.fs_rs = ws.fwd.sic_rs.get();
    w.fs_dst = ws.fwd.sic_dst.get();
    w.cap = ws.push_limit + 1;
    w.push_limit = ws.push_limit;
    w.astro_words = (rc.n_astro + 31) / 32;
    w.neuron_words = (rc.n_neurons + 31) / 32;
    w.W = ws.W;
    return w;
}

// Sorts deposits by (step, kind, key): the order in which the reference's dense
// gather meets them (row order within one step and kind).
template <typename R>
__device__ __forceinline__ void sort_deposits(Deposit<R>* d, int n) {
    for (int i = 1; i < n; ++i) {
        const Deposit<R> x = d[i];
        const unsigned long long kx = (static_cast<unsigned long long>(x.meta) << 32) | x.key;
        int k = i - 1;
        while (k >= 0 && ((static_cast<unsigned long long>(d[k].meta) << 32) | d[k].key) > kx) {
            d[k + 1] = d[k];
            --k;
        }
        d[k + 1] = x;
    }
}

// Per-step sums of one CSR row against the previous window's spike words, in row
// order (the exact fallback when deposits are not available).
template <typename R>
__device__ __forceinline__ void pull_row(const u32* __restrict__ rs, const u32* __restrict__ src, u32 row,
                                         const u32* __restrict__ words, const R* __restrict__ vals, u64 n_neurons,
                                         int s0, int s1, R* acc) {
    const u32 k1 = rs[row + 1];
    for (u32 k = rs[row]; k < k1; ++k) {
        const u32 s = src[k];
        u32 wd = words[s];
        if (!wd) continue;
        wd &= ((s1 >= 32 ? 0xFFFFFFFFu : ((1u << s1) - 1u)) & ~((1u << s0) - 1u));
        while (wd) {
            const int b = __ffs(wd) - 1;
            wd &= wd - 1;
            acc[b] += vals[static_cast<u64>(b) * n_neurons + s];
        }
    }
}

// Neuron j through steps [s_begin, s_end) of the window starting at win_start.
template <typename R, bool EXC>
__device__ __forceinline__ void neuron_window(const RunConsts& rc, const NetScalars& ns, const NeuronK& pk,
                                              const StepPtrs<R>& p,
                                              const WinPtrs<R>& w, u32 j, i64 win_start, int s_begin, int s_end,
                                              int buf, bool pull, bool window_done) {
    const int prev = buf ^ 1;
    const int W = w.W;
    const u64 nN = ns.n_neurons;

    // synaptic input of the window: deposits (push) or the row walk (pull); steps
    // whose bit in ex_mask / in_mask is clear have none (+0.0)
    R ex_acc[kMaxWindow], in_acc[kMaxWindow];
    u32 ex_mask = 0, in_mask = 0;
    const u64 slot_base = static_cast<u64>(buf) * nN + j;
    const u32 c = w.nin_cnt[slot_base];
    if (pull || c > kInboxSlots) {
        for (int i = 0; i < W; ++i) ex_acc[i] = in_acc[i] = static_cast<R>(0.0);
        ex_mask = in_mask = (1u << W) - 1u;
        const u32* words = w.spk_word + static_cast<u64>(prev) * nN;
        const R* vals = w.spk_val + static_cast<u64>(prev) * W * nN;
        pull_row<R>(p.exc_rs, p.exc_src, j, words, vals, nN, s_begin, s_end, ex_acc);
        pull_row<R>(p.inh_rs, p.inh_src, j, words, vals, nN, s_begin, s_end, in_acc);
    } else if (c > 0) {
        Deposit<R> d[kInboxSlots];
        for (u32 i = 0; i < c; ++i) d[i] = w.nin_ent[slot_base * kInboxSlots + i];
        sort_deposits<R>(d, static_cast<int>(c));
        for (u32 i = 0; i < c; ++i) {
            const int st = static_cast<int>(d[i].meta & 0xFFu);
            if (st < s_begin || st >= s_end) continue;
            const u32 bit = 1u << st;
            if ((d[i].meta >> 8) == 0) {
                ex_acc[st] = ((ex_mask & bit) ? ex_acc[st] : static_cast<R>(0.0)) + d[i].val;
                ex_mask |= bit;
            } else {
                in_acc[st] = ((in_mask & bit) ? in_acc[st] : static_cast<R>(0.0)) + d[i].val;
                in_mask |= bit;
            }
        }
    }
    if (window_done && c) w.nin_cnt[slot_base] = 0;

    // SIC factors of the previous window through the active-astrocyte bitmask, for a
    // neuron the push flagged (its a2n row holds an astrocyte that was active); for
    // the others every factor in the row is 0, the same as the walk would find
    R sic_acc[kMaxWindow];
    bool sic_input = false;
    u32* flag_word = w.sic_flag + static_cast<u64>(buf) * w.neuron_words + (j >> 5);
    const u32 flag_bit = 1u << (j & 31);
    if (*flag_word & flag_bit) {
        if (window_done) atomicAnd(flag_word, ~flag_bit);  // clean for the window after next
        const u32* act = w.astro_active + static_cast<u64>(prev) * w.astro_words;
        const R* fac = w.sic_win + static_cast<u64>(prev) * ns.n_astro * W;
        const u32 k1 = p.sic_rs[j + 1];
        for (u32 k = p.sic_rs[j]; k < k1; ++k) {
            const u32 a = p.sic_src[k];
            if (!((act[a >> 5] >> (a & 31)) & 1u)) continue;  // every factor of this astrocyte was 0
            if (!sic_input) {
                for (int i = 0; i < W; ++i) sic_acc[i] = static_cast<R>(0.0);
                sic_input = true;
            }
            const R* f = fac + static_cast<u64>(a) * W;
            for (int st = s_begin; st < s_end; ++st) sic_acc[st] += f[st];
        }
    }

    NeuronRegs<R> n{p.V[j], p.w[j], p.V_reset[j], p.b[j], p.g_ex[j], p.dg_ex[j], p.g_in[j], p.dg_in[j], p.I_sic[j],
                    p.refr[j]};
    const R hs = as_r<R>(rc.h_step, rc.f_h_step);
    const R ex_decay = exp_r(-hs / static_cast<R>(pk.tau_syn_ex));
    const R in_decay = exp_r(-hs / static_cast<R>(pk.tau_syn_in));
    const double nstd = EXC ? rc.noise_exc : rc.noise_inh;
    const bool has_noise = nstd > 0.0 && rc.independent_noise;
    // Per-step schedule by counters instead of divisions: the SIC refresh runs when
    // (t - d_a2n) >= 0 and (t - d_a2n) % sic_interval == 0, the noise index is
    // t / steps_per_noise (src/astrosim_fused.cu:1046-1050).
    const i64 t0 = win_start + s_begin;
    i64 since = t0 - rc.d_a2n;
    const int si = rc.sic_interval, spn = rc.steps_per_noise;
    int phase = static_cast<int>(((since % si) + si) % si);
    u64 nidx = static_cast<u64>(t0 / spn);
    int nphase = static_cast<int>(t0 % spn);
    double noise = 0.0;
    if (has_noise) noise = neuron_noise<R>(ns, nstd, nidx, j);
    u64 pbase = step_base(ns.seed, kNeuronPoissonKey, t0, j);
    u32 word = 0;
    R* vout = w.spk_val + static_cast<u64>(buf) * W * nN;
    for (int st = s_begin; st < s_end; ++st) {
        const i64 t = win_start + st;
        const bool refresh = since >= 0 && phase == 0;
        if (has_noise && nphase == 0 && st != s_begin) noise = neuron_noise<R>(ns, nstd, nidx, j);
        const R zero = static_cast<R>(0.0);
        const bool spiked = neuron_advance_step<R>(
            rc, ns, pk, EXC, n, ((ex_mask >> st) & 1u) ? ex_acc[st] : zero, ((in_mask >> st) & 1u) ? in_acc[st] : zero,
            refresh, sic_input ? sic_acc[st] : zero, has_noise, noise, pbase, ex_decay, in_decay);
        pbase += kStepAdvance;
        ++since;
        if (++phase == si) phase = 0;
        if (++nphase == spn) {
            nphase = 0;
            ++nidx;
        }
        if (spiked) {
            const R out = stp_on_spike<R>(rc, p.stp_x[j], p.stp_u[j], p.stp_t[j], t);
            vout[static_cast<u64>(st) * nN + j] = out;
            word |= 1u << st;
            const u32 slot = atomicAdd(&w.spk_count[buf], 1u);
            if (slot < w.cap) w.spk_list[static_cast<u64>(buf) * w.cap + slot] = (j << 5) | static_cast<u32>(st);
            atomicAdd(&p.counts[t], 1u);
            if (t < p.raster_steps) atomicOr(&p.raster[static_cast<u64>(t) * ns.words + (j >> 5)], 1u << (j & 31));
        }
    }
    p.V[j] = n.V;
    p.w[j] = n.w;
    p.g_ex[j] = n.g_ex;
    p.dg_ex[j] = n.dg_ex;
    p.g_in[j] = n.g_in;
    p.dg_in[j] = n.dg_in;
    p.I_sic[j] = n.I_sic;
    p.refr[j] = n.refr;
    u32* sw = w.spk_word + slot_base;
    *sw = s_begin == 0 ? word : (*sw | word);
}

// One block of 128 cells advances through steps [s_begin, s_end) of the window that
// starts at step win_start (buffer parity buf): block `blk` of the astrocytes when
// `astro`, else block `blk` of the neurons.
template <typename R>
__device__ __forceinline__ void window_cells(const RunConsts& rc, const NetScalars& ns, const StepPtrs<R>& p,
                                             const WinPtrs<R>& w,
                                             i64 win_start, int s_begin, int s_end, int buf, i64 mark, u32 blk,
                                             bool astro) {
    const int prev = buf ^ 1;
    const int W = w.W;
    const bool window_done = s_end == W;
    const bool pull = w.mode[buf] != 0;
    if (astro) {
        // ------------------------------------------------------------ astrocytes
        const u32 a = blk * blockDim.x + threadIdx.x;
        const bool valid = a < ns.n_astro;
        bool any_active = false;
        if (valid) {
            AstroRegs<R> s = load_astro<R>(p.Ca[a], p.IP3[a], p.h[a], p.Ca_tot[a], p.IP3_0[a], p.tau_IP3[a],
                                           p.delta_IP3[a]);
            // per-step IP3 input; steps whose bit in in_mask is clear have none (+0.0)
            R acc[kMaxWindow];
            u32 in_mask = 0;
            const u64 slot_base = (static_cast<u64>(buf) * ns.n_astro + a);
            const u32 c = w.ain_cnt[slot_base];
            if (pull || c > kInboxSlots) {
                for (int i = 0; i < W; ++i) acc[i] = static_cast<R>(0.0);
                in_mask = (1u << W) - 1u;
                pull_row<R>(p.e2a_rs, p.e2a_src, a, w.spk_word + static_cast<u64>(prev) * ns.n_neurons,
                            w.spk_val + static_cast<u64>(prev) * W * ns.n_neurons, ns.n_neurons, s_begin, s_end, acc);
            } else if (c > 0) {
                Deposit<R> d[kInboxSlots];
                for (u32 i = 0; i < c; ++i) d[i] = w.ain_ent[slot_base * kInboxSlots + i];
                sort_deposits<R>(d, static_cast<int>(c));
                for (u32 i = 0; i < c; ++i) {
                    const int st = static_cast<int>(d[i].meta & 0xFFu);
                    if (st < s_begin || st >= s_end) continue;
                    const u32 bit = 1u << st;
                    acc[st] = ((in_mask & bit) ? acc[st] : static_cast<R>(0.0)) + d[i].val;
                    in_mask |= bit;
                }
            }
            if (window_done && c) w.ain_cnt[slot_base] = 0;
            unsigned char ever = p.ever_active[a];
            R* out = w.sic_win + (static_cast<u64>(buf) * ns.n_astro + a) * W;
            R factor = static_cast<R>(0.0);
            u64 pbase = step_base(ns.seed, kAstroPoissonKey, win_start + s_begin, a);
            u64 nbase = step_base(ns.seed, kAstroNoiseKey, win_start + s_begin, a);
            // recording phase (t + 1) % rec_every, advanced by a counter
            i64 rphase = p.ca_rec ? (win_start + s_begin + 1) % p.rec_every : 1;
            for (int st = s_begin; st < s_end; ++st) {
                const i64 t = win_start + st;
                factor = astro_advance_step<R>(rc, ns, s, ((in_mask >> st) & 1u) ? acc[st] : static_cast<R>(0.0), a, t,
                                               pbase, nbase);
                pbase += kStepAdvance;
                nbase += kStepAdvance;
                if (p.ca_rec) {
                    record_ca<R>(p, a, t, rphase == 0, s.Ca);
                    if (++rphase == p.rec_every) rphase = 0;
                }
                out[st] = factor;
                if (factor > static_cast<R>(0.0)) {
                    ever = 1;
                    any_active = true;
                }
                if (t == mark) ever = 0;  // end of the pre-run (src/astrosim_fused.cu:1075)
            }
            p.Ca[a] = s.Ca;
            p.IP3[a] = s.IP3;
            p.h[a] = s.h;
            p.ever_active[a] = ever;
            p.sic_last[a] = factor;
        }
        const unsigned ballot = __ballot_sync(0xffffffffu, any_active);
        if ((threadIdx.x & 31) == 0 && a < ns.n_astro) {
            u32* word = w.astro_active + static_cast<u64>(buf) * w.astro_words + (a >> 5);
            if (s_begin == 0) *word = ballot; else if (ballot) atomicOr(word, ballot);
        }
        return;
    }
    // ---------------------------------------------------------------- neurons
    const u32 j = blk * blockDim.x + threadIdx.x;
    if (j >= ns.n_neurons) return;
    // one instantiation per population, so its constants are compile-time operands
    if (j < ns.n_exc)
        neuron_window<R, true>(rc, ns, rc.pe, p, w, j, win_start, s_begin, s_end, buf, pull, window_done);
    else
        neuron_window<R, false>(rc, ns, rc.pi, p, w, j, win_start, s_begin, s_end, buf, pull, window_done);
}

// After window `buf` completes: flag the neurons whose a2n rows hold an astrocyte
// that was active in it, then deliver its spikes into the inboxes of the next
// window (buffer buf ^ 1), or switch the next window to pull when it was busy.
// Blocks 0 .. n_blk-1 share the spike list and the active-astrocyte words.
// Targets outside [t_lo, t_hi) (neurons) and [a_lo, a_hi) (astrocytes) are skipped:
// a rank of a sharded network delivers only into the cells it owns.
template <typename R>
__device__ __forceinline__ void push_cells(const WinPtrs<R>& w, u32 n_exc, u32 n_inh, u64 n_neurons, u64 n_astro,
                                           int buf, u32 blk, u32 n_blk, u32 t_lo = 0, u32 t_hi = 0xFFFFFFFFu,
                                           u32 a_lo = 0, u32 a_hi = 0xFFFFFFFFu) {
    const int nxt = buf ^ 1;
    const u32 n = w.spk_count[buf];
    const bool busy = n > w.push_limit;
    if (blk == 0 && threadIdx.x == 0) {
        w.mode[nxt] = busy ? 1 : 0;
        w.spk_count[nxt] = 0;  // the next window appends its spikes there
    }
    const u32 lane = threadIdx.x & 31;
    const u64 warp = (static_cast<u64>(blk) * blockDim.x + threadIdx.x) >> 5;
    const u64 n_warps = (static_cast<u64>(n_blk) * blockDim.x) >> 5;
    {
        // a warp per active astrocyte: flag its a2n targets for the next window
        const u32* act = w.astro_active + static_cast<u64>(buf) * w.astro_words;
        u32* flags = w.sic_flag + static_cast<u64>(nxt) * w.neuron_words;
        for (u64 wd = warp; wd < w.astro_words; wd += n_warps) {
            u32 bits = act[wd];
            while (bits) {
                const u32 a = static_cast<u32>(wd * 32) + static_cast<u32>(__ffs(bits) - 1);
                bits &= bits - 1;
                for (u32 k = w.fs_rs[a] + lane; k < w.fs_rs[a + 1]; k += 32) {
                    const u32 t = w.fs_dst[k];
                    if (t < t_lo || t >= t_hi) continue;
                    atomicOr(&flags[t >> 5], 1u << (t & 31));
                }
            }
        }
    }
    if (busy) return;
    const R* vals = w.spk_val + static_cast<u64>(buf) * w.W * n_neurons;
    for (u64 e = warp; e < n; e += n_warps) {
        const u32 packed = w.spk_list[static_cast<u64>(buf) * w.cap + e];
        const u32 j = packed >> 5, st = packed & 31u;
        const R v = vals[static_cast<u64>(st) * n_neurons + j];
        if (j < n_exc) {
            for (u32 k = w.fe_rs[j] + lane; k < w.fe_rs[j + 1]; k += 32) {
                const u32 t = w.fe_dst[k];
                if (t < t_lo || t >= t_hi) continue;
                const u64 sb = static_cast<u64>(nxt) * n_neurons + t;
                const u32 slot = atomicAdd(&w.nin_cnt[sb], 1u);
                if (slot < kInboxSlots) w.nin_ent[sb * kInboxSlots + slot] = Deposit<R>{j, st, v};
            }
            for (u32 k = w.fa_rs[j] + lane; k < w.fa_rs[j + 1]; k += 32) {
                const u32 a = w.fa_astro[k];
                if (a < a_lo || a >= a_hi) continue;
                const u64 sb = static_cast<u64>(nxt) * n_astro + a;
                const u32 slot = atomicAdd(&w.ain_cnt[sb], 1u);
                if (slot < kInboxSlots) w.ain_ent[sb * kInboxSlots + slot] = Deposit<R>{w.fa_pos[k], st, v};
            }
        }
        // the inhibitory rows hold local inhibitory ids and read the spike ring by
        // global id (src/astrosim_fused.cu:458-463): neuron j feeds them when j < n_inh
        if (j < n_inh) {
            for (u32 k = w.fi_rs[j] + lane; k < w.fi_rs[j + 1]; k += 32) {
                const u32 t = w.fi_dst[k];
                if (t < t_lo || t >= t_hi) continue;
                const u64 sb = static_cast<u64>(nxt) * n_neurons + t;
                const u32 slot = atomicAdd(&w.nin_cnt[sb], 1u);
                if (slot < kInboxSlots) w.nin_ent[sb * kInboxSlots + slot] = Deposit<R>{j, st | (1u << 8), v};
            }
        }
    }
}

}  // namespace astrosim
