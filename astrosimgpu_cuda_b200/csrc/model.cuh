// model.cuh -- model definition shared by every kernel of the simulator:
// the counter RNG, the biology constants and the per-cell right-hand sides.
//
// The arithmetic follows the reference program (src/astrosim_fused.cu) operation
// for operation so that results agree with it to the last bit wherever the same
// math library is used; each function names the lines it follows.
#pragma once

#include <cmath>
#include <cstdint>

#ifndef __CUDACC__
#define __host__
#define __device__
#define __forceinline__ inline
#endif

namespace astrosim {

using u32 = std::uint32_t;
using u64 = std::uint64_t;
using i64 = std::int64_t;
using u8 = std::uint8_t;
using u16 = std::uint16_t;

// ------------------------------------------------------------------ RNG
// Stateless splitmix64-style hash of (seed, stream, counter):
// src/astrosim_fused.cu:127-135.  Every random quantity in the model is a
// pure function of these three integers, which is what lets the device
// generate any draw of the reference's sequential streams directly.
constexpr u64 kStreamMul = 0x9E3779B97F4A7C15ULL;
constexpr u64 kCounterMul = 0xBF58476D1CE4E5B9ULL;

// The mixing half of the hash, applied to seed + stream * kStreamMul + counter * kCounterMul.
__host__ __device__ __forceinline__ u64 rng_mix(u64 z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

__host__ __device__ __forceinline__ u64 rng_bits(u64 seed, u64 stream, u64 counter) {
    u64 z = seed;
    z += stream * kStreamMul;
    z += counter * kCounterMul;
    return rng_mix(z);
}

// Stream base seed + stream * kStreamMul: the draws of one (seed, stream) are
// rng_mix(base + counter * kCounterMul).  Per-step streams step * S + cell advance
// the base by S * kStreamMul each step, so a loop over steps needs one 64-bit add.
__host__ __device__ __forceinline__ u64 rng_base(u64 seed, u64 stream) { return seed + stream * kStreamMul; }
__host__ __device__ __forceinline__ double rng_uniform_at(u64 base, u64 counter) {
    return static_cast<double>(rng_mix(base + counter * kCounterMul) >> 11) * (1.0 / 9007199254740992.0);
}

// 53-bit uniform in [0, 1): src/astrosim_fused.cu:137-141 (double build).
__host__ __device__ __forceinline__ double rng_uniform(u64 seed, u64 stream, u64 counter) {
    return static_cast<double>(rng_bits(seed, stream, counter) >> 11) * (1.0 / 9007199254740992.0);
}

// True when the reference's Box-Muller redraw test (u1 <= 1e-300) rejects this draw:
// only an all-zero top 53 bits gives a uniform that small.
__host__ __device__ __forceinline__ bool rng_uniform_is_zero(u64 seed, u64 stream, u64 counter) {
    return (rng_bits(seed, stream, counter) >> 11) == 0;
}

constexpr double kTwoPi = 6.283185307179586476925286766559;

// Box-Muller cosine half from counters 0 and 1: src/astrosim_fused.cu:143-149.
__host__ __device__ __forceinline__ double rng_normal(u64 seed, u64 stream) {
    double u1 = rng_uniform(seed, stream, 0);
    if (u1 <= 1e-300) u1 = 1e-300;
    const double u2 = rng_uniform(seed, stream, 1);
    return sqrt(-2.0 * log(u1)) * cos(kTwoPi * u2);
}

// Knuth's product method with a fresh (seed, stream) per draw, normal
// approximation above lambda = 30: src/astrosim_fused.cu:154-175.
// `limit` must be exp(-lambda); callers hoist it because lambda is a per-run constant.
__host__ __device__ __forceinline__ int rng_poisson_knuth(u64 seed, u64 stream, double lambda, double limit) {
    if (lambda <= 0.0) return 0;
    if (lambda > 30.0) {
        double u1 = rng_uniform(seed, stream, 0);
        if (u1 <= 1e-300) u1 = 1e-300;
        const double u2 = rng_uniform(seed, stream, 1);
        const double z = sqrt(-2.0 * log(u1)) * cos(kTwoPi * u2);
        const double v = lambda + sqrt(lambda) * z;
        return v < 0.0 ? 0 : static_cast<int>(v + 0.5);
    }
    u64 c = 0;
    double product = rng_uniform(seed, stream, c++);
    int count = 0;
    while (product > limit) {
        ++count;
        product *= rng_uniform(seed, stream, c++);
    }
    return count;
}

// rng_poisson_knuth on a precomputed stream base.  `lim53` = floor(exp(-lambda) * 2^53):
// the first draw u0 = m * 2^-53 exceeds the limit exactly when m > lim53, so the
// common zero-event case needs no floating point at all.
__host__ __device__ __forceinline__ int rng_poisson_at(u64 base, double lambda, double limit, u64 lim53) {
    if (lambda <= 0.0) return 0;
    if (lambda > 30.0) {
        double u1 = rng_uniform_at(base, 0);
        if (u1 <= 1e-300) u1 = 1e-300;
        const double u2 = rng_uniform_at(base, 1);
        const double z = sqrt(-2.0 * log(u1)) * cos(kTwoPi * u2);
        const double v = lambda + sqrt(lambda) * z;
        return v < 0.0 ? 0 : static_cast<int>(v + 0.5);
    }
    const u64 m = rng_mix(base) >> 11;
    if (m <= lim53) return 0;
    double product = static_cast<double>(m) * (1.0 / 9007199254740992.0);
    int count = 0;
    u64 c = 1;
    do {
        ++count;
        product *= rng_uniform_at(base, c++);
    } while (product > limit);
    return count;
}

// Stream-selection constants of the per-step draws (src/astrosim_fused.cu:395, 404, 476, 499).
constexpr u64 kAstroPoissonKey = 0xC2B2AE3D27D4EB4FULL;
constexpr u64 kAstroNoiseKey = 0x9E3779B97F4A7C15ULL;
constexpr u64 kNeuronPoissonKey = 0x2545F4914F6CDD1DULL;
constexpr u64 kNeuronNoiseKey = 0x9E3779B185EBCA87ULL;
constexpr u64 kCellStride = 1000003ULL;   // step * 1000003 + cell (src/astrosim_fused.cu:396, 477)
constexpr u64 kNoiseStride = 1000033ULL;  // noise_idx * 1000033 + cell (src/astrosim_fused.cu:500)
constexpr u64 kSetupStream = 0x5EEDULL;   // setup stream id (src/astrosim_fused.cu:634, 917)

// ------------------------------------------------------------------ constants
// Fixed-in-degree scaling law (src/astrosim_fused.cu:595-615).
struct Sizes {
    u32 n_total = 0, n_exc = 0, n_inh = 0, n_astro = 0, n_neurons = 0;
    double p = 0.0;
};
inline Sizes scaling_law(u32 n_total) {
    Sizes s;
    s.n_total = n_total;
    const long e = std::lround(n_total * 0.8);
    s.n_exc = e < 1 ? 1u : static_cast<u32>(e);
    s.n_inh = n_total > s.n_exc ? n_total - s.n_exc : 1u;
    if (s.n_inh < 1) s.n_inh = 1;
    const long a = std::lround(n_total / 5.0);
    s.n_astro = a < 1 ? 1u : static_cast<u32>(a);
    s.n_neurons = s.n_exc + s.n_inh;
    const double p = 80.0 / static_cast<double>(s.n_exc);
    s.p = p < 1.0 ? p : 1.0;
    return s;
}

constexpr u32 kPoolSize = 5;                 // POOL_SIZE (src/astrosim_fused.cu:603)
constexpr double kPThird = 0.2;              // P_THIRD (src/astrosim_fused.cu:600)
constexpr u32 kMaxAstroOutDegree = 10000;    // MAX_ASTRO_OUT_DEGREE (src/astrosim_fused.cu:604)

// Li-Rinzel astrocyte constants (src/astrosim_fused.cu:222-226).
struct AstroK {
    double Kd_IP3_1, Kd_IP3_2, Kd_act, Kd_inh, Km_SERCA;
    double k_IP3R, rate_IP3R, rate_L, rate_SERCA, ratio_ER_cyt;
    double SIC_scale, SIC_th;
    // Folded constants of the FP32 form (its stages multiply by reciprocals).
    float f_inv_ratio, f_ratio_rate_IP3R, f_ratio_rate_L, f_k_Kd_inh, f_Km2;
    // 1 + 1 / ratio_ER_cyt and rate_SERCA * Km_SERCA^2, for the refolded FP32 form.
    float f_1p_inv_ratio, f_rate_Km2;
    // Float copies read by the FP32 stages (converted once here, not per use).
    float f_Kd_IP3_1, f_Kd_IP3_2, f_Kd_act, f_rate_SERCA, f_k_IP3R, f_SIC_scale;
    float pad_[3];     // explicit, zero: the struct has no implicit padding
    double rcp_ratio;  // RN(1 / ratio_ER_cyt), for the exact division by a constant (div_by)
};
static_assert(sizeof(AstroK) == 12 * 8 + 16 * 4 + 8, "AstroK has no implicit padding");

// AdEx neuron constants for one population (src/astrosim_fused.cu:228-232).
struct NeuronK {
    double C_m, g_L, E_L, V_th, Delta_T, a, tau_w;
    double V_peak, t_ref, E_ex, E_in, tau_syn_ex, tau_syn_in, I_e;
    double psc_init_ex, psc_init_in;
    // 1 / Delta_T when Delta_T is a power of two (then x / Delta_T == x * (1 / Delta_T)
    // exactly in IEEE arithmetic), else 0.
    double inv_Delta_T_pow2;
    // Folded constants of the FP32 form.
    float f_gL_DT, f_inv_DT, f_inv_Cm, f_inv_tauw;
    // Float copies read by the FP32 stages (converted once here, not per use).
    float f_V_peak, f_E_L, f_V_th, f_E_ex, f_E_in, f_g_L, f_I_e, f_a, f_psc_init_ex, f_psc_init_in;
    // The FP32 form's AdEx right-hand side refolded (adex_rhs_folded), around E_L and
    // V_th so that no two large terms cancel:  with u = Vc - E_L,
    //   dV = A u + B - w / C_m + 2^(K1 (Vc - V_th) + K2),  A = A0 - (g_ex + g_in) / C_m,
    //   B = C0 + (g_ex Eex_c + g_in Ein_c) + I_ext / C_m,   dw = Wa u - w / tau_w,
    // with K1 = log2(e) / Delta_T, K2 = log2(g_L Delta_T / C_m), A0 = -g_L / C_m,
    // C0 = I_e / C_m, Eex_c = (E_ex - E_L) / C_m, Ein_c = (E_in - E_L) / C_m and
    // Wa = a / tau_w (each computed in double, rounded once).
    float f_K1, f_K2, f_A0, f_C0, f_Eex_c, f_Ein_c, f_Wa, f_pad2;
    // Refractory length in steps, static_cast<int>(t_ref / h_step + 0.5) (src/astrosim_fused.cu:555);
    // set with the step size.
    int ref_steps;
    int pad_;  // explicit, zero: the struct has no implicit padding
    // RN(1 / x) of the constant divisors, for the exact division by a constant (div_by).
    double rcp_C_m, rcp_tau_w, rcp_Delta_T;
};
static_assert(sizeof(NeuronK) == 17 * 8 + 22 * 4 + 2 * 4 + 3 * 8, "NeuronK has no implicit padding");

// Biology defaults, compiled into the reference (src/astrosim_fused.cu:742-781).
struct Biology {
    double Ca_tot = 1.8958264782990153, IP3_0 = 0.010925583871830699;
    double tau_IP3 = 1058.7589568400845, delta_IP3 = 0.04911592657233997;
    double SIC_scale = 1.0, Kd_IP3_1 = 0.13, Kd_IP3_2 = 0.9434, Kd_act = 0.08234, Kd_inh = 1.049;
    double Km_SERCA = 0.1, SIC_th = 0.19669, k_IP3R = 0.0002, rate_IP3R = 0.006, rate_L = 0.00011;
    double rate_SERCA = 0.0009, ratio_ER_cyt = 0.185, Ca_init = 0.073, h_init = 0.793;
    double IP3_init = 0.010925583871830699;
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
    double noise_dt = 0.0;  // 0 resolves to 10 * dt (src/astrosim_fused.cu:848)
};

inline AstroK astro_constants(const Biology& b) {  // src/astrosim_fused.cu:935-938
    AstroK k{};
    k.Kd_IP3_1 = b.Kd_IP3_1; k.Kd_IP3_2 = b.Kd_IP3_2; k.Kd_act = b.Kd_act; k.Kd_inh = b.Kd_inh;
    k.Km_SERCA = b.Km_SERCA; k.k_IP3R = b.k_IP3R; k.rate_IP3R = b.rate_IP3R; k.rate_L = b.rate_L;
    k.rate_SERCA = b.rate_SERCA; k.ratio_ER_cyt = b.ratio_ER_cyt; k.SIC_scale = b.SIC_scale; k.SIC_th = b.SIC_th;
    k.f_inv_ratio = static_cast<float>(1.0 / b.ratio_ER_cyt);
    k.f_ratio_rate_IP3R = static_cast<float>(b.ratio_ER_cyt * b.rate_IP3R);
    k.f_ratio_rate_L = static_cast<float>(b.ratio_ER_cyt * b.rate_L);
    k.f_k_Kd_inh = static_cast<float>(b.k_IP3R * b.Kd_inh);
    k.f_Km2 = static_cast<float>(b.Km_SERCA * b.Km_SERCA);
    k.f_1p_inv_ratio = static_cast<float>(1.0 + 1.0 / b.ratio_ER_cyt);
    k.f_rate_Km2 = static_cast<float>(b.rate_SERCA * b.Km_SERCA * b.Km_SERCA);
    k.f_Kd_IP3_1 = static_cast<float>(b.Kd_IP3_1);
    k.f_Kd_IP3_2 = static_cast<float>(b.Kd_IP3_2);
    k.f_Kd_act = static_cast<float>(b.Kd_act);
    k.f_rate_SERCA = static_cast<float>(b.rate_SERCA);
    k.f_k_IP3R = static_cast<float>(b.k_IP3R);
    k.f_SIC_scale = static_cast<float>(b.SIC_scale);
    k.rcp_ratio = 1.0 / b.ratio_ER_cyt;
    return k;
}

inline NeuronK neuron_constants(const Biology& b, bool exc) {  // src/astrosim_fused.cu:940-951
    NeuronK k{};
    k.C_m = exc ? b.e_C_m : b.i_C_m;
    k.g_L = exc ? b.e_g_L : b.i_g_L;
    k.E_L = exc ? b.e_E_L : b.i_E_L;
    k.V_th = exc ? b.e_V_th : b.i_V_th;
    k.Delta_T = exc ? b.e_Delta_T : b.i_Delta_T;
    k.a = exc ? b.e_a : b.i_a;
    k.tau_w = exc ? b.e_tau_w : b.i_tau_w;
    k.V_peak = exc ? b.e_V_peak : b.i_V_peak;
    k.t_ref = exc ? b.e_t_ref : b.i_t_ref;
    k.E_ex = exc ? b.e_E_ex : b.i_E_ex;
    k.E_in = exc ? b.e_E_in : b.i_E_in;
    k.tau_syn_ex = exc ? b.e_tau_syn_ex : b.i_tau_syn_ex;
    k.tau_syn_in = exc ? b.e_tau_syn_in : b.i_tau_syn_in;
    k.I_e = 0.0;
    k.psc_init_ex = 2.7182818284590452353602874713527 / k.tau_syn_ex;
    k.psc_init_in = 2.7182818284590452353602874713527 / k.tau_syn_in;
    int ex = 0;
    const double mant = std::frexp(k.Delta_T, &ex);
    k.inv_Delta_T_pow2 = (k.Delta_T > 0.0 && mant == 0.5) ? 1.0 / k.Delta_T : 0.0;
    k.f_gL_DT = static_cast<float>(k.g_L * k.Delta_T);
    k.f_inv_DT = static_cast<float>(1.0 / k.Delta_T);
    k.f_inv_Cm = static_cast<float>(1.0 / k.C_m);
    k.f_inv_tauw = static_cast<float>(1.0 / k.tau_w);
    k.f_V_peak = static_cast<float>(k.V_peak);
    k.f_E_L = static_cast<float>(k.E_L);
    k.f_V_th = static_cast<float>(k.V_th);
    k.f_E_ex = static_cast<float>(k.E_ex);
    k.f_E_in = static_cast<float>(k.E_in);
    k.f_g_L = static_cast<float>(k.g_L);
    k.f_I_e = static_cast<float>(k.I_e);
    k.f_a = static_cast<float>(k.a);
    k.f_psc_init_ex = static_cast<float>(k.psc_init_ex);
    k.f_psc_init_in = static_cast<float>(k.psc_init_in);
    {
        const double log2e = 1.4426950408889634073599246810019;
        const double K1 = log2e / k.Delta_T;
        k.f_K1 = static_cast<float>(K1);
        k.f_K2 = static_cast<float>(std::log2(k.g_L * k.Delta_T / k.C_m));
        k.f_A0 = static_cast<float>(-k.g_L / k.C_m);
        k.f_C0 = static_cast<float>(k.I_e / k.C_m);
        k.f_Eex_c = static_cast<float>((k.E_ex - k.E_L) / k.C_m);
        k.f_Ein_c = static_cast<float>((k.E_in - k.E_L) / k.C_m);
        k.f_Wa = static_cast<float>(k.a / k.tau_w);
        k.f_pad2 = 0.0f;
    }
    k.ref_steps = 0;
    k.rcp_C_m = 1.0 / k.C_m;
    k.rcp_tau_w = 1.0 / k.tau_w;
    k.rcp_Delta_T = 1.0 / k.Delta_T;
    return k;
}

inline int delay_to_steps(double delay_ms, double dt) {  // src/astrosim_fused.cu:783-786
    const int s = static_cast<int>(delay_ms / dt + 0.5);
    return s < 1 ? 1 : s;
}

// ------------------------------------------------------------------ device arithmetic
#ifdef __CUDACC__
#ifdef ASTROSIM_FP32_IEEE
// Measurement build of the FP32 form (make fp32ieee): every float function below
// is CUDA's IEEE-conformant one (expf, logf, sqrtf, cosf, correctly rounded
// division) and the noise uniforms keep 53 bits, so that comparing it with the
// default build separates what the hardware approximations cost in agreement with
// FP64 from what float stages cost.  The default build is the product.
__device__ __forceinline__ float exp_fast(float x) { return expf(x); }
__device__ __forceinline__ float log_fast(float x) { return logf(x); }
__device__ __forceinline__ float div_fast(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float sqrt_ftz(float x) { return __fsqrt_rn(x); }
__device__ __forceinline__ float cos_ftz(float x) { return cosf(x); }
#else
// Hardware approximations of the FP32 form, denormals flushed to zero:
// exp(x) = 2^(x log2 e), log(x) = log2(x) ln 2, a / b = a * (1 / b).
__device__ __forceinline__ float ex2_ftz(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float lg2_ftz(float x) {
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rcp_ftz(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float sqrt_ftz(float x) {
    float y;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float cos_ftz(float x) {
    float y;
    asm("cos.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
constexpr float kLog2E = 1.44269504088896340736f;  // log2(e)
constexpr float kLn2 = 0.69314718055994530942f;    // ln(2)
__device__ __forceinline__ float exp_fast(float x) { return ex2_ftz(x * kLog2E); }
__device__ __forceinline__ float log_fast(float x) { return lg2_ftz(x) * kLn2; }
__device__ __forceinline__ float div_fast(float a, float b) { return a * rcp_ftz(b); }
#endif  // ASTROSIM_FP32_IEEE

// x / y rounded to nearest, for a divisor whose reciprocal ry = RN(1 / y) is known.
// q0 = RN(x ry) is within 1.5 ulp of x / y; one correction q1 = RN(q0 + (x - q0 y) ry)
// leaves an O(2^-106) relative error, so q1 is a faithful quotient; then by Markstein's
// theorem (faithful q, correctly rounded ry => the remainder x - q y is exact and
// RN(q + (x - q y) ry) = RN(x / y)) the second correction returns the rounded quotient.
// Holds while x / y neither overflows nor underflows; x = -0 keeps its sign.
__device__ __forceinline__ double div_by(double x, double y, double ry) {
    double q = x * ry;
    double r = fma(-q, y, x);
    q = fma(r, ry, q);
    r = fma(-q, y, x);
    const double out = fma(r, ry, q);
    return (__double_as_longlong(x) << 1) == 0 ? x : out;
}
#endif

// ------------------------------------------------------------------ right-hand sides
#ifdef __CUDACC__
// Li-Rinzel: src/astrosim_fused.cu:236-253 (operand order kept; the divisions by the
// constants ratio_ER_cyt and tau_IP3 are exact, see div_by; rcp_tau_IP3 = RN(1 / tau_IP3)).
__device__ __forceinline__ void astro_rhs(const AstroK& c, double Ca_tot, double IP3_0, double tau_IP3,
                                          double rcp_tau_IP3, double Ca, double IP3, double h, double noise,
                                          double& dCa, double& dIP3, double& dh) {
    const double ratio = c.ratio_ER_cyt;
    const double Ca_ER = div_by(Ca_tot - Ca, ratio, c.rcp_ratio);
    const double m_inf = IP3 / (IP3 + c.Kd_IP3_1);
    const double n_inf = Ca / (Ca + c.Kd_act);
    const double m3 = m_inf * m_inf * m_inf;
    const double n3 = n_inf * n_inf * n_inf;
    const double h3 = h * h * h;
    const double J_channel = ratio * c.rate_IP3R * m3 * n3 * h3 * (Ca_ER - Ca);
    const double J_pump = c.rate_SERCA * Ca * Ca / (c.Km_SERCA * c.Km_SERCA + Ca * Ca);
    const double J_leak = ratio * c.rate_L * (Ca_ER - Ca);
    const double alpha_h = c.k_IP3R * c.Kd_inh * (IP3 + c.Kd_IP3_1) / (IP3 + c.Kd_IP3_2);
    const double beta_h = c.k_IP3R * Ca;
    dCa = J_channel - J_pump + J_leak + noise;
    dIP3 = div_by(IP3_0 - IP3, tau_IP3, rcp_tau_IP3);
    dh = alpha_h * (1.0 - h) - beta_h * h;
}

__device__ __forceinline__ double exp_r(double x) { return exp(x); }
__device__ __forceinline__ float exp_r(float x) { return expf(x); }

// CUDA's double exp, kept out of line: inlined four times per RK4 step its expansion
// needs about 50 more registers than the rest of the step, which made the FP64 window
// kernel spill at every occupancy above 3 blocks per SM.  It is the same function, so
// the results are unchanged.
static __device__ __noinline__ double exp_outlined(double x) { return exp(x); }

// AdEx: src/astrosim_fused.cu:281-290 (operand order kept; the divisions by the
// constants C_m, tau_w and Delta_T are exact, see div_by).
__device__ __forceinline__ void neuron_rhs(const NeuronK& p, double V, double w, double g_ex, double g_in,
                                           double I_ext, double& dV, double& dw) {
    const double Vc = V < p.V_peak ? V : p.V_peak;
    const double arg = p.inv_Delta_T_pow2 != 0.0 ? (Vc - p.V_th) * p.inv_Delta_T_pow2
                                                 : div_by(Vc - p.V_th, p.Delta_T, p.rcp_Delta_T);
    const double I_spike = p.g_L * p.Delta_T * exp_outlined(arg);
    const double I_syn_ex = g_ex * (Vc - p.E_ex);
    const double I_syn_in = g_in * (Vc - p.E_in);
    dV = div_by(-p.g_L * (Vc - p.E_L) + I_spike - I_syn_ex - I_syn_in - w + p.I_e + I_ext, p.C_m, p.rcp_C_m);
    dw = div_by(p.a * (Vc - p.E_L) - w, p.tau_w, p.rcp_tau_w);
}

// The FP32 form of the same right-hand side: reciprocal multiplies and the
// hardware exponential (stage arithmetic only; V and w accumulate in double).
__device__ __forceinline__ void neuron_rhs(const NeuronK& p, float V, float w, float g_ex, float g_in, float I_ext,
                                           float& dV, float& dw) {
    const float Vc = V < p.f_V_peak ? V : p.f_V_peak;
#ifdef ASTROSIM_FP32_IEEE
    // the FP64 path's operations in float: divisions, not reciprocal multiplies
    const float DT = static_cast<float>(p.Delta_T);
    const float I_spike = p.f_g_L * DT * exp_fast((Vc - p.f_V_th) / DT);
    const float I_syn_ex = g_ex * (Vc - p.f_E_ex);
    const float I_syn_in = g_in * (Vc - p.f_E_in);
    dV = (-p.f_g_L * (Vc - p.f_E_L) + I_spike - I_syn_ex - I_syn_in - w + p.f_I_e + I_ext) / static_cast<float>(p.C_m);
    dw = (p.f_a * (Vc - p.f_E_L) - w) / static_cast<float>(p.tau_w);
#else
    const float I_spike = p.f_gL_DT * exp_fast((Vc - p.f_V_th) * p.f_inv_DT);
    const float I_syn_ex = g_ex * (Vc - p.f_E_ex);
    const float I_syn_in = g_in * (Vc - p.f_E_in);
    dV = (-p.f_g_L * (Vc - p.f_E_L) + I_spike - I_syn_ex - I_syn_in - w + p.f_I_e + I_ext) * p.f_inv_Cm;
    dw = (p.f_a * (Vc - p.f_E_L) - w) * p.f_inv_tauw;
#endif
}

#ifndef ASTROSIM_FP32_IEEE
// The conductance-dependent part of the FP32 form's refolded AdEx right-hand side:
// dV = A (Vc - E_L) + B - w / C_m + 2^(K1 (Vc - V_th) + K2) (see NeuronK).
// `iext_c` = C0 + I_ext / C_m.
struct AdexCoef {
    float A, B;
};
__device__ __forceinline__ AdexCoef adex_coef(const NeuronK& p, float g_ex, float g_in, float iext_c) {
    return AdexCoef{fmaf(-p.f_inv_Cm, g_ex + g_in, p.f_A0), fmaf(g_ex, p.f_Eex_c, fmaf(g_in, p.f_Ein_c, iext_c))};
}
// The FP32 form's AdEx right-hand side (src/astrosim_fused.cu:281-290 refolded): the
// same formula with the constants folded into two fused multiply-adds and the
// exponent, about half the operations of the term-by-term form.
__device__ __forceinline__ void adex_rhs_folded(const NeuronK& p, const AdexCoef& c, float V, float w, float& dV,
                                                float& dw) {
    const float Vc = fminf(V, p.f_V_peak);
    const float u = Vc - p.f_E_L;
    dV = fmaf(c.A, u, fmaf(-p.f_inv_Cm, w, c.B)) + ex2_ftz(fmaf(Vc - p.f_V_th, p.f_K1, p.f_K2));
    dw = fmaf(p.f_Wa, u, -p.f_inv_tauw * w);
}
#endif

// The FP32 form of the Li-Rinzel right-hand side (see astro_rhs).
__device__ __forceinline__ void astro_rhs_fast(const AstroK& c, float Ca_tot, float IP3_0, float tau_IP3, float inv_tau_IP3,
                                               float Ca, float IP3, float h, float noise, float& dCa, float& dIP3,
                                               float& dh) {
#ifdef ASTROSIM_FP32_IEEE
    // the FP64 formula's operations in float (the measurement build)
    const float Ca_ER = (Ca_tot - Ca) / static_cast<float>(c.ratio_ER_cyt);
    const float m_inf = div_fast(IP3, IP3 + c.f_Kd_IP3_1);
    const float n_inf = div_fast(Ca, Ca + c.f_Kd_act);
    const float m3 = m_inf * m_inf * m_inf;
    const float n3 = n_inf * n_inf * n_inf;
    const float h3 = h * h * h;
    const float J_channel =
        static_cast<float>(c.ratio_ER_cyt) * static_cast<float>(c.rate_IP3R) * m3 * n3 * h3 * (Ca_ER - Ca);
    const float J_pump = div_fast(c.f_rate_SERCA * Ca * Ca, c.f_Km2 + Ca * Ca);
    const float J_leak = c.f_ratio_rate_L * (Ca_ER - Ca);
    const float alpha_h = div_fast(c.f_k_Kd_inh * (IP3 + c.f_Kd_IP3_1), IP3 + c.f_Kd_IP3_2);
    const float beta_h = c.f_k_IP3R * Ca;
    dCa = J_channel - J_pump + J_leak + noise;
    dIP3 = (IP3_0 - IP3) / tau_IP3;
    dh = alpha_h * (1.0f - h) - beta_h * h;
    (void)inv_tau_IP3;
#else
    // Refolded (the same formula, fewer roundings and operations): with d = Ca_ER - Ca,
    // J_channel + J_leak = d (ratio rate_IP3R (m_inf n_inf)^3 h^3 + ratio rate_L),
    // m_inf n_inf = IP3 Ca / ((IP3 + Kd_IP3_1)(Ca + Kd_act)) with one reciprocal, and
    // J_pump = rate_SERCA - rate_SERCA Km^2 / (Km^2 + Ca^2).
    const float d = fmaf(-Ca, c.f_1p_inv_ratio, Ca_tot * c.f_inv_ratio);
    const float ip_k1 = IP3 + c.f_Kd_IP3_1;
    const float mn = (IP3 * Ca) * rcp_ftz(ip_k1 * (Ca + c.f_Kd_act));
    const float mn3 = mn * mn * mn;
    const float h3 = h * h * h;
    const float J_pump = fmaf(-c.f_rate_Km2, rcp_ftz(fmaf(Ca, Ca, c.f_Km2)), c.f_rate_SERCA);
    dCa = fmaf(d, fmaf(c.f_ratio_rate_IP3R * mn3, h3, c.f_ratio_rate_L), noise - J_pump);
    const float alpha_h = (c.f_k_Kd_inh * ip_k1) * rcp_ftz(IP3 + c.f_Kd_IP3_2);
    dIP3 = fmaf(-IP3, inv_tau_IP3, IP3_0 * inv_tau_IP3);
    dh = fmaf(-h, fmaf(c.f_k_IP3R, Ca, alpha_h), alpha_h);
    (void)tau_IP3;
#endif
}

#endif  // __CUDACC__ (the right-hand sides are device code)

// A run constant in the stage type: the double value, or its float copy.
template <typename R>
__host__ __device__ __forceinline__ R as_r(double d, float f);
template <>
__host__ __device__ __forceinline__ double as_r<double>(double d, float) { return d; }
template <>
__host__ __device__ __forceinline__ float as_r<float>(double, float f) { return f; }

#ifdef __CUDACC__
// Box-Muller in float from one stream (counters 0 and 1): the noise draws of the FP32 form.
__device__ __forceinline__ float normal_fast(u64 base) {
#ifdef ASTROSIM_FP32_IEEE
    // the FP64 path's 53-bit uniforms, rounded to float; its u1 <= 1e-300 clamp
    // (src/astrosim_fused.cu:146) becomes log(1e-300) for an all-zero draw
    const double d1 = rng_uniform_at(base, 0);
    const double d2 = rng_uniform_at(base, 1);
    const float l1 = d1 > 0.0 ? log_fast(static_cast<float>(d1)) : -690.775528f;
    return sqrt_ftz(-2.0f * l1) * cos_ftz(static_cast<float>(kTwoPi) * static_cast<float>(d2));
#else
    const u32 a = static_cast<u32>(rng_mix(base) >> 40);
    const u32 b = static_cast<u32>(rng_mix(base + kCounterMul) >> 40);
    const float u1 = (static_cast<float>(a) + 0.5f) * (1.0f / 16777216.0f);
    const float u2 = static_cast<float>(b) * (1.0f / 16777216.0f);
    return sqrt_ftz(-2.0f * log_fast(u1)) * cos_ftz(static_cast<float>(kTwoPi) * u2);
#endif
}

#endif  // __CUDACC__

}  // namespace astrosim
