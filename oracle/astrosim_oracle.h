/*
 * astrosim_oracle.h -- TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.
 *
 * C interface of the FP64 CPU oracle: a plain restatement of the reference
 * program's algorithm (src/astrosim_fused.cu) used only by tests/, by the
 * smoke check and by bench.py's CPU-baseline leg, always as the checker.
 * The shipped library never links, loads or calls it.
 */
#ifndef ASTROSIM_ORACLE_H
#define ASTROSIM_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#include "../include/astrosim.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_sim oracle_sim;

/* Raw counter RNG draws (src/astrosim_fused.cu:127-175). */
uint64_t oracle_rng_bits(uint64_t seed, uint64_t stream, uint64_t counter);
double oracle_rng_uniform(uint64_t seed, uint64_t stream, uint64_t counter);
double oracle_rng_normal(uint64_t seed, uint64_t stream);
int oracle_rng_poisson(uint64_t seed, uint64_t stream, double lambda);

/*
 * Sequential stream (src/astrosim_fused.cu:180-208): writes n successive
 * normal() draws of the stream (seed, stream) to out.
 */
void oracle_seq_normals(uint64_t seed, uint64_t stream, size_t n, double* out);

/*
 * Builds the network and state for cfg on the host, exactly as the reference's
 * host code does (src/astrosim_fused.cu:846-1018).  Returns NULL on bad input.
 * n_threads <= 0 uses every OpenMP thread.
 */
oracle_sim* oracle_create(const astrosim_config* cfg, int n_threads);

/*
 * Same, but with externally supplied connectivity (four target-keyed CSRs in the
 * layout astrosim_get_csr returns) instead of rebuilding it.  Used to time the
 * stepping at sizes where the serial builder would take minutes.
 */
oracle_sim* oracle_create_with_csr(const astrosim_config* cfg, int n_threads,
                                   const uint32_t* exc_rs, const uint32_t* exc_src,
                                   const uint32_t* inh_rs, const uint32_t* inh_src,
                                   const uint32_t* sic_rs, const uint32_t* sic_src,
                                   const uint32_t* e2a_rs, const uint32_t* e2a_src);

/*
 * oracle_create with biology constants overridden by name (the reference's
 * Biology fields, src/astrosim_fused.cu:742-781); cfg's fields apply after them,
 * as in the reference's main.  Returns NULL for an unknown name.
 */
oracle_sim* oracle_create_with_biology(const astrosim_config* cfg, int n_threads, const char* const* names,
                                       const double* values, size_t n);

void oracle_destroy(oracle_sim* s);

/* Advances n_steps time steps (src/astrosim_fused.cu:1042-1102). */
void oracle_step(oracle_sim* s, int64_t n_steps);

void oracle_summary(oracle_sim* s, astrosim_summary_t* out);

/* Copies one ASTROSIM_STATE_* array; returns the element count, or -1. */
int64_t oracle_get_state(oracle_sim* s, int which, double* dst, size_t cap);

/* CSR sizes / copies (ASTROSIM_CSR_*). row_start/src may be NULL to query sizes. */
int oracle_get_csr(oracle_sim* s, int which, uint32_t* row_start, uint32_t* src,
                   uint32_t* n_targets, uint64_t* n_edges);

/* Spike counts per step for steps [first, first + n). */
int oracle_spike_counts(oracle_sim* s, int64_t first, int64_t n, uint32_t* counts);

/* Raster bitmask in the astrosim_raster layout for the first cfg.raster_steps steps. */
int oracle_raster(oracle_sim* s, uint32_t* bits, size_t words);

/* Seconds spent in oracle_create's connectivity build. */
double oracle_build_seconds(oracle_sim* s);

/*
 * Sensitivity probe: from now on, the AdEx exponential (src/astrosim_fused.cu:286)
 * returns a result one ulp away from the host C library's for a fraction `rate` of
 * its arguments (chosen by a hash of the argument, so deterministic), standing in
 * for a second correct math library that disagrees in the last bit.  0 turns it off.
 */
void oracle_set_exp_perturbation(oracle_sim* s, double rate);

/*
 * Sensitivity probe: from now on, evaluate the AdEx right-hand side and the
 * neuron's RK4 stage arguments and update with fused multiply-adds (each product
 * fused into the sum that consumes it, as a GPU compiler contracts them), a second
 * correct rounding of the same formulas.  0 restores separate roundings.
 */
void oracle_set_contraction(oracle_sim* s, int on);

#ifdef __cplusplus
}
#endif

#endif
