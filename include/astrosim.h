/*
 * astrosim.h -- C ABI of the B200-native tripartite neuron-astrocyte simulator.
 *
 * The reference program (src/astrosim_fused.cu) has no library interface: it is
 * one `main` (src/astrosim_fused.cu:791) that parses flags, builds a network on
 * the host, steps it with two kernels per time step and prints a summary.  This
 * header is the library boundary that replaces that monolith.  Each entry point
 * names the part of the reference it stands in for.  All entry points:
 *   - take plain pointers and sizes (no C++ or torch types),
 *   - return an int status (ASTROSIM_OK == 0) and never abort the process,
 *   - leave a human-readable message for the calling thread in
 *     astrosim_last_error() when they fail.
 * One handle owns one simulated network (or one ensemble) and all of its device
 * memory; a handle must be used from one host thread at a time.
 */
#ifndef ASTROSIM_H
#define ASTROSIM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ASTROSIM_ABI_VERSION 1

/* Status codes. */
enum {
    ASTROSIM_OK = 0,
    ASTROSIM_ERR_INVALID_ARG = 1,   /* bad pointer, size or configuration value */
    ASTROSIM_ERR_CUDA = 2,          /* a CUDA runtime call failed */
    ASTROSIM_ERR_OUT_OF_MEMORY = 3, /* device allocation failed */
    ASTROSIM_ERR_UNSUPPORTED = 4,   /* configuration outside what the kernels implement */
    ASTROSIM_ERR_NO_DEVICE = 5,     /* no CUDA device visible (reference: src/astrosim_fused.cu:906-912) */
    ASTROSIM_ERR_TIMEOUT = 6,       /* a bounded wait gave up: device-side, or on the other ranks of a
                                       sharded network (a rank that died or left) */
    ASTROSIM_ERR_STATE = 7,         /* call not valid in the handle's current state */
    ASTROSIM_ERR_IO = 8,            /* a host file could not be written */
    ASTROSIM_ERR_PEER = 9           /* another rank of a sharded network failed (reported by the communicator) */
};

enum {
    ASTROSIM_PRECISION_FP64 = 0, /* every state variable and every RK4 stage in double (reference default) */
    ASTROSIM_PRECISION_FP32 = 1  /* RK4 stages in float; V, w, Ca, IP3 accumulators and the
                                    threshold/reset test in double */
};

/*
 * Run configuration.  Field defaults are the reference's flag defaults
 * (src/astrosim_fused.cu:792-805) and its compiled-in biology
 * (src/astrosim_fused.cu:742-781).  Always initialise with
 * astrosim_config_default() and then change fields.
 */
typedef struct astrosim_config {
    uint32_t struct_size;   /* sizeof(astrosim_config); set by astrosim_config_default */
    uint32_t n_total;       /* --n: total neurons; split by the fixed-in-degree law (src/astrosim_fused.cu:606-614) */
    uint64_t seed;          /* --seed */
    double dt;              /* --dt, ms */
    int32_t substeps;       /* --substeps: RK4 substeps per time step */
    int32_t block;          /* --block: CUDA block size of the cell kernels (a multiple of 32 in [32, 1024];
                               the reference's default is 128).  0 (the default here) = the autotuner
                               times block sizes 64/128/256 with three occupancy targets each on
                               the first windows and keeps the fastest; a given size is used as is
                               (64/128/256 still tune their occupancy target) */
    double pre_ms;          /* --pre-ms: discarded transient */
    double sim_ms;          /* --sim-ms: recorded window */
    double w_n2a;           /* --w-n2a: neuron->astrocyte weight; NaN keeps the default 0.2 */
    double w_a2n;           /* --w-a2n: astrocyte->neuron (SIC) weight; NaN keeps the default 1.0 */
    int32_t stp_enabled;    /* 1 = Tsodyks-Markram STP on; --no-stp sets 0 */
    int32_t precision;      /* ASTROSIM_PRECISION_FP64 or ASTROSIM_PRECISION_FP32 */
    double neuron_drive_scale; /* multiplies the excitatory and inhibitory Poisson background rates
                                  (2700 Hz / 2500 Hz); 1.0 reproduces the reference */
    int32_t device;         /* CUDA device ordinal */
    int32_t raster_steps;   /* record the full spike raster of the first raster_steps steps (0 = off) */
    int32_t reserved[8];    /* must be zero */
} astrosim_config;

/* Result of a run, mirroring the reference's printed summary (src/astrosim_fused.cu:1103-1141). */
typedef struct astrosim_summary_s {
    uint32_t n_total, n_exc, n_inh, n_astro;
    double p_primary;
    uint64_t n_exc_edges, n_inh_edges, n_e2a_edges, n_sic_edges;
    int64_t pre_steps, sim_steps, total_steps, steps_done;
    uint64_t spikes_total;      /* every spike since step 0 */
    uint64_t spikes_measured;   /* spikes in the recorded window ("spikes (recorded win)") */
    double mean_rate_hz;        /* spikes_measured / (n_neurons * sim_ms * 1e-3) */
    double mean_ca;             /* mean astrocyte calcium at the last completed step, uM */
    uint32_t active_astro;      /* astrocytes with (Ca - SIC_th) * 1000 > 1 at the last step */
    uint32_t engaged_astro;     /* astrocytes whose SIC factor was > 0 at any recorded step */
    double sic_th;              /* SIC threshold used by the two counts above */
    double build_seconds;       /* device connectivity + parameter build time */
    double run_seconds;         /* wall time of the stepping since the first astrosim_step */
} astrosim_summary_t;

typedef struct astrosim_handle astrosim_handle;

/* Fills *cfg with the reference defaults. */
void astrosim_config_default(astrosim_config* cfg);

/* Message describing the calling thread's most recent failure ("" if none). */
const char* astrosim_last_error(void);

/* Library ABI version (ASTROSIM_ABI_VERSION). */
int astrosim_abi_version(void);

/*
 * Builds the network on the device and allocates its state.
 * Replaces src/astrosim_fused.cu:846-1018: the scaling law (606-614), the host
 * connectivity builder (631-735) and CSR inversion (304-315), the per-cell
 * parameter draws (917-933), the initial state and the device allocations.
 * Here every one of those steps runs on the GPU; the connectivity and the
 * per-cell parameters are bit-identical to the reference's host code for the
 * same (n_total, seed).
 */
int astrosim_create(const astrosim_config* cfg, astrosim_handle** out);

/*
 * astrosim_create with non-default biology.  `biology_json` is one flat JSON
 * object mapping parameter names to values, e.g.
 *     {"exc_poiss_rate": 3000, "stp_U": 0.4, "independent_noise": true}
 * The names are the reference's biology constants (its Biology struct,
 * src/astrosim_fused.cu:742-781; astrosim_biology_names lists them); reals and
 * integers take numbers, flags take true / false.  The reference compiles these
 * constants in; upstream loads them from a JSON config (not part of the
 * reference).  cfg's own fields apply on top: w_n2a / w_a2n when not NaN,
 * stp_enabled = 0, neuron_drive_scale (multiplies the neuron Poisson rates).
 * NULL or "" keeps every default.  Unknown or repeated names, malformed text and
 * values the model cannot run with (a non-positive time constant, capacitance or
 * delay, sic_interval < 1, ...) return ASTROSIM_ERR_INVALID_ARG with the name in
 * astrosim_last_error().  Delays that are not all equal, or not 2-16 steps, run on
 * the per-step engine instead of the windowed one.
 */
int astrosim_create_with_biology(const astrosim_config* cfg, const char* biology_json, astrosim_handle** out);

/* Comma-separated biology parameter names into buf (cap bytes, NUL included);
   *needed (if not NULL) receives the size the list needs.  buf = NULL only sizes. */
int astrosim_biology_names(char* buf, size_t cap, size_t* needed);

/* The value of parameter `name` after applying biology_json (NULL = defaults). */
int astrosim_biology_value(const char* biology_json, const char* name, double* value);

/*
 * Advances the network by n_steps time steps, asynchronously on the handle's
 * stream.  Replaces the body of the reference time loop
 * (src/astrosim_fused.cu:1042-1102): the per-step scalars, the astrocyte and
 * neuron kernels, and the reset of the "engaged" flags when the pre-run ends.
 * Steps past the configured pre+sim length are allowed.
 */
int astrosim_step(astrosim_handle* h, int64_t n_steps);

/* Waits for the handle's stream and fills *out.  Replaces src/astrosim_fused.cu:1103-1141. */
int astrosim_summary(astrosim_handle* h, astrosim_summary_t* out);

/* Frees every device allocation the handle owns.  Accepts NULL. */
int astrosim_destroy(astrosim_handle* h);

/*
 * Spike counts per time step for steps [first_step, first_step + n) (each
 * step must already be done).  The reference only keeps a running total
 * (the atomicAdd at src/astrosim_fused.cu:584) and reads it at its windowed-rate
 * checkpoints (src/astrosim_fused.cu:1081-1095); per-step counts let a caller
 * form those windows at any granularity.
 */
int astrosim_spike_counts(astrosim_handle* h, int64_t first_step, int64_t n, uint32_t* counts);

/*
 * Spike raster of the first cfg.raster_steps steps as a bitmask: bit (j % 32)
 * of word [step * ceil(n_neurons / 32) + j / 32] is set when neuron j spiked at
 * that step.  `words` is the capacity of `bits` in 32-bit words.
 */
int astrosim_raster(astrosim_handle* h, uint32_t* bits, size_t words);

/* Which state array astrosim_get_state copies. */
enum {
    ASTROSIM_STATE_CA = 0,        /* astrocyte calcium, n_astro doubles */
    ASTROSIM_STATE_IP3 = 1,       /* n_astro doubles */
    ASTROSIM_STATE_H = 2,         /* IP3R gating h, n_astro doubles */
    ASTROSIM_STATE_V = 3,         /* membrane potential, n_neurons doubles */
    ASTROSIM_STATE_W = 4,         /* adaptation current, n_neurons doubles */
    ASTROSIM_STATE_G_EX = 5,      /* n_neurons doubles */
    ASTROSIM_STATE_DG_EX = 6,
    ASTROSIM_STATE_G_IN = 7,
    ASTROSIM_STATE_DG_IN = 8,
    ASTROSIM_STATE_I_SIC = 9,     /* held SIC current */
    ASTROSIM_STATE_STP_X = 10,
    ASTROSIM_STATE_STP_U = 11,
    ASTROSIM_STATE_STP_T_LAST = 12,
    ASTROSIM_STATE_CA_TOT = 13,   /* per-cell parameters (src/astrosim_fused.cu:917-933) */
    ASTROSIM_STATE_IP3_0 = 14,
    ASTROSIM_STATE_TAU_IP3 = 15,
    ASTROSIM_STATE_DELTA_IP3 = 16,
    ASTROSIM_STATE_V_RESET = 17,
    ASTROSIM_STATE_B = 18,
    ASTROSIM_STATE_SIC_FACTOR = 19, /* astrocyte SIC factor written at the last completed step */
    ASTROSIM_STATE_COUNT = 20
};

/* Copies one state array to host memory as doubles (count elements). */
int astrosim_get_state(astrosim_handle* h, int which, double* dst, size_t count);

/* Which connectivity CSR astrosim_get_csr copies (all keyed by TARGET, as in src/astrosim_fused.cu:296-315). */
enum {
    ASTROSIM_CSR_EXC = 0, /* per neuron: excitatory primary sources */
    ASTROSIM_CSR_INH = 1, /* per neuron: inhibitory primary sources, local inhibitory indices */
    ASTROSIM_CSR_SIC = 2, /* per neuron: astrocyte (SIC) sources */
    ASTROSIM_CSR_E2A = 3  /* per astrocyte: excitatory third-factor sources */
};

/*
 * Copies one CSR to host memory.  row_start receives n_targets + 1 entries,
 * src receives n_edges entries; either may be NULL to query the sizes only.
 */
int astrosim_get_csr(astrosim_handle* h, int which, uint32_t* row_start, size_t row_cap,
                     uint32_t* src, size_t src_cap, uint32_t* n_targets, uint64_t* n_edges);

/*
 * Writes the connectivity as CSV in the reference's --dump-edges format
 * (src/astrosim_fused.cu:873-902): header "type,source,target", types
 * exc_primary / inh_primary / n2a / a2n, inhibitory sources offset by n_exc,
 * astrocyte ids prefixed "A".
 */
int astrosim_dump_edges(astrosim_handle* h, const char* path);

/* Device time of the most recent astrosim_step call's kernels, ms (CUDA events, synchronises). */
int astrosim_last_step_ms(astrosim_handle* h, double* ms);

/*
 * Calcium recording into device memory (the reference records nothing beyond its
 * printed summary; upstream recording is out of its scope, README.md:120-123).
 * From the next step on, after every step t with (t + 1) % every_steps == 0, the
 * kernels store the calcium of astrocytes [first_astro, first_astro + n_astro) as
 * one sample (n_astro doubles) in a device buffer of max_samples samples; samples
 * past the buffer are dropped.  Starting a recording replaces the previous one and
 * its buffer.  Recording adds no launches: the astrocyte update writes the sample.
 */
int astrosim_record_calcium(astrosim_handle* h, int64_t every_steps, uint32_t first_astro, uint32_t n_astro,
                            int64_t max_samples);

/* Samples recorded so far (at most max_samples) and the step after which sample 0 was taken. */
int astrosim_calcium_samples(astrosim_handle* h, int64_t* n_samples, int64_t* first_step);

/*
 * Copies samples [first, first + n) to dst (n * n_astro doubles, sample-major).
 * wait = 1 returns once the copy is done.  wait = 0 enqueues the copy on the
 * handle's stream and returns at once; the data is in dst after astrosim_sync
 * (or any call that synchronises the handle).  Pinned host memory lets the copy
 * overlap host work.
 */
int astrosim_copy_calcium(astrosim_handle* h, int64_t first, int64_t n, double* dst, int wait);

/* Waits for everything enqueued on the handle's stream. */
int astrosim_sync(astrosim_handle* h);

/*
 * Name and compute capability of a CUDA device (the reference prints them after
 * its device check, src/astrosim_fused.cu:904-914).  Returns ASTROSIM_ERR_NO_DEVICE
 * when no device is visible.
 */
int astrosim_device_info(int device, char* name, size_t name_cap, int* major, int* minor);

/* ------------------------------------------------------------------ batched ensemble
 * Many independent networks (each described by its own astrosim_config: size,
 * seed, drive scale, weights) stepped together: one launch per 1 ms window covers
 * every cell of every network, and the window sequence is replayed from a CUDA
 * graph.  The reference has no batched form; it runs one network per process
 * (src/astrosim_fused.cu:791).  Every network's results are bit-identical to
 * running it alone through astrosim_create/astrosim_step.  All networks must share
 * dt, substeps, precision and device.
 */
typedef struct astrosim_ensemble astrosim_ensemble;

/* Builds every network (concurrently) and its state. */
int astrosim_ensemble_create(const astrosim_config* cfgs, uint32_t n_networks, astrosim_ensemble** out);

/* Same, with biology overrides per network (biology_json[i] as in astrosim_create_with_biology;
   the array or any entry may be NULL).  All networks must still share one window length:
   equal delays d_e = d_i = d_a2n. */
int astrosim_ensemble_create_with_biology(const astrosim_config* cfgs, uint32_t n_networks,
                                          const char* const* biology_json, astrosim_ensemble** out);

/* Advances every network by n_steps (a whole number of windows, 1 ms each); a
   network stops at its own pre_ms + sim_ms. */
int astrosim_ensemble_step(astrosim_ensemble* e, int64_t n_steps);

/* Summary of network `index`, as astrosim_summary. */
int astrosim_ensemble_summary(astrosim_ensemble* e, uint32_t index, astrosim_summary_t* out);

/* State array of network `index`, as astrosim_get_state. */
int astrosim_ensemble_get_state(astrosim_ensemble* e, uint32_t index, int which, double* dst, size_t count);

/* Spike counts of network `index`, as astrosim_spike_counts. */
int astrosim_ensemble_spike_counts(astrosim_ensemble* e, uint32_t index, int64_t first_step, int64_t n,
                                   uint32_t* counts);

/* Device time of the last astrosim_ensemble_step, ms. */
int astrosim_ensemble_last_step_ms(astrosim_ensemble* e, double* ms);

/* Wall time of astrosim_ensemble_create (all builds), seconds. */
int astrosim_ensemble_build_seconds(astrosim_ensemble* e, double* seconds);

/* *shared = 1 when every network of the batch has the same constants apart from its
 * seed, sizes, drive rates and astrocyte-to-neuron weight (the window launch then
 * passes the shared constants once as kernel parameters), 0 when the networks differ
 * further (each block then stages its own network's constants).  Results do not
 * depend on it.  No counterpart in the reference, which runs one network per process. */
int astrosim_ensemble_shared_constants(astrosim_ensemble* e, int* shared);

int astrosim_ensemble_destroy(astrosim_ensemble* e);

/* ------------------------------------------------------------------ serving
 * A request loop with continuous batching (no counterpart in the reference, which
 * runs one network per process).  Requests queue FIFO and are admitted when their
 * estimated device footprint fits the HBM budget; their networks are built on
 * builder threads (own CUDA streams, overlapping the running batch), join the
 * running ensemble between windows, and leave it when they reach their last step.
 * Each result is bit-identical to running the same configuration alone.
 */
typedef struct astrosim_server astrosim_server;

typedef struct astrosim_request_result {
    astrosim_summary_t summary;
    double latency_s;  /* submit -> result ready */
    double queue_s;    /* submit -> admitted (its footprint fit the budget) */
    double build_s;    /* device build of its network */
    double run_s;      /* joined the batch -> last step done */
} astrosim_request_result;

typedef struct astrosim_server_stats {
    uint64_t submitted, done, failed, pending, building, running;
    uint64_t bytes_in_use, budget_bytes;
    double uptime_s;
} astrosim_server_stats;

/* hbm_budget_bytes = 0 uses 85 % of the device's free memory.  Requests must use
   dt = 0.1 ms and the server's precision. */
int astrosim_server_create(int device, int precision, uint64_t hbm_budget_bytes, int builder_threads,
                           astrosim_server** out);
int astrosim_server_submit(astrosim_server* s, const astrosim_config* cfg, uint64_t* request_id);
/* Same, with biology overrides (checked here; the text is copied). */
int astrosim_server_submit_with_biology(astrosim_server* s, const astrosim_config* cfg, const char* biology_json,
                                        uint64_t* request_id);
/* Admits what fits, joins built networks, advances the batch by `windows` windows
   (1 ms each) and retires finished requests. */
int astrosim_server_pump(astrosim_server* s, int64_t windows);
/* *done = 0 while the request is still queued or running. */
int astrosim_server_result(astrosim_server* s, uint64_t request_id, astrosim_request_result* out, int* done);
int astrosim_server_get_stats(astrosim_server* s, astrosim_server_stats* out);
int astrosim_server_destroy(astrosim_server* s);

/*
 * Astrocyte summary totals over caller-provided device arrays (the layout the
 * library reduces internally for astrosim_summary).
 */
typedef struct astrosim_astro_totals {
    double sum_ca;     /* sum of calcium over all astrocytes */
    double mean_ca;    /* sum_ca / max(1, n_astro) */
    uint32_t active;   /* astrocytes with (Ca - sic_th) * 1000 > 1 */
    uint32_t engaged;  /* astrocytes whose engaged flag is non-zero */
} astrosim_astro_totals;

/* Largest n_astro astrosim_astro_totals_noalloc accepts (4096 partial sums of 2048 astrocytes). */
#define ASTROSIM_NOALLOC_MAX_ASTRO 8388608u

/*
 * The astrocyte summary reduction that allocates nothing.
 *
 * No counterpart in the reference: it is an extra entry point of this library.
 * It runs the same two-pass reduction astrosim_summary uses, on device arrays the
 * caller owns: `ca` (n_astro doubles), `engaged` (n_astro bytes, non-zero =
 * engaged) and `out` (one astrosim_astro_totals in device memory), enqueued on
 * `stream` (a cudaStream_t; NULL = the legacy default stream) without waiting.
 *
 * It is for callers that cannot allocate device memory at the point where they
 * need the totals: applications that hand all device memory to their own pool or
 * run under a fixed memory budget, and loops that must not enter the CUDA
 * allocator because cudaMalloc/cudaFree may synchronize the device or stall on
 * the driver.  Its scratch (the per-block partial sums) is a static array in the
 * library's device image, 64 KB on every GPU that loads the library, held until
 * the process exits; that bounds n_astro to ASTROSIM_NOALLOC_MAX_ASTRO, and larger
 * inputs return ASTROSIM_ERR_INVALID_ARG.
 *
 * The first call on a device (with that device current) looks up the scratch
 * address once per CUDA context: again after cudaDeviceReset or any other change
 * of the device's context, which can move the device image.  Make the first call
 * in each context before any stream capture.  All calls share
 * the one scratch array: calls that may overlap on the GPU (different streams,
 * or different host threads) race and must be serialised by the caller.  Each
 * call writes every partial it reads, so nothing left by an earlier call leaks
 * into a result.
 */
int astrosim_astro_totals_noalloc(const double* ca, const unsigned char* engaged, uint32_t n_astro, double sic_th,
                                  astrosim_astro_totals* out, void* stream);

/* ------------------------------------------------------------------ one network on several GPUs
 * A network split across `world` ranks (the reference
 * runs on one GPU).  Every rank owns contiguous ranges of neurons and astrocytes
 * (128-cell blocks, balanced) and builds and keeps only the connectivity rows of
 * its own cells (about 1 / world of the connectivity; the build walks the whole
 * deterministic stream but emits only those rows); per 1 ms window
 * it advances its own cells, then the ranks all-gather the window's spikes and the
 * SIC factors of their active astrocytes, and each rank delivers every spike into
 * its own cells.  Results (spike counts, raster, every state array, the summary)
 * are bit-identical to the single-GPU run.  Stepping is in whole windows.  The
 * windowed engine is required (equal delays of 2-16 steps).
 */

/* Owned ranges of rank `rank` of `world` for n_total (host only, no device). */
int astrosim_shard_plan(uint32_t n_total, int rank, int world, uint32_t* neuron_lo, uint32_t* neuron_hi,
                        uint32_t* astro_lo, uint32_t* astro_hi);

/* One rank per process over NCCL (libnccl.so.2, loaded when first used).
   astrosim_shard_create builds this rank's network without communicating; cfg (and
   biology_json) must be identical on every rank except cfg.device, the rank's GPU.
   Once every rank has created its part (the caller checks that, e.g. with
   torch.distributed, so that no rank waits for one that failed), rank 0 makes the
   128-byte id with astrosim_shard_unique_id, the caller hands the same bytes to
   every rank, and each calls astrosim_shard_connect (collective).  step, summary
   and get_state are collective: every rank calls them in the same order. */
typedef struct astrosim_shard astrosim_shard;
int astrosim_shard_unique_id(unsigned char id[128]);
int astrosim_shard_create(const astrosim_config* cfg, const char* biology_json, int rank, int world,
                          astrosim_shard** out);
int astrosim_shard_connect(astrosim_shard* s, const unsigned char id[128]);
int astrosim_shard_step(astrosim_shard* s, int64_t n_steps);
int astrosim_shard_summary(astrosim_shard* s, astrosim_summary_t* out);
int astrosim_shard_get_state(astrosim_shard* s, int which, double* dst, size_t count);
int astrosim_shard_spike_counts(astrosim_shard* s, int64_t first_step, int64_t n, uint32_t* counts);
/* Device time of this rank's last astrosim_shard_step, ms (take the max over ranks). */
int astrosim_shard_last_step_ms(astrosim_shard* s, double* ms);
/* Deadline, in seconds, of every wait on the other ranks (connect, each window's
   exchange, the gathers of summary and get_state); default ASTROSIM_SHARD_TIMEOUT_S
   from the environment, else 120.  The communicator is non-blocking: when a wait
   passes its deadline (a rank died or left between windows) the call aborts the
   communicator and returns ASTROSIM_ERR_TIMEOUT, and when the communicator reports
   a failed peer it returns ASTROSIM_ERR_PEER.  Either way this rank stays unusable
   (ASTROSIM_ERR_STATE) until destroyed.  The reference has no counterpart: it runs
   on one GPU and aborts the process on any CUDA error (src/astrosim_fused.cu:109-117). */
int astrosim_shard_set_timeout(astrosim_shard* s, double seconds);
int astrosim_shard_destroy(astrosim_shard* s);

/* The deadline logic of the waits above, run on a stand-in communicator with no
   device and no NCCL.  Scenario 0: four windows whose exchanges complete;
   1: the first window's exchange never completes; 2: the communicator reports a
   failed peer during the first exchange; 3: windows 0 and 1 complete, then a rank
   has left and window 2's exchange never completes.  Returns the status the wait
   returned and reports the windows that completed, whether the stand-in was
   aborted, and the seconds spent.  No counterpart in the reference. */
int astrosim_shard_selftest_wait(int scenario, double timeout_s, int* windows_done, int* aborted, double* waited_s);

/* All ranks in this process: rank r runs on devices[r] (NULL: every rank on
   cfg.device; ranks that share a device run one after another).  Same results. */
typedef struct astrosim_shard_group astrosim_shard_group;
int astrosim_shard_group_create(const astrosim_config* cfg, const char* biology_json, int world, const int* devices,
                                astrosim_shard_group** out);
int astrosim_shard_group_step(astrosim_shard_group* g, int64_t n_steps);
int astrosim_shard_group_summary(astrosim_shard_group* g, astrosim_summary_t* out);
int astrosim_shard_group_get_state(astrosim_shard_group* g, int which, double* dst, size_t count);
int astrosim_shard_group_spike_counts(astrosim_shard_group* g, int64_t first_step, int64_t n, uint32_t* counts);
/* The connectivity rank `rank` keeps: CSR `which` (ASTROSIM_CSR_*) restricted to the
   rank's own targets, row r being cell *first_row + r (neurons for exc/inh/sic,
   astrocytes for e2a).  Each rank keeps only these rows, about 1 / world of the
   network; every kept row equals the whole network's row.  Sizes as astrosim_get_csr. */
int astrosim_shard_group_get_csr(astrosim_shard_group* g, int rank, int which, uint32_t* row_start, size_t row_cap,
                                 uint32_t* src, size_t src_cap, uint32_t* first_row, uint32_t* n_rows,
                                 uint64_t* n_edges);
int astrosim_shard_group_destroy(astrosim_shard_group* g);

/*
 * Device arithmetic self-check: the FP64 right-hand sides divide by the model's
 * constants (C_m, tau_w, Delta_T, ratio_ER_cyt and each astrocyte's tau_IP3) with a
 * reciprocal and two FMA corrections instead of a hardware division sequence.
 * This runs that division and IEEE x / y side by side on `device` for each of the
 * `n_divisors` divisors over `samples` random dividends and `samples` dividends
 * whose quotients lie next to a rounding midpoint, and writes the number of
 * quotients that differ in any bit to *mismatches (0 on a correct device).
 * Divisors must be finite, non-zero and have |x / y| in the normal range for the
 * sampled x (|x| in [2^-40, 2^40]).  No counterpart in the reference.
 */
int astrosim_selfcheck_division(int device, const double* divisors, size_t n_divisors, uint64_t samples,
                                uint64_t seed, uint64_t* mismatches);

#ifdef __cplusplus
}
#endif

#endif /* ASTROSIM_H */
