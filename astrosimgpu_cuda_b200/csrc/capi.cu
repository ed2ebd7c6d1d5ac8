// capi.cu -- the extern "C" boundary declared in include/astrosim.h.
// Every entry point converts library status into an int code and a per-thread
// message; none of them aborts or throws across the boundary.

#include <cmath>
#include <cstring>
#include <exception>
#include <new>
#include <string>

#include <mutex>

#include <cuda.h>

#include "../../include/astrosim.h"
#include "biology.cuh"
#include "ensemble.cuh"
#include "shard.cuh"
#include "reduce.cuh"
#include "server.cuh"
#include "sim.cuh"

struct astrosim_handle {
    astrosim::Simulation sim;
};

struct astrosim_ensemble {
    astrosim::Ensemble ens;
};

struct astrosim_server {
    astrosim::Server srv;
};

namespace {

thread_local std::string g_last_error;

int report(const astrosim::Status& s) {
    g_last_error = s.ok() ? std::string() : s.msg;
    return s.code;
}

int fail(int code, const char* msg) {
    g_last_error = msg;
    return code;
}

template <typename F>
int guarded(F&& f) {
    try {
        return report(f());
    } catch (const std::bad_alloc&) {
        return fail(ASTROSIM_ERR_OUT_OF_MEMORY, "host allocation failed");
    } catch (const std::exception& e) {
        return fail(ASTROSIM_ERR_CUDA, e.what());
    } catch (...) {
        return fail(ASTROSIM_ERR_CUDA, "unknown exception");
    }
}

}  // namespace

extern "C" {

void astrosim_config_default(astrosim_config* cfg) {
    if (!cfg) return;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->struct_size = sizeof(astrosim_config);
    cfg->n_total = 1000;      // src/astrosim_fused.cu:792-805
    cfg->seed = 1;
    cfg->dt = 0.1;
    cfg->substeps = 1;
    cfg->block = 0;           // the reference launches 128-thread blocks; 0 = autotuned
    cfg->pre_ms = 1000.0;
    cfg->sim_ms = 5000.0;
    cfg->w_n2a = std::nan("");
    cfg->w_a2n = std::nan("");
    cfg->stp_enabled = 1;
    cfg->precision = ASTROSIM_PRECISION_FP64;
    cfg->neuron_drive_scale = 1.0;
    cfg->device = 0;
    cfg->raster_steps = 0;
}

const char* astrosim_last_error(void) { return g_last_error.c_str(); }

int astrosim_abi_version(void) { return ASTROSIM_ABI_VERSION; }

int astrosim_create(const astrosim_config* cfg, astrosim_handle** out) {
    return astrosim_create_with_biology(cfg, nullptr, out);
}

int astrosim_create_with_biology(const astrosim_config* cfg, const char* biology_json, astrosim_handle** out) {
    if (!cfg || !out) return fail(ASTROSIM_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    if (cfg->struct_size != sizeof(astrosim_config))
        return fail(ASTROSIM_ERR_INVALID_ARG, "astrosim_config.struct_size mismatch (use astrosim_config_default)");
    for (int r : cfg->reserved)
        if (r != 0) return fail(ASTROSIM_ERR_INVALID_ARG, "astrosim_config.reserved must be zero");
    astrosim_handle* h = nullptr;
    try {
        h = new astrosim_handle();
    } catch (...) {
        return fail(ASTROSIM_ERR_OUT_OF_MEMORY, "host allocation failed");
    }
    const int rc = guarded([&] { return h->sim.create(*cfg, biology_json); });
    if (rc != ASTROSIM_OK) {
        const std::string msg = g_last_error;
        delete h;
        g_last_error = msg;
        return rc;
    }
    *out = h;
    return ASTROSIM_OK;
}

int astrosim_step(astrosim_handle* h, int64_t n_steps) {
    if (!h) return fail(ASTROSIM_ERR_INVALID_ARG, "null handle");
    return guarded([&] { return h->sim.step(n_steps); });
}

int astrosim_summary(astrosim_handle* h, astrosim_summary_t* out) {
    if (!h || !out) return fail(ASTROSIM_ERR_INVALID_ARG, "null argument");
    return guarded([&] { return h->sim.summary(*out); });
}

int astrosim_destroy(astrosim_handle* h) {
    delete h;
    g_last_error.clear();
    return ASTROSIM_OK;
}

int astrosim_spike_counts(astrosim_handle* h, int64_t first_step, int64_t n, uint32_t* counts) {
    if (!h) return fail(ASTROSIM_ERR_INVALID_ARG, "null handle");
    return guarded([&] { return h->sim.spike_counts(first_step, n, counts); });
}

int astrosim_raster(astrosim_handle* h, uint32_t* bits, size_t words) {
    if (!h) return fail(ASTROSIM_ERR_INVALID_ARG, "null handle");
    return guarded([&] { return h->sim.raster(bits, words); });
}

int astrosim_get_state(astrosim_handle* h, int which, double* dst, size_t count) {
    if (!h) return fail(ASTROSIM_ERR_INVALID_ARG, "null handle");
    return guarded([&] { return h->sim.get_state(which, dst, count); });
}

int astrosim_get_csr(astrosim_handle* h, int which, uint32_t* row_start, size_t row_cap, uint32_t* src,
                     size_t src_cap, uint32_t* n_targets, uint64_t* n_edges) {
    if (!h) return fail(ASTROSIM_ERR_INVALID_ARG, "null handle");
    return guarded([&] {
        astrosim::u64 ne = 0;
        astrosim::Status s = h->sim.get_csr(which, row_start, row_cap, src, src_cap, n_targets, &ne);
        if (n_edges) *n_edges = ne;
        return s;
    });
}

int astrosim_dump_edges(astrosim_handle* h, const char* path) {
    if (!h) return fail(ASTROSIM_ERR_INVALID_ARG, "null handle");
    return guarded([&] { return h->sim.dump_edges(path); });
}

int astrosim_last_step_ms(astrosim_handle* h, double* ms) {
    if (!h || !ms) return fail(ASTROSIM_ERR_INVALID_ARG, "null argument");
    return guarded([&] { return h->sim.last_step_ms(ms); });
}

int astrosim_record_calcium(astrosim_handle* h, int64_t every_steps, uint32_t first_astro, uint32_t n_astro,
                            int64_t max_samples) {
    if (!h) return fail(ASTROSIM_ERR_INVALID_ARG, "null handle");
    return guarded([&] { return h->sim.record_calcium(every_steps, first_astro, n_astro, max_samples); });
}

int astrosim_calcium_samples(astrosim_handle* h, int64_t* n_samples, int64_t* first_step) {
    if (!h) return fail(ASTROSIM_ERR_INVALID_ARG, "null handle");
    return guarded([&] { return h->sim.calcium_samples(n_samples, first_step); });
}

int astrosim_copy_calcium(astrosim_handle* h, int64_t first, int64_t n, double* dst, int wait) {
    if (!h) return fail(ASTROSIM_ERR_INVALID_ARG, "null handle");
    return guarded([&] { return h->sim.copy_calcium(first, n, dst, wait != 0); });
}

int astrosim_sync(astrosim_handle* h) {
    if (!h) return fail(ASTROSIM_ERR_INVALID_ARG, "null handle");
    return guarded([&] { return h->sim.sync(); });
}

int astrosim_ensemble_create(const astrosim_config* cfgs, uint32_t n_networks, astrosim_ensemble** out) {
    return astrosim_ensemble_create_with_biology(cfgs, n_networks, nullptr, out);
}

int astrosim_ensemble_create_with_biology(const astrosim_config* cfgs, uint32_t n_networks,
                                          const char* const* biology_json, astrosim_ensemble** out) {
    if (!cfgs || !out) return fail(ASTROSIM_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    for (uint32_t i = 0; i < n_networks; ++i) {
        if (cfgs[i].struct_size != sizeof(astrosim_config))
            return fail(ASTROSIM_ERR_INVALID_ARG, "astrosim_config.struct_size mismatch");
        for (int r : cfgs[i].reserved)
            if (r != 0) return fail(ASTROSIM_ERR_INVALID_ARG, "astrosim_config.reserved must be zero");
    }
    astrosim_ensemble* e = nullptr;
    try {
        e = new astrosim_ensemble();
    } catch (...) {
        return fail(ASTROSIM_ERR_OUT_OF_MEMORY, "host allocation failed");
    }
    const int rc = guarded([&] { return e->ens.create(cfgs, n_networks, biology_json); });
    if (rc != ASTROSIM_OK) {
        const std::string msg = g_last_error;
        delete e;
        g_last_error = msg;
        return rc;
    }
    *out = e;
    return ASTROSIM_OK;
}

int astrosim_ensemble_step(astrosim_ensemble* e, int64_t n_steps) {
    if (!e) return fail(ASTROSIM_ERR_INVALID_ARG, "null ensemble");
    return guarded([&] { return e->ens.step(n_steps); });
}

int astrosim_ensemble_summary(astrosim_ensemble* e, uint32_t index, astrosim_summary_t* out) {
    if (!e || !out) return fail(ASTROSIM_ERR_INVALID_ARG, "null argument");
    return guarded([&] { return e->ens.summary(index, *out); });
}

int astrosim_ensemble_get_state(astrosim_ensemble* e, uint32_t index, int which, double* dst, size_t count) {
    if (!e) return fail(ASTROSIM_ERR_INVALID_ARG, "null ensemble");
    return guarded([&] { return e->ens.get_state(index, which, dst, count); });
}

int astrosim_ensemble_spike_counts(astrosim_ensemble* e, uint32_t index, int64_t first_step, int64_t n,
                                   uint32_t* counts) {
    if (!e) return fail(ASTROSIM_ERR_INVALID_ARG, "null ensemble");
    return guarded([&] { return e->ens.spike_counts(index, first_step, n, counts); });
}

int astrosim_ensemble_last_step_ms(astrosim_ensemble* e, double* ms) {
    if (!e || !ms) return fail(ASTROSIM_ERR_INVALID_ARG, "null argument");
    return guarded([&] { return e->ens.last_step_ms(ms); });
}

int astrosim_ensemble_build_seconds(astrosim_ensemble* e, double* seconds) {
    if (!e || !seconds) return fail(ASTROSIM_ERR_INVALID_ARG, "null argument");
    *seconds = e->ens.build_seconds();
    g_last_error.clear();
    return ASTROSIM_OK;
}

int astrosim_ensemble_shared_constants(astrosim_ensemble* e, int* shared) {
    if (!e || !shared) return fail(ASTROSIM_ERR_INVALID_ARG, "null argument");
    *shared = e->ens.uniform_constants() ? 1 : 0;
    g_last_error.clear();
    return ASTROSIM_OK;
}

int astrosim_ensemble_destroy(astrosim_ensemble* e) {
    delete e;
    g_last_error.clear();
    return ASTROSIM_OK;
}

int astrosim_server_create(int device, int precision, uint64_t hbm_budget_bytes, int builder_threads,
                           astrosim_server** out) {
    if (!out) return fail(ASTROSIM_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    astrosim_server* s = nullptr;
    try {
        s = new astrosim_server();
    } catch (...) {
        return fail(ASTROSIM_ERR_OUT_OF_MEMORY, "host allocation failed");
    }
    const int rc = guarded([&] { return s->srv.create(device, precision, hbm_budget_bytes, builder_threads); });
    if (rc != ASTROSIM_OK) {
        const std::string msg = g_last_error;
        delete s;
        g_last_error = msg;
        return rc;
    }
    *out = s;
    return ASTROSIM_OK;
}

int astrosim_server_submit(astrosim_server* s, const astrosim_config* cfg, uint64_t* request_id) {
    return astrosim_server_submit_with_biology(s, cfg, nullptr, request_id);
}

int astrosim_server_submit_with_biology(astrosim_server* s, const astrosim_config* cfg, const char* biology_json,
                                        uint64_t* request_id) {
    if (!s || !cfg || !request_id) return fail(ASTROSIM_ERR_INVALID_ARG, "null argument");
    if (cfg->struct_size != sizeof(astrosim_config))
        return fail(ASTROSIM_ERR_INVALID_ARG, "astrosim_config.struct_size mismatch");
    return guarded([&] {
        astrosim::u64 id = 0;
        astrosim::Status st = s->srv.submit(*cfg, &id, biology_json);
        *request_id = id;
        return st;
    });
}

int astrosim_server_pump(astrosim_server* s, int64_t windows) {
    if (!s) return fail(ASTROSIM_ERR_INVALID_ARG, "null server");
    return guarded([&] { return s->srv.pump(windows); });
}

int astrosim_server_result(astrosim_server* s, uint64_t request_id, astrosim_request_result* out, int* done) {
    if (!s || !out || !done) return fail(ASTROSIM_ERR_INVALID_ARG, "null argument");
    return guarded([&] {
        bool d = false;
        astrosim::Status st = s->srv.result(request_id, *out, &d);
        *done = d ? 1 : 0;
        return st;
    });
}

int astrosim_server_get_stats(astrosim_server* s, astrosim_server_stats* out) {
    if (!s || !out) return fail(ASTROSIM_ERR_INVALID_ARG, "null argument");
    s->srv.stats(*out);
    g_last_error.clear();
    return ASTROSIM_OK;
}

int astrosim_server_destroy(astrosim_server* s) {
    delete s;
    g_last_error.clear();
    return ASTROSIM_OK;
}

int astrosim_device_info(int device, char* name, size_t name_cap, int* major, int* minor) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return fail(ASTROSIM_ERR_NO_DEVICE, "no CUDA device visible");
    }
    if (device < 0 || device >= n) return fail(ASTROSIM_ERR_INVALID_ARG, "device ordinal out of range");
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess)
        return fail(ASTROSIM_ERR_CUDA, "cudaGetDeviceProperties failed");
    if (name && name_cap) {
        std::strncpy(name, prop.name, name_cap - 1);
        name[name_cap - 1] = '\0';
    }
    if (major) *major = prop.major;
    if (minor) *minor = prop.minor;
    g_last_error.clear();
    return ASTROSIM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- allocation-free summary reduction
namespace {

constexpr astrosim::u32 kNoAllocPartials = 4096;
static_assert(static_cast<unsigned long long>(kNoAllocPartials) * astrosim::kReduceItemsPerBlock ==
                  ASTROSIM_NOALLOC_MAX_ASTRO,
              "ASTROSIM_NOALLOC_MAX_ASTRO must match the scratch array");
static_assert(sizeof(astrosim_astro_totals) == sizeof(astrosim::AstroTotals), "totals layout");

// Scratch of astrosim_astro_totals_noalloc: 4096 partial sums (64 KB) in the device
// image of every GPU that loads the library.  In host code this name is only a
// stand-in for the symbol; the device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) astrosim::AstroPartial g_noalloc_partials[kNoAllocPartials];

constexpr int kMaxDevices = 128;

// The scratch address belongs to one CUDA context: after cudaDeviceReset (or any
// new primary context) the device image is loaded again, possibly elsewhere.  The
// cache is keyed by the driver's context id, which is unique for the life of the
// process (a context's address can be reused; its id is not).  The two driver
// calls are fetched through the runtime, so the library needs no driver link.
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);
struct NoAllocSlot {
    unsigned long long ctx_id = 0;
    astrosim::AstroPartial* addr = nullptr;
};
std::mutex g_noalloc_mu;
NoAllocSlot g_noalloc_slot[kMaxDevices];
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;

// Id of the current context (made current by a runtime call first); 0 on failure.
unsigned long long current_context_id() {
    if (!g_ctx_get_current || !g_ctx_get_id) {
        void* f1 = nullptr;
        void* f2 = nullptr;
        cudaDriverEntryPointQueryResult q1{}, q2{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) != cudaSuccess ||
            cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) != cudaSuccess ||
            q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !f1 || !f2) {
            cudaGetLastError();
            return 0;
        }
        g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(f1);
        g_ctx_get_id = reinterpret_cast<CtxGetIdFn>(f2);
    }
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (g_ctx_get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
    if (g_ctx_get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

}  // namespace

extern "C" int astrosim_astro_totals_noalloc(const double* ca, const unsigned char* engaged, uint32_t n_astro,
                                             double sic_th, astrosim_astro_totals* out, void* stream) {
    if (!out) return fail(ASTROSIM_ERR_INVALID_ARG, "null output pointer");
    if (n_astro > 0 && (!ca || !engaged)) return fail(ASTROSIM_ERR_INVALID_ARG, "null input pointer");
    if (n_astro > ASTROSIM_NOALLOC_MAX_ASTRO)
        return fail(ASTROSIM_ERR_INVALID_ARG,
                    "n_astro exceeds ASTROSIM_NOALLOC_MAX_ASTRO (8388608), the capacity of the static scratch");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(ASTROSIM_ERR_NO_DEVICE, "no current CUDA device");
    }
    if (dev < 0 || dev >= kMaxDevices) return fail(ASTROSIM_ERR_INVALID_ARG, "device ordinal too large");
    astrosim::AstroPartial* scratch = nullptr;
    {
        // once per device context, with that device current: the device address of
        // the scratch.  Before the first runtime call of a thread no context may be
        // current (id 0); cudaGetSymbolAddress then creates the device's primary
        // context, and the id is read again after it.
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        unsigned long long ctx = current_context_id();
        NoAllocSlot& slot = g_noalloc_slot[dev];
        if (ctx == 0 || !slot.addr || slot.ctx_id != ctx) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_partials);
            ctx = current_context_id();
            if (e != cudaSuccess || !p || ctx == 0) {
                cudaGetLastError();
                slot = NoAllocSlot{};
                return fail(ASTROSIM_ERR_CUDA, "cudaGetSymbolAddress of the no-alloc scratch failed");
            }
            slot.addr = static_cast<astrosim::AstroPartial*>(p);
            slot.ctx_id = ctx;
        }
        scratch = slot.addr;
    }
    return guarded([&] {
        return astrosim::astro_totals(ca, engaged, n_astro, sic_th, scratch,
                                      reinterpret_cast<astrosim::AstroTotals*>(out),
                                      static_cast<cudaStream_t>(stream));
    });
}

namespace astrosim {
Status selfcheck_division(int device, const double* divisors, size_t n, u64 samples, u64 seed, u64* mismatches);
}

extern "C" int astrosim_selfcheck_division(int device, const double* divisors, size_t n_divisors, uint64_t samples,
                                           uint64_t seed, uint64_t* mismatches) {
    return guarded([&] { return astrosim::selfcheck_division(device, divisors, n_divisors, samples, seed, mismatches); });
}

int astrosim_biology_names(char* buf, size_t cap, size_t* needed) {
    const std::string names = astrosim::biology_names();
    if (needed) *needed = names.size() + 1;
    if (!buf) return ASTROSIM_OK;
    if (cap < names.size() + 1) return fail(ASTROSIM_ERR_INVALID_ARG, "buffer too small for the name list");
    std::memcpy(buf, names.c_str(), names.size() + 1);
    return ASTROSIM_OK;
}

int astrosim_biology_value(const char* biology_json, const char* name, double* value) {
    return guarded([&] {
        astrosim::Biology b;
        AS_TRY(astrosim::apply_biology_json(biology_json, b));
        return astrosim::biology_get(b, name, value);
    });
}

struct astrosim_shard {
    astrosim::ShardRank r;
};

struct astrosim_shard_group {
    astrosim::ShardGroup g;
};

int astrosim_shard_plan(uint32_t n_total, int rank, int world, uint32_t* neuron_lo, uint32_t* neuron_hi,
                        uint32_t* astro_lo, uint32_t* astro_hi) {
    if (world < 1 || rank < 0 || rank >= world || n_total == 0)
        return fail(ASTROSIM_ERR_INVALID_ARG, "need n_total > 0 and 0 <= rank < world");
    const astrosim::Sizes sz = astrosim::scaling_law(n_total);
    const astrosim::ShardPlan p = astrosim::shard_plan(sz.n_neurons, sz.n_astro, rank, world);
    if (neuron_lo) *neuron_lo = p.n_lo;
    if (neuron_hi) *neuron_hi = p.n_hi;
    if (astro_lo) *astro_lo = p.a_lo;
    if (astro_hi) *astro_hi = p.a_hi;
    return ASTROSIM_OK;
}

int astrosim_shard_unique_id(unsigned char id[128]) {
    if (!id) return fail(ASTROSIM_ERR_INVALID_ARG, "null id");
    return guarded([&] { return astrosim::nccl_unique_id(id); });
}

int astrosim_shard_create(const astrosim_config* cfg, const char* biology_json, int rank, int world,
                          astrosim_shard** out) {
    if (!cfg || !out) return fail(ASTROSIM_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    if (cfg->struct_size != sizeof(astrosim_config))
        return fail(ASTROSIM_ERR_INVALID_ARG, "astrosim_config.struct_size mismatch");
    astrosim_shard* s = nullptr;
    try {
        s = new astrosim_shard();
    } catch (...) {
        return fail(ASTROSIM_ERR_OUT_OF_MEMORY, "host allocation failed");
    }
    const int rc = guarded([&] { return s->r.create(*cfg, biology_json, rank, world); });
    if (rc != ASTROSIM_OK) {
        const std::string msg = g_last_error;
        delete s;
        g_last_error = msg;
        return rc;
    }
    *out = s;
    return ASTROSIM_OK;
}

int astrosim_shard_connect(astrosim_shard* s, const unsigned char id[128]) {
    if (!s || !id) return fail(ASTROSIM_ERR_INVALID_ARG, "null argument");
    return guarded([&] { return s->r.connect(id); });
}

int astrosim_shard_step(astrosim_shard* s, int64_t n_steps) {
    if (!s) return fail(ASTROSIM_ERR_INVALID_ARG, "null handle");
    return guarded([&] { return s->r.step(n_steps); });
}

int astrosim_shard_summary(astrosim_shard* s, astrosim_summary_t* out) {
    if (!s || !out) return fail(ASTROSIM_ERR_INVALID_ARG, "null argument");
    return guarded([&] { return s->r.summary(*out); });
}

int astrosim_shard_get_state(astrosim_shard* s, int which, double* dst, size_t count) {
    if (!s) return fail(ASTROSIM_ERR_INVALID_ARG, "null handle");
    return guarded([&] { return s->r.get_state(which, dst, count); });
}

int astrosim_shard_spike_counts(astrosim_shard* s, int64_t first_step, int64_t n, uint32_t* counts) {
    if (!s) return fail(ASTROSIM_ERR_INVALID_ARG, "null handle");
    return guarded([&] {
        if (!s->r.has_shard()) return astrosim::make_error(ASTROSIM_ERR_STATE, "no shard");
        return s->r.shard().sim.spike_counts(first_step, n, counts);
    });
}

int astrosim_shard_last_step_ms(astrosim_shard* s, double* ms) {
    if (!s || !ms) return fail(ASTROSIM_ERR_INVALID_ARG, "null argument");
    *ms = s->r.last_step_ms();
    return ASTROSIM_OK;
}

int astrosim_shard_set_timeout(astrosim_shard* s, double seconds) {
    if (!s) return fail(ASTROSIM_ERR_INVALID_ARG, "null handle");
    if (!(seconds > 0.0) || !std::isfinite(seconds)) return fail(ASTROSIM_ERR_INVALID_ARG, "seconds must be > 0");
    s->r.set_timeout(seconds);
    g_last_error.clear();
    return ASTROSIM_OK;
}

int astrosim_shard_selftest_wait(int scenario, double timeout_s, int* windows_done, int* aborted, double* waited_s) {
    return guarded([&] { return astrosim::selftest_bounded_wait(scenario, timeout_s, windows_done, aborted, waited_s); });
}

int astrosim_shard_destroy(astrosim_shard* s) {
    delete s;
    return ASTROSIM_OK;
}

int astrosim_shard_group_create(const astrosim_config* cfg, const char* biology_json, int world, const int* devices,
                                astrosim_shard_group** out) {
    if (!cfg || !out) return fail(ASTROSIM_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    if (cfg->struct_size != sizeof(astrosim_config))
        return fail(ASTROSIM_ERR_INVALID_ARG, "astrosim_config.struct_size mismatch");
    astrosim_shard_group* g = nullptr;
    try {
        g = new astrosim_shard_group();
    } catch (...) {
        return fail(ASTROSIM_ERR_OUT_OF_MEMORY, "host allocation failed");
    }
    const int rc = guarded([&] { return g->g.create(*cfg, biology_json, world, devices); });
    if (rc != ASTROSIM_OK) {
        const std::string msg = g_last_error;
        delete g;
        g_last_error = msg;
        return rc;
    }
    *out = g;
    return ASTROSIM_OK;
}

int astrosim_shard_group_step(astrosim_shard_group* g, int64_t n_steps) {
    if (!g) return fail(ASTROSIM_ERR_INVALID_ARG, "null handle");
    return guarded([&] { return g->g.step(n_steps); });
}

int astrosim_shard_group_summary(astrosim_shard_group* g, astrosim_summary_t* out) {
    if (!g || !out) return fail(ASTROSIM_ERR_INVALID_ARG, "null argument");
    return guarded([&] { return g->g.summary(*out); });
}

int astrosim_shard_group_get_state(astrosim_shard_group* g, int which, double* dst, size_t count) {
    if (!g) return fail(ASTROSIM_ERR_INVALID_ARG, "null handle");
    return guarded([&] { return g->g.get_state(which, dst, count); });
}

int astrosim_shard_group_spike_counts(astrosim_shard_group* g, int64_t first_step, int64_t n, uint32_t* counts) {
    if (!g) return fail(ASTROSIM_ERR_INVALID_ARG, "null handle");
    return guarded([&] { return g->g.spike_counts(first_step, n, counts); });
}

int astrosim_shard_group_get_csr(astrosim_shard_group* g, int rank, int which, uint32_t* row_start, size_t row_cap,
                                 uint32_t* src, size_t src_cap, uint32_t* first_row, uint32_t* n_rows,
                                 uint64_t* n_edges) {
    if (!g) return fail(ASTROSIM_ERR_INVALID_ARG, "null handle");
    if (rank < 0 || rank >= g->g.world()) return fail(ASTROSIM_ERR_INVALID_ARG, "rank out of range");
    return guarded([&] {
        astrosim::Simulation& sim = g->g.shard(rank).sim;
        const astrosim::CellRange& own = sim.network().own;
        if (first_row) *first_row = which == ASTROSIM_CSR_E2A ? own.a_lo : own.n_lo;
        astrosim::u64 ne = 0;
        astrosim::Status s = sim.get_csr(which, row_start, row_cap, src, src_cap, n_rows, &ne);
        if (n_edges) *n_edges = ne;
        return s;
    });
}

int astrosim_shard_group_destroy(astrosim_shard_group* g) {
    delete g;
    return ASTROSIM_OK;
}
