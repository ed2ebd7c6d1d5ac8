// params.cu -- per-cell parameter draws on the device (src/astrosim_fused.cu:917-933).
//
// The reference draws, from a fresh sequential stream (seed, 0x5EED), four
// truncated normals per astrocyte (Ca_tot, IP3_0, tau_IP3, delta_IP3) and then two
// per neuron (V_reset, b), each by redrawing until the value falls inside its
// bounds (src/astrosim_fused.cu:196-216).  Normals come in Box-Muller pairs with
// the sine half cached (src/astrosim_fused.cu:184-194), so the k-th normal the
// stream hands out is a fixed function of k: the cosine (k even) or sine (k odd)
// half of the pair drawn from uniforms 2*(k/2) and 2*(k/2)+1.  What is
// sequential is only the mapping of normals to parameters, an automaton whose
// state is "which parameter type draws next".  Each chunk of normals is scanned
// once per possible entry state, the chunks are composed in order, and a last
// pass writes the accepted values.
//
// Gaussians use CUDA's log/sqrt/sin/cos, so values can differ from the
// reference's host C library in the last bit.  An accept/reject test that lands
// within a few ulps of a bound is settled by the host formula, so the mapping of
// normals to parameters is identical to the reference.

#include <algorithm>
#include <cmath>
#include <map>
#include <vector>

#include "builder_internal.cuh"

namespace astrosim {

namespace {

constexpr int kMaxTypes = 4;
constexpr u32 kMaxChunkNormals = 2048;  // normals per chunk at most (every length is even)

// Normals per chunk of a phase that budgets `budget` normals.  One thread scans each
// chunk, one normal after the other, and one thread then composes the chunks, one
// after the other; a step of either costs about the same, so the length follows the
// square root of the budget: 64 for a few thousand normals, the 2048 cap from
// about 4e6 on (the astrocyte phase of networks from N = 5e5 up).
u32 chunk_normals(u64 budget) {
    u32 c = 64;
    while (c < kMaxChunkNormals && static_cast<u64>(c) * c < budget) c *= 2;
    return c;
}

struct TypeSpec {
    double mean, sd, lo, hi;
    bool randomized;
};

struct Phase {
    TypeSpec t[kMaxTypes];
    int n_types;      // cycle length
    u64 n_units;      // draw_scaled calls in the phase
    u64 k_start;      // first normal index of the phase
    u32 chunk;        // normals per chunk (chunk_normals)
};

// src/astrosim_fused.cu:210-216
TypeSpec type_spec(double mean, bool on, double lower, double upper, double var) {
    TypeSpec s{};
    s.mean = mean;
    s.randomized = on && var > 0.0;
    s.lo = mean < 0.0 ? mean * upper : mean * lower;
    s.hi = mean < 0.0 ? mean * lower : mean * upper;
    s.sd = var * std::fabs(mean);
    return s;
}

struct AcceptTable {
    const u64* k = nullptr;
    const unsigned char* acc = nullptr;
    int n = 0;
};

__device__ __forceinline__ double normal_k(u64 seed, u64 k) {
    const u64 m = k >> 1;
    const double u1 = rng_uniform(seed, kSetupStream, 2 * m);
    const double u2 = rng_uniform(seed, kSetupStream, 2 * m + 1);
    const double r = sqrt(-2.0 * log(u1));
    const double th = kTwoPi * u2;
    return (k & 1) ? r * sin(th) : r * cos(th);
}

constexpr double kBoundRel = 64.0 * 2.220446049250313e-16;

__device__ __forceinline__ bool accept(const TypeSpec& s, u64 k, double z, const AcceptTable& tab, u64* amb_k,
                                       unsigned* amb_n, unsigned amb_cap) {
    const double v = s.mean + s.sd * z;
    const bool a = v >= s.lo && v <= s.hi;
    const double scale = fabs(s.mean) + 1e-300;
    if (fabs(v - s.lo) <= kBoundRel * scale || fabs(v - s.hi) <= kBoundRel * scale) {
        int lo = 0, hi = tab.n;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (tab.k[mid] < k) lo = mid + 1; else hi = mid;
        }
        if (lo < tab.n && tab.k[lo] == k) return tab.acc[lo] != 0;
        if (amb_n) {
            const unsigned i = atomicAdd(amb_n, 1u);
            if (i < amb_cap) amb_k[i] = k;
        }
    }
    return a;
}

struct ChunkResult {
    u32 accepts;   // completed units
    u8 exit_type;  // type index at the chunk end
    u8 tries;      // rejections of the unit in progress at the chunk end (capped)
    u16 lead;      // rejections before the chunk's first accept (the whole chunk if none)
};

// One thread per (chunk, entry type): run the automaton over the chunk.
__global__ void param_table_kernel(Phase ph, u64 seed, u32 n_chunks, ChunkResult* out, AcceptTable tab, u64* amb_k,
                                   unsigned* amb_n, unsigned amb_cap, int* err) {
    const u32 gid = blockIdx.x * blockDim.x + threadIdx.x;
    const u32 chunk = gid / kMaxTypes;
    const int entry = gid % kMaxTypes;
    if (chunk >= n_chunks || entry >= ph.n_types) return;
    const u64 k0 = ph.k_start + static_cast<u64>(chunk) * ph.chunk;
    int type = entry;
    u32 acc = 0, lead = 0;
    int tries = 0;
    for (u32 i = 0; i < ph.chunk; ++i) {
        const u64 k = k0 + i;
        const double z = normal_k(seed, k);
        if (accept(ph.t[type], k, z, tab, amb_k, amb_n, amb_cap)) {
            if (acc == 0) lead = i;
            ++acc;
            type = type + 1 == ph.n_types ? 0 : type + 1;
            tries = 0;
        } else if (++tries >= 200) {
            *err = 1;  // 200 straight rejections: probability below 1e-60 per unit
        }
    }
    ChunkResult r{};
    r.accepts = acc;
    r.exit_type = static_cast<u8>(type);
    r.tries = static_cast<u8>(tries > 255 ? 255 : tries);
    r.lead = static_cast<u16>(acc == 0 ? ph.chunk : lead);
    out[static_cast<u64>(chunk) * kMaxTypes + entry] = r;
}

// One thread composes the chunks in order.  It also follows the run of rejections
// of the unit in progress across chunk ends (the table scan sees runs inside a chunk).
__global__ void param_compose_kernel(Phase ph, u32 n_chunks, const ChunkResult* tabs, u8* entry_type,
                                     u64* unit_offset, u32* end_chunk, int* err) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int type = 0;
    u64 units = 0;
    u32 run = 0;
    u32 c = 0;
    for (; c < n_chunks; ++c) {
        entry_type[c] = static_cast<u8>(type);
        unit_offset[c] = units;
        const ChunkResult r = tabs[static_cast<u64>(c) * kMaxTypes + type];
        if (r.accepts == 0) {
            run += r.lead;
        } else {
            if (run + r.lead >= 200) *err = 1;
            run = r.tries;
        }
        if (run >= 200) *err = 1;
        if (units + r.accepts >= ph.n_units) break;
        units += r.accepts;
        type = r.exit_type;
    }
    *end_chunk = c;  // == n_chunks when the phase did not end inside the chunks
}

// One thread per chunk: replay from the known entry state and write the accepted values.
__global__ void param_emit_kernel(Phase ph, u64 seed, u32 n_chunks, const u8* entry_type, const u64* unit_offset,
                                  const u32* end_chunk, AcceptTable tab, double* const* dst, u64* k_end) {
    const u32 chunk = blockIdx.x * blockDim.x + threadIdx.x;
    const u32 last = *end_chunk;
    if (chunk >= n_chunks || chunk > last) return;
    const u64 k0 = ph.k_start + static_cast<u64>(chunk) * ph.chunk;
    int type = entry_type[chunk];
    u64 unit = unit_offset[chunk];
    for (u32 i = 0; i < ph.chunk && unit < ph.n_units; ++i) {
        const u64 k = k0 + i;
        const double z = normal_k(seed, k);
        if (accept(ph.t[type], k, z, tab, nullptr, nullptr, 0)) {
            const TypeSpec& s = ph.t[type];
            const u64 cell = unit / ph.n_types;
            dst[type][cell] = s.mean + s.sd * z;
            ++unit;
            type = type + 1 == ph.n_types ? 0 : type + 1;
            if (unit == ph.n_units) *k_end = k + 1;
        }
    }
}

__global__ void fill_kernel(double* dst, u64 n, double v) {
    const u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = v;
}

// Host settling of an ambiguous accept test with the reference's host formula.
bool host_accept(const TypeSpec& s, u64 seed, u64 k) {
    const u64 m = k >> 1;
    const double u1 = rng_uniform(seed, kSetupStream, 2 * m);
    const double u2 = rng_uniform(seed, kSetupStream, 2 * m + 1);
    const double r = std::sqrt(-2.0 * std::log(u1));
    const double th = kTwoPi * u2;
    const double z = (k & 1) ? r * std::sin(th) : r * std::cos(th);
    const double v = s.mean + s.sd * z;
    return v >= s.lo && v <= s.hi;
}

// Runs one phase (a cycle of parameter types over n_cells cells) starting at normal
// index ph.k_start; writes dst[type][cell] and returns the first normal after the phase.
Status run_phase(Phase ph, u64 seed, double* const* dst_host, u64 n_cells, u64* k_next, cudaStream_t st) {
    // A type that is not randomised returns its mean without drawing.
    bool any_random = false;
    for (int i = 0; i < ph.n_types; ++i) any_random |= ph.t[i].randomized;
    if (!any_random || ph.n_units == 0) {
        for (int i = 0; i < ph.n_types; ++i)
            if (n_cells) {
                fill_kernel<<<ceil_div(n_cells, 256), 256, 0, st>>>(dst_host[i], n_cells, ph.t[i].mean);
                AS_CUDA(cudaGetLastError());
            }
        *k_next = ph.k_start;
        return Status::Ok();
    }
    for (int i = 0; i < ph.n_types; ++i)
        if (!ph.t[i].randomized)
            return make_error(ASTROSIM_ERR_UNSUPPORTED, "mixed randomised and fixed parameter types in one phase");

    // Acceptance is about 0.53 for the astrocyte types and 0.95 for the neuron types.
    u64 budget = static_cast<u64>(static_cast<double>(ph.n_units) * 2.2) + 4096;
    DevBuf<double*> dst;
    AS_TRY(dst.alloc(ph.n_types));
    AS_CUDA(cudaMemcpyAsync(dst.get(), dst_host, ph.n_types * sizeof(double*), cudaMemcpyHostToDevice, st));
    std::map<u64, unsigned char> table;
    DevBuf<u64> tab_k, amb_k;
    DevBuf<unsigned char> tab_a;
    DevBuf<unsigned> amb_n;
    DevBuf<int> err;
    AS_TRY(amb_k.alloc(4096));
    AS_TRY(amb_n.alloc(1));
    AS_TRY(err.alloc(1));
    for (int attempt = 0; attempt < 8; ++attempt) {
        ph.chunk = chunk_normals(budget);
        const u32 n_chunks = ceil_div(budget, ph.chunk);
        DevBuf<ChunkResult> tabs;
        DevBuf<u8> entry;
        DevBuf<u64> offs, kend;
        DevBuf<u32> endc;
        AS_TRY(tabs.alloc(static_cast<size_t>(n_chunks) * kMaxTypes));
        AS_TRY(entry.alloc(n_chunks));
        AS_TRY(offs.alloc(n_chunks));
        AS_TRY(endc.alloc(1));
        AS_TRY(kend.alloc(1));
        // upload the settled accept decisions
        std::vector<u64> tk;
        std::vector<unsigned char> ta;
        for (const auto& kv : table) {
            tk.push_back(kv.first);
            ta.push_back(kv.second);
        }
        AS_TRY(tab_k.alloc(tk.size()));
        AS_TRY(tab_a.alloc(ta.size()));
        if (!tk.empty()) {
            AS_CUDA(cudaMemcpyAsync(tab_k.get(), tk.data(), tk.size() * sizeof(u64), cudaMemcpyHostToDevice, st));
            AS_CUDA(cudaMemcpyAsync(tab_a.get(), ta.data(), ta.size(), cudaMemcpyHostToDevice, st));
        }
        AcceptTable tab{tab_k.get(), tab_a.get(), static_cast<int>(tk.size())};
        AS_CUDA(cudaMemsetAsync(amb_n.get(), 0, sizeof(unsigned), st));
        AS_CUDA(cudaMemsetAsync(err.get(), 0, sizeof(int), st));
        const u64 threads = static_cast<u64>(n_chunks) * kMaxTypes;
        param_table_kernel<<<ceil_div(threads, 128), 128, 0, st>>>(ph, seed, n_chunks, tabs.get(), tab, amb_k.get(),
                                                                  amb_n.get(), 4096, err.get());
        AS_CUDA(cudaGetLastError());
        unsigned namb = 0;
        int herr = 0;
        AS_CUDA(cudaMemcpyAsync(&namb, amb_n.get(), sizeof(unsigned), cudaMemcpyDeviceToHost, st));
        AS_CUDA(cudaMemcpyAsync(&herr, err.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
        AS_CUDA(cudaStreamSynchronize(st));
        if (herr)
            return make_error(ASTROSIM_ERR_UNSUPPORTED, "parameter stream with 200 consecutive rejections");
        if (namb) {
            // Settle every logged test with the host formula, then scan again.  The
            // type of the unit drawing normal k is not known here, so every type's
            // decision is recorded; only types with a bound near v can differ.
            const unsigned m = std::min<unsigned>(namb, 4096);
            std::vector<u64> ks(m);
            AS_CUDA(cudaMemcpyAsync(ks.data(), amb_k.get(), m * sizeof(u64), cudaMemcpyDeviceToHost, st));
            AS_CUDA(cudaStreamSynchronize(st));
            bool added = false;
            for (u64 k : ks) {
                if (table.count(k)) continue;
                // ambiguous for one type; decide for the type whose bound is near
                unsigned char d = 0;
                for (int i = 0; i < ph.n_types; ++i) {
                    const TypeSpec& s = ph.t[i];
                    const u64 mm = k >> 1;
                    const double u1 = rng_uniform(seed, kSetupStream, 2 * mm);
                    const double u2 = rng_uniform(seed, kSetupStream, 2 * mm + 1);
                    const double r = std::sqrt(-2.0 * std::log(u1));
                    const double th = kTwoPi * u2;
                    const double z = (k & 1) ? r * std::sin(th) : r * std::cos(th);
                    const double v = s.mean + s.sd * z;
                    const double scale = std::fabs(s.mean) + 1e-300;
                    if (std::fabs(v - s.lo) <= 1e3 * kBoundRel * scale || std::fabs(v - s.hi) <= 1e3 * kBoundRel * scale)
                        d = host_accept(s, seed, k) ? 1 : 0;
                }
                table[k] = d;
                added = true;
            }
            if (added) {
                // Different types can share one normal index only if two bounds are
                // within a few ulps of the same value; the defaults never do this.
                continue;
            }
        }
        param_compose_kernel<<<1, 32, 0, st>>>(ph, n_chunks, tabs.get(), entry.get(), offs.get(), endc.get(),
                                                err.get());
        AS_CUDA(cudaGetLastError());
        u32 hend = 0;
        AS_CUDA(cudaMemcpyAsync(&hend, endc.get(), sizeof(u32), cudaMemcpyDeviceToHost, st));
        AS_CUDA(cudaMemcpyAsync(&herr, err.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
        AS_CUDA(cudaStreamSynchronize(st));
        if (herr)
            return make_error(ASTROSIM_ERR_UNSUPPORTED, "parameter stream with 200 consecutive rejections");
        if (hend >= n_chunks) {
            budget *= 2;  // the phase needed more normals than budgeted
            continue;
        }
        param_emit_kernel<<<ceil_div(hend + 1, 128), 128, 0, st>>>(ph, seed, n_chunks, entry.get(), offs.get(),
                                                                  endc.get(), tab, dst.get(), kend.get());
        AS_CUDA(cudaGetLastError());
        AS_CUDA(cudaMemcpyAsync(k_next, kend.get(), sizeof(u64), cudaMemcpyDeviceToHost, st));
        AS_CUDA(cudaStreamSynchronize(st));
        return Status::Ok();
    }
    return make_error(ASTROSIM_ERR_CUDA, "parameter scan did not settle");
}

__global__ void zero_scan_kernel(u64 seed, u64 n, unsigned* found) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        if (rng_uniform_is_zero(seed, kSetupStream, i)) atomicAdd(found, 1u);
}

}  // namespace

Status alloc_cell_parameters(const Sizes& sz, Network& net) {
    const u32 nA = sz.n_astro, nN = sz.n_neurons;
    AS_TRY(net.Ca_tot.alloc(nA));
    AS_TRY(net.IP3_0.alloc(nA));
    AS_TRY(net.tau_IP3.alloc(nA));
    AS_TRY(net.delta_IP3.alloc(nA));
    AS_TRY(net.V_reset.alloc(nN));
    AS_TRY(net.b.alloc(nN));
    return Status::Ok();
}

Status draw_cell_parameters(const Sizes& sz, u64 seed, const Biology& bio, Network& net, cudaStream_t st) {
    const u32 nA = sz.n_astro, nN = sz.n_neurons;

    // src/astrosim_fused.cu:919-924: four astrocyte parameters per cell, in this order
    Phase pa{};
    pa.n_types = 4;
    pa.t[0] = type_spec(bio.Ca_tot, bio.randomize_astro, bio.ra_lower, bio.ra_upper, bio.ra_var);
    pa.t[1] = type_spec(bio.IP3_0, bio.randomize_astro, bio.ra_lower, bio.ra_upper, bio.ra_var);
    pa.t[2] = type_spec(bio.tau_IP3, bio.randomize_astro, bio.ra_lower, bio.ra_upper, bio.ra_var);
    pa.t[3] = type_spec(bio.delta_IP3, bio.randomize_astro, bio.ra_lower, bio.ra_upper, bio.ra_var);
    pa.n_units = 4ull * nA;
    pa.k_start = 0;

    PhaseClock pc(st);
    // The normals k map to uniforms 2*(k/2), 2*(k/2)+1 only while no pair's first
    // uniform is exactly zero (the reference would redraw it).  Check the range used.
    {
        DevBuf<unsigned> found;
        AS_TRY(found.alloc_zero(1, st));
        const u64 n_uniforms = 2 * (static_cast<u64>((4.0 * nA * 2.2 + 2.0 * nN * 1.2)) + 8192);
        zero_scan_kernel<<<1184, 256, 0, st>>>(seed, n_uniforms, found.get());
        AS_CUDA(cudaGetLastError());
        unsigned f = 0;
        AS_CUDA(cudaMemcpyAsync(&f, found.get(), sizeof(unsigned), cudaMemcpyDeviceToHost, st));
        AS_CUDA(cudaStreamSynchronize(st));
        if (f)
            return make_error(ASTROSIM_ERR_UNSUPPORTED,
                              "seed %llu: a 53-bit zero draw occurs in the parameter stream; unsupported",
                              static_cast<unsigned long long>(seed));
    }

    pc.mark("  zero-draw scan");
    double* adst[4] = {net.Ca_tot.get(), net.IP3_0.get(), net.tau_IP3.get(), net.delta_IP3.get()};
    u64 k = 0;
    AS_TRY(run_phase(pa, seed, adst, nA, &k, st));
    pc.mark("  astrocyte parameters");

    // src/astrosim_fused.cu:927-933: V_reset then b per neuron; exc then inh means
    for (int pop = 0; pop < 2; ++pop) {
        const bool exc = pop == 0;
        const u64 n_cells = exc ? sz.n_exc : sz.n_inh;
        const u64 first = exc ? 0 : sz.n_exc;
        Phase pn{};
        pn.n_types = 2;
        pn.t[0] = type_spec(exc ? bio.e_V_reset : bio.i_V_reset, bio.randomize_neuron, bio.rn_lower, bio.rn_upper,
                            bio.rn_var);
        pn.t[1] = type_spec(exc ? bio.e_b : bio.i_b, bio.randomize_neuron, bio.rn_lower, bio.rn_upper, bio.rn_var);
        pn.n_units = 2 * n_cells;
        pn.k_start = k;
        double* ndst[2] = {net.V_reset.get() + first, net.b.get() + first};
        AS_TRY(run_phase(pn, seed, ndst, n_cells, &k, st));
        pc.mark(exc ? "  excitatory parameters" : "  inhibitory parameters");
    }
    return Status::Ok();
}

}  // namespace astrosim
