// network.cuh -- the device-resident network: four target-keyed CSRs and the
// per-cell parameters, plus the builder that makes them on the GPU.
#pragma once

#include <vector>

#include "common.cuh"
#include "model.cuh"

namespace astrosim {

// Target-keyed CSR (src/astrosim_fused.cu:296-301): row_start[n_targets + 1], src[n_edges].
struct DeviceCSR {
    DeviceCSR() = default;
    DeviceCSR(DeviceCSR&&) = default;
    DeviceCSR& operator=(DeviceCSR&&) = default;
    DevBuf<u32> row_start, src;
    u32 n_targets = 0;
    u64 n_edges = 0;
};

// The cells whose incoming connections a network keeps: neurons [n_lo, n_hi) and
// astrocytes [a_lo, a_hi).  A whole network owns every cell.  A rank of a sharded
// network owns its range: its exc, inh and sic CSRs hold only the rows of neurons
// [n_lo, n_hi) and its e2a CSR only those of astrocytes [a_lo, a_hi), row r being
// cell lo + r, so each rank keeps about 1 / world of the connectivity.  The rows it
// keeps are exactly the whole network's rows (same sources in the same order).
struct CellRange {
    u32 n_lo = 0, n_hi = 0xFFFFFFFFu;
    u32 a_lo = 0, a_hi = 0xFFFFFFFFu;
    CellRange clamped(const Sizes& sz) const {
        CellRange c = *this;
        c.n_hi = c.n_hi < sz.n_neurons ? c.n_hi : sz.n_neurons;
        c.a_hi = c.a_hi < sz.n_astro ? c.a_hi : sz.n_astro;
        c.n_lo = c.n_lo < c.n_hi ? c.n_lo : c.n_hi;
        c.a_lo = c.a_lo < c.a_hi ? c.a_lo : c.a_hi;
        return c;
    }
    bool whole(const Sizes& sz) const {
        const CellRange c = clamped(sz);
        return c.n_lo == 0 && c.n_hi == sz.n_neurons && c.a_lo == 0 && c.a_hi == sz.n_astro;
    }
};

struct Network {
    Network() = default;
    Network(Network&&) = default;
    Network& operator=(Network&&) = default;
    Sizes sz;
    u64 seed = 0;
    CellRange own;  // clamped to sz; the CSRs below hold these cells' rows
    DeviceCSR exc, inh, sic, e2a;
    // Edge counts of the whole network (exc, inh, e2a, sic), whatever `own` keeps.
    u64 total_edges[4] = {0, 0, 0, 0};
    bool partial() const { return !own.whole(sz); }
    // Source-major lists of the exc and inh CSRs, when the builder wrote them while
    // emitting the edges (the chunked builder): row r of fwd_exc (exc source r) and of
    // fwd_inh (inh source r) lists the target rows of its edges in ascending order,
    // the lists the windowed engine would otherwise derive by sorting the CSRs.
    DevBuf<u32> fwd_exc_rs, fwd_exc_dst, fwd_inh_rs, fwd_inh_dst;
    bool has_fwd = false;
    void drop_forward() {
        fwd_exc_rs.release();
        fwd_exc_dst.release();
        fwd_inh_rs.release();
        fwd_inh_dst.release();
        has_fwd = false;
    }
    // Per-cell parameters (src/astrosim_fused.cu:917-933), always double.
    DevBuf<double> Ca_tot, IP3_0, tau_IP3, delta_IP3, V_reset, b;
    double build_seconds = 0.0;
    int builder_path = 0;  // 0 = sequential walk, 1 = parallel chunked walk
};

struct BuildOptions {
    // Networks whose estimated connectivity stream is shorter than this many draws are
    // walked by one device thread (exact, no setup overhead); larger ones by the chunked
    // parallel builder.  0 forces the parallel builder, UINT64_MAX the sequential one.
    u64 sequential_max_draws = 50000ULL;
    // Targets whose rows the network keeps (a rank of a sharded network: its cells).
    CellRange own;
};

// Builds connectivity and per-cell parameters for (sizes, seed, biology) on `stream`,
// bit-identical in structure to the reference's host builder (src/astrosim_fused.cu:631-735)
// and parameter draws (src/astrosim_fused.cu:917-933).
Status build_network(const Sizes& sz, u64 seed, const Biology& bio, const BuildOptions& opt, Network& net,
                     cudaStream_t stream);

// Writes a CSR to host vectors (test and dump support).
Status download_csr(const DeviceCSR& c, std::vector<u32>& row_start, std::vector<u32>& src, cudaStream_t st);

// Expected number of setup-stream draws of the connectivity walk (for choosing the builder).
double estimated_walk_draws(const Sizes& sz);

}  // namespace astrosim
