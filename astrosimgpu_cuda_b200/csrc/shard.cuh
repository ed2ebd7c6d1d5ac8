// shard.cuh -- one network split across ranks (GPUs) by contiguous cell ranges.
//
// Every rank builds the whole network (the construction is deterministic in
// (N_total, seed), so all ranks hold identical connectivity and parameters) and
// owns a contiguous range of neurons and of astrocytes, cut at 128-cell block
// boundaries.  Per window of D steps a rank advances only its own cells; the ranks
// then exchange what the next window needs from other ranks' cells:
//   - every spike of the window as (neuron << 5 | step, STP value), and
//   - the D SIC factors of every astrocyte that was active in the window,
// all-gathered (variable sizes: a count exchange first, then the lists padded to
// the largest).  Each rank scatters the other ranks' spikes and factors into its
// window buffers (spike words and values, spike list and per-step counts, active
// mask and factors), so its push and pull read the same data a single-GPU run
// reads, and delivers every spike into the inboxes of its own cells only.  The
// results are bit-identical to the single-GPU run.
#pragma once

#include <memory>
#include <vector>

#include "sim.cuh"
#include "window.cuh"

namespace astrosim {

struct ShardPlan {
    u32 n_lo, n_hi;  // neurons [n_lo, n_hi)
    u32 a_lo, a_hi;  // astrocytes [a_lo, a_hi)
};

// Rank `rank` of `world`: blocks of 128 cells dealt in contiguous, balanced runs.
ShardPlan shard_plan(u32 n_neurons, u32 n_astro, int rank, int world);

// Collective exchange between the ranks of one sharded network (device memory,
// enqueued on the caller's stream).
class ShardComm {
public:
    virtual ~ShardComm() = default;
    // recv[r * bytes, (r + 1) * bytes) <- rank r's send[0, bytes), on every rank.
    virtual Status all_gather(const void* send, void* recv, size_t bytes, cudaStream_t st) = 0;
    virtual Status group_begin() { return Status::Ok(); }
    virtual Status group_end() { return Status::Ok(); }
};

// NCCL communicator (libnccl.so.2 loaded at run time) for one rank per process.
Status nccl_unique_id(unsigned char id[128]);
Status make_nccl_comm(const unsigned char id[128], int rank, int world, int device, std::unique_ptr<ShardComm>& out);

// One rank's part of a sharded network.
class ShardSim {
public:
    ~ShardSim();
    Status create(const astrosim_config& cfg, const char* biology_json, int rank, int world);

    // The phases of window k (whole windows only), in order.
    Status run_window(i64 k);
    Status pack(i64 k);  // export lists and counts; counts reach host_counts() after a stream sync
    Status import(i64 k, const u32* counts_all, u64 stride_spk, u64 stride_ast);  // counts_all: 2 per rank
    Status push(i64 k);
    void note_window(double seconds);

    const u32* host_counts() const { return h_cnt_; }
    cudaStream_t stream() const { return sim.stream(); }
    int device() const { return sim.config().device; }
    size_t real_bytes() const { return sim.fp32() ? sizeof(float) : sizeof(double); }
    int window() const { return W_; }

    Simulation sim;
    ShardPlan plan{};
    int rank = 0, world = 1;
    u64 cap_spk = 0, cap_ast = 0;
    DevBuf<u32> x_keys, x_ids, x_cnt;        // export: spike keys, active astrocyte ids, {n_spk, n_ast}
    DevBuf<unsigned char> x_vals, x_facs;    // export: spike values, W factors per astrocyte
    DevBuf<u32> r_keys, r_ids, r_cnt;        // receive: world x stride
    DevBuf<unsigned char> r_vals, r_facs;

private:
    int W_ = 0;
    u32* h_cnt_ = nullptr;  // pinned: this rank's {n_spk, n_ast}, or all ranks' after an exchange
};

// A sharded network driven by one process per rank over NCCL.
class ShardRank {
public:
    // Builds this rank's network (no communication yet).
    Status create(const astrosim_config& cfg, const char* biology_json, int rank, int world);
    // Joins the ranks' NCCL communicator (collective); a world of one needs none.
    Status connect(const unsigned char id[128]);
    Status step(i64 n);  // collective; whole windows
    Status summary(astrosim_summary_t& out);  // collective
    Status get_state(int which, double* dst, size_t count);  // collective; the whole network's array
    ShardSim& shard() { return *s_; }
    bool has_shard() const { return static_cast<bool>(s_); }
    double last_step_ms() const { return last_ms_; }

private:
    Status gather(int which);
    std::unique_ptr<ShardSim> s_;
    std::unique_ptr<ShardComm> comm_;
    double last_ms_ = 0.0;
};

// All ranks of a sharded network in one process: devices[r] runs rank r (devices
// may repeat; on one device the ranks run one after another, which exercises the
// exchange exactly as separate GPUs would).
class ShardGroup {
public:
    Status create(const astrosim_config& cfg, const char* biology_json, int world, const int* devices);
    Status step(i64 n);
    Status summary(astrosim_summary_t& out);
    Status get_state(int which, double* dst, size_t count);
    Status spike_counts(i64 first, i64 n, u32* dst) { return shards_[0]->sim.spike_counts(first, n, dst); }
    ShardSim& shard(int r) { return *shards_[r]; }
    int world() const { return static_cast<int>(shards_.size()); }
    double last_step_ms() const { return last_ms_; }

private:
    Status gather(int which);
    std::vector<std::unique_ptr<ShardSim>> shards_;
    std::vector<u32> counts_;
    double last_ms_ = 0.0;
};

}  // namespace astrosim
