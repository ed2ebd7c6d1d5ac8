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

#include <functional>
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
    // The communicator's own view of its peers: an ASTROSIM_ERR_PEER status once it
    // has seen a peer fail or leave; *pending while it is still setting up.
    virtual Status async_state(bool* pending) {
        *pending = false;
        return Status::Ok();
    }
    // Ends every operation of this communicator still in flight (the communicator
    // is unusable afterwards): the way out of a wait on a peer that never comes.
    virtual void abort() {}
};

// Polls `query` (0: the work is done, 1: still running, -1: it failed) until it
// reports done, the communicator reports a failed peer, or `timeout_s` passes.  On
// a failed peer or an expired deadline it aborts the communicator and returns
// ASTROSIM_ERR_PEER or ASTROSIM_ERR_TIMEOUT, so no rank waits for ever on a rank
// that died or left; `what` names the wait in the message.
Status bounded_wait(ShardComm* comm, const std::function<int()>& query, double timeout_s, const char* what);

// bounded_wait on everything enqueued on stream `st` so far.
Status bounded_stream_wait(ShardComm* comm, cudaStream_t st, double timeout_s, const char* what);

// Exercises bounded_wait with a stand-in communicator and stand-in exchanges (no
// device, no NCCL): scenario 0, four windows whose exchanges complete; 1, the first
// exchange never completes; 2, the communicator reports a failed peer during the
// first exchange; 3, the exchanges of windows 0 and 1 complete, then a rank has
// left and the exchange of window 2 never completes.
Status selftest_bounded_wait(int scenario, double timeout_s, int* windows_done, int* aborted, double* waited_s);

// Seconds a rank waits on the others before it gives up: ASTROSIM_SHARD_TIMEOUT_S,
// else 120.
double default_shard_timeout();

// NCCL communicator (libnccl.so.2 loaded at run time) for one rank per process;
// non-blocking, so that set-up and every exchange can be given a deadline.
Status nccl_unique_id(unsigned char id[128]);
Status make_nccl_comm(const unsigned char id[128], int rank, int world, int device, double timeout_s,
                      std::unique_ptr<ShardComm>& out);

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
    u32* host_counts_buffer() { return h_cnt_; }  // pinned, 2 * world entries
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
    // Deadline of every wait on the other ranks (set-up included), seconds.
    void set_timeout(double seconds) { timeout_s_ = seconds; }
    double timeout() const { return timeout_s_; }

private:
    Status gather(int which);
    Status wait(const char* what);  // bounded wait on this rank's stream
    Status usable() const;
    std::unique_ptr<ShardSim> s_;
    std::unique_ptr<ShardComm> comm_;
    double last_ms_ = 0.0;
    double timeout_s_ = default_shard_timeout();
    bool failed_ = false;  // a wait gave up: the communicator is aborted, the state is mid-window
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
