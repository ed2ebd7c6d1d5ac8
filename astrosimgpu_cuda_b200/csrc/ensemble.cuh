// ensemble.cuh -- many independent networks stepped together (the batched form).
//
// Each network keeps its own device state exactly as a single Simulation (its own
// windowed engine buffers).  One window launch covers every cell of every network:
// a tile table maps each block (a tile of 64, 128 or 256 cells: the autotuner times
// each size with three occupancy targets) to (network, population, tile), and each
// block reads its network's descriptor (constants and pointers) into shared memory.
// The constants that differ between networks (NetScalars) sit in the descriptor;
// when every network shares the rest (the same biology, dt and substeps) those come
// from the kernel parameters, else each block also stages its network's full
// constants.  Every network has its own window counter and stop step on the device, so the
// per-window sequence {window, push, advance} is identical for every window and is
// captured once in a CUDA graph and replayed.
#pragma once

#include <memory>
#include <vector>

#include "common.cuh"
#include "sim.cuh"

namespace astrosim {

constexpr int kNumTileSizes = 3;  // tiles of 64, 128 or 256 cells, chosen by the autotuner

class Ensemble {
public:
    ~Ensemble();
    Status create(const astrosim_config* cfgs, u32 n, const char* const* biology_json = nullptr);
    Status step(i64 n_steps);
    Status summary(u32 i, astrosim_summary_t& out);
    Status get_state(u32 i, int which, double* dst, size_t count);
    Status spike_counts(u32 i, i64 first, i64 n, u32* dst);
    Status last_step_ms(double* ms);
    u32 size() const { return static_cast<u32>(nets_.size()); }
    bool uniform_constants() const { return uniform_; }
    i64 steps_done() const { return steps_done_; }
    double build_seconds() const { return build_seconds_; }

    // Membership control used by the serving loop: networks can be appended and
    // retired between windows; descriptors and tiles are rebuilt on change.
    Status add(std::unique_ptr<Simulation> sim);
    Status retire(u32 i);  // frees network i (its slot stays, inactive)
    bool active(u32 i) const { return i < nets_.size() && nets_[i] != nullptr; }
    i64 net_steps_done(u32 i) const;
    Simulation* net(u32 i) { return nets_[i].get(); }
    Status init_empty(bool fp32, int window, int device);
    Status advance_windows(i64 windows);  // one window for every active unfinished network, `windows` times

private:
    Status rebuild();
    Status capture_graph();
    Status sync_progress();
    void launch_window(int v);  // window + push kernels for variant v

    std::vector<std::unique_ptr<Simulation>> nets_;
    std::vector<cudaStream_t> build_streams_;  // lent to the networks create() built
    int build_device_ = 0;
    std::vector<i64> win_host_;  // window index of each network at the last sync
    bool fp32_ = false;
    int W_ = 0;
    int device_ = 0;
    cudaStream_t stream_ = nullptr;
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    bool have_events_ = false;
    DevBuf<unsigned char> descs_;
    DevBuf<unsigned char> rcs_;  // RunConsts per network (read when !uniform_)
    RunConsts common_{};         // shared constants (NetScalars fields cleared)
    bool uniform_ = true;
    // tile tables for tiles of 64, 128 and 256 cells
    DevBuf<u32> tile_net_[kNumTileSizes], tile_blk_[kNumTileSizes];
    DevBuf<i64> win_, stop_;
    u32 n_tiles_[kNumTileSizes] = {0, 0, 0};
    bool dirty_ = true;
    int variant_ = -1;  // (tile size, launch bounds) variant; -1 while the autotuner times them
    int tune_step_ = 0;
    float tune_ms_[9] = {1e30f, 1e30f, 1e30f, 1e30f, 1e30f, 1e30f, 1e30f, 1e30f, 1e30f};
    cudaGraphExec_t graph_ = nullptr;
    int graph_windows_ = 0;
    i64 steps_done_ = 0;
    double build_seconds_ = 0.0;
};

}  // namespace astrosim
