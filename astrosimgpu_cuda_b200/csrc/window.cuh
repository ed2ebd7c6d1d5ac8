// window.cuh -- the windowed stepping engine.
//
// Every synaptic delay of the model is the same 1 ms (src/astrosim_fused.cu:766),
// D time steps.  Inside a window of D consecutive steps no cell needs anything
// produced in the same window: the spikes and SIC factors it reads were produced
// D steps earlier, i.e. in the previous window.  So one launch advances every cell
// through a whole window with its state in registers, and the window's spikes are
// delivered to their targets once, between windows:
//   - push (the normal case, activity is sparse): a warp per spike writes a deposit
//     {source key, step, STP value} into a fixed number of inbox slots per target;
//     the target sorts its deposits into CSR row order and sums them, which is
//     bit-identical to the reference's dense gather (its skipped terms are +0.0);
//   - pull (a busy window, or a target whose slots overflowed): the target walks its
//     CSR rows against the previous window's per-neuron spike words, exactly like
//     the per-step gather.
// SIC factors are pulled through a per-window "astrocyte active" bitmask, by the
// neurons that the push flagged: those whose a2n row holds an astrocyte that was
// active (the push walks each active astrocyte's forward a2n list), so a window
// without active astrocytes costs every other neuron one flag-word read.
#pragma once

#include "common.cuh"
#include "network.cuh"
#include "sim.cuh"

namespace astrosim {

constexpr int kMaxWindow = 16;  // windows up to 16 steps (D = 10 at dt = 0.1 ms)
constexpr int kInboxSlots = 8;  // deposits per target per window before it falls back to pull

template <typename R>
struct Deposit {
    u32 key;   // exc/inh: source neuron id (rows are sorted by it); e2a: position in the astrocyte's row
    u32 meta;  // step within the window | kind << 8 (0 excitatory, 1 inhibitory)
    R val;     // STP multiplier of the spike
};

// Source-keyed copies of the connectivity used by the push.
struct ForwardCSR {
    DevBuf<u32> exc_rs, exc_dst;            // excitatory source -> neuron targets
    DevBuf<u32> inh_rs, inh_dst;            // stored inhibitory id -> neuron targets
    DevBuf<u32> e2a_rs, e2a_astro, e2a_pos; // excitatory source -> (astrocyte, position in its row)
    DevBuf<u32> sic_rs, sic_dst;            // astrocyte -> neurons whose a2n rows hold it
    u32 max_fanout = 0;
};

struct WindowState {
    int W = 0;
    u32 push_limit = 0;
    ForwardCSR fwd;
    DevBuf<u32> nin_cnt, ain_cnt;             // [2][n] deposit counts
    DevBuf<unsigned char> nin_ent, ain_ent;   // [2][n][kInboxSlots] deposits
    DevBuf<u32> spk_word;                     // [2][n_neurons]: bit s = spiked at window step s
    DevBuf<unsigned char> spk_val;            // [2][W][n_neurons] real
    DevBuf<u32> spk_list;                     // [2][cap] (neuron << 5 | step)
    DevBuf<u32> spk_count;                    // [2]
    DevBuf<unsigned char> sic_win;            // [2][n_astro][W] real
    DevBuf<u32> astro_active;                 // [2][ceil(n_astro / 32)]
    DevBuf<u32> sic_flag;                     // [2][ceil(n_neurons / 32)]: a2n row holds an active astrocyte
    DevBuf<int> mode;                         // [2]: 0 push, 1 pull
    // autotuner: (block size, launch bounds) variant of window_kernel, an index into
    // its table; -1 while timing the candidates, -2 for the generic kernel (a block
    // size outside the table, nothing to tune)
    int variant = -1;
    int tune_step = 0;
    float tune_ms[9] = {1e30f, 1e30f, 1e30f, 1e30f, 1e30f, 1e30f, 1e30f, 1e30f, 1e30f};
    cudaEvent_t tune_ev[2] = {nullptr, nullptr};
    ~WindowState() {
        if (tune_ev[0]) cudaEventDestroy(tune_ev[0]);
        if (tune_ev[1]) cudaEventDestroy(tune_ev[1]);
    }
};

Status window_setup(const RunConsts& rc, Network& net, bool fp32, WindowState& ws, cudaStream_t st);

// Advances steps [first, first + count) with windows of ws.W steps.  `block` is the
// window kernel's block size (a multiple of 32); 0 lets the autotuner choose it.
Status window_launch(const RunConsts& rc, StateBuffers& sb, Network& net, bool fp32, WindowState& ws,
                     i64 raster_steps, i64 mark_step, i64 first, i64 count, cudaStream_t st, int block);

}  // namespace astrosim
