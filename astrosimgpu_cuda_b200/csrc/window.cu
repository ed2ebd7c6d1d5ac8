// window.cu -- windowed stepping: one launch per window of D steps plus one push
// launch between windows (see window.cuh).

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <map>
#include <tuple>
#include <mutex>
#include <type_traits>
#include <utility>

#include "window_kernels.cuh"

namespace astrosim {

namespace {

// Block and MinBlocks are the block size and the launch-bounds occupancy target
// (resident blocks per SM): the autotuner (window_launch) times the instantiated
// pairs on the first windows of a run and keeps the fastest.  The per-cell
// arithmetic is the same in every instantiation; the kernel indexes cells by
// blockDim.x, so Block = 1024 with MinBlocks = 1 serves any other block size.
template <typename R, int Block, int MinBlocks>
__global__ void __launch_bounds__(Block, MinBlocks) window_kernel(RunConsts rc, StepPtrs<R> p, WinPtrs<R> w,
                                                                  i64 win_start, int s_begin, int s_end, int buf,
                                                                  i64 mark, u32 astro_blocks) {
    const bool astro = blockIdx.x < astro_blocks;
    window_cells<R>(rc, net_scalars(rc), p, w, win_start, s_begin, s_end, buf, mark, astro ? blockIdx.x : blockIdx.x - astro_blocks,
                    astro);
}

template <typename R>
__global__ void push_kernel(WinPtrs<R> w, u32 n_exc, u32 n_inh, u64 n_neurons, u64 n_astro, int buf) {
    push_cells<R>(w, n_exc, n_inh, n_neurons, n_astro, buf, blockIdx.x, gridDim.x);
}

// ------------------------------------------------------------------ forward CSRs
// One warp per target row, so that a row's entries are written by adjacent lanes.
__global__ void edge_rows_kernel(const u32* rs, u32 n_rows, u32* row_of_edge) {
    const u64 r = (static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    if (r >= n_rows) return;
    const u32 end = rs[r + 1];
    for (u32 k = rs[r] + (threadIdx.x & 31u); k < end; k += 32) row_of_edge[k] = static_cast<u32>(r);
}

__global__ void iota_kernel(u32* v, u64 n) {
    const u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) v[i] = static_cast<u32>(i);
}

__global__ void lower_bound_rows_kernel(const u32* sorted_keys, u64 n, u32 n_rows, u32* rs) {
    const u64 t = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t > n_rows) return;
    u64 lo = 0, hi = n;
    while (lo < hi) {
        const u64 mid = (lo + hi) >> 1;
        if (sorted_keys[mid] < t) lo = mid + 1; else hi = mid;
    }
    rs[t] = static_cast<u32>(lo);
}

__global__ void gather_fwd_kernel(const u32* edge_idx, u64 n, const u32* row_of_edge, const u32* tgt_rs, u32 row0,
                                  u32* dst, u32* pos) {
    const u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const u32 e = edge_idx[i];
    const u32 r = row_of_edge[e];
    dst[i] = r + row0;
    if (pos) pos[i] = e - tgt_rs[r];
}

__global__ void add_offset_kernel(u32* v, u64 n, u32 off) {
    const u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) v[i] += off;
}

// Inverts a target-keyed CSR into a source-keyed one.  Within one source the
// targets come out in increasing edge order (stable sort), which the push does not
// depend on; positions let e2a deposits name their place in the target row.  Row r
// of `c` is target row0 + r (a network that keeps only its owned cells' rows), and
// the forward lists hold target ids.
Status invert_csr(const DeviceCSR& c, u32 row0, u32 n_sources, DevBuf<u32>& rs, DevBuf<u32>& dst, DevBuf<u32>* pos,
                  cudaStream_t st) {
    const u64 n = c.n_edges;
    AS_TRY(rs.alloc(static_cast<size_t>(n_sources) + 1));
    AS_TRY(dst.alloc(n));
    if (pos) AS_TRY(pos->alloc(n));
    if (n == 0) {
        AS_CUDA(cudaMemsetAsync(rs.get(), 0, rs.bytes(), st));
        return Status::Ok();
    }
    DevBuf<u32> row_of, keys_out;
    AS_TRY(row_of.alloc(n));
    AS_TRY(keys_out.alloc(n));
    edge_rows_kernel<<<ceil_div(static_cast<u64>(c.n_targets) * 32, 256), 256, 0, st>>>(c.row_start.get(), c.n_targets,
                                                                                     row_of.get());
    AS_CUDA(cudaGetLastError());
    int end_bit = 1;
    while (end_bit < 32 && (1ull << end_bit) < static_cast<u64>(n_sources) + 1) ++end_bit;
    size_t tb = 0;
    if (!pos) {
        // Sorting the target rows themselves by source gives the forward lists
        // directly (the same lists as the edge-index route below, without its index
        // arrays and gather pass).
        AS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, c.src.get(), keys_out.get(), row_of.get(), dst.get(), n,
                                                0, end_bit, st));
        DevBuf<unsigned char> tmp;
        AS_TRY(tmp.alloc(tb));
        AS_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tb, c.src.get(), keys_out.get(), row_of.get(), dst.get(),
                                                n, 0, end_bit, st));
        lower_bound_rows_kernel<<<ceil_div(static_cast<u64>(n_sources) + 1, 256), 256, 0, st>>>(keys_out.get(), n,
                                                                                              n_sources, rs.get());
        if (row0) add_offset_kernel<<<ceil_div(n, 256), 256, 0, st>>>(dst.get(), n, row0);
        AS_CUDA(cudaGetLastError());
        AS_CUDA(cudaStreamSynchronize(st));
        return Status::Ok();
    }
    DevBuf<u32> idx_in, idx_out;
    AS_TRY(idx_in.alloc(n));
    AS_TRY(idx_out.alloc(n));
    iota_kernel<<<ceil_div(n, 256), 256, 0, st>>>(idx_in.get(), n);
    AS_CUDA(cudaGetLastError());
    AS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, c.src.get(), keys_out.get(), idx_in.get(), idx_out.get(), n,
                                            0, end_bit, st));
    DevBuf<unsigned char> tmp;
    AS_TRY(tmp.alloc(tb));
    AS_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tb, c.src.get(), keys_out.get(), idx_in.get(), idx_out.get(), n,
                                            0, end_bit, st));
    lower_bound_rows_kernel<<<ceil_div(static_cast<u64>(n_sources) + 1, 256), 256, 0, st>>>(keys_out.get(), n,
                                                                                          n_sources, rs.get());
    gather_fwd_kernel<<<ceil_div(n, 256), 256, 0, st>>>(idx_out.get(), n, row_of.get(), c.row_start.get(), row0,
                                                        dst.get(), pos->get());
    AS_CUDA(cudaGetLastError());
    AS_CUDA(cudaStreamSynchronize(st));
    return Status::Ok();
}

}  // namespace

Status window_setup(const RunConsts& rc, Network& net, bool fp32, WindowState& ws, cudaStream_t st) {
    ws.W = rc.d_e;
    const u64 nN = rc.n_neurons, nA = rc.n_astro;
    const size_t rb = fp32 ? sizeof(float) : sizeof(double);
    const size_t db = fp32 ? sizeof(Deposit<float>) : sizeof(Deposit<double>);
    // a rank of a sharded network keeps its own cells' rows: its forward lists reach its own cells only
    if (net.has_fwd && net.fwd_exc_rs.size() == static_cast<size_t>(rc.n_exc) + 1 &&
        net.fwd_inh_rs.size() == static_cast<size_t>(net.sz.n_inh) + 1) {
        // the builder wrote these lists while emitting the edges, with the owned rows'
        // indices (cell - n_lo); the forward lists hold target ids
        ws.fwd.exc_rs = std::move(net.fwd_exc_rs);
        ws.fwd.exc_dst = std::move(net.fwd_exc_dst);
        ws.fwd.inh_rs = std::move(net.fwd_inh_rs);
        ws.fwd.inh_dst = std::move(net.fwd_inh_dst);
        net.has_fwd = false;
        if (net.own.n_lo) {
            if (net.exc.n_edges)
                add_offset_kernel<<<ceil_div(net.exc.n_edges, 256), 256, 0, st>>>(ws.fwd.exc_dst.get(),
                                                                                 net.exc.n_edges, net.own.n_lo);
            if (net.inh.n_edges)
                add_offset_kernel<<<ceil_div(net.inh.n_edges, 256), 256, 0, st>>>(ws.fwd.inh_dst.get(),
                                                                                 net.inh.n_edges, net.own.n_lo);
            AS_CUDA(cudaGetLastError());
        }
    } else {
        net.drop_forward();
        AS_TRY(invert_csr(net.exc, net.own.n_lo, rc.n_exc, ws.fwd.exc_rs, ws.fwd.exc_dst, nullptr, st));
        AS_TRY(invert_csr(net.inh, net.own.n_lo, net.sz.n_inh, ws.fwd.inh_rs, ws.fwd.inh_dst, nullptr, st));
    }
    AS_TRY(invert_csr(net.e2a, net.own.a_lo, rc.n_exc, ws.fwd.e2a_rs, ws.fwd.e2a_astro, &ws.fwd.e2a_pos, st));
    AS_TRY(invert_csr(net.sic, net.own.n_lo, rc.n_astro, ws.fwd.sic_rs, ws.fwd.sic_dst, nullptr, st));
    // Windows with more spikes than this use the pull gather instead of deposits.
    // ASTROSIM_PUSH_LIMIT overrides it (the tests force the pull path with 0).
    ws.push_limit = static_cast<u32>(std::max<u64>(1024, nN / 50));
    if (const char* env = std::getenv("ASTROSIM_PUSH_LIMIT")) ws.push_limit = static_cast<u32>(std::strtoul(env, nullptr, 10));
    const u32 cap = ws.push_limit + 1;
    AS_TRY(ws.nin_cnt.alloc_zero(2 * nN, st));
    AS_TRY(ws.ain_cnt.alloc_zero(2 * nA, st));
    AS_TRY(ws.nin_ent.alloc(2 * nN * kInboxSlots * db));
    AS_TRY(ws.ain_ent.alloc(2 * nA * kInboxSlots * db));
    AS_TRY(ws.spk_word.alloc_zero(2 * nN, st));
    AS_TRY(ws.spk_val.alloc_zero(2 * static_cast<u64>(ws.W) * nN * rb, st));
    AS_TRY(ws.spk_list.alloc(2 * static_cast<u64>(cap)));
    AS_TRY(ws.spk_count.alloc_zero(2, st));
    AS_TRY(ws.sic_win.alloc_zero(2 * nA * ws.W * rb, st));
    AS_TRY(ws.astro_active.alloc_zero(2 * ((nA + 31) / 32), st));
    AS_TRY(ws.sic_flag.alloc_zero(2 * ((nN + 31) / 32), st));
    AS_TRY(ws.mode.alloc_zero(2, st));
    AS_CUDA(cudaStreamSynchronize(st));
    return Status::Ok();
}

namespace {

// Variants the autotuner chooses from: (block size, minimum resident blocks per SM).
// Each block size comes with three occupancy targets (the same threads per SM as
// the 128-thread entries), trading registers (and a few spills) for occupancy.
struct Variant {
    int block, min_blocks;
};
constexpr Variant kVariantsF32[] = {{128, 6}, {128, 8}, {128, 4}, {64, 12}, {64, 16}, {64, 8},
                                    {256, 3}, {256, 4}, {256, 2}};
constexpr Variant kVariantsF64[] = {{128, 4}, {128, 5}, {128, 3}, {64, 8}, {64, 10}, {64, 6},
                                    {256, 2}, {256, 3}, {256, 1}};
constexpr int kNumVariants = 9;
constexpr int kVariantsPerBlock = 3;
constexpr int kTuneRounds = 2;
static_assert(sizeof(kVariantsF32) / sizeof(Variant) == kNumVariants, "variant table");
static_assert(sizeof(kVariantsF64) / sizeof(Variant) == kNumVariants, "variant table");

// The variants a run may use: every entry for block 0 (the autotuned choice), the
// three entries of a tuned block size, or the generic instantiation (index -1) for
// any other requested block size.
void variant_range(int block, int* first, int* count) {
    for (int b = 0; b < kNumVariants / kVariantsPerBlock; ++b)
        if (kVariantsF32[b * kVariantsPerBlock].block == block) {
            *first = b * kVariantsPerBlock;
            *count = kVariantsPerBlock;
            return;
        }
    if (block == 0) {
        *first = 0;
        *count = kNumVariants;
        return;
    }
    *first = -1;
    *count = 0;
}

std::mutex g_tune_mu;
std::map<std::tuple<int, int, int>, int> g_tuned;  // (precision, log2 size bucket, requested block) -> variant

template <typename R, int B, int M>
void launch_one(u32 cells_astro, u32 cells_neuron, cudaStream_t st, const RunConsts& rc, const StepPtrs<R>& p,
                const WinPtrs<R>& w, i64 start, int s0, int s1, int buf, i64 mark, int block) {
    const u32 astro_blocks = ceil_div(cells_astro, block);
    const u32 grid = astro_blocks + ceil_div(cells_neuron, block);
    window_kernel<R, B, M><<<grid, block, 0, st>>>(rc, p, w, start, s0, s1, buf, mark, astro_blocks);
}

// Launches variant `variant` (an index into the table; -1 = the generic kernel at
// `block` threads).
template <typename R>
void launch_window(int variant, int block, cudaStream_t st, const RunConsts& rc, const StepPtrs<R>& p,
                   const WinPtrs<R>& w, i64 start, int s0, int s1, int buf, i64 mark) {
    constexpr bool f32 = std::is_same<R, float>::value;
    const u32 nA = rc.n_astro, nN = rc.n_neurons;
#define AS_WIN(B, M) launch_one<R, B, M>(nA, nN, st, rc, p, w, start, s0, s1, buf, mark, B)
    if (variant < 0) {
        launch_one<R, 1024, 1>(nA, nN, st, rc, p, w, start, s0, s1, buf, mark, block);
        return;
    }
    const Variant v = f32 ? kVariantsF32[variant] : kVariantsF64[variant];
    if constexpr (f32) {
        switch (v.block * 100 + v.min_blocks) {
            case 12804: AS_WIN(128, 4); break;
            case 12808: AS_WIN(128, 8); break;
            case 6412: AS_WIN(64, 12); break;
            case 6416: AS_WIN(64, 16); break;
            case 6408: AS_WIN(64, 8); break;
            case 25603: AS_WIN(256, 3); break;
            case 25604: AS_WIN(256, 4); break;
            case 25602: AS_WIN(256, 2); break;
            default: AS_WIN(128, 6); break;
        }
    } else {
        switch (v.block * 100 + v.min_blocks) {
            case 12803: AS_WIN(128, 3); break;
            case 12805: AS_WIN(128, 5); break;
            case 6408: AS_WIN(64, 8); break;
            case 6410: AS_WIN(64, 10); break;
            case 6406: AS_WIN(64, 6); break;
            case 25602: AS_WIN(256, 2); break;
            case 25603: AS_WIN(256, 3); break;
            case 25601: AS_WIN(256, 1); break;
            default: AS_WIN(128, 4); break;
        }
    }
#undef AS_WIN
}

template <typename R>
Status launch_impl(const RunConsts& rc, StateBuffers& sb, Network& net, WindowState& ws, i64 raster_steps, i64 mark,
                   i64 first, i64 count, cudaStream_t st, int block) {
    constexpr bool f32 = std::is_same<R, float>::value;
    StepPtrs<R> p = make_ptrs<R>(sb, net, rc, raster_steps);
    WinPtrs<R> w = win_ptrs<R>(ws, rc);
    const int W = ws.W;
    const u32 push_blocks = std::max<u32>(1, std::min<u32>(sm_count() * 8, ceil_div(ws.push_limit, 8)));
    int v_first = 0, v_count = 0;
    variant_range(block, &v_first, &v_count);
    if (v_first < 0) ws.variant = -2;  // a block size outside the table: the generic kernel, nothing to tune
    int bucket = 0;
    while ((1ull << bucket) < rc.n_neurons) ++bucket;
    const std::tuple<int, int, int> key{f32 ? 1 : 0, bucket, block};
    if (ws.variant == -1) {
        if (const char* env = std::getenv("ASTROSIM_WINDOW_VARIANT")) {
            ws.variant = v_first + std::min(v_count - 1, std::max(0, std::atoi(env)));
        } else {
            std::lock_guard<std::mutex> lock(g_tune_mu);
            auto it = g_tuned.find(key);
            if (it != g_tuned.end()) ws.variant = it->second;
        }
    }
    i64 t = first;
    const i64 end = first + count;
    while (t < end) {
        const i64 k = t / W;
        const int s0 = static_cast<int>(t - k * W);
        const int s1 = static_cast<int>(std::min<i64>(W, end - k * W));
        const int buf = static_cast<int>(k & 1);
        const bool tuning = ws.variant == -1 && s0 == 0 && s1 == W;
        int v = ws.variant >= 0 ? ws.variant : (tuning ? v_first + ws.tune_step % v_count : v_first);
        if (ws.variant == -2) v = -1;
        if (tuning && !ws.tune_ev[0]) {  // made on the first tuned window only
            AS_CUDA(cudaEventCreate(&ws.tune_ev[0]));
            AS_CUDA(cudaEventCreate(&ws.tune_ev[1]));
        }
        if (tuning) AS_CUDA(cudaEventRecord(ws.tune_ev[0], st));
        launch_window<R>(v, block, st, rc, p, w, k * W, s0, s1, buf, mark);
        AS_CUDA(cudaGetLastError());
        if (tuning) {
            AS_CUDA(cudaEventRecord(ws.tune_ev[1], st));
            AS_CUDA(cudaEventSynchronize(ws.tune_ev[1]));
            float ms = 0.f;
            AS_CUDA(cudaEventElapsedTime(&ms, ws.tune_ev[0], ws.tune_ev[1]));
            float& slot = ws.tune_ms[v];
            slot = std::min(slot, ms);  // min over rounds: the first launch also loads the kernel
            if (++ws.tune_step == v_count * kTuneRounds) {
                int best = v_first;
                for (int i = v_first + 1; i < v_first + v_count; ++i)
                    if (ws.tune_ms[i] < ws.tune_ms[best]) best = i;
                ws.variant = best;
                std::lock_guard<std::mutex> lock(g_tune_mu);
                g_tuned[key] = best;
            }
        }
        if (s1 == W) {
            push_kernel<R><<<push_blocks, 256, 0, st>>>(w, rc.n_exc, net.sz.n_inh, rc.n_neurons, rc.n_astro, buf);
            AS_CUDA(cudaGetLastError());
        }
        t = k * W + s1;
    }
    return Status::Ok();
}
}  // namespace

Status window_launch(const RunConsts& rc, StateBuffers& sb, Network& net, bool fp32, WindowState& ws,
                     i64 raster_steps, i64 mark_step, i64 first, i64 count, cudaStream_t st, int block) {
    if (fp32) return launch_impl<float>(rc, sb, net, ws, raster_steps, mark_step, first, count, st, block);
    return launch_impl<double>(rc, sb, net, ws, raster_steps, mark_step, first, count, st, block);
}

}  // namespace astrosim
