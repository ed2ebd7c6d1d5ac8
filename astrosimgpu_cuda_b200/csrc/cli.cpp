// cli.cpp -- command-line driver with the reference program's flags and printed
// lines (src/astrosim_fused.cu:791-1141), running on the C ABI of libastrosim_b200.
//
// Flags, defaults and the NaN "not overridden" sentinel follow
// src/astrosim_fused.cu:792-844.  Three flags are added: --precision fp64|fp32,
// --device N and --biology FILE (a JSON object of biology constants).  The summary lines keep the reference's formats, which
// scripts/run_gh200.sbatch:56-61 scrapes.  Differences: connectivity is built on the
// GPU, so --dump-edges needs a device; the windowed-rate lines are printed at the
// same steps from per-step spike counts.

#include <algorithm>
#include <fstream>
#include <sstream>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/astrosim.h"

namespace {

int die(const char* what) {
    std::fprintf(stderr, "%s failed: %s\n", what, astrosim_last_error());
    return 1;
}

void print_help() {
    std::printf(
        "astrosim --n N_total [--seed S] [--dt 0.1] [--substeps 1] "
        "[--pre-ms 1000] [--sim-ms 5000] [--block N]\n"
        "         [--w-n2a W] [--w-a2n W] [--no-stp] [--dump-edges PATH]\n"
        "         [--precision fp64|fp32] [--device N] [--biology FILE.json]\n"
        "N_total is split by the fixed-in-degree scaling law: N_E=0.8*N, N_I=0.2*N,\n"
        "N_A=N/5, p_primary=80/N_E.  --w-n2a/--w-a2n override the neuron->astrocyte /\n"
        "astrocyte->neuron coupling weight (default 0.2 / 1.0); 0 disconnects that\n"
        "direction.  --no-stp disables Tsodyks-Markram short-term plasticity.\n"
        "--dump-edges PATH writes the network as type,source,target CSV and exits.\n"
        "--block N sets the CUDA block size of the cell kernels (the reference uses\n"
        "128); without it the autotuner picks the block size and occupancy.\n"
        "--precision fp32 runs RK4 stages in float with double accumulators.\n"
        "--biology FILE reads a JSON object of biology constants to override, e.g.\n"
        "{\"exc_poiss_rate\": 3000, \"stp_U\": 0.4}; the flags above apply on top.\n"
        "Connectivity and every time step run on the GPU.\n");
}

}  // namespace

int main(int argc, char** argv) {
    astrosim_config cfg;
    astrosim_config_default(&cfg);
    std::string dump_path, biology;
    bool w_over = false;
    for (int i = 1; i < argc; ++i) {
        auto arg = [&](const char* name) { return std::strcmp(argv[i], name) == 0; };
        auto next = [&]() -> const char* { return (i + 1 < argc) ? argv[++i] : ""; };
        if (arg("--n") || arg("-n")) cfg.n_total = static_cast<uint32_t>(std::atoll(next()));
        else if (arg("--seed")) cfg.seed = static_cast<uint64_t>(std::atoll(next()));
        else if (arg("--dt")) cfg.dt = std::atof(next());
        else if (arg("--substeps")) cfg.substeps = std::atoi(next());
        else if (arg("--pre-ms")) cfg.pre_ms = std::atof(next());
        else if (arg("--sim-ms")) cfg.sim_ms = std::atof(next());
        else if (arg("--block")) cfg.block = std::atoi(next());
        else if (arg("--w-n2a")) { cfg.w_n2a = std::atof(next()); w_over = true; }
        else if (arg("--w-a2n")) { cfg.w_a2n = std::atof(next()); w_over = true; }
        else if (arg("--no-stp")) cfg.stp_enabled = 0;
        else if (arg("--dump-edges")) dump_path = next();
        else if (arg("--precision")) {
            const std::string v = next();
            if (v == "fp64" || v == "double") cfg.precision = ASTROSIM_PRECISION_FP64;
            else if (v == "fp32" || v == "float") cfg.precision = ASTROSIM_PRECISION_FP32;
            else { std::fprintf(stderr, "unknown precision: %s\n", v.c_str()); return 1; }
        } else if (arg("--device")) cfg.device = std::atoi(next());
        else if (arg("--biology")) {
            const std::string path = next();
            std::ifstream f(path);
            if (!f) { std::fprintf(stderr, "cannot read %s for --biology\n", path.c_str()); return 1; }
            std::stringstream ss;
            ss << f.rdbuf();
            biology = ss.str();
            double probe = 0.0;
            if (astrosim_biology_value(biology.c_str(), "w_e", &probe) != ASTROSIM_OK) {
                std::fprintf(stderr, "--biology %s: %s\n", path.c_str(), astrosim_last_error());
                return 1;
            }
        }
        else if (arg("--help") || arg("-h")) { print_help(); return 0; }
        else {
            std::fprintf(stderr, "unknown argument: %s (try --help)\n", argv[i]);
            return 1;
        }
    }

    const uint32_t n_total = cfg.n_total;
    const uint32_t n_exc = std::max<uint32_t>(1, static_cast<uint32_t>(std::lround(n_total * 0.8)));
    const uint32_t n_inh = std::max<uint32_t>(1, n_total - n_exc);
    const uint32_t n_astro = std::max<uint32_t>(1, static_cast<uint32_t>(std::lround(n_total / 5.0)));
    const double p = std::min(1.0, 80.0 / static_cast<double>(n_exc));
    double w_n2a = cfg.w_n2a, w_a2n = cfg.w_a2n;
    if (std::isnan(w_n2a)) astrosim_biology_value(biology.c_str(), "w_n2a", &w_n2a);
    if (std::isnan(w_a2n)) astrosim_biology_value(biology.c_str(), "w_a2n", &w_a2n);
    std::printf("=== astrosim: tripartite neuron-astrocyte network on B200 ===\n");
    std::printf("N_total=%u  N_E=%u  N_I=%u  N_A=%u  p_primary=%.6g  (fixed in-degree law, K_SYN=%.0f)\n", n_total,
                n_exc, n_inh, n_astro, p, 80.0);
    std::printf("w_n2a=%g  w_a2n=%g%s\n", w_n2a, w_a2n, w_over ? "  (overridden)" : "");
    std::printf("dt=%g ms  substeps=%d  pre=%g ms  sim=%g ms  seed=%llu  precision=%s\n", cfg.dt, cfg.substeps,
                cfg.pre_ms, cfg.sim_ms, static_cast<unsigned long long>(cfg.seed),
                cfg.precision == ASTROSIM_PRECISION_FP32 ? "float" : "double");
    std::fflush(stdout);

    astrosim_handle* h = nullptr;
    if (astrosim_create_with_biology(&cfg, biology.empty() ? nullptr : biology.c_str(), &h) != ASTROSIM_OK) {
        if (std::strstr(astrosim_last_error(), "no CUDA device")) {
            std::fprintf(stderr, "No CUDA device visible: connectivity and stepping run on the GPU.\n");
            return 1;
        }
        return die("astrosim_create");
    }
    astrosim_summary_t s;
    if (astrosim_summary(h, &s) != ASTROSIM_OK) return die("astrosim_summary");
    std::printf("connectivity: exc=%llu inh=%llu e2a=%llu sic=%llu edges, built in %.3f s\n",
                static_cast<unsigned long long>(s.n_exc_edges), static_cast<unsigned long long>(s.n_inh_edges),
                static_cast<unsigned long long>(s.n_e2a_edges), static_cast<unsigned long long>(s.n_sic_edges),
                s.build_seconds);
    if (!dump_path.empty()) {
        if (astrosim_dump_edges(h, dump_path.c_str()) != ASTROSIM_OK) {
            std::fprintf(stderr, "cannot open %s for --dump-edges\n", dump_path.c_str());
            astrosim_destroy(h);
            return 1;
        }
        std::printf("Wrote edge list to %s\n", dump_path.c_str());
        astrosim_destroy(h);
        return 0;
    }
    char name[256];
    int major = 0, minor = 0;
    if (astrosim_device_info(cfg.device, name, sizeof(name), &major, &minor) == ASTROSIM_OK)
        std::printf("GPU: %s (sm_%d%d)\n", name, major, minor);

    // time loop with the reference's checkpoints (src/astrosim_fused.cu:1029-1102)
    const int64_t pre = s.pre_steps, sim = s.sim_steps, total = s.total_steps;
    const int64_t checkpoint_every = std::max<int64_t>(1, sim / 10);
    const uint32_t n_neurons = s.n_exc + s.n_inh;
    std::vector<int64_t> marks;  // steps after which a windowed rate is printed
    for (int64_t st = pre + checkpoint_every; st < total; st += checkpoint_every) marks.push_back(st);
    int64_t done = 0, last_cp = pre;
    uint64_t spikes_at_last = 0;
    std::vector<uint32_t> counts;
    auto spikes_upto = [&](int64_t inclusive) -> uint64_t {
        uint64_t t = 0;
        counts.resize(static_cast<size_t>(inclusive + 1));
        if (astrosim_spike_counts(h, 0, inclusive + 1, counts.data()) != ASTROSIM_OK) return 0;
        for (uint32_t c : counts) t += c;
        return t;
    };
    auto run_to = [&](int64_t upto) -> bool {  // run steps [done, upto)
        if (upto <= done) return true;
        if (astrosim_step(h, upto - done) != ASTROSIM_OK) return false;
        done = upto;
        return true;
    };
    const int64_t pre_mark = pre == 0 ? 0 : pre - 1;
    if (total > 0) {
        if (!run_to(std::min(total, pre_mark + 1))) return die("astrosim_step");
        spikes_at_last = spikes_upto(std::min(total - 1, pre_mark));
    }
    for (int64_t m : marks) {
        if (!run_to(m + 1)) return die("astrosim_step");
        if (m <= last_cp) continue;
        const uint64_t now = spikes_upto(m);
        const int64_t window_steps = m - last_cp;
        const double window_s = window_steps * cfg.dt * 1e-3;
        const double hz = static_cast<double>(now - spikes_at_last) / (static_cast<double>(n_neurons) * window_s);
        std::printf("  step %8lld / %8lld (%5.1f%%)  windowed rate: %.4f Hz\n", static_cast<long long>(m),
                    static_cast<long long>(total), 100.0 * m / total, hz);
        std::fflush(stdout);
        spikes_at_last = now;
        last_cp = m;
    }
    if (!run_to(total)) return die("astrosim_step");
    if (astrosim_summary(h, &s) != ASTROSIM_OK) return die("astrosim_summary");

    // src/astrosim_fused.cu:1131-1141
    std::printf("\n=== done ===\n");
    std::printf("wall time            : %.3f s for %lld steps (%.2f us/step, both kernels)\n", s.run_seconds,
                static_cast<long long>(total), total ? s.run_seconds * 1e6 / static_cast<double>(total) : 0.0);
    std::printf("spikes (recorded win): %llu\n", static_cast<unsigned long long>(s.spikes_measured));
    std::printf("mean firing rate     : %.4f Hz\n", s.mean_rate_hz);
    std::printf("mean calcium (final) : %.6g uM  (SIC_th=%.6g uM)\n", s.mean_ca, s.sic_th);
    std::printf("astrocytes active    : %u / %u (Ca above SIC threshold at the final step only)\n", s.active_astro,
                s.n_astro);
    std::printf("astrocytes engaged   : %u / %u (Ca crossed SIC threshold at ANY point in the "
                "recorded window -- comparable to astrosimgpu's 'astrocytes with transients')\n",
                s.engaged_astro, s.n_astro);
    astrosim_destroy(h);
    return 0;
}
