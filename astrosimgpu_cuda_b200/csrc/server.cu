// server.cu -- the serving loop: continuous batching of simulation requests.
//
// Requests (one astrosim_config each) queue FIFO.  A request is admitted when its
// estimated device footprint fits the HBM budget next to everything admitted
// before it; builder threads then build its network on their own streams, which
// overlap the batch that is stepping.  Built networks join the running ensemble
// between windows, every running network advances one window per window launch,
// and a network that reaches its last step is summarised and retired, returning
// its memory to the budget.  A request's result is bit-identical to running it
// alone (the batch shares launches, not arithmetic).

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "biology.cuh"
#include "ensemble.cuh"
#include "server.cuh"

namespace astrosim {

namespace {
double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
}  // namespace

u64 Server::estimate_bytes(const astrosim_config& cfg) {
    // Resident: target and source-keyed CSRs (~8 B per synapse, 116 synapses per
    // neuron), state and window buffers (~300 B per neuron); while building, edge
    // lists, the skip cache and sort buffers roughly double that.  Measured at
    // N = 1e7 the resident total is about 15 GB.
    const double n = cfg.n_total;
    return static_cast<u64>(n * 3200.0) + (64ull << 20);
}

Server::~Server() {
    {
        std::lock_guard<std::mutex> lk(mu_);
        stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : builders_) t.join();
    ens_.reset();
}

Status Server::create(int device, int precision, u64 budget, int builder_threads) {
    if (precision != ASTROSIM_PRECISION_FP64 && precision != ASTROSIM_PRECISION_FP32)
        return make_error(ASTROSIM_ERR_INVALID_ARG, "unknown precision");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return make_error(ASTROSIM_ERR_NO_DEVICE, "no CUDA device visible");
    }
    if (device < 0 || device >= ndev) return make_error(ASTROSIM_ERR_INVALID_ARG, "device out of range");
    device_ = device;
    precision_ = precision;
    AS_CUDA(cudaSetDevice(device_));
    if (budget == 0) {
        size_t free_b = 0, total_b = 0;
        AS_CUDA(cudaMemGetInfo(&free_b, &total_b));
        budget = static_cast<u64>(static_cast<double>(free_b) * 0.85);
    }
    budget_ = budget;
    ens_ = std::make_unique<Ensemble>();
    // the window is fixed by dt; requests must share the default 0.1 ms step
    AS_TRY(ens_->init_empty(precision == ASTROSIM_PRECISION_FP32, delay_to_steps(1.0, 0.1), device_));
    const int nb = std::max(1, std::min(32, builder_threads));
    for (int i = 0; i < nb; ++i) builders_.emplace_back([this] { builder_loop(); });
    t0_ = now_s();
    return Status::Ok();
}

void Server::builder_loop() {
    cudaSetDevice(device_);
    for (;;) {
        std::shared_ptr<Request> r;
        {
            std::unique_lock<std::mutex> lk(mu_);
            cv_.wait(lk, [&] { return stop_ || !build_queue_.empty(); });
            if (stop_) return;
            r = build_queue_.front();
            build_queue_.pop_front();
            ++n_inflight_;
        }
        const double tb = now_s();
        auto sim = std::make_unique<Simulation>();
        Status s = sim->create(r->cfg, r->biology.empty() ? nullptr : r->biology.c_str());
        std::lock_guard<std::mutex> lk(mu_);
        --n_inflight_;
        r->build_s = now_s() - tb;
        if (!s.ok()) {
            r->status = s;
            r->done = true;
            r->done_t = now_s();
            in_use_ -= r->bytes;
            ++n_done_;
            ++n_failed_;
        } else {
            r->sim = std::move(sim);
            built_.push_back(r);
        }
    }
}

Status Server::submit(const astrosim_config& cfg, u64* id, const char* biology_json) {
    if (cfg.dt != 0.1 || cfg.substeps < 1 || cfg.precision != precision_)
        return make_error(ASTROSIM_ERR_INVALID_ARG, "requests must use dt 0.1 ms and the server's precision");
    auto r = std::make_shared<Request>();
    r->cfg = cfg;
    r->cfg.device = device_;
    if (biology_json) {
        Biology check;  // reject bad overrides at submission, not in a builder thread
        AS_TRY(apply_biology_json(biology_json, check));
        r->biology = biology_json;
    }
    r->bytes = estimate_bytes(cfg);
    if (r->bytes > budget_)
        return make_error(ASTROSIM_ERR_OUT_OF_MEMORY, "request needs about %llu bytes, more than the budget",
                          static_cast<unsigned long long>(r->bytes));
    std::lock_guard<std::mutex> lk(mu_);
    r->id = next_id_++;
    r->submit_t = now_s();
    requests_[r->id] = r;
    pending_.push_back(r);
    *id = r->id;
    return Status::Ok();
}

Status Server::pump(i64 windows) {
    AS_CUDA(cudaSetDevice(device_));
    // 1. admission by footprint, FIFO
    {
        std::lock_guard<std::mutex> lk(mu_);
        bool woke = false;
        while (!pending_.empty() && in_use_ + pending_.front()->bytes <= budget_) {
            auto r = pending_.front();
            pending_.pop_front();
            in_use_ += r->bytes;
            r->admit_t = now_s();
            build_queue_.push_back(r);
            woke = true;
        }
        if (woke) cv_.notify_all();
    }
    // 2. built networks join the batch between windows
    std::vector<std::shared_ptr<Request>> joined;
    {
        std::lock_guard<std::mutex> lk(mu_);
        joined.swap(built_);
    }
    for (auto& r : joined) {
        r->start_t = now_s();
        AS_TRY(ens_->add(std::move(r->sim)));
        // the slot is the one add() filled: find it by scanning for an unowned active slot
        for (u32 i = 0; i < ens_->size(); ++i) {
            if (ens_->active(i) && slot_owner_.count(i) == 0) {
                slot_owner_[i] = r;
                break;
            }
        }
    }
    // 3. one window per launch for every running network
    if (!slot_owner_.empty() && windows > 0) AS_TRY(ens_->advance_windows(windows));
    // 4. finished networks: summary, retire, release their budget
    std::vector<u32> finished;
    for (auto& kv : slot_owner_) {
        Simulation* s = ens_->net(kv.first);
        if (s->steps_done() >= s->total_steps()) finished.push_back(kv.first);
    }
    for (u32 slot : finished) {
        auto r = slot_owner_[slot];
        AS_TRY(ens_->summary(slot, r->summary));
        AS_TRY(ens_->retire(slot));
        slot_owner_.erase(slot);
        std::lock_guard<std::mutex> lk(mu_);
        r->done = true;
        r->done_t = now_s();
        in_use_ -= r->bytes;
        ++n_done_;
    }
    return Status::Ok();
}

Status Server::result(u64 id, astrosim_request_result& out, bool* done) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = requests_.find(id);
    if (it == requests_.end()) return make_error(ASTROSIM_ERR_INVALID_ARG, "unknown request %llu",
                                                 static_cast<unsigned long long>(id));
    const Request& r = *it->second;
    *done = r.done;
    if (!r.done) return Status::Ok();
    if (!r.status.ok()) return r.status;
    out.summary = r.summary;
    out.latency_s = r.done_t - r.submit_t;
    out.queue_s = r.admit_t - r.submit_t;
    out.build_s = r.build_s;
    out.run_s = r.done_t - r.start_t;
    return Status::Ok();
}

void Server::stats(astrosim_server_stats& s) {
    std::lock_guard<std::mutex> lk(mu_);
    s.submitted = next_id_ - 1;
    s.done = n_done_;
    s.failed = n_failed_;
    s.pending = pending_.size();
    s.building = build_queue_.size() + n_inflight_ + built_.size();
    s.running = slot_owner_.size();
    s.bytes_in_use = in_use_;
    s.budget_bytes = budget_;
    s.uptime_s = now_s() - t0_;
}

}  // namespace astrosim
