// server.cuh -- continuous-batching request loop over the ensemble engine.
#pragma once

#include <string>

#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "common.cuh"
#include "ensemble.cuh"
#include "sim.cuh"

namespace astrosim {

class Server {
public:
    ~Server();
    Status create(int device, int precision, u64 budget_bytes, int builder_threads);
    Status submit(const astrosim_config& cfg, u64* id, const char* biology_json = nullptr);
    Status pump(i64 windows);
    Status result(u64 id, astrosim_request_result& out, bool* done);
    void stats(astrosim_server_stats& s);
    static u64 estimate_bytes(const astrosim_config& cfg);

private:
    struct Request {
        u64 id = 0;
        astrosim_config cfg{};
        std::string biology;  // JSON overrides of the biology constants ("" = none)
        u64 bytes = 0;
        double submit_t = 0, admit_t = 0, start_t = 0, done_t = 0, build_s = 0;
        std::unique_ptr<Simulation> sim;
        astrosim_summary_t summary{};
        Status status;
        bool done = false;
    };
    void builder_loop();

    int device_ = 0;
    int precision_ = 0;
    u64 budget_ = 0, in_use_ = 0;
    u64 next_id_ = 1, n_done_ = 0, n_failed_ = 0, n_inflight_ = 0;
    double t0_ = 0;
    std::unique_ptr<Ensemble> ens_;
    std::mutex mu_;
    std::condition_variable cv_;
    bool stop_ = false;
    std::deque<std::shared_ptr<Request>> pending_, build_queue_;
    std::vector<std::shared_ptr<Request>> built_;
    std::map<u64, std::shared_ptr<Request>> requests_;
    std::map<u32, std::shared_ptr<Request>> slot_owner_;
    std::vector<std::thread> builders_;
};

}  // namespace astrosim
