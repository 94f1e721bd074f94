// ne2b_handles.h — the opaque handle types behind include/ne2b.h (internal).
#pragma once
#include <cuda_runtime.h>

#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "ne2b_engine.h"

struct ne2b_sim {
    ne2b::Engine eng;
    uint32_t slot = 0;
};

struct ne2b_batch {
    ne2b::Engine eng;
    std::vector<uint32_t> slots;
};

struct ne2b_server {
    struct Req {
        uint32_t slot = 0, n = 0, n_pad = 0, windows = 0;
        uint64_t steps = 0, fp_neurons = 0, fp_syn = 0, fp_ring = 0;
        bool queued = false;                 // admission thread has not attached it yet
        bool done = false;
        ne2b_status fail = NE2B_OK;          // build error, reported by take_result
        std::string fail_msg;
        uint16_t *d_win = nullptr;           // window counts, kept on device until taken
        unsigned long long *d_spk = nullptr; // spike total copied at retirement
        cudaEvent_t ev = nullptr;            // retirement copies complete
    };
    // asynchronous admission: jobs built by builder threads on their own
    // streams, attached by ne2b_server_step on the engine's stream
    struct Job {
        uint64_t id;
        ne2b_net_desc desc;
        ne2b_config cfg;
        const float *inputs;
        uint64_t steps;
    };
    struct Built {
        uint64_t id = 0;
        ne2b::NetHost *h = nullptr;
        cudaEvent_t ev = nullptr;  // the build's stream work is complete
        ne2b_status st = NE2B_OK;
        std::string msg;
    };
    struct Builder {
        std::thread th;
        cudaStream_t st = nullptr;
        ne2b::Stager sg;
    };
    ne2b::Engine eng;
    ne2b_server_config cfg{};
    std::map<uint64_t, Req> reqs;
    std::vector<uint64_t> finished;
    uint64_t used_neurons = 0, used_syn = 0, used_ring = 0;
    uint64_t next_id = 1, admitted = 0, retired = 0;
    cudaStream_t rstream = nullptr;  // result copies
    cudaEvent_t step_ev[2] = {nullptr, nullptr};
    uint64_t step_no = 0;
    std::vector<std::unique_ptr<Builder>> builders;
    std::mutex mu;  // jobs, built, stop
    std::condition_variable cv_job, cv_built;
    std::deque<Job> jobs;
    std::vector<Built> built;
    bool stop = false;

    void stop_builders() {
        {
            std::lock_guard<std::mutex> g(mu);
            stop = true;
        }
        cv_job.notify_all();
        for (auto &b : builders)
            if (b->th.joinable()) b->th.join();
        for (auto &b : builders)
            if (b->st) cudaStreamSynchronize(b->st);
        for (Built &r : built) {
            if (r.ev) cudaEventDestroy(r.ev);
            if (r.h) eng.discard_net(r.h, eng.stream());
        }
        built.clear();
    }
    ~ne2b_server() {
        stop_builders();
        eng.sync();
        for (auto &b : builders)
            if (b->st) cudaStreamDestroy(b->st);
        for (auto &kv : reqs) {
            if (kv.second.d_win) cudaFree(kv.second.d_win);
            if (kv.second.d_spk) cudaFree(kv.second.d_spk);
            if (kv.second.ev) cudaEventDestroy(kv.second.ev);
        }
        for (cudaEvent_t e : step_ev)
            if (e) cudaEventDestroy(e);
        if (rstream) cudaStreamDestroy(rstream);
    }
};
