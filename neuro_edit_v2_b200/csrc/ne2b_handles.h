// ne2b_handles.h — the opaque handle types behind include/ne2b.h (internal).
#pragma once
#include <cuda_runtime.h>

#include <map>
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
        bool done = false;
        uint16_t *d_win = nullptr;           // window counts, kept on device until taken
        unsigned long long *d_spk = nullptr; // spike total copied at retirement
        cudaEvent_t ev = nullptr;            // retirement copies complete
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
    ~ne2b_server() {
        eng.sync();
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

