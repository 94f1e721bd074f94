// ne2b_net.h — the host-side network behind the opaque ne2b_net handle
// (internal): source-major CSR, per-neuron model rows, stimulus routing.
#pragma once
#include <stdint.h>

#include <utility>
#include <vector>

struct ne2b_net {
    uint32_t n = 0;
    std::vector<uint8_t> model, kind;
    std::vector<float> params;  // n * 10
    std::vector<float> pos;     // n * 3
    std::vector<uint32_t> src_ptr, tgt;
    std::vector<float> w;
    std::vector<uint16_t> delay;
    std::vector<float> tau;  // per-synapse tau in ms (empty: none is custom)
    uint32_t n_inputs = 0;
    std::vector<uint32_t> stim_ptr, stim_input;
    std::vector<float> stim_w;
};

namespace ne2b_hostnet {
// network.rs:674-685: steps = max(1, round(delay/dt)); above u16 is an error
bool delay_steps(float ms, float dt, uint16_t *out);
// StimMap::from_network (sim/src/stim.rs:26-48) from per-input target lists
void build_stim(ne2b_net &net, const std::vector<std::vector<std::pair<uint32_t, float>>> &inputs);
}  // namespace ne2b_hostnet
