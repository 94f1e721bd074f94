// ne2b_csr.h — the synapse CSR built on the device (ne2b_csr.cu), for sims
// created from a plain synapse list (ne2b_create_from_synapses).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "ne2b_layout.h"

namespace ne2b {

// The synapse list and the per-neuron kinds, in device memory.
struct DevSynapses {
    const uint32_t *src = nullptr, *tgt = nullptr;
    const float *w = nullptr, *delay_ms = nullptr;
    const uint8_t *kind = nullptr;  // [n], 1 = inhibitory (Dale's sign)
    uint64_t n_syn = 0;
    uint32_t n = 0;
    float dt_ms = 0.1f;
};

// Prepass results (device memory; zero bad indices mean "none" only after
// the host sets them to ~0).
struct CsrScalars {
    unsigned long long bad_ref;    // first synapse with src or tgt >= n
    unsigned long long bad_delay;  // first synapse whose delay exceeds 65535 steps
    uint32_t max_delay;            // largest delay in steps (>= 1)
    uint32_t timeout;              // a scatter block gave up waiting for its predecessor
};

// Checks references, rounds delays to steps, counts synapses per source
// (counts zeroed by the caller) and finds the largest delay.
cudaError_t csr_prepass(const DevSynapses &ds, uint32_t *counts, uint16_t *steps, CsrScalars *sc, cudaStream_t st);
// Row pointers [n + 1] from the counts; cursor [n] = rowptr[0..n).  `sums`
// holds csr_scan_blocks(n) words.
cudaError_t csr_scan(const uint32_t *counts, uint32_t n, uint32_t e, uint32_t *rowptr, uint32_t *cursor,
                     uint32_t *sums, cudaStream_t st);
uint32_t csr_scan_blocks(uint32_t n);
// Scatter blocks (8192 synapses each); `ticket` (one word) and `done`
// (csr_chunks words) zeroed by the caller.
uint64_t csr_chunks(uint64_t n_syn);
cudaError_t csr_scatter(const DevSynapses &ds, const uint16_t *steps, uint32_t *cursor, SynRec *syn_out,
                        uint16_t *delay16_out, bool int_w, bool wide, uint32_t *ticket, uint32_t *done,
                        CsrScalars *sc, unsigned long long limit_ns, cudaStream_t st);

}  // namespace ne2b
