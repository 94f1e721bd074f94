// ne2b_layout.h — device-resident layout shared by the step kernel and the
// host engine.
//
// HBM layout per network (every array is the net's own allocation, so nets
// can be admitted and retired independently):
//   neuron state, structure-of-arrays, n_pad = round_up(n, 64) entries:
//     v, u (model state slots 0/1), s (merged synaptic current), tk (u16
//     steps since the last spike: trace = trace_tab[tk], 0xFFFF = trace 0),
//     ext, v0/u0 (reset rows), pidx (u16 index into the param table, bit 15
//     set for AdEx rows),
//     pn_total (u64 lifetime spike counts), wcount (u32 current-window counts)
//   delay ring: D x n_pad words (int32 fixed point or f32), slot-major, so the
//     neuron pass reads one contiguous slot row per step
//   CSR by source: rowptr[n+1] (u32, local) and one 8-byte record per
//     synapse, syn[E] = {target | delay << 24, weight bits (int32 =
//     lrintf(w*4096) or f32)}, read with one 64-bit load; a net whose delays
//     exceed 255 steps or whose targets exceed 24 bits (kNetDelayWide) keeps
//     the bare target in the record and its delays in delay16[E] (u16)
//   stimulus: neuron-major (input, weight) rows and a [steps x n_inputs] f32
//     value buffer; spike record: rows x n_pad/32 u32 words; window counts:
//     max_windows x n_pad u16.
#pragma once
#include <stdint.h>

namespace ne2b {

constexpr uint32_t kNeuronAlign = 64;  // n_pad multiple: one u64 record word never spans nets
constexpr uint32_t kMaxParams = 12;

enum NetFlags : uint32_t {
    kNetHasExt = 1u << 0,
    kNetDelayWide = 1u << 1,  // delays in delay16[], bare targets in the records
    kNetRecord = 1u << 2,
    kNetWindows = 1u << 3,
    kNetActive = 1u << 4,
    kNetHasAdex = 1u << 5,  // at least one AdEx neuron
    kNetXsyn = 1u << 6,     // some synapses have their own tau (XSyn)
    kNetWatch = 1u << 7,    // watched neurons record their state every step
    kNetGridWatch = 1u << 8,  // grid groups record each member's last spike step
    kNetTraceF32 = 1u << 9,   // readout trace kept as f32 (its step table would be too long)
};

enum TileFlags : uint32_t {
    kTileHasStim = 1u << 0,
};

struct alignas(16) ParamRow {
    float p[kMaxParams];
    uint32_t model;  // registry id: 0 izh, 1 AdEx
    uint32_t pad[3];
};

struct alignas(16) Tile {
    uint32_t net;
    uint32_t start;     // first local neuron
    uint32_t count;     // neurons in this tile (<= tile size)
    uint32_t flags;
    uint32_t smem_off;  // resident kernel: offset of the tile's state in its block's shared memory
    uint32_t pad[3];
};

// One synapse of the CSR: td = target | delay_steps << 24 (or the bare
// target with kNetDelayWide), w = weight bits.
struct alignas(8) SynRec {
    uint32_t td;
    uint32_t w;
};
constexpr uint32_t kSynTgtBits = 24;
constexpr uint32_t kSynTgtMask = (1u << kSynTgtBits) - 1u;
constexpr uint32_t kSynMaxPackedDelay = 255u;

constexpr uint16_t kTraceZero = 0xFFFFu;  // tk value of a zero trace
constexpr uint32_t kNoXsyn = 0xFFFFFFFFu;  // xmap value of a synapse on the merged ring
constexpr uint32_t kWatchCap = 4096;       // samples kept per watched neuron (cpu.rs:78 V_HIST_CAP)
constexpr uint32_t kNoWatch = 0xFFFFFFFFu; // watch_idx of an unwatched neuron
constexpr uint32_t kNeverSpiked = 0xFFFFFFFFu;  // gw_ls of a texel that never spiked
constexpr uint32_t kParamAdexBit = 0x8000u;  // pidx bit: the row is an AdEx row
constexpr uint32_t kSmemParamRows = 32;      // param tables up to this size are staged in shared memory

// Per-network descriptor.  Device copy read by the kernels; the host keeps a
// mirror and rewrites the fields it changes.
struct alignas(16) NetDev {
    // neuron arrays
    float *v, *u, *s, *ext;
    uint16_t *tk;              // steps since last spike (trace_tab index), kTraceZero = 0
    float *trace_f;            // kNetTraceF32 only: the f32 trace itself
    const float *trace_tab;    // trace_tab[k] = decay_t applied k times to 1.0 (f32, in order)
    const float *v0, *u0;
    const uint16_t *pidx;
    unsigned long long *pn_total;
    uint32_t *wcount;
    // ring (int32 or f32 words)
    void *ring;
    // csr
    const uint32_t *rowptr;
    const SynRec *syn;        // [E]
    const uint16_t *delay16;  // [E], kNetDelayWide only
    // stimulus
    const uint32_t *stim_ptr;
    const uint32_t *stim_in;
    const float *stim_w;
    const float *stim_buf;  // [stim_len x n_inputs]
    // spike record + windows
    uint32_t *rec_bits;     // [rec_rows x n_pad/32]
    uint16_t *win_out;      // [max_windows x n_pad]
    // synapses with their own tau (sim/src/state.rs:231-275), kNetXsyn only
    const uint32_t *xmap;   // [E] custom-synapse id of CSR synapse j, or kNoXsyn
    const uint32_t *xt_ptr; // [n+1] each target's range in xt_idx
    const uint32_t *xt_idx; // [nx] custom-synapse ids grouped by target, CSR order within
    float *xsyn;            // [nx] each custom synapse's current
    const float *xdecay;    // [nx] exp(-dt / tau)
    const float *xw;        // [nx] arrival weight (rt_get(rt_put(w)) with the int ring)
    uint32_t *xpend;        // [D x xwords] arrival bits: bit k of slot s = synapse k arrives at s
    // editor watches (cpu.rs:63-95, 290-420), kNetWatch / kNetGridWatch only
    const uint32_t *watch_idx;  // [n_pad] ring row of a watched neuron, or kNoWatch
    float *watch_ring;          // [2][watch_n][kWatchCap] state slots after step t at t % kWatchCap
    const int32_t *gw_map;      // [gw_n][n_pad] member-list position of neuron i in group g, or -1
    const uint32_t *gw_off;     // [gw_n + 1] group ranges in gw_ls
    uint32_t *gw_ls;            // last spike step per texel (min(t, 2^32-2)), kNeverSpiked
    uint32_t watch_n, gw_n;
    // scalars
    unsigned long long t;       // step index of the next launch group's k = 0
    unsigned long long t_end;   // steps at or beyond this are skipped (serving)
    long long stim_t0;          // step of stim_buf row 0
    unsigned long long seed;
    unsigned long long noise_step;  // step part of the noise base at t (set_step)
    uint32_t n, n_pad, D, tmod;  // tmod = t % D
    uint32_t n_inputs, stim_len;
    uint32_t rec_rows, win_steps, max_windows, flags;
    float dt, pkick, kick, decay_s, decay_t, gauss_k;
    uint32_t trace_last;  // last index of trace_tab (saturation)
    uint32_t xwords;      // ceil(nx / 32)
    // phases of t kept beside it (set_step), so a step finds its record row
    // and window without a division: rphase = t % rec_rows, wphase =
    // (t + 1) % win_steps, widx0 = (t + 1) / win_steps
    uint32_t rphase, wphase, widx0;
};

#ifdef __CUDACC__
#define NE2B_HD __host__ __device__
#else
#define NE2B_HD
#endif
// The noise counter hash's multipliers of the step and the seed
// (sim/src/state.rs:285-288).
constexpr unsigned long long kNoiseStepMul = 0xBF58476D1CE4E5B9ull;
constexpr unsigned long long kNoiseSeedMul = 0x94D049BB133111EBull;

// Sets t and every phase derived from it (tmod, rphase, wphase, widx0, and
// the noise base's step part t * kNoiseStepMul + seed * kNoiseSeedMul, from
// which a kernel reaches step t + k with one multiply-add).
NE2B_HD inline void set_step(NetDev &d, unsigned long long t) {
    d.t = t;
    d.noise_step = t * kNoiseStepMul + d.seed * kNoiseSeedMul;
    d.tmod = (uint32_t)(t % d.D);
    d.rphase = d.rec_rows ? (uint32_t)(t % d.rec_rows) : 0u;
    if (d.win_steps) {
        d.wphase = (uint32_t)((t + 1) % d.win_steps);
        const unsigned long long w = (t + 1) / d.win_steps;
        d.widx0 = w > 0xffffffffull ? 0xffffffffu : (uint32_t)w;
    } else {
        d.wphase = d.widx0 = 0u;
    }
}

// Mutable per-net counters, kept apart from the read-mostly descriptor.
struct NetCounters {
    unsigned long long spikes_total;
};

// Everything a step launch needs, in device memory so that a captured CUDA
// graph stays valid when nets are admitted or retired.
struct EngineDev {
    const Tile *tiles;
    uint32_t n_tiles;
    uint32_t n_nets;
    NetDev *nets;
    const ParamRow *ptab;
    NetCounters *counters;
    // resident kernel: block b owns tiles [block_tiles[b], block_tiles[b+1])
    const uint32_t *block_tiles;
    uint32_t block_neurons;  // shared-memory state capacity per block
    uint32_t n_params;       // rows of ptab on the device
    unsigned int *barrier;   // grid-barrier arrival counter (zeroed before each launch)
    unsigned int *err;       // nonzero: a device wait gave up (kErrBarrier, kErrDeliveryQueue)
};
constexpr unsigned int kErrBarrier = 1u;        // a resident kernel's grid barrier
constexpr unsigned int kErrDeliveryQueue = 2u;  // a delivery-queue wait of step_kernel_ws

}  // namespace ne2b
