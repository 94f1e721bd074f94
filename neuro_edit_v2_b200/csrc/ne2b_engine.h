// ne2b_engine.h — host runtime of the B200 simulation core.
//
// An Engine owns one CUDA stream and a set of independent networks that are
// stepped together: one persistent step kernel per dt step covers every
// active net's tiles, and launch groups of `graph_steps` steps are replayed
// from a captured CUDA graph.  A single sim (ne2b_sim) is an Engine with one
// net; the batch runner and the serving loop are Engines with many.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <array>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ne2b.h"
#include "ne2b_csr.h"
#include "ne2b_layout.h"

namespace ne2b {

// A synapse list on the device, checked by csr_prepass, with the scratch
// its CSR build uses (all device memory, owned by the caller).
struct DevCsrBuild {
    DevSynapses syn;
    const uint16_t *steps = nullptr;   // delay steps per list entry
    const uint32_t *counts = nullptr;  // synapses per source
    uint32_t max_delay = 1;
    uint32_t *cursor = nullptr;        // [n]
    uint32_t *sums = nullptr;          // [csr_scan_blocks(n)]
    uint32_t *ticket = nullptr;        // [1], zeroed
    uint32_t *done = nullptr;          // [csr_chunks(n_syn)], zeroed
    CsrScalars *sc = nullptr;
};

ne2b_status set_error(ne2b_status st, const char *fmt, ...);
ne2b_status cuda_error(cudaError_t e, const char *what);
ne2b_status noalloc_setup(int device);  // ne2b_noalloc.cu

// Host mirror of one network's stimulus program (sim/src/stim.rs:9-127).
struct Stimulus {
    std::vector<float> constants;
    std::vector<std::vector<float>> series;
    std::vector<uint64_t> play_start;
    std::vector<uint8_t> looped;
    float value(uint32_t k, uint64_t t) const;
    void play(uint32_t k, uint64_t t, const float *v, uint64_t len, bool loop);
};

struct NetHost {
    ne2b_config cfg{};
    NetDev dev{};             // host mirror of the device descriptor
    uint32_t slot = 0;        // index in the engine's net array
    uint32_t n = 0, n_pad = 0, D = 0, n_inputs = 0;
    uint64_t e = 0;
    uint32_t nx = 0;          // synapses with their own tau (XSyn)
    uint64_t t = 0;           // host mirror of dev.t
    uint64_t t_end = ~0ull;
    uint64_t dev_bytes = 0;
    bool fixed_stim = false;  // serving: the input matrix is uploaded once
    uint32_t stim_cap = 0;    // rows of stim_buf
    Stimulus stim;
    std::vector<float> ext_host;
    std::vector<uint32_t> stim_ptr_host;  // for tile flags
    std::vector<void *> allocs;
    std::vector<float> pack_buf;
    // editor watches (cpu.rs:63-95)
    std::vector<uint32_t> watch_ids;   // as set
    std::vector<int32_t> watch_row;    // watch k -> ring row, -1 for an id beyond n (records 0)
    uint64_t watch_t0 = 0;             // first step of the undrained history
    std::vector<void *> watch_allocs;
    std::vector<uint32_t> gw_ptr, gw_members;
    std::vector<void *> gw_allocs;
    uint64_t build_launches = 0;  // kernels queued by build_net
};

enum KernelMode { kModeAuto = 0, kModeStream = 1, kModeResident = 2 };

struct EngineSnapshot {
    struct Item {
        void *live, *backup;
        size_t bytes;
    };
    struct Host {
        uint32_t slot;
        uint64_t t;
        NetDev dev;
    };
    std::vector<Item> items;
    std::vector<Host> hosts;
};

struct PinnedBlock {
    void *p = nullptr;
    size_t cap = 0, used = 0;
    cudaEvent_t ev = nullptr;
};

// Host-to-device copies on one stream through a pool of pinned staging
// blocks: the source is copied into pinned memory and the DMA is issued
// asynchronously, so a large upload never waits for kernels in flight.
// Blocks used since the last close() stay "open": they are not handed out
// again until close() has recorded, after every copy from them was enqueued,
// the event that marks them reusable.  The owner synchronises the stream
// before destroying a Stager.
class Stager {
  public:
    Stager() = default;
    Stager(const Stager &) = delete;
    Stager &operator=(const Stager &) = delete;
    ~Stager();
    void set_stream(cudaStream_t st) { st_ = st; }
    cudaStream_t stream() const { return st_; }
    ne2b_status reserve(size_t bytes, void **host);
    ne2b_status issue(void *dst, const void *host, size_t bytes);
    ne2b_status copy(void *dst, const void *src, size_t bytes);  // small copies go from pageable memory
    ne2b_status close();

    // Copies larger than two ring blocks stream through a fixed ring of
    // pinned blocks, each refilled once its previous DMA has completed, so
    // a multi-GB upload pins no more than the ring and overlaps the host
    // copy with the transfer.  ring_next hands out the next block (kRingBytes)
    // once it is free; ring_issue sends its first `bytes` to `dst`.
    static constexpr size_t kRingBytes = (size_t)32 << 20;
    ne2b_status ring_next(void **host);
    ne2b_status ring_issue(void *dst, size_t bytes);

  private:
    static constexpr int kRing = 4;
    ne2b_status copy_streamed(void *dst, const void *src, size_t bytes);
    int ring_cur_ = -1;
    PinnedBlock ring_[kRing];
    int ring_next_ = 0;
    cudaStream_t st_ = nullptr;
    std::vector<PinnedBlock> pin_;
    int cur_ = -1;
    std::vector<int> open_;
};

struct TileShape {
    uint32_t block = 256;
    uint32_t npt = 2;
    uint32_t blocks_per_sm = 0;  // 0 = occupancy limit
    bool ws = false;             // separate delivery warps (step_kernel_ws), engines of one net
};

class Engine {
  public:
    Engine() = default;
    ~Engine();
    ne2b_status init(int device, bool int_ring, uint32_t max_nets);

    // Adds a net (slot returned).  inputs/steps: a fixed [steps x n_inputs]
    // input matrix (serving); NULL = host-packed stimulus program.
    ne2b_status add_net(const ne2b_net_desc *net, const ne2b_config *cfg, const float *inputs, uint64_t steps,
                        uint32_t *slot, bool rebuild = true);
    // add_net in two halves.  build_net validates the net and creates its
    // device arrays (reset to the initial state) with copies and kernels on
    // `sg`'s stream; it touches no other engine state than the parameter
    // dictionary (under its lock), so it may run on another host thread
    // while this engine steps.  attach_net publishes a built net (slot,
    // descriptor, counters, parameter rows) on the engine's stream, which
    // must already be ordered after the build's stream work.
    // `dc`: the synapses are a list already on the device (checked by
    // csr_prepass), whose CSR the build sorts into place on the device; the
    // CSR fields of `net` are then unused.
    ne2b_status build_net(const ne2b_net_desc *net, const ne2b_config *cfg, const float *inputs, uint64_t steps,
                          Stager &sg, NetHost **out, const DevCsrBuild *dc = nullptr);
    ne2b_status add_net_device_csr(const ne2b_net_desc *net, const ne2b_config *cfg, const DevCsrBuild &dc,
                                   uint32_t *slot);
    // The device CSR of a net copied out (weights as stored, delays widened).
    ne2b_status read_csr(NetHost &h, uint32_t *rowptr, uint32_t *tgt, uint32_t *w_bits, uint16_t *delay_steps);
    ne2b_status attach_net(NetHost *h, uint32_t *slot, bool rebuild = true);
    void discard_net(NetHost *h, cudaStream_t st);  // a built net that is never attached
    ne2b_status remove_net(uint32_t slot, bool rebuild = true, const void *keep = nullptr);
    ne2b_status pin_copy(void *dst, const void *src, size_t bytes) { return stager_.copy(dst, src, bytes); }
    ne2b_status pin_close() { return stager_.close(); }
    ne2b_status run_steps(uint64_t steps);
    ne2b_status reset_net(uint32_t slot);
    ne2b_status sync();
    ne2b_status set_shape(const TileShape &s);
    ne2b_status autotune(uint32_t steps_per_trial);
    ne2b_status rebuild_tiles();
    ne2b_status upload_net(NetHost &h);

    ne2b_status read_f32(const float *dev, uint32_t n, float *out);
    ne2b_status read_trace(NetHost &h, float *out);
    ne2b_status check_err();
    ne2b_status spike_counts(NetHost &h, uint64_t rows, uint32_t *out);
    ne2b_status spike_row(NetHost &h, uint32_t back, uint64_t *out);
    ne2b_status spikes_total(NetHost &h, uint64_t *out);
    ne2b_status window_counts(NetHost &h, uint32_t window, uint16_t *out);
    ne2b_status set_ext(NetHost &h, const float *ext, uint32_t len);
    ne2b_status set_input_matrix(NetHost &h, const float *x, uint64_t steps);
    ne2b_status refresh_noise(NetHost &h);
    // editor watches (lib.rs:164-176, cpu.rs:308-407)
    ne2b_status set_v_watch(NetHost &h, const uint32_t *ids, uint32_t count);
    ne2b_status drain_watch(NetHost &h, float *out, uint32_t *count);  // out: [2][nwatch][count]
    ne2b_status set_grid_watches(NetHost &h, const uint32_t *members, const uint32_t *group_ptr, uint32_t ngroups);
    ne2b_status grid_traces(NetHost &h, float tau_ms, float *out);
    ne2b_status snapshot(EngineSnapshot &snap);
    ne2b_status restore(const EngineSnapshot &snap);
    void drop(EngineSnapshot &snap);

    NetHost *net(uint32_t slot) { return slot < nets_.size() ? nets_[slot] : nullptr; }
    unsigned long long *counter_ptr(uint32_t slot) { return &d_counters_[slot].spikes_total; }
    uint32_t active_nets() const;
    uint64_t dev_bytes() const;
    float last_ms() const { return last_ms_; }
    const TileShape &shape() const { return shape_; }
    cudaStream_t stream() const { return stream_; }
    int device() const { return device_; }
    bool int_ring() const { return int_ring_; }
    uint64_t launches() const { return launches_; }
    void count_launches(uint64_t k) { launches_ += k; }  // kernels launched by entry points outside the engine
    bool resident() const { return resident_; }
    int mode() const { return mode_; }
    ne2b_status set_mode(int m);
    // the streaming kernel runs separate delivery warps for shape `s`
    bool ws_applies(const TileShape &s) const;
    bool fixed_grid = false;  // grid independent of the tile count (serving)
    bool multi_net = false;   // many nets (batch, server): the streaming kernel stages tiles ahead
    uint32_t graph_steps = 256;
    uint32_t resident_steps = 4096;  // max steps per resident launch
    uint64_t stim_chunk = 2048;

  private:
    ne2b_status launch_group(uint32_t steps);
    ne2b_status pack_stim(const std::vector<NetHost *> &nets);
    ne2b_status stage_reserve(size_t bytes);
    ne2b_status param_index(uint32_t model, const float *p, uint32_t np, uint16_t *idx);
    ne2b_status upload_ptab();
    ne2b_status upload_eng();
    uint32_t grid() const;
    // the streaming kernel instance for the engine's nets (StepVariant)
    int step_variant() const;
    int step_variant(const TileShape &s) const;  // with `s`'s delivery warps where they apply
    bool plan_resident(std::vector<Tile> &tiles, std::vector<uint32_t> &block_tiles);
    void clear_graphs();

    int device_ = 0;
    int sm_count_ = 148;
    bool int_ring_ = true;
    cudaStream_t stream_ = nullptr;
    std::vector<NetHost *> nets_;
    NetDev *d_nets_ = nullptr;
    NetCounters *d_counters_ = nullptr;
    uint32_t nets_cap_ = 0;
    std::vector<ParamRow> h_ptab_;
    std::map<std::array<uint32_t, kMaxParams + 1>, uint16_t> ptab_index_;
    std::array<uint32_t, kMaxParams + 1> last_key_{};
    uint16_t last_idx_ = 0;
    bool last_key_valid_ = false;
    ParamRow *d_ptab_ = nullptr;
    uint32_t ptab_cap_ = 0;
    bool ptab_dirty_ = false;
    uint32_t ptab_rows_dev_ = 0;  // rows copied to the device (EngineDev::n_params)
    Tile *d_tiles_ = nullptr;
    uint32_t tiles_cap_ = 0;
    uint32_t n_tiles_ = 0;
    EngineDev *d_eng_ = nullptr;
    TileShape shape_;
    std::map<uint32_t, cudaGraphExec_t> graphs_;
    int graph_variant_ = -1;   // the step instance the cached graphs launch
    uint32_t stim_tiles_ = 0;  // tiles with stimulus entries
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    float last_ms_ = 0.0f;
    uint64_t launches_ = 0;  // kernels launched (graph nodes counted per replay)
    // resident kernel
    int mode_ = kModeAuto;
    bool resident_ = false;
    bool adex_ = false;  // some net holds AdEx rows: the kernels with the AdEx path run
    uint32_t *d_block_tiles_ = nullptr;
    uint32_t block_tiles_cap_ = 0;
    uint32_t res_neurons_ = 0;
    size_t res_smem_ = 0;
    uint32_t res_grid_ = 0;
    unsigned int *d_barrier_ = nullptr;
    unsigned int *d_err_ = nullptr;
    Stager stager_;  // uploads on the engine's own stream
    std::mutex ptab_mu_;  // the parameter dictionary (builds may run on other threads)
    void *stage_ = nullptr;  // pinned staging for stimulus chunks and descriptors
    size_t stage_bytes_ = 0;
};

}  // namespace ne2b
