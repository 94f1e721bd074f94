// ne2b_engine.cu — host runtime: per-net device allocations, the param
// dictionary, tiles, CUDA-graph replay of launch groups, stimulus packing,
// readbacks, snapshots for the tile-shape autotuner.
#include "ne2b_engine.h"

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <mutex>
#include <thread>

#include "ne2b_kernels.h"
#include "ne2b_step_kind.h"
#include "ne2b_parallel.h"

namespace ne2b {

static thread_local std::string g_err;

ne2b_status set_error(ne2b_status st, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return st;
}

ne2b_status cuda_error(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return NE2B_OK;
    if (e == cudaErrorMemoryAllocation)
        return set_error(NE2B_ENOMEM, "%s: %s", what, cudaGetErrorString(e));
    return set_error(NE2B_ECUDA, "%s: %s", what, cudaGetErrorString(e));
}

const char *last_error_str() { return g_err.c_str(); }

#define NE2B_CUDA(call)                                                  \
    do {                                                                 \
        cudaError_t _e = (call);                                         \
        if (_e != cudaSuccess) return cuda_error(_e, #call);             \
    } while (0)
#define NE2B_TRY(call)                                                   \
    do {                                                                 \
        ne2b_status _s = (call);                                         \
        if (_s != NE2B_OK) return _s;                                    \
    } while (0)

// ------------------------------------------------------------ Stimulus
// stim.rs:102-115
float Stimulus::value(uint32_t k, uint64_t t) const {
    if (k < series.size() && !series[k].empty()) {
        const std::vector<float> &s = series[k];
        const uint64_t start = k < play_start.size() ? play_start[k] : 0;
        if (k < looped.size() && looped[k]) {
            const int64_t m = (int64_t)s.size();
            int64_t d = ((int64_t)t - (int64_t)start) % m;
            if (d < 0) d += m;
            return s[(size_t)d];
        }
        const uint64_t idx = t - start;  // wrapping_sub
        return idx < s.size() ? s[(size_t)idx] : 0.0f;
    }
    return k < constants.size() ? constants[k] : 0.0f;
}

// stim.rs:71-96
void Stimulus::play(uint32_t k, uint64_t t, const float *v, uint64_t len, bool loop) {
    if (k >= series.size()) series.resize(k + 1);
    if (k >= play_start.size()) play_start.resize(k + 1, 0);
    if (k >= looped.size()) looped.resize(k + 1, 0);
    series[k].assign(v, v + len);
    play_start[k] = t;
    looped[k] = loop ? 1 : 0;
}

// -------------------------------------------------------------- Engine
Engine::~Engine() {
    if (stream_) cudaStreamSynchronize(stream_);
    clear_graphs();
    for (NetHost *h : nets_) {
        if (!h) continue;
        for (void *p : h->allocs) cudaFreeAsync(p, stream_);
        for (void *p : h->watch_allocs) cudaFreeAsync(p, stream_);
        for (void *p : h->gw_allocs) cudaFreeAsync(p, stream_);
        delete h;
    }
    if (stream_) cudaStreamSynchronize(stream_);
    if (stage_) cudaFreeHost(stage_);
    cudaFree(d_nets_);
    cudaFree(d_counters_);
    cudaFree(d_ptab_);
    cudaFree(d_tiles_);
    cudaFree(d_eng_);
    cudaFree(d_block_tiles_);
    cudaFree(d_barrier_);
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
    if (stream_) cudaStreamDestroy(stream_);
}

void Engine::clear_graphs() {
    for (auto &kv : graphs_) cudaGraphExecDestroy(kv.second);
    graphs_.clear();
}

ne2b_status Engine::init(int device, bool int_ring, uint32_t max_nets) {
    device_ = device;
    int_ring_ = int_ring;
    NE2B_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    NE2B_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10)
        return set_error(NE2B_UNSUPPORTED, "device %d is sm_%d%d; this library is built for sm_100a", device,
                         prop.major, prop.minor);
    noalloc_setup(device);  // scratch address of ne2b_spike_counts_noalloc; a failure only disables that entry point
    sm_count_ = prop.multiProcessorCount;
    NE2B_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    stager_.set_stream(stream_);
    {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
            uint64_t thr = ~0ull;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
    }
    nets_cap_ = max_nets ? max_nets : 1;
    NE2B_CUDA(cudaMalloc(&d_nets_, sizeof(NetDev) * nets_cap_));
    NE2B_CUDA(cudaMemset(d_nets_, 0, sizeof(NetDev) * nets_cap_));
    NE2B_CUDA(cudaMalloc(&d_counters_, sizeof(NetCounters) * nets_cap_));
    NE2B_CUDA(cudaMemset(d_counters_, 0, sizeof(NetCounters) * nets_cap_));
    NE2B_CUDA(cudaMalloc(&d_eng_, sizeof(EngineDev)));
    ptab_cap_ = 64;
    NE2B_CUDA(cudaMalloc(&d_ptab_, sizeof(ParamRow) * ptab_cap_));
    tiles_cap_ = 1024;
    NE2B_CUDA(cudaMalloc(&d_tiles_, sizeof(Tile) * tiles_cap_));
    NE2B_CUDA(cudaEventCreate(&ev0_));
    NE2B_CUDA(cudaEventCreate(&ev1_));
    NE2B_CUDA(cudaMalloc(&d_barrier_, 2 * sizeof(unsigned int)));
    NE2B_CUDA(cudaMemset(d_barrier_, 0, 2 * sizeof(unsigned int)));
    d_err_ = d_barrier_ + 1;
    if (const char *pdl = getenv("NE2B_PDL")) set_pdl(strcmp(pdl, "0") != 0);
    if (const char *m = getenv("NE2B_KERNEL")) {
        if (!strcmp(m, "stream")) mode_ = kModeStream;
        else if (!strcmp(m, "resident")) mode_ = kModeResident;
    }
    nets_.assign(nets_cap_, nullptr);
    return upload_eng();
}

ne2b_status Engine::upload_eng() {
    EngineDev e;
    e.tiles = d_tiles_;
    e.n_tiles = n_tiles_;
    e.n_nets = nets_cap_;
    e.nets = d_nets_;
    e.ptab = d_ptab_;
    e.counters = d_counters_;
    e.block_tiles = d_block_tiles_;
    e.block_neurons = res_neurons_;
    e.n_params = ptab_rows_dev_;
    e.barrier = d_barrier_;
    e.err = d_err_;
    // pageable source: the runtime copies it to staging before returning, so
    // the stack frame may go away without waiting for the device
    NE2B_CUDA(cudaMemcpyAsync(d_eng_, &e, sizeof e, cudaMemcpyHostToDevice, stream_));
    return NE2B_OK;
}

ne2b_status Engine::param_index(uint32_t model, const float *p, uint32_t np, uint16_t *idx) {
    std::array<uint32_t, kMaxParams + 1> key{};
    key[0] = model;
    for (uint32_t k = 0; k < np && k < kMaxParams; ++k) memcpy(&key[k + 1], &p[k], 4);
    if (last_key_valid_ && key == last_key_) {  // consecutive neurons usually share a row
        *idx = last_idx_;
        return NE2B_OK;
    }
    auto it = ptab_index_.find(key);
    if (it != ptab_index_.end()) {
        last_key_ = key;
        last_idx_ = it->second;
        last_key_valid_ = true;
    }
    if (it != ptab_index_.end()) {
        *idx = it->second;
        return NE2B_OK;
    }
    if (h_ptab_.size() >= kParamAdexBit)
        return set_error(NE2B_UNSUPPORTED, "more than 32768 distinct parameter rows in one engine");
    ParamRow r;
    memset(&r, 0, sizeof r);
    for (uint32_t k = 0; k < np && k < kMaxParams; ++k) r.p[k] = p[k];
    r.model = model;
    *idx = (uint16_t)(h_ptab_.size() | (model == NE2B_MODEL_ADEX ? kParamAdexBit : 0u));
    h_ptab_.push_back(r);
    ptab_index_[key] = *idx;
    ptab_dirty_ = true;
    last_key_ = key;
    last_idx_ = *idx;
    last_key_valid_ = true;
    return NE2B_OK;
}

ne2b_status Engine::upload_ptab() {
    if (!ptab_dirty_) return NE2B_OK;
    if (h_ptab_.size() > ptab_cap_) {
        uint32_t cap = ptab_cap_;
        while (cap < h_ptab_.size()) cap *= 2;
        NE2B_CUDA(cudaStreamSynchronize(stream_));
        NE2B_CUDA(cudaFree(d_ptab_));
        d_ptab_ = nullptr;
        NE2B_CUDA(cudaMalloc(&d_ptab_, sizeof(ParamRow) * cap));
        ptab_cap_ = cap;
        NE2B_TRY(upload_eng());
    }
    NE2B_CUDA(cudaMemcpyAsync(d_ptab_, h_ptab_.data(), sizeof(ParamRow) * h_ptab_.size(), cudaMemcpyHostToDevice,
                              stream_));
    ptab_dirty_ = false;
    if (ptab_rows_dev_ != (uint32_t)h_ptab_.size()) {
        ptab_rows_dev_ = (uint32_t)h_ptab_.size();
        NE2B_TRY(upload_eng());
    }
    return NE2B_OK;
}

static float host_decay(float dt, float tau) {
    // cpu.rs:203-204: (-dt / tau.max(1e-6)).exp() in f32 (libm expf)
    const float t = tau > 1e-6f ? tau : 1e-6f;
    return expf(-dt / t);
}

static void fill_noise(NetDev &d, const ne2b_config &c) {
    d.pkick = c.noise_rate_hz * c.dt_ms / 1000.0f;                 // cpu.rs:197
    d.kick = c.noise_kick_mv != 0.0f ? c.noise_kick_mv / c.dt_ms : 0.0f;  // cpu.rs:198-202
    d.gauss_k = c.gauss_sd != 0.0f ? (float)((double)c.gauss_sd * 1.7320508075688772 / 256.0) : 0.0f;
}

Stager::~Stager() {
    for (PinnedBlock &b : pin_) {
        cudaFreeHost(b.p);
        cudaEventDestroy(b.ev);
    }
    for (PinnedBlock &b : ring_) {
        if (b.ev) cudaEventSynchronize(b.ev);
        if (b.p) cudaFreeHost(b.p);
        if (b.ev) cudaEventDestroy(b.ev);
    }
}

ne2b_status Stager::ring_next(void **host) {
    ring_cur_ = ring_next_;
    ring_next_ = (ring_next_ + 1) % kRing;
    PinnedBlock &b = ring_[ring_cur_];
    if (!b.p) {
        NE2B_CUDA(cudaMallocHost(&b.p, kRingBytes));
        NE2B_CUDA(cudaEventCreateWithFlags(&b.ev, cudaEventDisableTiming));
        b.cap = kRingBytes;
    } else {
        NE2B_CUDA(cudaEventSynchronize(b.ev));  // its previous transfer has left the block
    }
    *host = b.p;
    return NE2B_OK;
}

ne2b_status Stager::ring_issue(void *dst, size_t bytes) {
    PinnedBlock &b = ring_[ring_cur_];
    NE2B_CUDA(cudaMemcpyAsync(dst, b.p, bytes, cudaMemcpyHostToDevice, st_));
    NE2B_CUDA(cudaEventRecord(b.ev, st_));
    return NE2B_OK;
}

ne2b_status Stager::copy_streamed(void *dst, const void *src, size_t bytes) {
    for (size_t off = 0; off < bytes; off += kRingBytes) {
        const size_t len = std::min(kRingBytes, bytes - off);
        void *hb = nullptr;
        NE2B_TRY(ring_next(&hb));
        const uint8_t *s = (const uint8_t *)src + off;
        parallel_for(len, [&](uint64_t lo, uint64_t hi) { memcpy((uint8_t *)hb + lo, s + lo, hi - lo); });
        NE2B_TRY(ring_issue((uint8_t *)dst + off, len));
    }
    return NE2B_OK;
}

ne2b_status Stager::reserve(size_t bytes, void **host) {
    const size_t need = (bytes + 255) / 256 * 256;
    if (cur_ >= 0 && pin_[cur_].used + need > pin_[cur_].cap) {
        open_.push_back(cur_);
        cur_ = -1;
    }
    if (cur_ < 0) {
        for (size_t k = 0; k < pin_.size(); ++k) {
            if (std::find(open_.begin(), open_.end(), (int)k) != open_.end()) continue;
            if (pin_[k].cap >= need && cudaEventQuery(pin_[k].ev) == cudaSuccess) {
                cur_ = (int)k;
                break;
            }
        }
        if (cur_ < 0) {
            PinnedBlock b;
            b.cap = std::max<size_t>(need, (size_t)64 << 20);
            NE2B_CUDA(cudaMallocHost(&b.p, b.cap));
            NE2B_CUDA(cudaEventCreateWithFlags(&b.ev, cudaEventDisableTiming));
            pin_.push_back(b);
            cur_ = (int)pin_.size() - 1;
        }
        pin_[cur_].used = 0;
    }
    PinnedBlock &b = pin_[cur_];
    *host = (uint8_t *)b.p + b.used;
    b.used += need;
    return NE2B_OK;
}

ne2b_status Stager::issue(void *dst, const void *host, size_t bytes) {
    NE2B_CUDA(cudaMemcpyAsync(dst, host, bytes, cudaMemcpyHostToDevice, st_));
    return NE2B_OK;
}

ne2b_status Stager::copy(void *dst, const void *src, size_t bytes) {
    if (!bytes) return NE2B_OK;
    if (bytes <= (64u << 10)) {
        NE2B_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st_));
        return NE2B_OK;
    }
    if (bytes > 2 * kRingBytes) return copy_streamed(dst, src, bytes);
    void *stage = nullptr;
    NE2B_TRY(reserve(bytes, &stage));
    parallel_for(bytes, [&](uint64_t lo, uint64_t hi) { memcpy((uint8_t *)stage + lo, (const uint8_t *)src + lo, hi - lo); });
    return issue(dst, stage, bytes);
}

ne2b_status Stager::close() {
    if (cur_ >= 0) open_.push_back(cur_);
    for (int k : open_) NE2B_CUDA(cudaEventRecord(pin_[k].ev, st_));
    open_.clear();
    cur_ = -1;
    return NE2B_OK;
}

static double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

ne2b_status Engine::add_net(const ne2b_net_desc *net, const ne2b_config *cfg, const float *inputs, uint64_t steps,
                            uint32_t *slot_out, bool rebuild) {
    NetHost *h = nullptr;
    NE2B_TRY(build_net(net, cfg, inputs, steps, stager_, &h));
    const ne2b_status st = attach_net(h, slot_out, rebuild);
    if (st != NE2B_OK) discard_net(h, stream_);
    return st;
}

void Engine::discard_net(NetHost *h, cudaStream_t st) {
    if (!h) return;
    for (void *p : h->allocs) cudaFreeAsync(p, st);
    delete h;
}

ne2b_status Engine::attach_net(NetHost *h, uint32_t *slot_out, bool rebuild) {
    uint32_t slot = nets_cap_;
    for (uint32_t j = 0; j < nets_cap_; ++j)
        if (!nets_[j]) {
            slot = j;
            break;
        }
    if (slot == nets_cap_) return set_error(NE2B_EFULL, "all %u net slots are in use", nets_cap_);
    {
        std::lock_guard<std::mutex> g(ptab_mu_);
        NE2B_TRY(upload_ptab());
    }
    NE2B_CUDA(cudaMemsetAsync(d_counters_ + slot, 0, sizeof(NetCounters), stream_));
    h->slot = slot;
    nets_[slot] = h;
    launches_ += h->build_launches;
    h->build_launches = 0;
    NE2B_TRY(upload_net(*h));
    if (rebuild) NE2B_TRY(rebuild_tiles());
    *slot_out = slot;
    return NE2B_OK;
}

ne2b_status Engine::add_net_device_csr(const ne2b_net_desc *net, const ne2b_config *cfg, const DevCsrBuild &dc,
                                       uint32_t *slot_out) {
    NetHost *h = nullptr;
    NE2B_TRY(build_net(net, cfg, nullptr, 0, stager_, &h, &dc));
    const ne2b_status st = attach_net(h, slot_out, true);
    if (st != NE2B_OK) discard_net(h, stream_);
    return st;
}

ne2b_status Engine::build_net(const ne2b_net_desc *net, const ne2b_config *cfg, const float *inputs, uint64_t steps,
                              Stager &sg, NetHost **out, const DevCsrBuild *dc) {
    *out = nullptr;
    if (!net || !cfg) return set_error(NE2B_EINVAL, "add_net: null net or config");
    const cudaStream_t bst = sg.stream();
    const bool dbg = getenv("NE2B_DEBUG") != nullptr;
    double tp[8] = {now_ms()};
    const uint32_t n = net->n;
    if (!(cfg->dt_ms >= 0.001f && cfg->dt_ms <= 100.0f))  // lib.rs:35-39 valid_dt_ms
        return set_error(NE2B_EINVAL, "dt_ms %g outside [0.001, 100]", (double)cfg->dt_ms);
    if (n > 0 && (!net->model || !net->params || (!net->src_ptr && !dc)))
        return set_error(NE2B_EINVAL, "net: model, params and src_ptr are required");
    if (net->param_stride < 4 && n > 0) return set_error(NE2B_EINVAL, "param_stride %u < 4", net->param_stride);
    const uint64_t n_syn = dc ? dc->syn.n_syn : net->n_syn;
    if (n_syn > 0xffffffffull) return set_error(NE2B_UNSUPPORTED, "more than 2^32-1 synapses in one net");
    if (!dc) {
        if (n > 0 && net->src_ptr[n] != net->n_syn)
            return set_error(NE2B_EINVAL, "src_ptr[n] = %u but n_syn = %llu", net->src_ptr[n],
                             (unsigned long long)net->n_syn);
        for (uint32_t i = 0; i < n; ++i)
            if (net->src_ptr[i] > net->src_ptr[i + 1]) return set_error(NE2B_EINVAL, "src_ptr not monotone at %u", i);
    }
    // one parallel pass over the synapses: target range, delay range, tau
    // (a device list was checked by its prepass)
    uint32_t maxd = dc ? dc->max_delay : 1, mind = dc ? 1 : 0xffff, maxt = 0;
    bool any_tau = false;
    if (!dc) {
        std::mutex mu;
        parallel_for(net->n_syn, [&](uint64_t lo, uint64_t hi) {
            uint32_t mx = 1, mn = 0xffff, mt = 0;
            bool tau = false;
            for (uint64_t j = lo; j < hi; ++j) {
                const uint32_t d = net->delay_steps[j];
                mx = d > mx ? d : mx;
                mn = d < mn ? d : mn;
                mt = net->tgt[j] > mt ? net->tgt[j] : mt;
            }
            if (net->tau_ms)
                for (uint64_t j = lo; j < hi; ++j) tau |= net->tau_ms[j] > 0.0f;
            std::lock_guard<std::mutex> g(mu);
            maxd = std::max(maxd, mx);
            mind = std::min(mind, mn);
            maxt = std::max(maxt, mt);
            any_tau |= tau;
        });
    }
    if (!dc && net->n_syn && maxt >= n) {
        for (uint64_t j = 0; j < net->n_syn; ++j)
            if (net->tgt[j] >= n)
                return set_error(NE2B_EINVAL, "synapse %llu targets %u >= n %u", (unsigned long long)j, net->tgt[j], n);
    }
    if (!dc && net->n_syn && mind < 1) return set_error(NE2B_EINVAL, "a synapse has delay 0 steps");
    for (uint32_t i = 0; i < n; ++i)
        if (net->model[i] > 1) return set_error(NE2B_EINVAL, "neuron %u: unknown model id %u", i, net->model[i]);
    if (n > 0 && net->n_inputs > 0 && net->stim_ptr) {
        if (net->stim_ptr[0] != 0) return set_error(NE2B_EINVAL, "stim_ptr[0] != 0");
        for (uint32_t i = 0; i < n; ++i)
            if (net->stim_ptr[i] > net->stim_ptr[i + 1]) return set_error(NE2B_EINVAL, "stim_ptr not monotone");
        for (uint32_t j = 0; j < net->stim_ptr[n]; ++j)
            if (net->stim_input[j] >= net->n_inputs) return set_error(NE2B_EINVAL, "stim entry %u names input %u", j, net->stim_input[j]);
    }
    if (cfg->window_steps > 0 && cfg->window_steps > 131070u)
        return set_error(NE2B_EINVAL, "window_steps %u would overflow the u16 window counts", cfg->window_steps);
    if (inputs && net->n_inputs == 0) inputs = nullptr;
    tp[1] = now_ms();

    NetHost *h = new NetHost();
    h->cfg = *cfg;
    h->n = n;
    h->n_pad = (n + kNeuronAlign - 1) / kNeuronAlign * kNeuronAlign;
    h->D = maxd + 1 < 2 ? 2 : maxd + 1;  // state.rs:221-224
    h->e = n_syn;
    h->n_inputs = net->n_inputs;
    h->t_end = inputs ? steps : ~0ull;
    h->fixed_stim = inputs != nullptr;
    h->stim.constants.assign(net->n_inputs, 0.0f);
    h->stim.series.assign(net->n_inputs, {});
    h->stim.play_start.assign(net->n_inputs, 0);
    h->stim.looped.assign(net->n_inputs, 0);
    h->ext_host.assign(n, 0.0f);

    auto alloc = [&](void **p, size_t bytes) -> ne2b_status {
        *p = nullptr;
        if (bytes == 0) return NE2B_OK;
        cudaError_t e = cudaMallocAsync(p, bytes, bst);
        if (e != cudaSuccess) return cuda_error(e, "cudaMallocAsync (net arrays)");
        h->allocs.push_back(*p);
        h->dev_bytes += bytes;
        return NE2B_OK;
    };
    auto fail = [&](ne2b_status st) {
        for (void *p : h->allocs) cudaFreeAsync(p, bst);
        sg.close();
        cudaStreamSynchronize(bst);
        delete h;
        return st;
    };
    auto up = [&](void *dst, const void *src, size_t bytes) -> ne2b_status { return sg.copy(dst, src, bytes); };
#define NET_TRY(x)                          \
    do {                                    \
        ne2b_status _s = (x);               \
        if (_s != NE2B_OK) return fail(_s); \
    } while (0)

    const uint32_t np = h->n_pad;
    NetDev &d = h->dev;
    memset(&d, 0, sizeof d);
    void *p = nullptr;
    NET_TRY(alloc(&p, sizeof(float) * np)); d.v = (float *)p;
    NET_TRY(alloc(&p, sizeof(float) * np)); d.u = (float *)p;
    NET_TRY(alloc(&p, sizeof(float) * np)); d.s = (float *)p;
    NET_TRY(alloc(&p, sizeof(uint16_t) * np)); d.tk = (uint16_t *)p;
    NET_TRY(alloc(&p, sizeof(float) * np)); d.ext = (float *)p;
    NET_TRY(alloc(&p, sizeof(float) * np)); d.v0 = (const float *)p;
    NET_TRY(alloc(&p, sizeof(float) * np)); d.u0 = (const float *)p;
    NET_TRY(alloc(&p, sizeof(uint16_t) * np)); d.pidx = (const uint16_t *)p;
    NET_TRY(alloc(&p, sizeof(unsigned long long) * np)); d.pn_total = (unsigned long long *)p;
    NET_TRY(alloc(&p, sizeof(uint32_t) * (size_t)h->D * np)); d.ring = p;
    NET_TRY(alloc(&p, sizeof(uint32_t) * ((size_t)n + 1))); d.rowptr = (const uint32_t *)p;
    NET_TRY(alloc(&p, sizeof(SynRec) * h->e)); d.syn = (const SynRec *)p;
    // delays past 8 bits, or targets past 24, do not fit the packed record
    const bool wide = h->D > kSynMaxPackedDelay + 1u || n > kSynTgtMask + 1u;
    if (wide) {
        NET_TRY(alloc(&p, sizeof(uint16_t) * h->e));
        d.delay16 = (const uint16_t *)p;
    }

    tp[2] = now_ms();
    // host-side rows: params -> dictionary, x0
    std::vector<uint16_t> pidx(np, 0);
    std::vector<float> v0(np, 0.0f), u0(np, 0.0f);
    bool any_adex = false;
    std::unique_lock<std::mutex> ptab_lock(ptab_mu_);
    for (uint32_t i = 0; i < n; ++i) {
        const float *row = net->params + (size_t)i * net->param_stride;
        const uint32_t m = net->model[i];
        any_adex |= m == NE2B_MODEL_ADEX;
        const uint32_t width = std::min<uint32_t>(net->param_stride, 10);
        NET_TRY(param_index(m, row, width, &pidx[i]));
        if (net->x0) {
            v0[i] = net->x0[2 * (size_t)i];
            u0[i] = net->x0[2 * (size_t)i + 1];
        } else if (m == NE2B_MODEL_ADEX) {  // adex.rs:149-152
            v0[i] = row[2];
            u0[i] = 0.0f;
        } else {  // izh.rs:175-178
            v0[i] = -65.0f;
            u0[i] = row[1] * v0[i];
        }
    }
    ptab_lock.unlock();  // the rows reach the device when the net is attached
    tp[3] = now_ms();
    NET_TRY(up((void *)d.pidx, pidx.data(), sizeof(uint16_t) * np));
    NET_TRY(up((void *)d.v0, v0.data(), sizeof(float) * np));
    NET_TRY(up((void *)d.u0, u0.data(), sizeof(float) * np));
    NET_TRY(cuda_error(cudaMemsetAsync(d.ext, 0, sizeof(float) * np, bst), "memset ext"));
    if (dc) {
        // the list's CSR sorted into place on the device (csrc/ne2b_csr.cu)
        NET_TRY(cuda_error(csr_scan(dc->counts, n, (uint32_t)h->e, (uint32_t *)d.rowptr, dc->cursor, dc->sums, bst),
                           "device CSR: row pointers"));
        NET_TRY(cuda_error(csr_scatter(dc->syn, dc->steps, dc->cursor, (SynRec *)d.syn, (uint16_t *)d.delay16, int_ring_, wide,
                                       dc->ticket, dc->done, dc->sc, 5000000000ull, bst),
                           "device CSR: scatter"));
        h->build_launches += (n ? 3 : 0) + (h->e ? 1 : 0);
    } else {
        NET_TRY(up((void *)d.rowptr, net->src_ptr, sizeof(uint32_t) * ((size_t)n + 1)));
    }
    if (h->e && !dc) {
        // one parallel pass over the synapses into pinned staging: each
        // record packs the target with its delay (u8) and the weight,
        // quantised (kernels.rs:61 rt_put: lrintf(w * 4096)) for the
        // fixed-point ring; a wide net's delays go to their own u16 array;
        // synapses [j0, j0 + m) into host buffers at their offset 0
        const bool iq = int_ring_;
        auto fill = [&](SynRec *rec, uint16_t *d16, uint64_t j0, uint64_t m) {
            parallel_for(m, [&](uint64_t lo, uint64_t hi) {
                if (rec)
                    for (uint64_t j = lo; j < hi; ++j) {
                        const uint64_t k = j0 + j;
                        const float wf = net->w[k];
                        uint32_t wb;
                        if (iq) wb = (uint32_t)(int32_t)lrintf(wf * 4096.0f);
                        else memcpy(&wb, &wf, 4);
                        const uint32_t tg = net->tgt[k];
                        rec[j].td = wide ? tg : tg | ((uint32_t)net->delay_steps[k] << kSynTgtBits);
                        rec[j].w = wb;
                    }
                if (d16) memcpy(d16 + lo, net->delay_steps + j0 + lo, 2 * (hi - lo));
            });
        };
        if (sizeof(SynRec) * h->e > 2 * Stager::kRingBytes) {
            // a large net streams through the stager's ring of pinned blocks
            const uint64_t per = Stager::kRingBytes / sizeof(SynRec);
            for (uint64_t j0 = 0; j0 < h->e; j0 += per) {
                const uint64_t m = std::min<uint64_t>(per, h->e - j0);
                void *hb = nullptr;
                NET_TRY(sg.ring_next(&hb));
                fill((SynRec *)hb, nullptr, j0, m);
                NET_TRY(sg.ring_issue((SynRec *)d.syn + j0, sizeof(SynRec) * m));
                if (wide) {
                    NET_TRY(sg.ring_next(&hb));
                    fill(nullptr, (uint16_t *)hb, j0, m);
                    NET_TRY(sg.ring_issue((uint16_t *)d.delay16 + j0, sizeof(uint16_t) * m));
                }
            }
        } else {
            SynRec *rec = nullptr;
            uint16_t *d16 = nullptr;
            NET_TRY(sg.reserve(sizeof(SynRec) * h->e, (void **)&rec));
            if (wide) NET_TRY(sg.reserve(sizeof(uint16_t) * h->e, (void **)&d16));
            fill(rec, d16, 0, h->e);
            NET_TRY(sg.issue((void *)d.syn, rec, sizeof(SynRec) * h->e));
            if (wide) NET_TRY(sg.issue((void *)d.delay16, d16, sizeof(uint16_t) * h->e));
        }
    }
    if (any_tau) {
        // XSyn::build (sim/src/state.rs:245-274): synapses with tau > 0 get
        // their own current, numbered in CSR order; the neuron pass reads
        // them grouped by target (CSR order within a target)
        std::vector<uint32_t> xmap(h->e), xt_ptr((size_t)n + 1, 0);
        uint32_t nx = 0;
        for (uint64_t j = 0; j < h->e; ++j) xmap[j] = net->tau_ms[j] > 0.0f ? nx++ : kNoXsyn;
        std::vector<float> xdecay(nx), xw(nx);
        std::vector<uint32_t> xt_idx(nx);
        for (uint64_t j = 0; j < h->e; ++j) {
            const uint32_t k = xmap[j];
            if (k == kNoXsyn) continue;
            xdecay[k] = host_decay(cfg->dt_ms, net->tau_ms[j]);  // state.rs:262-264
            // the arrival adds w; with the int ring it is rt_get(rt_put(w)),
            // the value the fixed-point path delivers (kernels.rs:57-66)
            xw[k] = int_ring_ ? (float)(int32_t)lrintf(net->w[j] * 4096.0f) / 4096.0f : net->w[j];
            xt_ptr[net->tgt[j] + 1]++;
        }
        for (uint32_t i = 0; i < n; ++i) xt_ptr[i + 1] += xt_ptr[i];
        {
            std::vector<uint32_t> fill(xt_ptr.begin(), xt_ptr.end() - 1);
            for (uint64_t j = 0; j < h->e; ++j)
                if (xmap[j] != kNoXsyn) xt_idx[fill[net->tgt[j]]++] = xmap[j];
        }
        h->nx = nx;
        d.xwords = (nx + 31) / 32;
        NET_TRY(alloc(&p, sizeof(uint32_t) * h->e)); d.xmap = (const uint32_t *)p;
        NET_TRY(up(p, xmap.data(), sizeof(uint32_t) * h->e));
        NET_TRY(alloc(&p, sizeof(uint32_t) * ((size_t)n + 1))); d.xt_ptr = (const uint32_t *)p;
        NET_TRY(up(p, xt_ptr.data(), sizeof(uint32_t) * ((size_t)n + 1)));
        NET_TRY(alloc(&p, sizeof(uint32_t) * nx)); d.xt_idx = (const uint32_t *)p;
        NET_TRY(up(p, xt_idx.data(), sizeof(uint32_t) * nx));
        NET_TRY(alloc(&p, sizeof(float) * nx)); d.xdecay = (const float *)p;
        NET_TRY(up(p, xdecay.data(), sizeof(float) * nx));
        NET_TRY(alloc(&p, sizeof(float) * nx)); d.xw = (const float *)p;
        NET_TRY(up(p, xw.data(), sizeof(float) * nx));
        NET_TRY(alloc(&p, sizeof(float) * nx)); d.xsyn = (float *)p;
        NET_TRY(alloc(&p, sizeof(uint32_t) * (size_t)h->D * d.xwords)); d.xpend = (uint32_t *)p;
    }
    tp[4] = now_ms();
    // stimulus routing
    const bool has_stim = n > 0 && net->n_inputs > 0 && net->stim_ptr && net->stim_ptr[n] > 0;
    if (has_stim) {
        const uint32_t ne = net->stim_ptr[n];
        NET_TRY(alloc(&p, sizeof(uint32_t) * ((size_t)n + 1))); d.stim_ptr = (const uint32_t *)p;
        NET_TRY(alloc(&p, sizeof(uint32_t) * ne)); d.stim_in = (const uint32_t *)p;
        NET_TRY(alloc(&p, sizeof(float) * ne)); d.stim_w = (const float *)p;
        NET_TRY(up((void *)d.stim_ptr, net->stim_ptr, sizeof(uint32_t) * ((size_t)n + 1)));
        NET_TRY(up((void *)d.stim_in, net->stim_input, sizeof(uint32_t) * ne));
        NET_TRY(up((void *)d.stim_w, net->stim_w, sizeof(float) * ne));
        h->stim_ptr_host.assign(net->stim_ptr, net->stim_ptr + n + 1);
        if (inputs) {
            NET_TRY(alloc(&p, sizeof(float) * (size_t)steps * net->n_inputs)); d.stim_buf = (const float *)p;
            NET_TRY(up((void *)d.stim_buf, inputs, sizeof(float) * (size_t)steps * net->n_inputs));
            d.stim_t0 = 0;
            d.stim_len = (uint32_t)std::min<uint64_t>(steps, 0xffffffffull);
        } else {
            h->stim_cap = (uint32_t)stim_chunk;
            NET_TRY(alloc(&p, sizeof(float) * (size_t)h->stim_cap * net->n_inputs)); d.stim_buf = (const float *)p;
            d.stim_t0 = 0;
            d.stim_len = 0;  // packed before the first launch
        }
    }
    // spike record + windows
    uint32_t rec_rows = 0;
    if (cfg->record_spikes) rec_rows = cfg->spike_record_steps < 2 ? 2 : cfg->spike_record_steps;  // cpu.rs:112-116
    if (rec_rows) {
        NET_TRY(alloc(&p, sizeof(uint32_t) * (size_t)rec_rows * (np / 32))); d.rec_bits = (uint32_t *)p;
    }
    if (cfg->window_steps > 0) {
        NET_TRY(alloc(&p, sizeof(uint32_t) * np)); d.wcount = (uint32_t *)p;
        const uint32_t mw = cfg->max_windows ? cfg->max_windows : 1;
        NET_TRY(alloc(&p, sizeof(uint16_t) * (size_t)mw * np)); d.win_out = (uint16_t *)p;
        d.win_steps = cfg->window_steps;
        d.max_windows = mw;
    }
    d.n = n;
    d.n_pad = np;
    d.D = h->D;
    d.t_end = h->t_end;
    d.seed = cfg->seed;
    d.n_inputs = net->n_inputs;
    d.rec_rows = rec_rows;
    set_step(d, 0);
    d.dt = cfg->dt_ms;
    d.decay_s = host_decay(cfg->dt_ms, cfg->synapse_tau_ms);
    d.decay_t = host_decay(cfg->dt_ms, cfg->readout_tau_ms);
    {
        // trace after k non-spiking steps = 1.0 * decay_t * ... * decay_t (k
        // f32 multiplies in order, cpu.rs:252-256); the table stops at 0 or
        // at the subnormal fixed point, where the trace stays forever
        // (a u16 step counter); a readout tau whose table would pass 65534
        // entries keeps the f32 trace per neuron instead
        std::vector<float> tab(1, 1.0f);
        bool trace_f32 = false;
        while (true) {
            const float nx = tab.back() * d.decay_t;
            if (nx == tab.back()) break;
            tab.push_back(nx);
            if (nx == 0.0f) break;
            if (tab.size() > 65534) {
                trace_f32 = true;
                tab.resize(1);
                break;
            }
        }
        if (trace_f32) {
            NET_TRY(alloc(&p, sizeof(float) * np)); d.trace_f = (float *)p;
            NET_TRY(cuda_error(cudaMemsetAsync(d.trace_f, 0, sizeof(float) * np, bst), "memset trace"));
        }
        NET_TRY(alloc(&p, sizeof(float) * tab.size())); d.trace_tab = (const float *)p;
        NET_TRY(up((void *)d.trace_tab, tab.data(), sizeof(float) * tab.size()));
        d.trace_last = (uint32_t)tab.size() - 1;
    }
    fill_noise(d, *cfg);
    d.flags = kNetActive | (wide ? kNetDelayWide : 0u) | (rec_rows ? kNetRecord : 0u) |
              (cfg->window_steps ? kNetWindows : 0u) | (any_adex ? kNetHasAdex : 0u) | (h->nx ? kNetXsyn : 0u) |
              (d.trace_f ? kNetTraceF32 : 0u);
    tp[5] = now_ms();
    // initial state (cpu.rs:158-183), on the build stream
    NET_TRY(cuda_error(launch_reset_neurons(d, bst), "reset kernel"));
    h->build_launches += np ? 1 : 0;
    NET_TRY(cuda_error(cudaMemsetAsync(d.ring, 0, sizeof(uint32_t) * (size_t)h->D * np, bst), "memset ring"));
    if (d.rec_bits)
        NET_TRY(cuda_error(cudaMemsetAsync(d.rec_bits, 0, sizeof(uint32_t) * (size_t)rec_rows * (np / 32), bst),
                           "memset record"));
    if (d.win_out)
        NET_TRY(cuda_error(cudaMemsetAsync(d.win_out, 0, sizeof(uint16_t) * (size_t)d.max_windows * np, bst),
                           "memset windows"));
    if (h->nx) {
        NET_TRY(cuda_error(cudaMemsetAsync(d.xsyn, 0, sizeof(float) * h->nx, bst), "memset xsyn"));
        NET_TRY(cuda_error(cudaMemsetAsync(d.xpend, 0, sizeof(uint32_t) * (size_t)h->D * d.xwords, bst),
                           "memset xsyn arrivals"));
    }
    NET_TRY(sg.close());
    tp[6] = now_ms();
    if (dbg)
        fprintf(stderr, "ne2b build_net n=%u e=%llu: validate %.3f alloc %.3f params %.3f csr %.3f rest %.3f reset %.3f ms\n",
                n, (unsigned long long)h->e, tp[1] - tp[0], tp[2] - tp[1], tp[3] - tp[2], tp[4] - tp[3], tp[5] - tp[4],
                tp[6] - tp[5]);
#undef NET_TRY
    *out = h;
    return NE2B_OK;
}

// Stream-ordered removal: the descriptor is cleared and the net's arrays
// freed after every kernel already queued; `keep` (if not null) is an
// allocation handed over to the caller instead of being freed.
ne2b_status Engine::remove_net(uint32_t slot, bool rebuild, const void *keep) {
    NetHost *h = net(slot);
    if (!h) return set_error(NE2B_EINVAL, "no net in slot %u", slot);
    NetDev z;
    memset(&z, 0, sizeof z);
    NE2B_CUDA(cudaMemcpyAsync(d_nets_ + slot, &z, sizeof z, cudaMemcpyHostToDevice, stream_));
    for (void *p : h->allocs)
        if (p != keep) NE2B_CUDA(cudaFreeAsync(p, stream_));
    for (void *p : h->watch_allocs) NE2B_CUDA(cudaFreeAsync(p, stream_));
    for (void *p : h->gw_allocs) NE2B_CUDA(cudaFreeAsync(p, stream_));
    nets_[slot] = nullptr;
    delete h;
    return rebuild ? rebuild_tiles() : NE2B_OK;
}

ne2b_status Engine::upload_net(NetHost &h) {
    // pageable source, staged by the runtime before the call returns
    NE2B_CUDA(cudaMemcpyAsync(d_nets_ + h.slot, &h.dev, sizeof(NetDev), cudaMemcpyHostToDevice, stream_));
    return NE2B_OK;
}

uint32_t Engine::active_nets() const {
    uint32_t c = 0;
    for (NetHost *h : nets_) c += h != nullptr;
    return c;
}

uint64_t Engine::dev_bytes() const {
    uint64_t b = 0;
    for (NetHost *h : nets_)
        if (h) b += h->dev_bytes;
    return b;
}

uint32_t Engine::grid() const {
    uint32_t bps = shape_.blocks_per_sm;
    const int occ = step_occupancy(int_ring_, adex_, step_variant(), shape_.block, shape_.npt);
    if (bps == 0 || (int)bps > occ) bps = (uint32_t)(occ > 0 ? occ : 1);
    uint32_t g = (uint32_t)sm_count_ * bps;
    if (fixed_grid) return g;  // serving: graphs stay valid as nets come and go
    // never more blocks than tiles: idle blocks still cost launch time
    const uint32_t nt = n_tiles_ ? n_tiles_ : 1;
    return g < nt ? g : nt;
}

int Engine::step_variant() const { return step_variant(shape_); }

// The warp-specialised kernel serves streaming engines of exactly one net
// (its tile warps never restage a net descriptor) in the shapes it is
// compiled for.
bool Engine::ws_applies(const TileShape &s) const {
    return s.ws && !multi_net && active_nets() == 1 && ws_shape_supported(s.block, s.npt);
}

int Engine::step_variant(const TileShape &s) const {
    constexpr uint32_t kDebug = kNetRecord | kNetXsyn | kNetWatch | kNetGridWatch | kNetTraceF32;
    constexpr uint32_t kInput = kNetHasExt | kNetWindows;
    uint32_t used = 0;
    for (const NetHost *h : nets_)
        if (h) used |= h->dev.flags;
    if (multi_net) return (used & kDebug) ? kStepMulti : kStepMultiLean;
    const int ws = ws_applies(s) ? kStepWS : 0;
    if (stim_tiles_ || (used & (kDebug | kInput))) return kStepSingle | ws;
    return kStepPlain | ws;
}

// Resident plan: G co-resident blocks, each owning a contiguous range of
// tiles balanced by neuron count, with the owned state (v, u, s: 12 B;
// tk, pidx: 4 B per neuron) in dynamic shared memory.  Chooses the most
// blocks per SM whose shared memory still fits; false when nothing fits.
bool Engine::plan_resident(std::vector<Tile> &tiles, std::vector<uint32_t> &block_tiles) {
    // AUTO streams: on B200 the resident kernel's software grid barrier
    // (an arrival atomic and an acquire poll, two L2 round trips) costs more
    // than a kernel boundary in a graph with programmatic dependent launch
    // (10k neurons: 2.9 against 1.4 us per step; 100k: 3.1 against 1.9).
    // It runs when forced, or when ne2b_autotune finds it faster.
    if (tiles.empty() || mode_ != kModeResident) return false;
    uint64_t total = 0;
    for (const Tile &t : tiles) total += t.count;
    const uint32_t head = resident_head(shape_.block, shape_.npt);
    const uint32_t max_bps = std::max<uint32_t>(1, 2048 / shape_.block);
    for (uint32_t bps = shape_.blocks_per_sm ? shape_.blocks_per_sm : max_bps; bps >= 1; --bps) {
        const uint32_t G = (uint32_t)std::min<uint64_t>((uint64_t)sm_count_ * bps, tiles.size());
        // tile k goes to block floor(prefix_k * G / total): contiguous,
        // never more than G blocks, balanced to within one tile
        std::vector<uint32_t> bt(G + 1, (uint32_t)tiles.size());
        std::vector<uint64_t> sum(G, 0);
        uint64_t prefix = 0;
        uint32_t prev = 0;
        bt[0] = 0;
        for (uint32_t k = 0; k < tiles.size(); ++k) {
            uint32_t blk = (uint32_t)std::min<uint64_t>(G - 1, prefix * G / total);
            if (blk < prev) blk = prev;
            for (uint32_t b2 = prev + 1; b2 <= blk; ++b2) bt[b2] = k;
            prev = blk;
            sum[blk] += tiles[k].count;
            prefix += tiles[k].count;
        }
        for (uint32_t b2 = prev + 1; b2 <= G; ++b2) bt[b2] = (uint32_t)tiles.size();
        uint64_t m = 0;
        for (uint64_t x : sum) m = std::max(m, x);
        const size_t smem = head + 16 * (size_t)((m + 3) / 4 * 4);
        const int occ = smem > 227 * 1024 ? 0 : resident_occupancy(int_ring_, adex_, shape_.block, shape_.npt, smem);
        const uint32_t blocks = (uint32_t)bt.size() - 1;
        if (getenv("NE2B_DEBUG"))
            fprintf(stderr, "ne2b plan: block %u npt %u bps %u -> %u blocks, %llu neurons/block, smem %zu, occ %d\n",
                    shape_.block, shape_.npt, bps, blocks, (unsigned long long)m, smem, occ);
        if (occ < 1 || (uint64_t)occ * sm_count_ < blocks) continue;
        // smem offsets within each block
        for (uint32_t b = 0; b + 1 < bt.size(); ++b) {
            uint32_t off = 0;
            for (uint32_t k = bt[b]; k < bt[b + 1]; ++k) {
                tiles[k].smem_off = off;
                off += tiles[k].count;
            }
        }
        block_tiles = bt;
        res_neurons_ = (uint32_t)((m + 3) / 4 * 4);
        res_smem_ = smem;
        res_grid_ = blocks;
        return true;
    }
    return false;
}

ne2b_status Engine::rebuild_tiles() {
    const uint32_t tile = shape_.block * shape_.npt;
    std::vector<Tile> tiles;
    bool adex = false;
    for (NetHost *h : nets_)
        if (h) adex |= (h->dev.flags & kNetHasAdex) != 0u;
    if (adex != adex_) {
        adex_ = adex;
        clear_graphs();
    }
    for (NetHost *h : nets_) {
        if (!h) continue;
        for (uint32_t start = 0; start < h->n_pad; start += tile) {
            Tile t;
            memset(&t, 0, sizeof t);
            t.net = h->slot;
            t.start = start;
            t.count = std::min(tile, h->n_pad - start);
            t.flags = 0;
            if (!h->stim_ptr_host.empty()) {
                const uint32_t lo = std::min(start, h->n), hi = std::min(start + t.count, h->n);
                if (h->stim_ptr_host[hi] > h->stim_ptr_host[lo]) t.flags |= kTileHasStim;
            }
            tiles.push_back(t);
        }
    }
    stim_tiles_ = 0;
    for (const Tile &t : tiles) stim_tiles_ += (t.flags & kTileHasStim) ? 1u : 0u;
    const uint32_t old_grid = grid();
    std::vector<uint32_t> block_tiles;
    resident_ = plan_resident(tiles, block_tiles);
    if (mode_ == kModeResident && !resident_ && !tiles.empty())
        return set_error(NE2B_UNSUPPORTED, "the nets do not fit the resident kernel's shared memory");
    if (tiles.size() > tiles_cap_ || block_tiles.size() > block_tiles_cap_) NE2B_CUDA(cudaStreamSynchronize(stream_));
    if (tiles.size() > tiles_cap_) {
        uint32_t cap = tiles_cap_;
        while (cap < tiles.size()) cap *= 2;
        NE2B_CUDA(cudaFree(d_tiles_));
        d_tiles_ = nullptr;
        NE2B_CUDA(cudaMalloc(&d_tiles_, sizeof(Tile) * cap));
        tiles_cap_ = cap;
    }
    if (block_tiles.size() > block_tiles_cap_) {
        uint32_t cap = std::max<uint32_t>(block_tiles_cap_, 64);
        while (cap < block_tiles.size()) cap *= 2;
        NE2B_CUDA(cudaFree(d_block_tiles_));
        d_block_tiles_ = nullptr;
        NE2B_CUDA(cudaMalloc(&d_block_tiles_, sizeof(uint32_t) * cap));
        block_tiles_cap_ = cap;
    }
    if (!tiles.empty()) NE2B_TRY(pin_copy(d_tiles_, tiles.data(), sizeof(Tile) * tiles.size()));
    if (!block_tiles.empty())
        NE2B_TRY(pin_copy(d_block_tiles_, block_tiles.data(), sizeof(uint32_t) * block_tiles.size()));
    NE2B_TRY(pin_close());
    n_tiles_ = (uint32_t)tiles.size();
    NE2B_TRY(upload_eng());
    if (grid() != old_grid) clear_graphs();
    return NE2B_OK;
}

ne2b_status Engine::set_mode(int m) {
    if (m < kModeAuto || m > kModeResident) return set_error(NE2B_EINVAL, "kernel mode %d", m);
    NE2B_CUDA(cudaStreamSynchronize(stream_));
    const int old = mode_;
    mode_ = m;
    clear_graphs();
    ne2b_status st = rebuild_tiles();
    if (st != NE2B_OK) {
        mode_ = old;
        rebuild_tiles();
    }
    return st;
}

ne2b_status Engine::set_shape(const TileShape &s) {
    if (!shape_supported(s.block, s.npt))
        return set_error(NE2B_EINVAL, "tile shape block=%u npt=%u is not compiled in", s.block, s.npt);
    NE2B_CUDA(cudaStreamSynchronize(stream_));
    shape_ = s;
    clear_graphs();
    return rebuild_tiles();
}

ne2b_status Engine::reset_net(uint32_t slot) {
    NetHost *hp = net(slot);
    if (!hp) return set_error(NE2B_EINVAL, "no net in slot %u", slot);
    NetHost &h = *hp;
    NetDev &d = h.dev;
    NE2B_CUDA(launch_reset_neurons(d, stream_));
    launches_ += d.n_pad ? 1 : 0;
    NE2B_CUDA(cudaMemsetAsync(d.ring, 0, sizeof(uint32_t) * (size_t)h.D * h.n_pad, stream_));
    if (d.rec_bits) NE2B_CUDA(cudaMemsetAsync(d.rec_bits, 0, sizeof(uint32_t) * (size_t)d.rec_rows * (h.n_pad / 32), stream_));
    if (d.win_out) NE2B_CUDA(cudaMemsetAsync(d.win_out, 0, sizeof(uint16_t) * (size_t)d.max_windows * h.n_pad, stream_));
    if (d.trace_f) NE2B_CUDA(cudaMemsetAsync(d.trace_f, 0, sizeof(float) * h.n_pad, stream_));
    if (h.nx) {
        NE2B_CUDA(cudaMemsetAsync(d.xsyn, 0, sizeof(float) * h.nx, stream_));
        NE2B_CUDA(cudaMemsetAsync(d.xpend, 0, sizeof(uint32_t) * (size_t)h.D * d.xwords, stream_));
    }
    // cpu.rs:176-183: the watch history and the grid marks start over
    h.watch_t0 = 0;
    if (d.gw_ls) NE2B_CUDA(cudaMemsetAsync(d.gw_ls, 0xFF, sizeof(uint32_t) * std::max<uint32_t>(h.gw_ptr.back(), 1), stream_));
    NE2B_CUDA(cudaMemsetAsync(d_counters_ + slot, 0, sizeof(NetCounters), stream_));
    h.t = 0;
    set_step(d, 0);
    if (!h.fixed_stim) d.stim_len = 0;  // repack from t = 0
    return upload_net(h);
}

ne2b_status Engine::sync() {
    NE2B_CUDA(cudaStreamSynchronize(stream_));
    return check_err();
}

// A grid barrier of the resident kernel that timed out leaves a flag; the
// state of that launch is not trustworthy, so the next sync reports it.
ne2b_status Engine::check_err() {
    unsigned int e = 0;
    NE2B_CUDA(cudaMemcpy(&e, d_err_, sizeof e, cudaMemcpyDeviceToHost));
    if (e) {
        NE2B_CUDA(cudaMemset(d_err_, 0, sizeof e));
        if (e == kErrDeliveryQueue)
            return set_error(NE2B_ECUDA, "step kernel: a delivery-queue wait exceeded its limit; state is invalid");
        return set_error(NE2B_ECUDA, "resident kernel: a grid barrier wait exceeded its limit; state is invalid");
    }
    return NE2B_OK;
}

ne2b_status Engine::stage_reserve(size_t bytes) {
    if (bytes <= stage_bytes_) return NE2B_OK;
    NE2B_CUDA(cudaStreamSynchronize(stream_));
    if (stage_) cudaFreeHost(stage_);
    stage_ = nullptr;
    stage_bytes_ = 0;
    size_t cap = 1 << 20;
    while (cap < bytes) cap *= 2;
    NE2B_CUDA(cudaMallocHost(&stage_, cap));
    stage_bytes_ = cap;
    return NE2B_OK;
}

// Pack the stimulus program of every net in `nets` for steps [t, t + rows)
// (stim.rs:118-127 Stimulus::pack) into one pinned staging buffer, copy each
// to its device buffer, then copy every net descriptor, and synchronise once.
ne2b_status Engine::pack_stim(const std::vector<NetHost *> &nets) {
    size_t bytes = 0;
    for (NetHost *h : nets) bytes += sizeof(float) * (size_t)h->stim_cap * h->n_inputs;
    bytes = (bytes + 255) / 256 * 256;
    NE2B_TRY(stage_reserve(bytes + sizeof(NetDev) * nets_cap_));
    uint8_t *base = (uint8_t *)stage_;
    size_t off = 0;
    for (NetHost *h : nets) {
        const uint32_t ni = h->n_inputs;
        const uint64_t rows = h->stim_cap;
        float *dst = (float *)(base + off);
        for (uint64_t r = 0; r < rows; ++r)
            for (uint32_t k = 0; k < ni; ++k) dst[(size_t)r * ni + k] = h->stim.value(k, h->t + r);
        const size_t b = sizeof(float) * (size_t)rows * ni;
        NE2B_CUDA(cudaMemcpyAsync((void *)h->dev.stim_buf, dst, b, cudaMemcpyHostToDevice, stream_));
        h->dev.stim_t0 = (long long)h->t;
        h->dev.stim_len = (uint32_t)rows;
        off += b;
    }
    NetDev *mirror = (NetDev *)(base + bytes);
    for (uint32_t j = 0; j < nets_cap_; ++j) {
        if (nets_[j]) mirror[j] = nets_[j]->dev;
        else memset(&mirror[j], 0, sizeof(NetDev));
    }
    NE2B_CUDA(cudaMemcpyAsync(d_nets_, mirror, sizeof(NetDev) * nets_cap_, cudaMemcpyHostToDevice, stream_));
    NE2B_CUDA(cudaStreamSynchronize(stream_));
    return NE2B_OK;
}

// A fixed [steps x n_inputs] input matrix, device-resident from the current
// step on: nothing is packed during runs (batched and served trials).
ne2b_status Engine::set_input_matrix(NetHost &h, const float *x, uint64_t steps) {
    if (!h.n_inputs || h.stim_ptr_host.empty()) return NE2B_OK;  // no stimulus routing
    if (steps == 0 || !x) return set_error(NE2B_EINVAL, "empty input matrix");
    if (steps > 0xffffffffull) return set_error(NE2B_EINVAL, "input matrix longer than 2^32-1 steps");
    const size_t bytes = sizeof(float) * (size_t)steps * h.n_inputs;
    void *p = nullptr;
    NE2B_CUDA(cudaMallocAsync(&p, bytes, stream_));
    ne2b_status cs = pin_copy(p, x, bytes);
    if (cs == NE2B_OK) cs = pin_close();
    if (cs != NE2B_OK) {
        cudaFreeAsync(p, stream_);
        return cs;
    }
    void *old = (void *)h.dev.stim_buf;
    for (auto &a : h.allocs)
        if (a == old) {
            NE2B_CUDA(cudaFreeAsync(old, stream_));
            h.dev_bytes -= sizeof(float) * (size_t)(h.fixed_stim ? h.dev.stim_len : h.stim_cap) * h.n_inputs;
            a = p;
            old = nullptr;
            break;
        }
    if (old) h.allocs.push_back(p);
    h.dev_bytes += bytes;
    h.dev.stim_buf = (const float *)p;
    h.dev.stim_t0 = (long long)h.t;
    h.dev.stim_len = (uint32_t)steps;
    h.fixed_stim = true;
    return upload_net(h);
}

ne2b_status Engine::launch_group(uint32_t steps) {
    if (n_tiles_ == 0 || steps == 0) return NE2B_OK;
    if (resident_) {
        NE2B_CUDA(cudaMemsetAsync(d_barrier_, 0, sizeof(unsigned int), stream_));
        NE2B_CUDA(launch_resident(int_ring_, adex_, shape_.block, shape_.npt, d_eng_, 0, steps, res_grid_, res_smem_, stream_));
        NE2B_CUDA(launch_advance(d_nets_, nets_cap_, steps, stream_));
        launches_ += 2;
        return NE2B_OK;
    }
    // the instance follows the nets' features (an external current or a
    // watch can be switched on and off between launches)
    const int var = step_variant();
    if (var != graph_variant_) {
        clear_graphs();
        graph_variant_ = var;
    }
    const uint32_t g = grid();
    if (steps == graph_steps) {
        auto it = graphs_.find(steps);
        if (it == graphs_.end()) {
            cudaGraph_t gr;
            NE2B_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
            cudaError_t err = cudaSuccess;
            for (uint32_t k = 0; k < steps && err == cudaSuccess; ++k)
                err = launch_step(int_ring_, adex_, var, shape_.block, shape_.npt, d_eng_, k, g, stream_);
            if (err == cudaSuccess) err = launch_advance(d_nets_, nets_cap_, steps, stream_);
            cudaError_t e2 = cudaStreamEndCapture(stream_, &gr);
            if (err != cudaSuccess) return cuda_error(err, "step launch during capture");
            NE2B_CUDA(e2);
            cudaGraphExec_t ex;
            cudaError_t e3 = cudaGraphInstantiate(&ex, gr, 0);
            cudaGraphDestroy(gr);
            NE2B_CUDA(e3);
            it = graphs_.emplace(steps, ex).first;
        }
        NE2B_CUDA(cudaGraphLaunch(it->second, stream_));
        launches_ += steps + 1;
        return NE2B_OK;
    }
    for (uint32_t k = 0; k < steps; ++k) NE2B_CUDA(launch_step(int_ring_, adex_, var, shape_.block, shape_.npt, d_eng_, k, g, stream_));
    NE2B_CUDA(launch_advance(d_nets_, nets_cap_, steps, stream_));
    launches_ += steps + 1;
    return NE2B_OK;
}

ne2b_status Engine::run_steps(uint64_t steps) {
    NE2B_CUDA(cudaSetDevice(device_));
    while (steps > 0) {
        uint64_t chunk = steps;
        for (NetHost *h : nets_)
            if (h && h->stim_cap && !h->fixed_stim) chunk = std::min<uint64_t>(chunk, h->stim_cap);
        std::vector<NetHost *> repack;
        for (NetHost *h : nets_) {
            if (!h || !h->stim_cap || h->fixed_stim) continue;
            const uint64_t lo = (uint64_t)h->dev.stim_t0, hi = lo + h->dev.stim_len;
            if (!(h->dev.stim_len > 0 && h->t >= lo && h->t + chunk <= hi)) repack.push_back(h);
        }
        if (!repack.empty()) NE2B_TRY(pack_stim(repack));
        uint64_t left = chunk;
        const uint64_t group = resident_ ? std::max<uint64_t>(graph_steps, resident_steps) : graph_steps;
        while (left > 0) {
            const uint32_t g = (uint32_t)std::min<uint64_t>(left, group);
            NE2B_TRY(launch_group(g));
            left -= g;
        }
        for (NetHost *h : nets_)
            if (h) {
                h->t = std::min<uint64_t>(h->t + chunk, h->t_end);
                set_step(h->dev, h->t);
            }
        steps -= chunk;
    }
    return NE2B_OK;
}

ne2b_status Engine::read_csr(NetHost &h, uint32_t *rowptr, uint32_t *tgt, uint32_t *w_bits, uint16_t *delay_steps) {
    const NetDev &d = h.dev;
    if (rowptr) NE2B_CUDA(cudaMemcpyAsync(rowptr, d.rowptr, sizeof(uint32_t) * ((size_t)h.n + 1), cudaMemcpyDeviceToHost, stream_));
    const bool wide = d.flags & kNetDelayWide;
    if (delay_steps && wide && h.e)
        NE2B_CUDA(cudaMemcpyAsync(delay_steps, d.delay16, sizeof(uint16_t) * h.e, cudaMemcpyDeviceToHost, stream_));
    if (h.e && (tgt || w_bits || delay_steps)) {
        // unpack the records (target | delay << 24, weight bits) through a
        // bounded host buffer, a chunk at a time
        const uint64_t chunk = std::min<uint64_t>(h.e, 1ull << 22);
        std::vector<SynRec> rec(chunk);
        for (uint64_t j0 = 0; j0 < h.e; j0 += chunk) {
            const uint64_t m = std::min<uint64_t>(chunk, h.e - j0);
            NE2B_CUDA(cudaMemcpyAsync(rec.data(), d.syn + j0, sizeof(SynRec) * m, cudaMemcpyDeviceToHost, stream_));
            NE2B_CUDA(cudaStreamSynchronize(stream_));
            for (uint64_t j = 0; j < m; ++j) {
                if (tgt) tgt[j0 + j] = wide ? rec[j].td : rec[j].td & kSynTgtMask;
                if (w_bits) w_bits[j0 + j] = rec[j].w;
                if (delay_steps && !wide) delay_steps[j0 + j] = (uint16_t)(rec[j].td >> kSynTgtBits);
            }
        }
    }
    NE2B_CUDA(cudaStreamSynchronize(stream_));
    return NE2B_OK;
}

ne2b_status Engine::read_f32(const float *dev, uint32_t n, float *out) {
    if (n == 0) return NE2B_OK;
    NE2B_CUDA(cudaMemcpyAsync(out, dev, sizeof(float) * n, cudaMemcpyDeviceToHost, stream_));
    NE2B_CUDA(cudaStreamSynchronize(stream_));
    return check_err();
}

ne2b_status Engine::read_trace(NetHost &h, float *out) {
    if (h.n == 0) return NE2B_OK;
    if (h.dev.trace_f) return read_f32(h.dev.trace_f, h.n, out);
    float *tmp = nullptr;
    NE2B_CUDA(cudaMallocAsync((void **)&tmp, sizeof(float) * h.n, stream_));
    cudaError_t e = launch_trace(h.dev.tk, h.dev.trace_tab, h.n, tmp, stream_);
    launches_ += 1;
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, tmp, sizeof(float) * h.n, cudaMemcpyDeviceToHost, stream_);
    cudaFreeAsync(tmp, stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    NE2B_TRY(cuda_error(e, "trace readback"));
    return check_err();
}

ne2b_status Engine::spike_counts(NetHost &h, uint64_t rows, uint32_t *out) {
    const uint32_t n = h.n;
    if (!h.dev.rec_rows || h.t == 0) {  // cpu.rs:425-428
        memset(out, 0, sizeof(uint32_t) * n);
        return NE2B_OK;
    }
    if (rows < h.t && rows > h.dev.rec_rows)
        return set_error(NE2B_EWINDOW, "spike_counts window %llu exceeds the recorded %u steps",
                         (unsigned long long)rows, h.dev.rec_rows);
    if (n == 0) return NE2B_OK;
    uint32_t *tmp = nullptr;
    NE2B_CUDA(cudaMallocAsync((void **)&tmp, sizeof(uint32_t) * n, stream_));
    cudaError_t e;
    if (rows >= h.t) e = launch_pn_total(h.dev.pn_total, n, tmp, stream_);
    else e = launch_window_count(h.dev.rec_bits, h.dev.rec_rows, h.n_pad, n, h.t, (uint32_t)rows, tmp, stream_);
    launches_ += 1;
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, tmp, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, stream_);
    cudaFreeAsync(tmp, stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    return cuda_error(e, "spike_counts");
}

ne2b_status Engine::spike_row(NetHost &h, uint32_t back, uint64_t *out) {
    const uint32_t rr = h.dev.rec_rows;
    if (!rr || h.t == 0 || back >= h.t || back >= rr)  // cpu.rs:399-406
        return set_error(NE2B_ENODATA, "spike_row %u is outside the recorded window", back);
    const uint64_t t = h.t - 1 - back;
    const uint32_t row = (uint32_t)(t % rr);
    const uint32_t words = (h.n + 63) / 64;
    NE2B_CUDA(cudaMemcpyAsync(out, h.dev.rec_bits + (size_t)row * (h.n_pad / 32), sizeof(uint64_t) * words,
                              cudaMemcpyDeviceToHost, stream_));
    NE2B_CUDA(cudaStreamSynchronize(stream_));
    return NE2B_OK;
}

ne2b_status Engine::spikes_total(NetHost &h, uint64_t *out) {
    NE2B_CUDA(cudaMemcpyAsync(out, &d_counters_[h.slot].spikes_total, sizeof(uint64_t), cudaMemcpyDeviceToHost, stream_));
    NE2B_CUDA(cudaStreamSynchronize(stream_));
    return NE2B_OK;
}

ne2b_status Engine::window_counts(NetHost &h, uint32_t window, uint16_t *out) {
    if (!h.dev.win_out) return set_error(NE2B_EINVAL, "window counts are off (window_steps = 0)");
    if (window >= h.dev.max_windows) return set_error(NE2B_EINVAL, "window %u >= max_windows %u", window, h.dev.max_windows);
    if (h.n == 0) return NE2B_OK;
    NE2B_CUDA(cudaMemcpyAsync(out, h.dev.win_out + (size_t)window * h.n_pad, sizeof(uint16_t) * h.n,
                              cudaMemcpyDeviceToHost, stream_));
    NE2B_CUDA(cudaStreamSynchronize(stream_));
    return NE2B_OK;
}

ne2b_status Engine::set_ext(NetHost &h, const float *ext, uint32_t len) {
    const uint32_t m = std::min(len, h.n);
    for (uint32_t i = 0; i < m; ++i) h.ext_host[i] = ext[i];
    bool any = false;
    for (float x : h.ext_host) {
        uint32_t b;
        memcpy(&b, &x, 4);
        if (b) { any = true; break; }
    }
    if (h.n) NE2B_CUDA(cudaMemcpyAsync(h.dev.ext, h.ext_host.data(), sizeof(float) * h.n, cudaMemcpyHostToDevice, stream_));
    h.dev.flags = any ? (h.dev.flags | kNetHasExt) : (h.dev.flags & ~kNetHasExt);
    return upload_net(h);
}

ne2b_status Engine::refresh_noise(NetHost &h) {
    fill_noise(h.dev, h.cfg);
    return upload_net(h);
}

// cpu.rs:330-338: a new list starts an empty history; the same list keeps it.
// Each distinct id below n gets a ring row; an id beyond n records 0.
ne2b_status Engine::set_v_watch(NetHost &h, const uint32_t *ids, uint32_t count) {
    if (count && !ids) return set_error(NE2B_EINVAL, "null ids");
    if (count == h.watch_ids.size() && std::equal(h.watch_ids.begin(), h.watch_ids.end(), ids)) return NE2B_OK;
    NE2B_CUDA(cudaStreamSynchronize(stream_));  // no launch in flight writes the old ring
    for (void *p : h.watch_allocs) NE2B_CUDA(cudaFreeAsync(p, stream_));
    h.watch_allocs.clear();
    h.watch_ids.assign(ids, ids + count);
    h.watch_row.assign(count, -1);
    std::vector<uint32_t> idx(h.n_pad, kNoWatch);
    uint32_t rows = 0;
    for (uint32_t k = 0; k < count; ++k) {
        const uint32_t i = ids[k];
        if (i >= h.n) continue;
        if (idx[i] == kNoWatch) idx[i] = rows++;
        h.watch_row[k] = (int32_t)idx[i];
    }
    h.watch_t0 = h.t;
    h.dev.watch_idx = nullptr;
    h.dev.watch_ring = nullptr;
    h.dev.watch_n = rows;
    h.dev.flags &= ~kNetWatch;
    if (rows) {
        void *p = nullptr;
        NE2B_CUDA(cudaMallocAsync(&p, sizeof(uint32_t) * h.n_pad, stream_));
        h.watch_allocs.push_back(p);
        NE2B_TRY(pin_copy(p, idx.data(), sizeof(uint32_t) * h.n_pad));
        h.dev.watch_idx = (const uint32_t *)p;
        NE2B_CUDA(cudaMallocAsync(&p, sizeof(float) * 2 * (size_t)rows * kWatchCap, stream_));
        h.watch_allocs.push_back(p);
        h.dev.watch_ring = (float *)p;
        NE2B_TRY(pin_close());
        h.dev.flags |= kNetWatch;
    }
    return upload_net(h);
}

// drain_state for both slots (cpu.rs:350-357): the samples of steps
// [max(t0, t - kWatchCap), t), oldest first, then an empty history.
ne2b_status Engine::drain_watch(NetHost &h, float *out, uint32_t *count) {
    const uint64_t span = h.t - std::min(h.watch_t0, h.t);
    const uint32_t c = (uint32_t)std::min<uint64_t>(span, kWatchCap);
    const uint32_t w = (uint32_t)h.watch_ids.size();
    *count = c;
    if (c && w && out) {
        std::vector<float> ring(2 * (size_t)h.dev.watch_n * kWatchCap);
        if (h.dev.watch_n) {
            NE2B_CUDA(cudaMemcpyAsync(ring.data(), h.dev.watch_ring, sizeof(float) * ring.size(),
                                      cudaMemcpyDeviceToHost, stream_));
            NE2B_CUDA(cudaStreamSynchronize(stream_));
        }
        const uint64_t first = h.t - c;
        for (uint32_t slot = 0; slot < 2; ++slot)
            for (uint32_t k = 0; k < w; ++k) {
                float *o = out + ((size_t)slot * w + k) * c;
                const int32_t row = h.watch_row[k];
                for (uint32_t j = 0; j < c; ++j)
                    o[j] = row < 0 ? 0.0f
                                   : ring[((size_t)slot * h.dev.watch_n + (uint32_t)row) * kWatchCap +
                                          ((first + j) & (kWatchCap - 1u))];
            }
    }
    h.watch_t0 = h.t;
    return NE2B_OK;
}

// cpu.rs:361-387: member lists in texel order (a neuron's texel is its
// last position in the list); the same lists keep their marks.
ne2b_status Engine::set_grid_watches(NetHost &h, const uint32_t *members, const uint32_t *group_ptr,
                                     uint32_t ngroups) {
    if (ngroups && !group_ptr) return set_error(NE2B_EINVAL, "null group_ptr");
    const uint32_t total = ngroups ? group_ptr[ngroups] : 0;
    if (total && !members) return set_error(NE2B_EINVAL, "null members");
    for (uint32_t g = 0; g < ngroups; ++g)
        if (group_ptr[g] > group_ptr[g + 1]) return set_error(NE2B_EINVAL, "group_ptr not monotone");
    if (ngroups && group_ptr[0] != 0) return set_error(NE2B_EINVAL, "group_ptr[0] != 0");
    const bool same = ngroups == 0 ? h.gw_ptr.empty()
                                   : (h.gw_ptr.size() == (size_t)ngroups + 1 &&
                                      std::equal(h.gw_ptr.begin(), h.gw_ptr.end(), group_ptr) &&
                                      h.gw_members.size() == total &&
                                      std::equal(h.gw_members.begin(), h.gw_members.end(), members));
    if (same) return NE2B_OK;
    NE2B_CUDA(cudaStreamSynchronize(stream_));
    for (void *p : h.gw_allocs) NE2B_CUDA(cudaFreeAsync(p, stream_));
    h.gw_allocs.clear();
    h.gw_ptr.assign(group_ptr, group_ptr + (ngroups ? ngroups + 1 : 0));
    h.gw_members.assign(members, members + total);
    h.dev.gw_map = nullptr;
    h.dev.gw_off = nullptr;
    h.dev.gw_ls = nullptr;
    h.dev.gw_n = ngroups;
    h.dev.flags &= ~kNetGridWatch;
    if (ngroups) {
        std::vector<int32_t> map((size_t)ngroups * h.n_pad, -1);
        for (uint32_t g = 0; g < ngroups; ++g)
            for (uint32_t k = group_ptr[g]; k < group_ptr[g + 1]; ++k)
                if (members[k] < h.n) map[(size_t)g * h.n_pad + members[k]] = (int32_t)(k - group_ptr[g]);
        void *p = nullptr;
        NE2B_CUDA(cudaMallocAsync(&p, sizeof(int32_t) * map.size(), stream_));
        h.gw_allocs.push_back(p);
        NE2B_TRY(pin_copy(p, map.data(), sizeof(int32_t) * map.size()));
        h.dev.gw_map = (const int32_t *)p;
        NE2B_CUDA(cudaMallocAsync(&p, sizeof(uint32_t) * ((size_t)ngroups + 1), stream_));
        h.gw_allocs.push_back(p);
        NE2B_TRY(pin_copy(p, group_ptr, sizeof(uint32_t) * ((size_t)ngroups + 1)));
        h.dev.gw_off = (const uint32_t *)p;
        NE2B_CUDA(cudaMallocAsync(&p, sizeof(uint32_t) * std::max<uint32_t>(total, 1), stream_));
        h.gw_allocs.push_back(p);
        NE2B_CUDA(cudaMemsetAsync(p, 0xFF, sizeof(uint32_t) * std::max<uint32_t>(total, 1), stream_));
        h.dev.gw_ls = (uint32_t *)p;
        NE2B_TRY(pin_close());
        h.dev.flags |= kNetGridWatch;
    }
    return upload_net(h);
}

// cpu.rs:391-407: exp(-(t - last) * dt / tau) per texel (f32, libm expf),
// 0 for a texel that never spiked; groups concatenated in order.
ne2b_status Engine::grid_traces(NetHost &h, float tau_ms, float *out) {
    const uint32_t ng = h.gw_ptr.empty() ? 0 : (uint32_t)h.gw_ptr.size() - 1;
    const uint32_t total = ng ? h.gw_ptr[ng] : 0;
    if (!total) return NE2B_OK;
    std::vector<uint32_t> ls(total);
    NE2B_CUDA(cudaMemcpyAsync(ls.data(), h.dev.gw_ls, sizeof(uint32_t) * total, cudaMemcpyDeviceToHost, stream_));
    NE2B_CUDA(cudaStreamSynchronize(stream_));
    const float k = h.cfg.dt_ms / (tau_ms > 1e-6f ? tau_ms : 1e-6f);
    for (uint32_t j = 0; j < total; ++j)
        out[j] = ls[j] == kNeverSpiked ? 0.0f : expf(-(float)(h.t > ls[j] ? h.t - ls[j] : 0) * k);
    return NE2B_OK;
}

// Snapshot of every mutable device array (state, ring, record, windows,
// descriptors, counters) in device memory, for the autotuner's trials.
ne2b_status Engine::snapshot(EngineSnapshot &snap) {
    snap.items.clear();
    snap.hosts.clear();
    auto grab = [&](void *live, size_t bytes) -> ne2b_status {
        if (!live || !bytes) return NE2B_OK;
        void *b = nullptr;
        NE2B_CUDA(cudaMallocAsync(&b, bytes, stream_));
        snap.items.push_back({live, b, bytes});
        NE2B_CUDA(cudaMemcpyAsync(b, live, bytes, cudaMemcpyDeviceToDevice, stream_));
        return NE2B_OK;
    };
    NE2B_TRY(grab(d_nets_, sizeof(NetDev) * nets_cap_));
    NE2B_TRY(grab(d_counters_, sizeof(NetCounters) * nets_cap_));
    for (NetHost *h : nets_) {
        if (!h) continue;
        NetDev &d = h->dev;
        const size_t np = h->n_pad;
        NE2B_TRY(grab(d.v, 4 * np));
        NE2B_TRY(grab(d.u, 4 * np));
        NE2B_TRY(grab(d.s, 4 * np));
        NE2B_TRY(grab(d.tk, 2 * np));
        NE2B_TRY(grab(d.trace_f, d.trace_f ? 4 * np : 0));
        NE2B_TRY(grab(d.pn_total, 8 * np));
        NE2B_TRY(grab(d.ring, 4 * (size_t)h->D * np));
        NE2B_TRY(grab(d.rec_bits, d.rec_bits ? 4 * (size_t)d.rec_rows * (np / 32) : 0));
        NE2B_TRY(grab(d.wcount, d.wcount ? 4 * np : 0));
        NE2B_TRY(grab(d.win_out, d.win_out ? 2 * (size_t)d.max_windows * np : 0));
        NE2B_TRY(grab(d.xsyn, 4 * (size_t)h->nx));
        NE2B_TRY(grab(d.watch_ring, d.watch_ring ? 8 * (size_t)d.watch_n * kWatchCap : 0));
        NE2B_TRY(grab(d.gw_ls, d.gw_ls ? 4 * (size_t)std::max<uint32_t>(h->gw_ptr.back(), 1) : 0));
        NE2B_TRY(grab(d.xpend, 4 * (size_t)h->D * d.xwords));
        snap.hosts.push_back({h->slot, h->t, h->dev});
    }
    return NE2B_OK;
}

ne2b_status Engine::restore(const EngineSnapshot &snap) {
    for (const auto &it : snap.items)
        NE2B_CUDA(cudaMemcpyAsync(it.live, it.backup, it.bytes, cudaMemcpyDeviceToDevice, stream_));
    for (const auto &hs : snap.hosts) {
        NetHost *h = net(hs.slot);
        if (!h) continue;
        h->t = hs.t;
        h->dev = hs.dev;
    }
    return NE2B_OK;
}

void Engine::drop(EngineSnapshot &snap) {
    for (const auto &it : snap.items) cudaFreeAsync(it.backup, stream_);
    snap.items.clear();
    snap.hosts.clear();
}

// Time every (kernel, tile shape, occupancy) candidate on the live nets for
// `steps_per_trial` steps, restoring the state after each trial, and keep
// the fastest.  Candidates: the streaming kernel at full and half
// occupancy, the resident kernel wherever its shared-memory plan fits.
ne2b_status Engine::autotune(uint32_t steps_per_trial) {
    if (steps_per_trial == 0) steps_per_trial = graph_steps;
    EngineSnapshot snap;
    NE2B_TRY(snapshot(snap));
    // bring the clocks up from idle and size the trials: every candidate runs
    // at least ~3 ms of steps, twice, and keeps its faster repetition
    {
        float ms = 0.0f;
        for (int rep = 0; rep < 8 && ms < 30.0f; ++rep) {
            NE2B_TRY(restore(snap));
            NE2B_CUDA(cudaEventRecord(ev0_, stream_));
            NE2B_TRY(run_steps(steps_per_trial));
            NE2B_CUDA(cudaEventRecord(ev1_, stream_));
            NE2B_CUDA(cudaEventSynchronize(ev1_));
            float one = 0.0f;
            NE2B_CUDA(cudaEventElapsedTime(&one, ev0_, ev1_));
            ms += one;
            if (one > 0.0f && one < 3.0f) steps_per_trial = (uint32_t)std::min<double>(65536.0, steps_per_trial * 3.0 / one + 1);
        }
    }
    uint32_t blocks[32], npts[32], count = 0;
    shape_list(blocks, npts, &count);
    const int saved_mode = mode_;
    TileShape best = shape_;
    int best_mode = mode_ == kModeAuto ? (resident_ ? kModeResident : kModeStream) : mode_;
    float best_ms = 1e30f;
    for (int m : {(int)kModeStream, (int)kModeResident}) {
        if (saved_mode != kModeAuto && m != saved_mode) continue;  // a forced kernel keeps its mode
        for (uint32_t c = 0; c < 2 * count; ++c) {
            // candidates c >= count: the same shapes with delivery warps
            TileShape s;
            s.block = blocks[c % count];
            s.npt = npts[c % count];
            s.ws = c >= count;
            if (s.ws && (m == kModeResident || !ws_applies(s))) continue;
            const int occ = step_occupancy(int_ring_, adex_, step_variant(s), s.block, s.npt);
            for (int half = 0; half < 2; ++half) {
                if (half && (m == kModeResident || occ < 2)) continue;
                s.blocks_per_sm = half ? (uint32_t)std::max(1, occ / 2) : 0;
                mode_ = m;
                shape_ = s;
                clear_graphs();
                if (rebuild_tiles() != NE2B_OK) continue;  // resident plan does not fit
                NE2B_TRY(restore(snap));
                NE2B_TRY(run_steps(graph_steps));  // capture + warm
                float ms = 1e30f;
                for (int rep = 0; rep < 2; ++rep) {
                    NE2B_TRY(restore(snap));
                    NE2B_CUDA(cudaEventRecord(ev0_, stream_));
                    NE2B_TRY(run_steps(steps_per_trial));
                    NE2B_CUDA(cudaEventRecord(ev1_, stream_));
                    NE2B_CUDA(cudaEventSynchronize(ev1_));
                    NE2B_TRY(check_err());
                    float one = 0.0f;
                    NE2B_CUDA(cudaEventElapsedTime(&one, ev0_, ev1_));
                    ms = std::min(ms, one);
                }
                if (ms < best_ms) {
                    best_ms = ms;
                    best = s;
                    best_mode = m;
                }
            }
        }
    }
    mode_ = saved_mode == kModeAuto ? best_mode : saved_mode;
    shape_ = best;
    clear_graphs();
    NE2B_TRY(rebuild_tiles());
    NE2B_TRY(restore(snap));
    drop(snap);
    NE2B_CUDA(cudaStreamSynchronize(stream_));
    last_ms_ = best_ms;
    return NE2B_OK;
}

}  // namespace ne2b
