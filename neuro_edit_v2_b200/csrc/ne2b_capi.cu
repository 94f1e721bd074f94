// ne2b_capi.cu — the extern "C" entry points declared in include/ne2b.h.
// Each entry point validates its handle and arguments, calls the Engine and
// returns a status; no exception or abort crosses the boundary.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <map>
#include <new>
#include <vector>

#include "ne2b_engine.h"
#include "ne2b_kernels.h"
#include "ne2b_parallel.h"

using ne2b::Engine;
using ne2b::NetHost;
using ne2b::set_error;

namespace ne2b {
const char *last_error_str();
}

#include "ne2b_handles.h"

#define GUARD(expr)                                                            \
    do {                                                                       \
        try {                                                                  \
            return (expr);                                                     \
        } catch (const std::bad_alloc &) {                                     \
            return set_error(NE2B_ENOMEM, "host allocation failed");           \
        } catch (...) {                                                        \
            return set_error(NE2B_ECUDA, "unexpected internal exception");     \
        }                                                                      \
    } while (0)

#define CHECK_SIM(sim)                                                         \
    if (!(sim)) return set_error(NE2B_EINVAL, "null sim handle");              \
    NetHost *h = (sim)->eng.net((sim)->slot);                                  \
    if (!h) return set_error(NE2B_EINVAL, "sim has no network");

extern "C" {

void ne2b_config_default(ne2b_config *c) {
    if (!c) return;
    memset(c, 0, sizeof *c);
    c->dt_ms = 0.1f;            // net-format/src/lib.rs:39
    c->synapse_tau_ms = 2.0f;   // lib.rs:26
    c->readout_tau_ms = 2.0f;   // lib.rs:29
    c->noise_rate_hz = 0.0f;    // state.rs:41
    c->noise_kick_mv = 20.0f;   // state.rs:42
    c->seed = 1;
    c->record_spikes = 0;
    c->spike_record_steps = 512;
    c->int_weights = 0;
    c->gauss_sd = 0.0f;
    c->window_steps = 0;
    c->max_windows = 0;
}

const char *ne2b_last_error(void) { return ne2b::last_error_str(); }
const char *ne2b_version(void) { return "ne2b 0.1 sm_100a"; }

// ------------------------------------------------------------------- sim
ne2b_status ne2b_create(const ne2b_net_desc *net, const ne2b_config *cfg, int device, ne2b_sim **out) {
    if (!out || !net || !cfg) return set_error(NE2B_EINVAL, "ne2b_create: null argument");
    *out = nullptr;
    GUARD(([&]() -> ne2b_status {
        ne2b_sim *s = new ne2b_sim();
        ne2b_status st = s->eng.init(device, cfg->int_weights != 0, 1);
        if (st == NE2B_OK) st = s->eng.add_net(net, cfg, nullptr, 0, &s->slot);
        if (st != NE2B_OK) {
            delete s;
            return st;
        }
        *out = s;
        return NE2B_OK;
    })());
}

ne2b_status ne2b_destroy(ne2b_sim *sim) {
    delete sim;
    return NE2B_OK;
}

}  // extern "C"

// The synapse list on the device, checked by the prepass, then the net
// built with its CSR sorted into place there (csrc/ne2b_csr.cu).  Errors
// are the host build's (ne2b_net_from_synapses).
static ne2b_status create_from_list(ne2b::Engine &eng, const ne2b_net_desc *net, const uint8_t *kind, uint64_t E,
                                    const uint32_t *src, const uint32_t *tgt, const float *w, const float *dly,
                                    const ne2b_config *cfg, uint32_t *slot) {
    using namespace ne2b;
    const cudaStream_t st = eng.stream();
    const uint32_t n = net->n;
    std::vector<void *> tmp;
    auto release = [&]() {
        for (void *p : tmp) cudaFreeAsync(p, st);
        cudaStreamSynchronize(st);
    };
    auto dalloc = [&](size_t bytes, void **p) -> ne2b_status {
        *p = nullptr;
        const cudaError_t e = cudaMallocAsync(p, bytes ? bytes : 16, st);
        if (e != cudaSuccess) return cuda_error(e, "cudaMallocAsync (synapse list)");
        tmp.push_back(*p);
        return NE2B_OK;
    };
#define LIST_TRY(x)                          \
    do {                                     \
        const ne2b_status _s = (x);          \
        if (_s != NE2B_OK) {                 \
            release();                       \
            return _s;                       \
        }                                    \
    } while (0)
    // arrays already in device memory are read where they are; host arrays
    // are copied (through the stager's pinned ring when large)
    bool foreign = false;  // device memory of another GPU
    auto on_device = [&](const void *q) {
        cudaPointerAttributes a{};
        const bool dev = q && cudaPointerGetAttributes(&a, q) == cudaSuccess && a.type == cudaMemoryTypeDevice;
        cudaGetLastError();
        if (dev && a.device != eng.device()) foreign = true;
        return dev;
    };
    const bool d_src = on_device(src), d_tgt = on_device(tgt), d_w = on_device(w), d_dly = on_device(dly),
               d_kind = on_device(kind);
    if (foreign) return set_error(NE2B_EINVAL, "a synapse-list array is in another GPU's memory (the sim is on GPU %d)",
                                  eng.device());
    auto value_at = [&](const void *base, bool dev, uint64_t j) -> uint32_t {  // one 4-byte entry, for messages
        uint32_t v = 0;
        if (!dev) memcpy(&v, (const uint8_t *)base + 4 * j, 4);
        else cudaMemcpy(&v, (const uint8_t *)base + 4 * j, 4, cudaMemcpyDeviceToHost);
        return v;
    };
    DevCsrBuild dc;
    void *p = nullptr;
    if (d_src) dc.syn.src = src; else { LIST_TRY(dalloc(4 * E, &p)); dc.syn.src = (const uint32_t *)p; }
    if (d_tgt) dc.syn.tgt = tgt; else { LIST_TRY(dalloc(4 * E, &p)); dc.syn.tgt = (const uint32_t *)p; }
    if (d_w) dc.syn.w = w; else { LIST_TRY(dalloc(4 * E, &p)); dc.syn.w = (const float *)p; }
    if (d_dly) dc.syn.delay_ms = dly; else { LIST_TRY(dalloc(4 * E, &p)); dc.syn.delay_ms = (const float *)p; }
    if (d_kind) dc.syn.kind = kind; else { LIST_TRY(dalloc(n, &p)); dc.syn.kind = (const uint8_t *)p; }
    LIST_TRY(dalloc(2 * E, &p)); dc.steps = (const uint16_t *)p;
    LIST_TRY(dalloc(4 * (size_t)n, &p)); dc.counts = (const uint32_t *)p;
    LIST_TRY(dalloc(4 * (size_t)n, &p)); dc.cursor = (uint32_t *)p;
    LIST_TRY(dalloc(4 * (size_t)csr_scan_blocks(n), &p)); dc.sums = (uint32_t *)p;
    const uint64_t chunks = csr_chunks(E);
    LIST_TRY(dalloc(4 * (chunks + 1), &p)); dc.ticket = (uint32_t *)p;
    dc.done = dc.ticket + 1;
    LIST_TRY(dalloc(sizeof(CsrScalars), &p)); dc.sc = (CsrScalars *)p;
    dc.syn.n_syn = E;
    dc.syn.n = n;
    dc.syn.dt_ms = cfg->dt_ms;
    CsrScalars sc{~0ull, ~0ull, 1u, 0u};
    if (E) {
        if (!d_src) LIST_TRY(eng.pin_copy((void *)dc.syn.src, src, 4 * E));
        if (!d_tgt) LIST_TRY(eng.pin_copy((void *)dc.syn.tgt, tgt, 4 * E));
        if (!d_w) LIST_TRY(eng.pin_copy((void *)dc.syn.w, w, 4 * E));
        if (!d_dly) LIST_TRY(eng.pin_copy((void *)dc.syn.delay_ms, dly, 4 * E));
    }
    if (n && !d_kind) LIST_TRY(eng.pin_copy((void *)dc.syn.kind, kind, n));
    LIST_TRY(eng.pin_copy(dc.sc, &sc, sizeof sc));
    LIST_TRY(eng.pin_close());
    LIST_TRY(cuda_error(cudaMemsetAsync((void *)dc.counts, 0, 4 * (size_t)n, st), "memset counts"));
    LIST_TRY(cuda_error(cudaMemsetAsync(dc.ticket, 0, 4 * (chunks + 1), st), "memset tickets"));
    LIST_TRY(cuda_error(csr_prepass(dc.syn, (uint32_t *)dc.counts, (uint16_t *)dc.steps, dc.sc, st), "csr prepass"));
    LIST_TRY(cuda_error(cudaMemcpyAsync(&sc, dc.sc, sizeof sc, cudaMemcpyDeviceToHost, st), "prepass readback"));
    LIST_TRY(cuda_error(cudaStreamSynchronize(st), "prepass"));
    if (sc.bad_ref != ~0ull) {
        const uint64_t j = sc.bad_ref;
        LIST_TRY(set_error(NE2B_EINVAL, "synapse %llu references %u -> %u but only %u neurons exist",
                           (unsigned long long)j, value_at(src, d_src, j), value_at(tgt, d_tgt, j), n));
    }
    if (sc.bad_delay != ~0ull) {
        const uint64_t j = sc.bad_delay;
        const uint32_t db = value_at(dly, d_dly, j);
        float dv;
        memcpy(&dv, &db, sizeof dv);
        LIST_TRY(set_error(NE2B_EINVAL, "synapse %u -> %u: delay %g ms at dt %g ms exceeds the 65535-step ring",
                           value_at(src, d_src, j), value_at(tgt, d_tgt, j), (double)dv, (double)cfg->dt_ms));
    }
    dc.max_delay = sc.max_delay;
    LIST_TRY(eng.add_net_device_csr(net, cfg, dc, slot));
    LIST_TRY(cuda_error(cudaMemcpyAsync(&sc, dc.sc, sizeof sc, cudaMemcpyDeviceToHost, st), "scatter readback"));
    LIST_TRY(cuda_error(cudaStreamSynchronize(st), "device CSR build"));
    release();
#undef LIST_TRY
    if (sc.timeout) return set_error(NE2B_ECUDA, "device CSR build: a scatter block's wait exceeded its limit");
    return NE2B_OK;
}

extern "C" {

ne2b_status ne2b_create_from_synapses(const ne2b_net_desc *net, const uint8_t *kind, uint64_t n_syn,
                                      const uint32_t *src, const uint32_t *tgt, const float *w,
                                      const float *delay_ms, const ne2b_config *cfg, int device, ne2b_sim **out) {
    if (!out || !net || !cfg) return set_error(NE2B_EINVAL, "ne2b_create_from_synapses: null argument");
    *out = nullptr;
    if (net->n_syn || net->src_ptr || net->tgt || net->w || net->delay_steps || net->tau_ms)
        return set_error(NE2B_EINVAL, "the net's CSR fields must be empty: its synapses come as a list");
    if (net->n && (!net->model || !net->params || !kind))
        return set_error(NE2B_EINVAL, "model, params and kind are required");
    if (n_syn && (!src || !tgt || !w || !delay_ms)) return set_error(NE2B_EINVAL, "synapse arrays are required");
    if (n_syn > 0xffffffffull) return set_error(NE2B_UNSUPPORTED, "more than 2^32-1 synapses");
    if (!(cfg->dt_ms >= 0.001f && cfg->dt_ms <= 100.0f))  // lib.rs:35-39 valid_dt_ms
        return set_error(NE2B_EINVAL, "dt_ms %g outside [0.001, 100]", (double)cfg->dt_ms);
    GUARD(([&]() -> ne2b_status {
        ne2b_sim *s = new ne2b_sim();
        ne2b_status st = s->eng.init(device, cfg->int_weights != 0, 1);
        if (st == NE2B_OK) st = create_from_list(s->eng, net, kind, n_syn, src, tgt, w, delay_ms, cfg, &s->slot);
        if (st != NE2B_OK) {
            delete s;
            return st;
        }
        *out = s;
        return NE2B_OK;
    })());
}

ne2b_status ne2b_syn_count(const ne2b_sim *sim, uint64_t *e) {
    CHECK_SIM(const_cast<ne2b_sim *>(sim));
    if (!e) return set_error(NE2B_EINVAL, "null argument");
    *e = h->e;
    return NE2B_OK;
}

ne2b_status ne2b_read_csr(ne2b_sim *sim, uint32_t *rowptr, uint32_t *tgt, uint32_t *w_bits, uint16_t *delay_steps) {
    CHECK_SIM(sim);
    GUARD(sim->eng.read_csr(*h, rowptr, tgt, w_bits, delay_steps));
}

ne2b_status ne2b_n(const ne2b_sim *sim, uint32_t *n) {
    CHECK_SIM(const_cast<ne2b_sim *>(sim));
    *n = h->n;
    return NE2B_OK;
}

ne2b_status ne2b_step_count(const ne2b_sim *sim, uint64_t *t) {
    CHECK_SIM(const_cast<ne2b_sim *>(sim));
    *t = h->t;
    return NE2B_OK;
}

ne2b_status ne2b_time_ms(const ne2b_sim *sim, double *ms) {
    CHECK_SIM(const_cast<ne2b_sim *>(sim));
    *ms = (double)h->t * (double)h->cfg.dt_ms;  // cpu.rs:385-387
    return NE2B_OK;
}

ne2b_status ne2b_ring_depth(const ne2b_sim *sim, uint32_t *d) {
    CHECK_SIM(const_cast<ne2b_sim *>(sim));
    *d = h->D;
    return NE2B_OK;
}

ne2b_status ne2b_run_steps(ne2b_sim *sim, uint64_t steps) {
    CHECK_SIM(sim);
    GUARD(sim->eng.run_steps(steps));
}

ne2b_status ne2b_run_ms(ne2b_sim *sim, float ms) {
    CHECK_SIM(sim);
    // cpu.rs:379-382: (ms / dt).round() as usize (saturating at 0)
    float st = roundf(ms / h->cfg.dt_ms);
    uint64_t steps = (st > 0.0f && st == st) ? (uint64_t)st : 0;
    GUARD(sim->eng.run_steps(steps));
}

ne2b_status ne2b_reset_state(ne2b_sim *sim) {
    CHECK_SIM(sim);
    GUARD(sim->eng.reset_net(sim->slot));
}

ne2b_status ne2b_synchronize(ne2b_sim *sim) {
    if (!sim) return set_error(NE2B_EINVAL, "null sim handle");
    return sim->eng.sync();
}

ne2b_status ne2b_dev_mem_bytes(const ne2b_sim *sim, uint64_t *bytes) {
    if (!sim || !bytes) return set_error(NE2B_EINVAL, "null argument");
    *bytes = sim->eng.dev_bytes();
    return NE2B_OK;
}

ne2b_status ne2b_read_trace(ne2b_sim *sim, float *out) {
    CHECK_SIM(sim);
    return sim->eng.read_trace(*h, out);
}

ne2b_status ne2b_read_state(ne2b_sim *sim, uint32_t slot, float *out) {
    CHECK_SIM(sim);
    if (slot >= 2) return set_error(NE2B_EINVAL, "state slot %u >= 2", slot);
    return sim->eng.read_f32(slot == 0 ? h->dev.v : h->dev.u, h->n, out);
}

ne2b_status ne2b_read_syn_current(ne2b_sim *sim, float *out) {
    CHECK_SIM(sim);
    return sim->eng.read_f32(h->dev.s, h->n, out);
}

ne2b_status ne2b_last_spikes(ne2b_sim *sim, uint32_t *out, uint32_t cap, uint32_t *count) {
    CHECK_SIM(sim);
    if (!count) return set_error(NE2B_EINVAL, "null count");
    *count = 0;
    std::vector<uint64_t> row((h->n + 63) / 64);
    ne2b_status st = sim->eng.spike_row(*h, 0, row.data());
    if (st == NE2B_ENODATA) return NE2B_OK;  // cpu.rs:546-548: empty
    if (st != NE2B_OK) return st;
    uint32_t c = 0;
    for (size_t wi = 0; wi < row.size(); ++wi) {
        uint64_t w = row[wi];
        while (w) {
            const uint32_t i = (uint32_t)(wi * 64 + __builtin_ctzll(w));
            w &= w - 1;
            if (i < h->n) {
                if (c < cap && out) out[c] = i;
                ++c;
            }
        }
    }
    *count = c;
    return NE2B_OK;
}

ne2b_status ne2b_spike_counts(ne2b_sim *sim, uint64_t rows, uint32_t *out) {
    CHECK_SIM(sim);
    if (!out && h->n) return set_error(NE2B_EINVAL, "null out");
    GUARD(sim->eng.spike_counts(*h, rows, out));
}

ne2b_status ne2b_spike_row(ne2b_sim *sim, uint32_t back, uint64_t *out) {
    CHECK_SIM(sim);
    return sim->eng.spike_row(*h, back, out);
}

ne2b_status ne2b_spikes_total(ne2b_sim *sim, uint64_t *total) {
    CHECK_SIM(sim);
    return sim->eng.spikes_total(*h, total);
}

ne2b_status ne2b_mean_rate_hz(ne2b_sim *sim, double *hz) {
    CHECK_SIM(sim);
    if (h->t == 0) {  // cpu.rs:389-396
        *hz = 0.0;
        return NE2B_OK;
    }
    uint64_t tot = 0;
    ne2b_status st = sim->eng.spikes_total(*h, &tot);
    if (st != NE2B_OK) return st;
    const double n = h->n ? (double)h->n : 1.0;
    *hz = (double)tot / n / ((double)h->t * (double)h->cfg.dt_ms / 1000.0);
    return NE2B_OK;
}

ne2b_status ne2b_window_counts(ne2b_sim *sim, uint32_t window, uint16_t *out) {
    CHECK_SIM(sim);
    return sim->eng.window_counts(*h, window, out);
}

ne2b_status ne2b_windows_done(ne2b_sim *sim, uint32_t *count) {
    CHECK_SIM(sim);
    *count = h->cfg.window_steps ? (uint32_t)std::min<uint64_t>(h->t / h->cfg.window_steps, h->dev.max_windows) : 0;
    return NE2B_OK;
}

ne2b_status ne2b_set_input_constant(ne2b_sim *sim, uint32_t input, float value) {
    CHECK_SIM(sim);
    if (input >= h->n_inputs) return set_error(NE2B_EINVAL, "input %u out of range (%u inputs)", input, h->n_inputs);
    h->stim.constants[input] = value;
    h->dev.stim_len = 0;  // repack at the next run
    return NE2B_OK;
}

ne2b_status ne2b_input_values(ne2b_sim *sim, float *out) {
    CHECK_SIM(sim);
    for (uint32_t k = 0; k < h->n_inputs; ++k) out[k] = h->stim.constants[k];
    return NE2B_OK;
}

static ne2b_status play(ne2b_sim *sim, uint32_t input, const float *series, uint64_t len, bool loop) {
    CHECK_SIM(sim);
    if (input >= h->n_inputs) return set_error(NE2B_EINVAL, "input %u out of range (%u inputs)", input, h->n_inputs);
    if (len && !series) return set_error(NE2B_EINVAL, "null series");
    GUARD(([&]() -> ne2b_status {
        h->stim.play(input, h->t, series, len, loop);
        h->dev.stim_len = 0;
        return NE2B_OK;
    })());
}

ne2b_status ne2b_play_input(ne2b_sim *sim, uint32_t input, const float *series, uint64_t len) {
    return play(sim, input, series, len, false);
}

ne2b_status ne2b_loop_input(ne2b_sim *sim, uint32_t input, const float *series, uint64_t len) {
    return play(sim, input, series, len, true);
}

ne2b_status ne2b_set_external(ne2b_sim *sim, uint32_t neuron, float amps) {
    CHECK_SIM(sim);
    if (neuron >= h->n) return NE2B_OK;  // cpu.rs:588-592: out of range is a no-op
    std::vector<float> ext = h->ext_host;
    ext[neuron] = amps;
    return sim->eng.set_ext(*h, ext.data(), (uint32_t)ext.size());
}

ne2b_status ne2b_set_external_all(ne2b_sim *sim, const float *ext, uint32_t len) {
    CHECK_SIM(sim);
    if (len && !ext) return set_error(NE2B_EINVAL, "null ext");
    return sim->eng.set_ext(*h, ext, len);
}

ne2b_status ne2b_external(ne2b_sim *sim, float *out) {
    CHECK_SIM(sim);
    for (uint32_t i = 0; i < h->n; ++i) out[i] = h->ext_host[i];
    return NE2B_OK;
}

ne2b_status ne2b_set_noise(ne2b_sim *sim, float rate_hz, float kick_mv) {
    CHECK_SIM(sim);
    h->cfg.noise_rate_hz = rate_hz;  // cuda.rs:807-810
    h->cfg.noise_kick_mv = kick_mv;
    return sim->eng.refresh_noise(*h);
}

ne2b_status ne2b_set_gauss_noise(ne2b_sim *sim, float sd) {
    CHECK_SIM(sim);
    h->cfg.gauss_sd = sd;
    return sim->eng.refresh_noise(*h);
}

ne2b_status ne2b_set_kernel_mode(ne2b_sim *sim, int32_t mode) {
    if (!sim) return set_error(NE2B_EINVAL, "null sim handle");
    GUARD(sim->eng.set_mode(mode));
}

ne2b_status ne2b_kernel_mode(ne2b_sim *sim, int32_t *mode, int32_t *resident) {
    if (!sim || !mode || !resident) return set_error(NE2B_EINVAL, "null argument");
    *mode = sim->eng.mode();
    *resident = sim->eng.resident() ? 1 : 0;
    return NE2B_OK;
}

ne2b_status ne2b_autotune(ne2b_sim *sim, uint32_t steps_per_trial) {
    CHECK_SIM(sim);
    GUARD(sim->eng.autotune(steps_per_trial));
}

ne2b_status ne2b_set_tile_shape(ne2b_sim *sim, uint32_t block, uint32_t npt, uint32_t bps) {
    if (!sim) return set_error(NE2B_EINVAL, "null sim handle");
    ne2b::TileShape sh;
    sh.block = block;
    sh.npt = npt;
    sh.blocks_per_sm = bps;
    sh.ws = sim->eng.shape().ws;  // the delivery-warp setting is kept
    GUARD(sim->eng.set_shape(sh));
}

ne2b_status ne2b_tile_shape(ne2b_sim *sim, uint32_t *block, uint32_t *npt, uint32_t *bps) {
    if (!sim || !block || !npt || !bps) return set_error(NE2B_EINVAL, "null argument");
    *block = sim->eng.shape().block;
    *npt = sim->eng.shape().npt;
    *bps = sim->eng.shape().blocks_per_sm;
    return NE2B_OK;
}

ne2b_status ne2b_set_delivery_warps(ne2b_sim *sim, int32_t on) {
    if (!sim) return set_error(NE2B_EINVAL, "null sim handle");
    ne2b::TileShape sh = sim->eng.shape();
    sh.ws = on != 0;
    GUARD(sim->eng.set_shape(sh));
}

ne2b_status ne2b_delivery_warps(ne2b_sim *sim, int32_t *on, int32_t *active) {
    if (!sim || !on || !active) return set_error(NE2B_EINVAL, "null argument");
    *on = sim->eng.shape().ws ? 1 : 0;
    *active = (!sim->eng.resident() && sim->eng.ws_applies(sim->eng.shape())) ? 1 : 0;
    return NE2B_OK;
}

ne2b_status ne2b_stream(ne2b_sim *sim, void **stream) {
    if (!sim || !stream) return set_error(NE2B_EINVAL, "null argument");
    *stream = (void *)sim->eng.stream();
    return NE2B_OK;
}

ne2b_status ne2b_kernel_launches(ne2b_sim *sim, uint64_t *launches) {
    if (!sim || !launches) return set_error(NE2B_EINVAL, "null argument");
    *launches = sim->eng.launches();
    return NE2B_OK;
}

ne2b_status ne2b_set_v_watch(ne2b_sim *sim, const uint32_t *ids, uint32_t count) {
    if (!sim) return set_error(NE2B_EINVAL, "null sim handle");
    GUARD(sim->eng.set_v_watch(*sim->eng.net(sim->slot), ids, count));
}

ne2b_status ne2b_watch_count(ne2b_sim *sim, uint32_t *watches, uint32_t *samples) {
    if (!sim) return set_error(NE2B_EINVAL, "null sim handle");
    NetHost &h = *sim->eng.net(sim->slot);
    const uint64_t span = h.t - std::min(h.watch_t0, h.t);
    if (watches) *watches = (uint32_t)h.watch_ids.size();
    if (samples) *samples = (uint32_t)std::min<uint64_t>(span, ne2b::kWatchCap);
    return NE2B_OK;
}

ne2b_status ne2b_drain_watch(ne2b_sim *sim, float *out, uint32_t *samples) {
    if (!sim || !samples) return set_error(NE2B_EINVAL, "null argument");
    GUARD(sim->eng.drain_watch(*sim->eng.net(sim->slot), out, samples));
}

ne2b_status ne2b_set_grid_watches(ne2b_sim *sim, const uint32_t *members, const uint32_t *group_ptr,
                                  uint32_t groups) {
    if (!sim) return set_error(NE2B_EINVAL, "null sim handle");
    GUARD(sim->eng.set_grid_watches(*sim->eng.net(sim->slot), members, group_ptr, groups));
}

ne2b_status ne2b_grid_traces(ne2b_sim *sim, float tau_ms, float *out) {
    if (!sim) return set_error(NE2B_EINVAL, "null sim handle");
    GUARD(sim->eng.grid_traces(*sim->eng.net(sim->slot), tau_ms, out));
}

// ----------------------------------------------------------------- batch
ne2b_status ne2b_batch_create(const ne2b_net_desc *nets, const ne2b_config *cfgs, uint32_t count, int device,
                              ne2b_batch **out) {
    if (!out || (!nets && count) || (!cfgs && count)) return set_error(NE2B_EINVAL, "ne2b_batch_create: null argument");
    *out = nullptr;
    if (count == 0) return set_error(NE2B_EINVAL, "empty batch");
    for (uint32_t k = 1; k < count; ++k)
        if ((cfgs[k].int_weights != 0) != (cfgs[0].int_weights != 0))
            return set_error(NE2B_EINVAL, "all nets of a batch share one ring mode");
    GUARD(([&]() -> ne2b_status {
        ne2b_batch *b = new ne2b_batch();
        b->eng.multi_net = true;
        ne2b_status st = b->eng.init(device, cfgs[0].int_weights != 0, count);
        for (uint32_t k = 0; k < count && st == NE2B_OK; ++k) {
            uint32_t slot = 0;
            st = b->eng.add_net(&nets[k], &cfgs[k], nullptr, 0, &slot);
            b->slots.push_back(slot);
        }
        if (st != NE2B_OK) {
            delete b;
            return st;
        }
        *out = b;
        return NE2B_OK;
    })());
}

ne2b_status ne2b_batch_destroy(ne2b_batch *b) {
    delete b;
    return NE2B_OK;
}

#define CHECK_BATCH_NET(b, k)                                                        \
    if (!(b)) return set_error(NE2B_EINVAL, "null batch handle");                    \
    if ((k) >= (b)->slots.size()) return set_error(NE2B_EINVAL, "net %u out of range", (k)); \
    NetHost *h = (b)->eng.net((b)->slots[(k)]);                                      \
    if (!h) return set_error(NE2B_EINVAL, "batch net %u missing", (k));

ne2b_status ne2b_batch_play_input(ne2b_batch *b, uint32_t net, uint32_t input, const float *series, uint64_t len) {
    CHECK_BATCH_NET(b, net);
    if (input >= h->n_inputs) return set_error(NE2B_EINVAL, "input %u out of range (%u inputs)", input, h->n_inputs);
    GUARD(([&]() -> ne2b_status {
        h->stim.play(input, h->t, series, len, false);
        h->dev.stim_len = 0;
        return NE2B_OK;
    })());
}

ne2b_status ne2b_batch_set_input_matrix(ne2b_batch *b, uint32_t net, const float *inputs, uint64_t steps) {
    CHECK_BATCH_NET(b, net);
    GUARD(b->eng.set_input_matrix(*h, inputs, steps));
}

ne2b_status ne2b_batch_run_steps(ne2b_batch *b, uint64_t steps) {
    if (!b) return set_error(NE2B_EINVAL, "null batch handle");
    GUARD(b->eng.run_steps(steps));
}

ne2b_status ne2b_batch_reset_state(ne2b_batch *b) {
    if (!b) return set_error(NE2B_EINVAL, "null batch handle");
    for (uint32_t s : b->slots) {
        ne2b_status st = b->eng.reset_net(s);
        if (st != NE2B_OK) return st;
    }
    return NE2B_OK;
}

ne2b_status ne2b_batch_synchronize(ne2b_batch *b) {
    if (!b) return set_error(NE2B_EINVAL, "null batch handle");
    return b->eng.sync();
}

ne2b_status ne2b_batch_window_counts(ne2b_batch *b, uint32_t net, uint32_t window, uint16_t *out) {
    CHECK_BATCH_NET(b, net);
    return b->eng.window_counts(*h, window, out);
}

ne2b_status ne2b_batch_spikes_total(ne2b_batch *b, uint32_t net, uint64_t *total) {
    CHECK_BATCH_NET(b, net);
    return b->eng.spikes_total(*h, total);
}

ne2b_status ne2b_batch_read_state(ne2b_batch *b, uint32_t net, uint32_t slot, float *out) {
    CHECK_BATCH_NET(b, net);
    if (slot >= 2) return set_error(NE2B_EINVAL, "state slot %u >= 2", slot);
    return b->eng.read_f32(slot == 0 ? h->dev.v : h->dev.u, h->n, out);
}

ne2b_status ne2b_batch_autotune(ne2b_batch *b, uint32_t steps_per_trial) {
    if (!b) return set_error(NE2B_EINVAL, "null batch handle");
    GUARD(b->eng.autotune(steps_per_trial));
}

ne2b_status ne2b_batch_tile_shape(ne2b_batch *b, uint32_t *block, uint32_t *npt, uint32_t *bps) {
    if (!b) return set_error(NE2B_EINVAL, "null batch handle");
    *block = b->eng.shape().block;
    *npt = b->eng.shape().npt;
    *bps = b->eng.shape().blocks_per_sm;
    return NE2B_OK;
}

ne2b_status ne2b_batch_set_tile_shape(ne2b_batch *b, uint32_t block, uint32_t npt, uint32_t bps) {
    if (!b) return set_error(NE2B_EINVAL, "null batch handle");
    ne2b::TileShape s;
    s.block = block;
    s.npt = npt;
    s.blocks_per_sm = bps;
    GUARD(b->eng.set_shape(s));
}

ne2b_status ne2b_batch_dev_mem_bytes(ne2b_batch *b, uint64_t *bytes) {
    if (!b) return set_error(NE2B_EINVAL, "null batch handle");
    *bytes = b->eng.dev_bytes();
    return NE2B_OK;
}

ne2b_status ne2b_batch_last_step_ms(ne2b_batch *b, float *ms) {
    if (!b) return set_error(NE2B_EINVAL, "null batch handle");
    *ms = b->eng.last_ms();
    return NE2B_OK;
}

ne2b_status ne2b_batch_set_kernel_mode(ne2b_batch *b, int32_t mode) {
    if (!b) return set_error(NE2B_EINVAL, "null batch handle");
    GUARD(b->eng.set_mode(mode));
}

ne2b_status ne2b_batch_kernel_mode(ne2b_batch *b, int32_t *mode, int32_t *resident) {
    if (!b || !mode || !resident) return set_error(NE2B_EINVAL, "null argument");
    *mode = b->eng.mode();
    *resident = b->eng.resident() ? 1 : 0;
    return NE2B_OK;
}

ne2b_status ne2b_batch_stream(ne2b_batch *b, void **stream) {
    if (!b || !stream) return set_error(NE2B_EINVAL, "null argument");
    *stream = (void *)b->eng.stream();
    return NE2B_OK;
}

ne2b_status ne2b_batch_kernel_launches(ne2b_batch *b, uint64_t *launches) {
    if (!b || !launches) return set_error(NE2B_EINVAL, "null argument");
    *launches = b->eng.launches();
    return NE2B_OK;
}

// --------------------------------------------------------------- serving
ne2b_status ne2b_request_footprint(const ne2b_net_desc *net, const ne2b_config *cfg, uint64_t *neurons,
                                   uint64_t *synapses, uint64_t *ring_words) {
    if (!net || !cfg) return set_error(NE2B_EINVAL, "null argument");
    const uint64_t np = (net->n + ne2b::kNeuronAlign - 1) / ne2b::kNeuronAlign * ne2b::kNeuronAlign;
    std::atomic<uint32_t> maxd{1};
    if (net->n_syn && !net->delay_steps) return set_error(NE2B_EINVAL, "net has synapses but no delays");
    ne2b::parallel_for(net->n_syn, [&](uint64_t lo, uint64_t hi) {
        uint16_t m = 1;
        for (uint64_t j = lo; j < hi; ++j) m = std::max(m, net->delay_steps[j]);
        uint32_t cur = maxd.load();
        while (m > cur && !maxd.compare_exchange_weak(cur, m)) {
        }
    });
    const uint64_t D = std::max<uint32_t>(2, maxd.load() + 1);
    if (neurons) *neurons = np;
    if (synapses) *synapses = net->n_syn;
    if (ring_words) *ring_words = D * np;
    return NE2B_OK;
}

// Admission thread: builds queued requests on its own stream (validation,
// parameter rows, CSR staging, uploads, initial state) and hands them to
// ne2b_server_step, which attaches them on the engine's stream.
static void server_builder(ne2b_server *s, ne2b_server::Builder *b) {
    cudaSetDevice(s->eng.device());
    for (;;) {
        ne2b_server::Job j;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_job.wait(lk, [&] { return s->stop || !s->jobs.empty(); });
            if (s->stop) return;
            j = s->jobs.front();
            s->jobs.pop_front();
        }
        ne2b_server::Built r;
        r.id = j.id;
        try {
            r.st = s->eng.build_net(&j.desc, &j.cfg, j.inputs, j.steps, b->sg, &r.h);
        } catch (const std::bad_alloc &) {
            r.st = set_error(NE2B_ENOMEM, "host allocation failed");
        } catch (...) {
            r.st = set_error(NE2B_ECUDA, "unexpected host exception while building a request");
        }
        if (r.st == NE2B_OK) {
            cudaError_t e = cudaEventCreateWithFlags(&r.ev, cudaEventDisableTiming);
            if (e == cudaSuccess) e = cudaEventRecord(r.ev, b->st);
            if (e != cudaSuccess) {
                r.st = ne2b::cuda_error(e, "build event");
                if (r.ev) cudaEventDestroy(r.ev);
                r.ev = nullptr;
                cudaStreamSynchronize(b->st);
                s->eng.discard_net(r.h, b->st);
                r.h = nullptr;
            }
        }
        if (r.st != NE2B_OK) r.msg = ne2b::last_error_str();
        {
            std::lock_guard<std::mutex> g(s->mu);
            s->built.push_back(std::move(r));
        }
        s->cv_built.notify_all();
    }
}

ne2b_status ne2b_server_create(const ne2b_server_config *cfg, int device, ne2b_server **out) {
    if (!cfg || !out) return set_error(NE2B_EINVAL, "null argument");
    *out = nullptr;
    if (cfg->max_requests == 0) return set_error(NE2B_EINVAL, "max_requests must be > 0");
    GUARD(([&]() -> ne2b_status {
        ne2b_server *s = new ne2b_server();
        s->cfg = *cfg;
        if (s->cfg.steps_per_launch == 0) s->cfg.steps_per_launch = 64;
        ne2b_status st = s->eng.init(device, cfg->int_weights != 0, cfg->max_requests);
        if (st == NE2B_OK) st = s->eng.set_mode(ne2b::kModeStream);
        if (st == NE2B_OK) st = ne2b::cuda_error(cudaStreamCreateWithFlags(&s->rstream, cudaStreamNonBlocking), "result stream");
        for (int k = 0; k < 2 && st == NE2B_OK; ++k)
            st = ne2b::cuda_error(cudaEventCreateWithFlags(&s->step_ev[k], cudaEventDisableTiming), "event");
        if (st != NE2B_OK) {
            delete s;
            return st;
        }
        s->eng.graph_steps = s->cfg.steps_per_launch;
        s->eng.fixed_grid = true;
        s->eng.multi_net = true;
        {
            // small tiles: the most blocks per SM, so the latency chains of
            // active tiles (state loads, scans, CSR loads) overlap; measured
            // 1.6x faster than 256x2 on the served request mix
            ne2b::TileShape sh;
            sh.block = 128;
            sh.npt = 1;
            st = s->eng.set_shape(sh);
            if (st != NE2B_OK) {
                delete s;
                return st;
            }
        }
        for (uint32_t k = 0; k < std::min<uint32_t>(cfg->admission_threads, 16u); ++k) {
            auto b = std::make_unique<ne2b_server::Builder>();
            st = ne2b::cuda_error(cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking), "admission stream");
            if (st != NE2B_OK) {
                delete s;
                return st;
            }
            b->sg.set_stream(b->st);
            ne2b_server::Builder *bp = b.get();
            s->builders.push_back(std::move(b));
            bp->th = std::thread(server_builder, s, bp);
        }
        *out = s;
        return NE2B_OK;
    })());
}

ne2b_status ne2b_server_destroy(ne2b_server *s) {
    delete s;
    return NE2B_OK;
}

ne2b_status ne2b_server_submit(ne2b_server *s, const ne2b_net_desc *net, const ne2b_config *cfg_in,
                               const float *inputs, uint64_t steps, uint64_t *request_id) {
    if (!s || !net || !cfg_in || !request_id) return set_error(NE2B_EINVAL, "null argument");
    if (steps == 0) return set_error(NE2B_EINVAL, "a request needs steps > 0");
    if (cfg_in->window_steps == 0) return set_error(NE2B_EINVAL, "a request needs window_steps > 0");
    if ((cfg_in->int_weights != 0) != (s->cfg.int_weights != 0))
        return set_error(NE2B_EINVAL, "request ring mode differs from the server's");
    uint64_t fn = 0, fs = 0, fr = 0;
    ne2b_status st = ne2b_request_footprint(net, cfg_in, &fn, &fs, &fr);
    if (st != NE2B_OK) return st;
    if (fn > s->cfg.neuron_capacity || fs > s->cfg.synapse_capacity || fr > s->cfg.ring_capacity)
        return set_error(NE2B_EINVAL, "request footprint exceeds the server's total capacity");
    uint32_t active = 0;
    for (auto &kv : s->reqs) active += !kv.second.done;
    if (active >= s->cfg.max_requests || s->used_neurons + fn > s->cfg.neuron_capacity ||
        s->used_syn + fs > s->cfg.synapse_capacity || s->used_ring + fr > s->cfg.ring_capacity)
        return set_error(NE2B_EFULL, "no capacity for this request now");
    GUARD(([&]() -> ne2b_status {
        ne2b_config cfg = *cfg_in;
        cfg.max_windows = (uint32_t)((steps + cfg.window_steps - 1) / cfg.window_steps);
        ne2b_server::Req r;
        if (!s->builders.empty()) {
            r.queued = true;
        } else {
            ne2b_status st2 = s->eng.add_net(net, &cfg, inputs, steps, &r.slot);
            if (st2 != NE2B_OK) return st2;
        }
        r.n = net->n;
        r.n_pad = (uint32_t)fn;
        r.windows = (uint32_t)(steps / cfg.window_steps);
        r.steps = steps;
        r.fp_neurons = fn;
        r.fp_syn = fs;
        r.fp_ring = fr;
        s->used_neurons += fn;
        s->used_syn += fs;
        s->used_ring += fr;
        const uint64_t id = s->next_id++;
        s->reqs.emplace(id, std::move(r));
        s->admitted++;
        if (!s->builders.empty()) {
            {
                std::lock_guard<std::mutex> g(s->mu);
                s->jobs.push_back(ne2b_server::Job{id, *net, cfg, inputs, steps});
            }
            s->cv_job.notify_one();
        }
        *request_id = id;
        return NE2B_OK;
    })());
}

// Attach the requests the admission threads have built: the engine's
// stream waits for each build's stream work, then the net is published.  A
// failed build finishes its request with the error.  When nothing runs on
// the device yet, waits for the first build instead of stepping an empty
// engine.
static ne2b_status server_attach_built(ne2b_server *s) {
    if (s->builders.empty()) return NE2B_OK;
    std::vector<ne2b_server::Built> got;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        bool queued = false;
        for (auto &kv : s->reqs) queued |= kv.second.queued;
        if (queued && s->built.empty() && s->eng.active_nets() == 0)
            s->cv_built.wait(lk, [&] { return !s->built.empty(); });
        got.swap(s->built);
    }
    bool attached = false;
    ne2b_status first_err = NE2B_OK;
    for (ne2b_server::Built &r : got) {
        auto it = s->reqs.find(r.id);
        ne2b_status st = r.st;
        std::string msg = r.msg;
        if (st == NE2B_OK && it != s->reqs.end()) {
            st = ne2b::cuda_error(cudaStreamWaitEvent(s->eng.stream(), r.ev, 0), "admission wait");
            if (st == NE2B_OK) st = s->eng.attach_net(r.h, &it->second.slot, false);
            if (st != NE2B_OK) {
                msg = ne2b::last_error_str();
                s->eng.discard_net(r.h, s->eng.stream());
            }
            r.h = nullptr;
        } else if (r.h) {
            s->eng.discard_net(r.h, s->eng.stream());
            r.h = nullptr;
        }
        if (r.ev) cudaEventDestroy(r.ev);
        if (it == s->reqs.end()) continue;
        ne2b_server::Req &q = it->second;
        q.queued = false;
        if (st == NE2B_OK) {
            attached = true;
            continue;
        }
        if (st == NE2B_ECUDA && first_err == NE2B_OK) first_err = st;
        q.done = true;
        q.fail = st;
        q.fail_msg = msg;
        s->used_neurons -= q.fp_neurons;
        s->used_syn -= q.fp_syn;
        s->used_ring -= q.fp_ring;
        s->retired++;
        s->finished.push_back(r.id);
    }
    if (attached) {
        ne2b_status st = s->eng.rebuild_tiles();
        if (st != NE2B_OK) return st;
    }
    if (first_err != NE2B_OK) return set_error(first_err, "admission: %s", ne2b::last_error_str());
    return NE2B_OK;
}

ne2b_status ne2b_server_step(ne2b_server *s, uint32_t *active_out, uint32_t *finished_out) {
    if (!s) return set_error(NE2B_EINVAL, "null server handle");
    GUARD(([&]() -> ne2b_status {
        ne2b_status sa = server_attach_built(s);
        if (sa != NE2B_OK) return sa;
        // at most two launch groups in flight: host admission and retirement
        // work overlaps the device without queueing unboundedly ahead of it
        cudaEvent_t &ev = s->step_ev[s->step_no & 1];
        if (s->step_no >= 2) {
            ne2b_status st0 = ne2b::cuda_error(cudaEventSynchronize(ev), "step event");
            if (st0 != NE2B_OK) return st0;
        }
        ne2b_status st = s->eng.run_steps(s->cfg.steps_per_launch);
        if (st != NE2B_OK) return st;
        st = ne2b::cuda_error(cudaEventRecord(ev, s->eng.stream()), "step event");
        if (st != NE2B_OK) return st;
        s->step_no++;
        uint32_t fin = 0, act = 0;
        for (auto &kv : s->reqs) {
            ne2b_server::Req &r = kv.second;
            if (r.done) continue;
            if (r.queued) {
                ++act;
                continue;
            }
            NetHost *h = s->eng.net(r.slot);
            if (!(h && h->t >= h->t_end)) {
                ++act;
                continue;
            }
            // retire, stream-ordered after the launch that finished it: the
            // spike total is copied out of the shared counter array, the
            // window counts stay allocated until the result is taken
            r.d_win = h->dev.win_out;
            cudaStream_t st_main = s->eng.stream();
            st = ne2b::cuda_error(cudaMallocAsync((void **)&r.d_spk, sizeof(unsigned long long), st_main), "result");
            if (st == NE2B_OK)
                st = ne2b::cuda_error(cudaMemcpyAsync(r.d_spk, s->eng.counter_ptr(r.slot), sizeof(unsigned long long),
                                                      cudaMemcpyDeviceToDevice, st_main), "result");
            if (st == NE2B_OK) st = s->eng.remove_net(r.slot, false, r.d_win);
            if (st == NE2B_OK) st = ne2b::cuda_error(cudaEventCreateWithFlags(&r.ev, cudaEventDisableTiming), "event");
            if (st == NE2B_OK) st = ne2b::cuda_error(cudaEventRecord(r.ev, st_main), "event");
            if (st != NE2B_OK) return st;
            r.done = true;
            s->used_neurons -= r.fp_neurons;
            s->used_syn -= r.fp_syn;
            s->used_ring -= r.fp_ring;
            s->retired++;
            s->finished.push_back(kv.first);
            ++fin;
        }
        if (fin) {
            st = s->eng.rebuild_tiles();
            if (st != NE2B_OK) return st;
        }
        if (active_out) *active_out = act;
        if (finished_out) *finished_out = fin;
        return NE2B_OK;
    })());
}

ne2b_status ne2b_server_result_shape(ne2b_server *s, uint64_t id, uint32_t *n, uint32_t *windows) {
    if (!s) return set_error(NE2B_EINVAL, "null server handle");
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return set_error(NE2B_EINVAL, "unknown request %llu", (unsigned long long)id);
    *n = it->second.n;
    *windows = it->second.windows;
    return NE2B_OK;
}

ne2b_status ne2b_server_take_result(ne2b_server *s, uint64_t id, uint16_t *counts, uint64_t *spikes_total) {
    if (!s) return set_error(NE2B_EINVAL, "null server handle");
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return set_error(NE2B_EINVAL, "unknown request %llu", (unsigned long long)id);
    ne2b_server::Req &r = it->second;
    if (!r.done) return set_error(NE2B_ENODATA, "request %llu is still running", (unsigned long long)id);
    if (r.fail != NE2B_OK) {
        const ne2b_status st = set_error(r.fail, "request %llu was not admitted: %s", (unsigned long long)id,
                                         r.fail_msg.c_str());
        s->reqs.erase(it);
        s->finished.erase(std::remove(s->finished.begin(), s->finished.end(), id), s->finished.end());
        return st;
    }
    GUARD(([&]() -> ne2b_status {
        // the copies wait only for this request's retirement, not for the
        // launches queued after it
        ne2b_status st = ne2b::cuda_error(cudaStreamWaitEvent(s->rstream, r.ev, 0), "result wait");
        std::vector<uint16_t> rows((size_t)r.windows * r.n_pad);
        unsigned long long tot = 0;
        if (st == NE2B_OK && !rows.empty() && r.d_win)
            st = ne2b::cuda_error(cudaMemcpyAsync(rows.data(), r.d_win, sizeof(uint16_t) * rows.size(),
                                                  cudaMemcpyDeviceToHost, s->rstream), "result copy");
        if (st == NE2B_OK && r.d_spk)
            st = ne2b::cuda_error(cudaMemcpyAsync(&tot, r.d_spk, sizeof tot, cudaMemcpyDeviceToHost, s->rstream),
                                  "result copy");
        if (st == NE2B_OK) st = ne2b::cuda_error(cudaStreamSynchronize(s->rstream), "result copy");
        if (st != NE2B_OK) return st;
        if (counts)
            for (uint32_t w = 0; w < r.windows; ++w)
                memcpy(counts + (size_t)w * r.n, rows.data() + (size_t)w * r.n_pad, sizeof(uint16_t) * r.n);
        if (spikes_total) *spikes_total = tot;
        if (r.d_win) cudaFreeAsync(r.d_win, s->rstream);
        if (r.d_spk) cudaFreeAsync(r.d_spk, s->rstream);
        cudaEventDestroy(r.ev);
        s->reqs.erase(it);
        s->finished.erase(std::remove(s->finished.begin(), s->finished.end(), id), s->finished.end());
        return NE2B_OK;
    })());
}

// Finished requests whose results can be taken without waiting: the
// device has completed the launch that retired them (or they failed to
// build).  Requests retired by launches still in flight are listed once
// those launches complete.
ne2b_status ne2b_server_finished_ids(ne2b_server *s, uint64_t *ids, uint32_t cap, uint32_t *count) {
    if (!s || !count) return set_error(NE2B_EINVAL, "null argument");
    uint32_t c = 0;
    for (uint64_t id : s->finished) {
        auto it = s->reqs.find(id);
        if (it == s->reqs.end()) continue;
        const ne2b_server::Req &r = it->second;
        if (r.ev && cudaEventQuery(r.ev) != cudaSuccess) continue;
        if (ids && c < cap) ids[c] = id;
        ++c;
    }
    *count = c;
    return NE2B_OK;
}

ne2b_status ne2b_server_stats(ne2b_server *s, uint64_t *admitted, uint64_t *retired, uint32_t *active,
                              uint64_t *neurons_used, uint64_t *synapses_used) {
    if (!s) return set_error(NE2B_EINVAL, "null server handle");
    uint32_t act = 0;
    for (auto &kv : s->reqs) act += !kv.second.done;
    if (admitted) *admitted = s->admitted;
    if (retired) *retired = s->retired;
    if (active) *active = act;
    if (neurons_used) *neurons_used = s->used_neurons;
    if (synapses_used) *synapses_used = s->used_syn;
    return NE2B_OK;
}

ne2b_status ne2b_server_set_tile_shape(ne2b_server *s, uint32_t block, uint32_t npt, uint32_t bps) {
    if (!s) return set_error(NE2B_EINVAL, "null server handle");
    ne2b::TileShape sh;
    sh.block = block;
    sh.npt = npt;
    sh.blocks_per_sm = bps;
    GUARD(s->eng.set_shape(sh));
}

ne2b_status ne2b_selftest_barrier_timeout(int device, uint32_t limit_ms, int32_t *timed_out) {
    if (!timed_out) return set_error(NE2B_EINVAL, "null argument");
    if (limit_ms == 0 || limit_ms > 2000) return set_error(NE2B_EINVAL, "limit_ms must be in 1..2000");
    *timed_out = 0;
    GUARD(([&]() -> ne2b_status {
        ne2b_status st = ne2b::cuda_error(cudaSetDevice(device), "cudaSetDevice");
        if (st != NE2B_OK) return st;
        unsigned int *d = nullptr;
        st = ne2b::cuda_error(cudaMalloc(&d, 2 * sizeof(unsigned int)), "cudaMalloc");
        if (st != NE2B_OK) return st;
        unsigned int h[2] = {0u, 0u};
        st = ne2b::cuda_error(cudaMemset(d, 0, sizeof h), "cudaMemset");
        if (st == NE2B_OK)
            st = ne2b::cuda_error(ne2b::launch_barrier_selftest(d, d + 1, 4, 2, 1000000ull * limit_ms, 0),
                                  "self-test launch");
        if (st == NE2B_OK) st = ne2b::cuda_error(cudaMemcpy(h, d, sizeof h, cudaMemcpyDeviceToHost), "readback");
        cudaFree(d);
        if (st != NE2B_OK) return st;
        *timed_out = h[1] != 0u ? 1 : 0;
        return NE2B_OK;
    })());
}

ne2b_status ne2b_server_synchronize(ne2b_server *s) {
    if (!s) return set_error(NE2B_EINVAL, "null server handle");
    GUARD(s->eng.sync());
}

ne2b_status ne2b_server_stream(ne2b_server *s, void **stream) {
    if (!s || !stream) return set_error(NE2B_EINVAL, "null argument");
    *stream = (void *)s->eng.stream();
    return NE2B_OK;
}

ne2b_status ne2b_server_kernel_launches(ne2b_server *s, uint64_t *launches) {
    if (!s || !launches) return set_error(NE2B_EINVAL, "null argument");
    *launches = s->eng.launches();
    return NE2B_OK;
}

}  // extern "C"
