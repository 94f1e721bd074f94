/*
 * ne2b.h — C ABI of the B200 simulation core for neuro_edit v2 networks.
 *
 * This is the drop-in boundary for the reference's `sim::Backend` trait
 * (sim/src/lib.rs:119-184).  A Rust `impl Backend for B200Sim` binds these
 * entry points one-to-one; every other caller (the Python mirror in neuro_edit_v2_b200, the batch
 * runner, the serving loop) uses the same symbols.
 *
 * Conventions
 *   - Every entry point returns an ne2b_status (0 = NE2B_OK).  On failure
 *     ne2b_last_error() returns a thread-local message.  Nothing panics or
 *     throws across this boundary.
 *   - The caller owns every buffer it passes in; the library copies what it
 *     keeps.  Output buffers are caller-allocated with the documented size.
 *   - One handle is used from one host thread at a time.  Stepping calls are
 *     asynchronous on the handle's CUDA stream (like the reference CUDA
 *     backend, sim/src/cuda.rs:584-604); every read synchronises first.
 *   - Plain pointers and sizes only; no CUDA, torch or C++ types.
 */
#ifndef NE2B_H
#define NE2B_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    NE2B_OK = 0,
    NE2B_EINVAL = 1,      /* bad argument, index out of range, malformed net */
    NE2B_ENOMEM = 2,      /* device or host allocation failed */
    NE2B_ECUDA = 3,       /* CUDA runtime error (message names the call) */
    NE2B_EWINDOW = 4,     /* spike_counts window between record depth and t */
    NE2B_UNSUPPORTED = 5, /* feature not provided by this backend */
    NE2B_EFULL = 6,       /* admission refused: footprint exceeds free capacity */
    NE2B_ENODATA = 7      /* nothing to return (e.g. spike_row outside the window) */
} ne2b_status;

/* Neuron model registry ids, sim/src/model/mod.rs:117 (MODELS order). */
enum { NE2B_MODEL_IZH = 0, NE2B_MODEL_ADEX = 1 };

/* A network in the flat layout the reference builds before a sim:
 * NeuronParams::from_network (sim/src/state.rs:98-153), SynCsr from
 * Network::synapse_csr (net-format/src/network.rs:654-692) and StimMap
 * (sim/src/stim.rs:26-48). */
typedef struct {
    uint32_t n;                  /* neurons */
    const uint8_t *model;        /* [n] registry id per neuron */
    const float *params;         /* [n * param_stride] param rows (izh: a,b,c,d; AdEx: 10) */
    uint32_t param_stride;       /* row width, >= the widest model's param count */
    const float *x0;             /* [n * 2] initial state rows, or NULL = model init */
    uint64_t n_syn;
    const uint32_t *src_ptr;     /* [n + 1] source-major CSR row pointers */
    const uint32_t *tgt;         /* [n_syn] target neuron */
    const float *w;              /* [n_syn] weight, Dale's-law signed */
    const uint16_t *delay_steps; /* [n_syn] delay in steps, >= 1 */
    const float *tau_ms;         /* [n_syn] per-synapse tau in ms or NULL: tau > 0 gives the synapse its own
                                    current (XSyn, sim/src/state.rs:231-275), 0 the merged ring */
    uint32_t n_inputs;           /* stimulus inputs (Network::inputs) */
    const uint32_t *stim_ptr;    /* [n + 1] neuron-major (input, weight) rows, or NULL */
    const uint32_t *stim_input;  /* [stim_ptr[n]] */
    const float *stim_w;         /* [stim_ptr[n]] */
} ne2b_net_desc;

/* SimConfig (sim/src/state.rs:8-49) plus the project's additions. */
typedef struct {
    float dt_ms;
    float synapse_tau_ms;
    float readout_tau_ms;
    float noise_rate_hz;         /* Poisson kicks (state.rs:15-22) */
    float noise_kick_mv;
    uint64_t seed;
    int32_t record_spikes;
    uint32_t spike_record_steps;
    int32_t int_weights;         /* fixed-point ring, scale 4096 (kernels.rs:57-66) */
    float gauss_sd;              /* Gaussian current noise sd, 0 = off (new) */
    uint32_t window_steps;       /* on-device per-neuron spike counts per window, 0 = off (new) */
    uint32_t max_windows;        /* windows kept on device when window_steps > 0 */
} ne2b_config;

/* sim/src/state.rs:35-49 defaults (dt 0.1, tau 2/2, kick 20 mV, seed 1, ...). */
void ne2b_config_default(ne2b_config *cfg);

const char *ne2b_last_error(void);
const char *ne2b_version(void);

/* ------------------------------------------------------------------ sim */
/* One network on one GPU: the B200 counterpart of CpuSim / CudaSim. */
typedef struct ne2b_sim ne2b_sim;

/* Sim::with_params (sim/src/lib.rs:217-233), CudaSim::with_params
 * (sim/src/cuda.rs:130-239).  device = CUDA ordinal. */
ne2b_status ne2b_create(const ne2b_net_desc *net, const ne2b_config *cfg, int device, ne2b_sim **out);
ne2b_status ne2b_destroy(ne2b_sim *sim);

/* Network::synapse_csr (net-format/src/network.rs:654-692) built on the
 * GPU, straight into a new sim.  `net` carries the neurons (n, model, params,
 * param_stride, x0) and the stimulus map; its CSR fields (n_syn, src_ptr,
 * tgt, w, delay_steps, tau_ms) must be 0/NULL.  The synapse list
 * src/tgt/w/delay_ms[n_syn], in any order, is copied to the device and
 * sorted there by source, stably (a source's synapses keep their list
 * order), with Dale's sign from kind[n] (1 = inhibitory) and delays of
 * max(1, roundf(ms / cfg->dt_ms)) steps, at most 65535.  The sim equals
 * ne2b_net_from_synapses (same arrays, dt = cfg->dt_ms) followed by
 * ne2b_create, bit for bit, and the same errors are reported.  No
 * per-synapse tau: nets with their own synapse currents use the host
 * build. */
/* The list arrays and `kind` may each be in host or device memory; device
 * arrays are read in place (no upload), and must stay valid until the call
 * returns. */
ne2b_status ne2b_create_from_synapses(const ne2b_net_desc *net, const uint8_t *kind, uint64_t n_syn,
                                      const uint32_t *src, const uint32_t *tgt, const float *w,
                                      const float *delay_ms, const ne2b_config *cfg, int device, ne2b_sim **out);
/* The sim's synapse CSR as it sits on the device: rowptr[n + 1], tgt[E],
 * w_bits[E] (the int32 fixed-point weight with the int ring, else the f32
 * bits) and delay_steps[E]; E from ne2b_syn_count.  NULL skips an array. */
ne2b_status ne2b_syn_count(const ne2b_sim *sim, uint64_t *e);
ne2b_status ne2b_read_csr(ne2b_sim *sim, uint32_t *rowptr, uint32_t *tgt, uint32_t *w_bits, uint16_t *delay_steps);

ne2b_status ne2b_n(const ne2b_sim *sim, uint32_t *n);                 /* Backend::n */
ne2b_status ne2b_step_count(const ne2b_sim *sim, uint64_t *t);        /* Backend::step_count */
ne2b_status ne2b_time_ms(const ne2b_sim *sim, double *ms);            /* Backend::time_ms */
ne2b_status ne2b_ring_depth(const ne2b_sim *sim, uint32_t *d);        /* state.rs:221 ring_depth */
/* Backend::run_steps / run_ms (lib.rs:126-127; cuda.rs:584-609): asynchronous */
ne2b_status ne2b_run_steps(ne2b_sim *sim, uint64_t steps);
ne2b_status ne2b_run_ms(ne2b_sim *sim, float ms);
ne2b_status ne2b_reset_state(ne2b_sim *sim);                          /* Backend::reset_state */
ne2b_status ne2b_synchronize(ne2b_sim *sim);                          /* Backend::synchronize */
ne2b_status ne2b_dev_mem_bytes(const ne2b_sim *sim, uint64_t *bytes); /* Backend::dev_mem_bytes */

/* Readbacks (lib.rs:136-151).  Buffers hold n values unless noted. */
ne2b_status ne2b_read_trace(ne2b_sim *sim, float *out);                    /* Backend::trace */
ne2b_status ne2b_read_state(ne2b_sim *sim, uint32_t slot, float *out);     /* Backend::state */
ne2b_status ne2b_read_syn_current(ne2b_sim *sim, float *out);              /* merged s[i] (cpu.rs:31) */
/* Backend::last_spikes: ascending ids; *count = spikes, at most cap written */
ne2b_status ne2b_last_spikes(ne2b_sim *sim, uint32_t *out, uint32_t cap, uint32_t *count);
/* Backend::spike_counts (lib.rs:143-146): NE2B_EWINDOW between depth and t */
ne2b_status ne2b_spike_counts(ne2b_sim *sim, uint64_t rows, uint32_t *out);
/* Backend::spike_row: out holds ceil(n/64) words; NE2B_ENODATA outside the window */
ne2b_status ne2b_spike_row(ne2b_sim *sim, uint32_t back, uint64_t *out);
/* No counterpart in the reference.  ne2b_spike_counts without any device
 * allocation, for callers that cannot allocate: a thread serving under a
 * fixed device-memory budget (any allocation would fail), or one that must
 * not stall on cudaMalloc/cudaFree, which synchronise the device.  Same
 * window rules and results as ne2b_spike_counts; the scratch is a 4 MiB
 * array compiled into the library (held by every GPU that loads it until
 * exit), so a sim of more than 1,048,576 neurons gets NE2B_EINVAL whenever
 * its counts need the device (recording on and t > 0).  The array's device
 * address is looked up when the first sim on a device is created.  Calls
 * share that array: calls whose work overlaps on the GPU race. */
ne2b_status ne2b_spike_counts_noalloc(ne2b_sim *sim, uint64_t rows, uint32_t *out);
ne2b_status ne2b_spikes_total(ne2b_sim *sim, uint64_t *total);             /* Backend::spikes_total */
ne2b_status ne2b_mean_rate_hz(ne2b_sim *sim, double *hz);                  /* Backend::mean_rate_hz */
/* On-device window counts (new): window w, n values */
ne2b_status ne2b_window_counts(ne2b_sim *sim, uint32_t window, uint16_t *out);
ne2b_status ne2b_windows_done(ne2b_sim *sim, uint32_t *count);

/* Drive (lib.rs:152-183; stim.rs:60-127) */
ne2b_status ne2b_set_input_constant(ne2b_sim *sim, uint32_t input, float value);
ne2b_status ne2b_input_values(ne2b_sim *sim, float *out);                  /* [n_inputs] */
ne2b_status ne2b_play_input(ne2b_sim *sim, uint32_t input, const float *series, uint64_t len);
ne2b_status ne2b_loop_input(ne2b_sim *sim, uint32_t input, const float *series, uint64_t len);
ne2b_status ne2b_set_external(ne2b_sim *sim, uint32_t neuron, float amps);
ne2b_status ne2b_set_external_all(ne2b_sim *sim, const float *ext, uint32_t len);
ne2b_status ne2b_external(ne2b_sim *sim, float *out);
ne2b_status ne2b_set_noise(ne2b_sim *sim, float rate_hz, float kick_mv);
ne2b_status ne2b_set_gauss_noise(ne2b_sim *sim, float sd);                 /* new */

/* Step kernel selection (new): NE2B_KERNEL_AUTO runs the streaming kernel
 * (one launch per step), which ne2b_autotune may replace by the resident
 * persistent kernel where that measures faster; the other two force one
 * (RESIDENT fails with NE2B_UNSUPPORTED when the nets' state does not fit
 * in shared memory).  *resident reports which kernel runs.  The environment variable NE2B_KERNEL=stream|resident sets
 * the initial mode of every handle. */
enum { NE2B_KERNEL_AUTO = 0, NE2B_KERNEL_STREAM = 1, NE2B_KERNEL_RESIDENT = 2 };
ne2b_status ne2b_set_kernel_mode(ne2b_sim *sim, int32_t mode);
ne2b_status ne2b_kernel_mode(ne2b_sim *sim, int32_t *mode, int32_t *resident);
/* Time every (kernel, tile shape, occupancy) candidate on this sim for
 * steps_per_trial steps from a device snapshot of its state and keep the
 * fastest (the state is restored afterwards; AUTO mode may switch kernel). */
ne2b_status ne2b_autotune(ne2b_sim *sim, uint32_t steps_per_trial);
/* The step kernels' tile shape: threads per block x neurons per thread,
 * one of 64 x {1, 2, 4}, {128, 256} x {1, 2, 4, 8} and 512 x {1, 2, 4};
 * blocks_per_sm 0 = as many as fit. */
ne2b_status ne2b_tile_shape(ne2b_sim *sim, uint32_t *block, uint32_t *neurons_per_thread,
                            uint32_t *blocks_per_sm);
ne2b_status ne2b_set_tile_shape(ne2b_sim *sim, uint32_t block, uint32_t neurons_per_thread,
                                uint32_t blocks_per_sm);
/* Delivery warps (new; no reference counterpart, the reference delivers
 * with one warp per spike in a second kernel, kernels.rs:174-204): with
 * `on`, the streaming step kernel of a one-net sim runs separate delivery
 * warps beside the tile threads, which queue their spiking neurons' rows
 * in shared memory, so delivery overlaps the neuron pass (tile blocks of
 * 128, 256 and 512 threads).  ne2b_autotune tries both and keeps the faster.
 * ne2b_set_tile_shape keeps this setting.  *active reports whether the
 * kernel that runs uses them.  Results are the same either way (bit for bit
 * with the int32 ring). */
ne2b_status ne2b_set_delivery_warps(ne2b_sim *sim, int32_t on);
ne2b_status ne2b_delivery_warps(ne2b_sim *sim, int32_t *on, int32_t *active);

/* Instrumentation (new): the CUDA stream the handle launches on (a
 * cudaStream_t, for timing with events on the launching stream) and the
 * number of kernels the handle has launched so far. */
ne2b_status ne2b_stream(ne2b_sim *sim, void **stream);
ne2b_status ne2b_kernel_launches(ne2b_sim *sim, uint64_t *launches);

/* Editor observability (lib.rs:164-176; cpu.rs:308-407).
 * set_v_watch: the neurons whose state slots 0 and 1 are recorded after
 * every step (an id beyond n records 0); a new list starts an empty
 * history, the same list keeps it; the last 4096 samples are kept.
 * watch_count: the watch count and the samples drain_watch would return.
 * drain_watch: out = [slot 0..1][watch][samples], oldest first, sized by
 * watch_count; empties the history.  set_grid_watches: member lists in
 * texel order (members[group_ptr[g] .. group_ptr[g+1]]); grid_traces: one
 * value per texel, groups concatenated, exp(-(t - last spike) * dt / tau)
 * and 0 for a texel that never spiked.  reset_state clears both. */
ne2b_status ne2b_set_v_watch(ne2b_sim *sim, const uint32_t *ids, uint32_t count);
ne2b_status ne2b_watch_count(ne2b_sim *sim, uint32_t *watches, uint32_t *samples);
ne2b_status ne2b_drain_watch(ne2b_sim *sim, float *out, uint32_t *samples);
ne2b_status ne2b_set_grid_watches(ne2b_sim *sim, const uint32_t *members, const uint32_t *group_ptr,
                                  uint32_t groups);
ne2b_status ne2b_grid_traces(ne2b_sim *sim, float tau_ms, float *out);

/* ---------------------------------------------------------------- batch */
/* Many independent networks of uneven size stepped together: one
 * persistent kernel per step over every net's tiles, the multi-step loop
 * replayed from a CUDA graph.  Results per net are those of the net run
 * alone (bit-identical in fixed-point mode). */
typedef struct ne2b_batch ne2b_batch;
ne2b_status ne2b_batch_create(const ne2b_net_desc *nets, const ne2b_config *cfgs, uint32_t count,
                              int device, ne2b_batch **out);
ne2b_status ne2b_batch_destroy(ne2b_batch *b);
ne2b_status ne2b_batch_play_input(ne2b_batch *b, uint32_t net, uint32_t input, const float *series,
                                  uint64_t len);
/* A fixed [steps x n_inputs] input matrix for one net, uploaded once and
 * read on the device from the net's current step on (new; replaces the
 * host-packed stimulus program for that net). */
ne2b_status ne2b_batch_set_input_matrix(ne2b_batch *b, uint32_t net, const float *inputs, uint64_t steps);
ne2b_status ne2b_batch_run_steps(ne2b_batch *b, uint64_t steps);
ne2b_status ne2b_batch_reset_state(ne2b_batch *b);
ne2b_status ne2b_batch_synchronize(ne2b_batch *b);
ne2b_status ne2b_batch_window_counts(ne2b_batch *b, uint32_t net, uint32_t window, uint16_t *out);
ne2b_status ne2b_batch_spikes_total(ne2b_batch *b, uint32_t net, uint64_t *total);
ne2b_status ne2b_batch_read_state(ne2b_batch *b, uint32_t net, uint32_t slot, float *out);
/* As ne2b_autotune, over every net of the batch. */
ne2b_status ne2b_batch_autotune(ne2b_batch *b, uint32_t steps_per_trial);
ne2b_status ne2b_batch_tile_shape(ne2b_batch *b, uint32_t *block, uint32_t *neurons_per_thread,
                                  uint32_t *blocks_per_sm);
ne2b_status ne2b_batch_set_tile_shape(ne2b_batch *b, uint32_t block, uint32_t neurons_per_thread,
                                      uint32_t blocks_per_sm);
ne2b_status ne2b_batch_dev_mem_bytes(ne2b_batch *b, uint64_t *bytes);
ne2b_status ne2b_batch_last_step_ms(ne2b_batch *b, float *ms);
ne2b_status ne2b_batch_set_kernel_mode(ne2b_batch *b, int32_t mode);
ne2b_status ne2b_batch_kernel_mode(ne2b_batch *b, int32_t *mode, int32_t *resident);
ne2b_status ne2b_batch_stream(ne2b_batch *b, void **stream);
ne2b_status ne2b_batch_kernel_launches(ne2b_batch *b, uint64_t *launches);
/* ne2b_fit_ridge_multi on features that stay on the device: trial r is net
 * nets[r] of the batch, its features the spike counts of its first
 * `windows` windows, window-major ([windows][n], F = windows x n; all the
 * nets the same size, each with those windows done).  Ordered after the
 * batch's queued steps; *n_features receives F. */
ne2b_status ne2b_batch_fit_ridge_multi(ne2b_batch *b, const uint32_t *nets, uint32_t t, uint32_t windows,
                                       const uint32_t *labels, uint32_t k, double lambda, uint32_t *n_features,
                                       double *w);
/* ne2b_fit_ridge on the same device-resident features, host targets y[T]. */
ne2b_status ne2b_batch_fit_ridge(ne2b_batch *b, const uint32_t *nets, uint32_t t, uint32_t windows, const float *y,
                                 float lambda, uint32_t *n_features, double *w);

/* -------------------------------------------------------------- serving */
/* Continuous batching of trial requests: requests are admitted into free
 * device capacity between steps, stepped together, and retired when their
 * duration is reached; all state stays on the device. */
typedef struct ne2b_server ne2b_server;
typedef struct {
    uint64_t neuron_capacity;    /* padded neurons resident at once */
    uint64_t synapse_capacity;   /* synapses resident at once */
    uint64_t ring_capacity;      /* ring words (depth x padded neurons) resident at once */
    uint32_t max_requests;       /* concurrent request slots */
    uint32_t steps_per_launch;   /* steps per graph replay between admissions */
    int32_t int_weights;
    /* 0: ne2b_server_submit builds the request's device arrays before it
     * returns.  k > 0: k host threads build them while the device steps;
     * submit only checks and reserves capacity, the request joins at a later
     * ne2b_server_step, and the caller's net arrays and input matrix must
     * stay valid until its result is taken.  A request that fails to build
     * is reported finished; ne2b_server_take_result returns its error. */
    uint32_t admission_threads;
} ne2b_server_config;
ne2b_status ne2b_server_create(const ne2b_server_config *cfg, int device, ne2b_server **out);
ne2b_status ne2b_server_destroy(ne2b_server *s);
/* Footprint of a request in the three capacities, for admission control. */
ne2b_status ne2b_request_footprint(const ne2b_net_desc *net, const ne2b_config *cfg, uint64_t *neurons,
                                   uint64_t *synapses, uint64_t *ring_words);
/* Admit a request: net + cfg + a [steps x n_inputs] input matrix.  cfg
 * must set window_steps; steps is the trial duration.  NE2B_EFULL when it
 * does not fit now (retry after ne2b_server_step retires requests). */
ne2b_status ne2b_server_submit(ne2b_server *s, const ne2b_net_desc *net, const ne2b_config *cfg,
                               const float *inputs, uint64_t steps, uint64_t *request_id);
/* Run one launch of steps_per_launch steps over every admitted request and
 * retire the finished ones; *finished = number of requests finished. */
ne2b_status ne2b_server_step(ne2b_server *s, uint32_t *active, uint32_t *finished);
/* Pop one finished request: its id, neuron count and windows; counts is
 * [windows x n] u16 (caller sizes it via ne2b_server_result_shape). */
ne2b_status ne2b_server_result_shape(ne2b_server *s, uint64_t request_id, uint32_t *n, uint32_t *windows);
ne2b_status ne2b_server_take_result(ne2b_server *s, uint64_t request_id, uint16_t *counts,
                                    uint64_t *spikes_total);
/* Ids of finished requests whose results are ready (taking them does not
 * wait for the device); *count is the number ready, ids[0..min(cap,count))
 * are filled.  A request retired by a launch still in flight appears once
 * that launch completes. */
ne2b_status ne2b_server_finished_ids(ne2b_server *s, uint64_t *ids, uint32_t cap, uint32_t *count);
ne2b_status ne2b_server_stats(ne2b_server *s, uint64_t *admitted, uint64_t *retired, uint32_t *active,
                              uint64_t *neurons_used, uint64_t *synapses_used);
/* Wait for every launch queued so far (no counterpart in the reference:
 * the serving loop is new). */
ne2b_status ne2b_server_synchronize(ne2b_server *s);
/* Tile shape of the server's step kernel (default 128 threads x 1 neuron);
 * same shapes as ne2b_set_tile_shape.  Waits for queued launches. */
ne2b_status ne2b_server_set_tile_shape(ne2b_server *s, uint32_t block, uint32_t npt, uint32_t blocks_per_sm);
ne2b_status ne2b_server_stream(ne2b_server *s, void **stream);
ne2b_status ne2b_server_kernel_launches(ne2b_server *s, uint64_t *launches);

/* ------------------------------------------------------ readout training */
/* fit_ridge_multi (sim/src/readout.rs:190-252): multi-class ridge solved in
 * the dual on the column-centred design x[T x F] (row-major f32, in host or
 * device memory), labels[T] in 0..k-1; w[k x (F + 1)] receives one weight
 * row per class, bias last.  The Gram matrix, its Cholesky factor and the
 * weights are computed on `device` with the reference's f64 operations in
 * the reference's order, so w equals the reference's bit for bit; a Gram
 * matrix that is not positive definite gives zero dual weights, as there.
 * T at most 32768 (the T x T Gram matrix is f64). */
ne2b_status ne2b_fit_ridge_multi(const float *x, uint32_t t, uint32_t f, const uint32_t *labels, uint32_t k,
                                 double lambda, int device, double *w);
/* fit_ridge (readout.rs:103-141): binary ridge in the primal on x[T x F]
 * (host or device memory) and host targets y[T]; w[F + 1], bias last, equal
 * to the reference's bit for bit (the (F + 1)^2 normal matrix, its
 * Cholesky factor and the fallback with 1e-3 + lambda more on the diagonal
 * as there).  F at most 32767. */
ne2b_status ne2b_fit_ridge(const float *x, uint32_t t, uint32_t f, const float *y, float lambda, int device,
                           double *w);

/* ----------------------------------------------------------- net building */
/* A host-side network owned by the library, in the ne2b_net_desc layout. */
typedef struct ne2b_net ne2b_net;
/* Network::synapse_csr (net-format/src/network.rs:654-692): stable sort by
 * source, Dale's-law sign from the source kind (kind[i]: 0 exc, 1 inh,
 * 2 regular), steps = max(1, round(delay/dt)), overflow of u16 is
 * NE2B_EINVAL. Inputs are synapse lists in insertion order. */
ne2b_status ne2b_net_from_synapses(uint32_t n, const uint8_t *model, const float *params,
                                   uint32_t param_stride, const uint8_t *kind, uint64_t n_syn,
                                   const uint32_t *src, const uint32_t *tgt, const float *w,
                                   const float *delay_ms, const float *tau_ms, float dt_ms,
                                   ne2b_net **out);
/* The reference's `.ne2` network files (net-format/src/io.rs:427-467 load):
 * format versions 1-7, checked by the rules of Network::validate
 * (network.rs:1007-1236), then built as Sim::new sees the network: model
 * rows by NeuronParams::from_network (sim/src/state.rs:98-153; models "izh"
 * and "adex", others NE2B_UNSUPPORTED), the CSR of Network::synapse_csr at
 * the file's dt, per-synapse tau kept, stimulus routing by
 * StimMap::from_network (stim.rs:26-48).  `meta` (may be NULL) receives the
 * file's Meta (network.rs:381-392) for the sim config.  A malformed file is
 * NE2B_EINVAL with the decoder's message. */
typedef struct {
    uint32_t version;
    float dt_ms;
    uint64_t seed;
    float conduction_speed;
    float synapse_tau_ms;
    float readout_tau_ms;
    float noise_rate_hz;
    float noise_kick_mv;
    uint32_t n_types, n_groups, n_samples, n_readouts, n_scripts;
} ne2b_ne2_meta;
ne2b_status ne2b_net_load_ne2(const char *path, ne2b_net **out, ne2b_ne2_meta *meta);
ne2b_status ne2b_net_from_ne2(const uint8_t *bytes, uint64_t len, ne2b_net **out, ne2b_ne2_meta *meta);
/* Self-test of the resident kernel's bounded grid barrier (no counterpart in
 * the reference): 4 cooperative blocks of which one never arrives; the
 * other three give up after limit_ms (1..2000), flag the error and return,
 * and *timed_out reports it.  The device stays usable; nothing faults. */
ne2b_status ne2b_selftest_barrier_timeout(int device, uint32_t limit_ms, int32_t *timed_out);
/* Random K-out workload net (10k/100k/1M configurations). */
ne2b_status ne2b_gen_random_kout(uint32_t n, uint32_t k, uint64_t seed, float w_scale, float exc_hi,
                                 float inh_hi, float delay_cap_ms, float dt_ms, ne2b_net **out);
/* Local 3-D liquid workload net (batched / served configurations). */
ne2b_status ne2b_gen_liquid(uint32_t side, uint64_t seed, double lambda_units, int32_t radius_units,
                            float w_rec, uint32_t n_inputs, uint32_t targets_per_input, float w_in,
                            int32_t model, float dt_ms, ne2b_net **out);
/* Convert every neuron of a net to a model with the given param rows
 * (exc_row for kind 0/2, inh_row for kind 1). */
ne2b_status ne2b_net_set_model_all(ne2b_net *net, int32_t model, const float *exc_row,
                                   const float *inh_row, uint32_t row_len);
ne2b_status ne2b_net_desc_of(const ne2b_net *net, ne2b_net_desc *out);
ne2b_status ne2b_net_kinds(const ne2b_net *net, uint8_t *kind);
ne2b_status ne2b_net_free(ne2b_net *net);

/* Deterministic exp used by the AdEx step (host copy of the device code). */
float ne2b_expf(float x);

#ifdef __cplusplus
}
#endif
#endif /* NE2B_H */
