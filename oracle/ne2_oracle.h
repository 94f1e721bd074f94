/*
 * ne2_oracle.h — CPU restatement of the neuro_edit v2 simulation step.
 *
 * TEST INFRASTRUCTURE ONLY. This is the parity oracle for the B200 kernels:
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg are the
 * only callers.  The shipped library (neuro_edit_v2_b200) never links it.
 *
 * Every function restates the reference Rust code it cites (paths are
 * relative to the lucksus/neuro_edit_v2 tree).  The reference is Rust and
 * cannot be compiled in this environment, so parity of this restatement is
 * pinned by the reference's own known-answer tests, chiefly the FNV
 * fingerprint 0x9d792bd233132f5d of sim/tests/cpu_ref.rs:208-244, which
 * covers Rng, create_2d_grid, create_connections, synapse_csr, Poisson
 * noise and the Izhikevich step bit-for-bit.
 *
 * Arithmetic contract: compiled with -O2 -ffp-contract=off and no fast-math,
 * SSE float, so every f32/f64 operation rounds exactly as Rust's does.
 */
#ifndef NE2_ORACLE_H
#define NE2_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- Rng */
/* net-format/src/rng.rs:8-82 — splitmix64 seed expansion into xoshiro256** */
typedef struct { uint64_t s[4]; } ne2o_rng;
void     ne2o_rng_seed(ne2o_rng *r, uint64_t seed);
uint64_t ne2o_rng_next_u64(ne2o_rng *r);
double   ne2o_rng_f64(ne2o_rng *r);
float    ne2o_rng_f32(ne2o_rng *r);
double   ne2o_rng_uniform(ne2o_rng *r, double lo, double hi);
uint64_t ne2o_rng_below(ne2o_rng *r, uint64_t n);
double   ne2o_rng_gauss(ne2o_rng *r, double mean, double sd);
void     ne2o_rng_shuffle_u32(ne2o_rng *r, uint32_t *v, size_t n);

/* ------------------------------------------------------------ Network */
enum { NE2O_EXC = 0, NE2O_INH = 1, NE2O_REGULAR = 2 };
enum { NE2O_MODEL_IZH = 0, NE2O_MODEL_ADEX = 1 };
#define NE2O_PMAX 10

typedef struct {
    /* neurons */
    uint32_t n, ncap;
    float   *pos;      /* n*3 */
    uint8_t *kind;     /* NE2O_EXC / INH / REGULAR */
    uint8_t *model;    /* registry id */
    float   *params;   /* n*NE2O_PMAX, effective param row */
    uint8_t *nparams;  /* row width per neuron */
    /* synapses (insertion order) */
    uint64_t ns, scap;
    uint32_t *s_src, *s_tgt;
    float    *s_w, *s_delay, *s_tau;
    /* inputs: input k targets in_tgt[in_ptr[k]..in_ptr[k+1]] */
    uint32_t ninputs, in_cap, nin_entries, in_ecap;
    uint32_t *in_ptr;
    uint32_t *in_tgt;
    float    *in_w;
    float conduction_speed;  /* net-format/src/lib.rs:36 default 100 */
} ne2o_net;

ne2o_net *ne2o_net_new(void);
void      ne2o_net_free(ne2o_net *net);
uint32_t  ne2o_net_add_neuron(ne2o_net *net, float x, float y, float z, int kind);
void      ne2o_net_set_model(ne2o_net *net, uint32_t id, int model, const float *p, int np);
void      ne2o_net_set_kind(ne2o_net *net, uint32_t id, int kind);
float     ne2o_net_conduction_delay_ms(const ne2o_net *net, uint32_t a, uint32_t b);
uint64_t  ne2o_net_connect(ne2o_net *net, uint32_t src, uint32_t tgt, float w);
void      ne2o_net_push_synapse(ne2o_net *net, uint32_t src, uint32_t tgt, float w,
                                float delay_ms, float tau_ms);
uint32_t  ne2o_net_add_input(ne2o_net *net, const uint32_t *tgt, const float *w, uint32_t m);

/* builders (net-format/src/builders.rs); grids write member ids to `members` */
uint32_t ne2o_create_2d_grid(ne2o_net *net, uint32_t w, uint32_t h, float dist,
                             float cx, float cy, float cz, uint32_t *members);
uint32_t ne2o_create_3d_grid(ne2o_net *net, uint32_t w, uint32_t h, uint32_t d, float dist,
                             float cx, float cy, float cz, uint32_t *members);
void ne2o_create_connections(ne2o_net *net, const uint32_t *members, uint32_t m,
                             double scaling, double lambda, float weight, ne2o_rng *rng);
void ne2o_set_exc_inh(ne2o_net *net, const uint32_t *members, uint32_t m,
                      double inh_fraction, ne2o_rng *rng);
void ne2o_set_exc_inh_exact(ne2o_net *net, const uint32_t *members, uint32_t m,
                            uint32_t n_inh, ne2o_rng *rng);
/* sim/src/bench.rs:10-52 */
ne2o_net *ne2o_bench_net(uint32_t n, uint32_t k, uint64_t seed, float w_scale, float w_inh);

/* Synthetic generators of the measured workloads (not in the reference;
 * defined by this project, restated identically by the product library). */
ne2o_net *ne2o_gen_random_kout(uint32_t n, uint32_t k, uint64_t seed, float w_scale,
                               float exc_hi, float inh_hi, float delay_cap_ms);
ne2o_net *ne2o_gen_liquid(uint32_t side, uint64_t seed, double lambda_units,
                          int radius_units, float w_rec, uint32_t n_inputs,
                          uint32_t targets_per_input, float w_in, int model);

/* -------------------------------------------------------------- CSR */
/* net-format/src/network.rs:654-692 */
typedef struct {
    uint32_t n;
    uint64_t e;
    uint32_t *src_ptr;   /* n+1 */
    uint32_t *tgt;
    float    *w;         /* signed by Dale's law */
    uint16_t *delay;     /* steps */
    float    *tau;
} ne2o_csr;
/* returns 0 on success, -1 when a delay exceeds u16 (message in err) */
int  ne2o_synapse_csr(const ne2o_net *net, float dt_ms, ne2o_csr *out, char *err, size_t errlen);
void ne2o_csr_free(ne2o_csr *c);

/* ------------------------------------------------------------ noise */
/* sim/src/state.rs:284-301 */
uint32_t ne2o_noise_hash(uint32_t i, uint64_t t, uint64_t seed);
int      ne2o_noise_fires(uint32_t i, uint64_t t, uint64_t seed, float p);
/* Gaussian current noise (project definition): Irwin-Hall sum of four
 * 16-bit fields of one counter hash; returns the integer numerator
 * S - 131070 (multiply by ne2o_gauss_scale(sd) for the current). */
int64_t  ne2o_gauss_numer(uint32_t i, uint64_t t, uint64_t seed);
float    ne2o_gauss_scale(float sd);

/* deterministic exp shared with the device kernels */
float ne2o_det_expf(float x);
/* test support: compares f with ne2o_det_expf bit for bit on every
 * `stride`-th float in [lo, hi] (by bit pattern, both signs), split over
 * `threads` threads; returns the mismatches and stores the values checked */
/* readout training, sim/src/readout.rs:190-252 fit_ridge_multi: multi-class
 * ridge in the dual on the column-centred design x[T*F] (f32), labels[T] in
 * 0..k-1; w_out[k][F + 1] (bias last).  A Gram matrix that is not positive
 * definite gives zero dual weights, as the reference does. */
void ne2o_fit_ridge_multi(const float *x, uint32_t t, uint32_t f, const uint32_t *labels, uint32_t k, double lambda,
                          double *w_out);
/* readout.rs:103-141 fit_ridge: binary ridge in the primal (normal
 * equations with a bias column, the bias unregularised); w_out[F + 1] */
void ne2o_fit_ridge(const float *x, uint32_t t, uint32_t f, const float *y, float lambda, double *w_out);
/* readout.rs:144-188 cholesky_solve (row-major n x n); 0 when not PD */
int ne2o_cholesky_solve(const double *a, const double *b, uint32_t n, double *w);
uint64_t ne2o_expf_mismatches(float (*f)(float), float lo, float hi, uint32_t stride, uint32_t threads,
                              uint64_t *checked);
/* test support: the largest distance, in representable floats, between f
 * and ne2o_det_expf on the same inputs as ne2o_expf_mismatches */
uint64_t ne2o_expf_max_ulp(float (*f)(float), float lo, float hi, uint32_t stride, uint32_t threads,
                           uint64_t *checked);
float    ne2o_expf_ref(float x);  /* (float)exp((double)x) */

/* --------------------------------------------------------------- sim */
typedef struct {
    float    dt_ms, synapse_tau_ms, readout_tau_ms, noise_rate_hz, noise_kick_mv;
    uint64_t seed;
    int      record_spikes;
    uint32_t spike_record_steps;
    int      int_weights;      /* fixed-point ring, scale 4096 */
    float    gauss_sd;         /* 0 = off (project feature) */
    int      exp_mode;         /* 0 = libm expf (reference), 1 = deterministic exp */
} ne2o_cfg;
void ne2o_cfg_default(ne2o_cfg *c);  /* sim/src/state.rs:35-49 */

typedef struct ne2o_sim ne2o_sim;
ne2o_sim *ne2o_sim_new(const ne2o_net *net, const ne2o_cfg *cfg, char *err, size_t errlen);
void      ne2o_sim_free(ne2o_sim *s);
void      ne2o_sim_step(ne2o_sim *s);
void      ne2o_sim_run_steps(ne2o_sim *s, uint64_t steps);
void      ne2o_sim_reset_state(ne2o_sim *s);
/* editor watches (cpu.rs:63-95, 308-407) */
#define NE2O_V_HIST_CAP 4096u
void      ne2o_sim_set_v_watch(ne2o_sim *s, const uint32_t *ids, uint32_t count);
uint32_t  ne2o_sim_drain_watch(ne2o_sim *s, float *out); /* out: [2][nwatch][returned count] */
void      ne2o_sim_set_grid_watches(ne2o_sim *s, const uint32_t *members, const uint32_t *group_ptr, uint32_t ngroups);
void      ne2o_sim_grid_traces(const ne2o_sim *s, float tau_ms, float *out);
uint64_t  ne2o_sim_t(const ne2o_sim *s);
uint32_t  ne2o_sim_n(const ne2o_sim *s);
uint32_t  ne2o_sim_ring_depth(const ne2o_sim *s);
uint64_t  ne2o_sim_spikes_total(const ne2o_sim *s);
double    ne2o_sim_mean_rate_hz(const ne2o_sim *s);
/* copies: state slot column, s, trace, pn_total */
int       ne2o_sim_state(const ne2o_sim *s, uint32_t slot, float *out);
void      ne2o_sim_syn_current(const ne2o_sim *s, float *out);
void      ne2o_sim_trace(const ne2o_sim *s, float *out);
void      ne2o_sim_pn_total(const ne2o_sim *s, uint64_t *out);
/* spike_row: returns words copied, 0 when unavailable */
uint32_t  ne2o_sim_spike_row(const ne2o_sim *s, uint32_t back, uint64_t *out);
/* 0 ok, -1 window error (message in err) */
int       ne2o_sim_spike_counts(const ne2o_sim *s, uint64_t rows, uint32_t *out,
                                char *err, size_t errlen);
/* number of spikes emitted by the last step, ascending neuron ids */
uint32_t  ne2o_sim_last_step_spikes(const ne2o_sim *s, uint32_t *out);
void      ne2o_sim_set_external(ne2o_sim *s, uint32_t i, float amps);
void      ne2o_sim_set_input_constant(ne2o_sim *s, uint32_t k, float v);
void      ne2o_sim_play_input(ne2o_sim *s, uint32_t k, const float *series, uint64_t len);
void      ne2o_sim_loop_input(ne2o_sim *s, uint32_t k, const float *series, uint64_t len);
void      ne2o_sim_set_noise(ne2o_sim *s, float rate_hz, float kick_mv);
float     ne2o_sim_stim_value(const ne2o_sim *s, uint32_t k, uint64_t t);
/* FNV-1a fold of 400 record rows + v bits (sim/tests/cpu_ref.rs:230-243) */
uint64_t  ne2o_sim_fingerprint(const ne2o_sim *s, uint32_t rows);

/* flattened views used to feed the product library the same net */
uint32_t  ne2o_net_n(const ne2o_net *net);
uint64_t  ne2o_net_ns(const ne2o_net *net);
void      ne2o_net_models(const ne2o_net *net, uint8_t *model, float *params_padded10);
void      ne2o_net_kinds(const ne2o_net *net, uint8_t *kind);
uint32_t  ne2o_net_ninputs(const ne2o_net *net);
uint32_t  ne2o_net_input_entries(const ne2o_net *net);
void      ne2o_net_inputs(const ne2o_net *net, uint32_t *in_ptr, uint32_t *in_tgt, float *in_w);
void      ne2o_net_synapses(const ne2o_net *net, uint32_t *src, uint32_t *tgt, float *w,
                            float *delay_ms, float *tau_ms);
void      ne2o_net_positions(const ne2o_net *net, float *pos);

#ifdef __cplusplus
}
#endif
#endif
