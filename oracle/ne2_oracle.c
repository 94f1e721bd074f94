/*
 * ne2_oracle.c — CPU restatement of the neuro_edit v2 `sim` step loop.
 *
 * TEST INFRASTRUCTURE ONLY (parity oracle).  See ne2_oracle.h.  Each
 * function cites the reference Rust code it restates; paths are relative to
 * the lucksus/neuro_edit_v2 source tree.
 *
 * Parity of this restatement is pinned by the reference's known-answer tests
 * (fingerprint 0x9d792bd233132f5d, sim/tests/cpu_ref.rs:208-244, and the
 * hand-computed traces of cpu_ref.rs:16-114); the fixed-point ring has no CPU
 * counterpart in the reference and follows the CUDA text of
 * sim/src/kernels.rs:57-66 applied to the CPU step order.
 */
#include "ne2_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define XMALLOC(T, n) ((T *)xmalloc_n(sizeof(T), (size_t)(n)))
static void *xmalloc(size_t b) {
    void *p = malloc(b ? b : 1);
    if (!p) { fprintf(stderr, "ne2_oracle: out of memory (%zu bytes)\n", b); abort(); }
    return p;
}
static void *xmalloc_n(size_t sz, size_t n) { return xmalloc(sz * (n ? n : 1)); }
static void *xrealloc(void *p, size_t b) {
    void *q = realloc(p, b ? b : 1);
    if (!q) { fprintf(stderr, "ne2_oracle: out of memory (%zu bytes)\n", b); abort(); }
    return q;
}

/* ================================================================ Rng */
/* net-format/src/rng.rs:17-30 */
void ne2o_rng_seed(ne2o_rng *r, uint64_t seed) {
    uint64_t z = seed;
    for (int k = 0; k < 4; ++k) {
        z += 0x9E3779B97F4A7C15ull;
        uint64_t x = z;
        x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
        x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
        r->s[k] = x ^ (x >> 31);
    }
}
static inline uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
/* net-format/src/rng.rs:32-42 (xoshiro256**) */
uint64_t ne2o_rng_next_u64(ne2o_rng *r) {
    uint64_t *s = r->s;
    uint64_t result = rotl64(s[1] * 5, 7) * 9;
    uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl64(s[3], 45);
    return result;
}
/* rng.rs:45-47 */
double ne2o_rng_f64(ne2o_rng *r) {
    return (double)(ne2o_rng_next_u64(r) >> 11) * (1.0 / 9007199254740992.0);
}
/* rng.rs:50-52 */
float ne2o_rng_f32(ne2o_rng *r) {
    return (float)(ne2o_rng_next_u64(r) >> 40) * (1.0f / 16777216.0f);
}
/* rng.rs:55-57 */
double ne2o_rng_uniform(ne2o_rng *r, double lo, double hi) {
    return lo + (hi - lo) * ne2o_rng_f64(r);
}
/* rng.rs:60-62 */
uint64_t ne2o_rng_below(ne2o_rng *r, uint64_t n) {
    return ne2o_rng_next_u64(r) % (n ? n : 1);
}
/* rng.rs:65-69 (Box-Muller, glibc log/sqrt/cos as Rust std uses) */
double ne2o_rng_gauss(ne2o_rng *r, double mean, double sd) {
    double u1 = 1.0 - ne2o_rng_f64(r);
    if (u1 < 1e-300) u1 = 1e-300;
    double u2 = ne2o_rng_f64(r);
    return mean + sd * sqrt(-2.0 * log(u1)) * cos(2.0 * 3.141592653589793 * u2);
}
/* rng.rs:77-81 (Fisher-Yates) */
void ne2o_rng_shuffle_u32(ne2o_rng *r, uint32_t *v, size_t n) {
    for (size_t i = n; i-- > 1;) {
        size_t j = (size_t)ne2o_rng_below(r, (uint64_t)(i + 1));
        uint32_t tmp = v[i]; v[i] = v[j]; v[j] = tmp;
    }
}

/* ============================================================ Network */
/* net-format/src/network.rs:53-54; sim/src/model/adex.rs:22-26 */
static const float IZH_RS[4] = {0.02f, 0.2f, -65.0f, 8.0f};
static const float IZH_FS[4] = {0.1f, 0.2f, -65.0f, 2.0f};

ne2o_net *ne2o_net_new(void) {
    ne2o_net *net = (ne2o_net *)calloc(1, sizeof(ne2o_net));
    if (!net) abort();
    net->conduction_speed = 100.0f; /* net-format/src/lib.rs:36 */
    net->in_ptr = XMALLOC(uint32_t, 1);
    net->in_ptr[0] = 0;
    net->in_cap = 1;
    return net;
}

void ne2o_net_free(ne2o_net *net) {
    if (!net) return;
    free(net->pos); free(net->kind); free(net->model); free(net->params); free(net->nparams);
    free(net->s_src); free(net->s_tgt); free(net->s_w); free(net->s_delay); free(net->s_tau);
    free(net->in_ptr); free(net->in_tgt); free(net->in_w);
    free(net);
}

static void net_grow_neurons(ne2o_net *net, uint32_t need) {
    if (need <= net->ncap) return;
    uint32_t cap = net->ncap ? net->ncap : 64;
    while (cap < need) cap *= 2;
    net->pos = (float *)xrealloc(net->pos, sizeof(float) * 3 * cap);
    net->kind = (uint8_t *)xrealloc(net->kind, cap);
    net->model = (uint8_t *)xrealloc(net->model, cap);
    net->params = (float *)xrealloc(net->params, sizeof(float) * NE2O_PMAX * cap);
    net->nparams = (uint8_t *)xrealloc(net->nparams, cap);
    net->ncap = cap;
}

static void set_row(ne2o_net *net, uint32_t id, int model, const float *p, int np) {
    net->model[id] = (uint8_t)model;
    net->nparams[id] = (uint8_t)np;
    float *row = net->params + (size_t)id * NE2O_PMAX;
    for (int k = 0; k < NE2O_PMAX; ++k) row[k] = k < np ? p[k] : 0.0f;
}

/* network.rs:451-461 + default_type_for (465-493): the kind's stock izh row */
uint32_t ne2o_net_add_neuron(ne2o_net *net, float x, float y, float z, int kind) {
    net_grow_neurons(net, net->n + 1);
    uint32_t id = net->n++;
    net->pos[3 * id + 0] = x;
    net->pos[3 * id + 1] = y;
    net->pos[3 * id + 2] = z;
    net->kind[id] = (uint8_t)kind;
    set_row(net, id, NE2O_MODEL_IZH, kind == NE2O_INH ? IZH_FS : IZH_RS, 4);
    return id;
}

void ne2o_net_set_model(ne2o_net *net, uint32_t id, int model, const float *p, int np) {
    set_row(net, id, model, p, np);
}

/* network.rs:530-541: a neuron still on a stock izh row picks up the new
 * kind's stock row; custom rows are kept as overrides. */
void ne2o_net_set_kind(ne2o_net *net, uint32_t id, int kind) {
    const float *row = net->params + (size_t)id * NE2O_PMAX;
    int stock = 0;
    if (net->model[id] == NE2O_MODEL_IZH && net->nparams[id] == 4) {
        stock = (memcmp(row, IZH_RS, sizeof IZH_RS) == 0) || (memcmp(row, IZH_FS, sizeof IZH_FS) == 0);
    }
    net->kind[id] = (uint8_t)kind;
    if (stock) set_row(net, id, NE2O_MODEL_IZH, kind == NE2O_INH ? IZH_FS : IZH_RS, 4);
}

/* network.rs:596-601 (f32 squares, f32 sqrt, /speed, floor 1e-3 ms) */
float ne2o_net_conduction_delay_ms(const ne2o_net *net, uint32_t a, uint32_t b) {
    const float *pa = net->pos + 3 * (size_t)a, *pb = net->pos + 3 * (size_t)b;
    float dx = pa[0] - pb[0], dy = pa[1] - pb[1], dz = pa[2] - pb[2];
    float d = sqrtf(dx * dx + dy * dy + dz * dz);
    float ms = d / net->conduction_speed;
    return ms > 1e-3f ? ms : 1e-3f;
}

void ne2o_net_push_synapse(ne2o_net *net, uint32_t src, uint32_t tgt, float w, float delay_ms,
                           float tau_ms) {
    if (net->ns == net->scap) {
        uint64_t cap = net->scap ? net->scap * 2 : 256;
        net->s_src = (uint32_t *)xrealloc(net->s_src, sizeof(uint32_t) * cap);
        net->s_tgt = (uint32_t *)xrealloc(net->s_tgt, sizeof(uint32_t) * cap);
        net->s_w = (float *)xrealloc(net->s_w, sizeof(float) * cap);
        net->s_delay = (float *)xrealloc(net->s_delay, sizeof(float) * cap);
        net->s_tau = (float *)xrealloc(net->s_tau, sizeof(float) * cap);
        net->scap = cap;
    }
    uint64_t j = net->ns++;
    net->s_src[j] = src;
    net->s_tgt[j] = tgt;
    net->s_w[j] = w;
    net->s_delay[j] = delay_ms;
    net->s_tau[j] = tau_ms;
}

/* network.rs:604-614 */
uint64_t ne2o_net_connect(ne2o_net *net, uint32_t src, uint32_t tgt, float w) {
    ne2o_net_push_synapse(net, src, tgt, w, ne2o_net_conduction_delay_ms(net, src, tgt), 0.0f);
    return net->ns - 1;
}

/* network.rs:719-731 (a new input; names are not modelled here) */
uint32_t ne2o_net_add_input(ne2o_net *net, const uint32_t *tgt, const float *w, uint32_t m) {
    if (net->ninputs + 2 > net->in_cap) {
        net->in_cap = net->in_cap * 2 + 2;
        net->in_ptr = (uint32_t *)xrealloc(net->in_ptr, sizeof(uint32_t) * net->in_cap);
    }
    if (net->nin_entries + m > net->in_ecap) {
        uint32_t cap = net->in_ecap ? net->in_ecap : 64;
        while (cap < net->nin_entries + m) cap *= 2;
        net->in_tgt = (uint32_t *)xrealloc(net->in_tgt, sizeof(uint32_t) * cap);
        net->in_w = (float *)xrealloc(net->in_w, sizeof(float) * cap);
        net->in_ecap = cap;
    }
    for (uint32_t j = 0; j < m; ++j) {
        net->in_tgt[net->nin_entries + j] = tgt[j];
        net->in_w[net->nin_entries + j] = w[j];
    }
    net->nin_entries += m;
    net->ninputs += 1;
    net->in_ptr[net->ninputs] = net->nin_entries;
    return net->ninputs - 1;
}

/* ============================================================ builders */
/* net-format/src/builders.rs:22-68 (create_2d_grid: w x h in the y-z plane) */
uint32_t ne2o_create_2d_grid(ne2o_net *net, uint32_t w, uint32_t h, float dist, float cx, float cy,
                             float cz, uint32_t *members) {
    uint32_t m = 0;
    for (uint32_t x = 0; x < w; ++x) {
        for (uint32_t y = 0; y < h; ++y) {
            float py = cy + ((float)y - (float)h / 2.0f) * dist;
            float pz = cz + ((float)x - (float)w / 2.0f) * dist;
            uint32_t id = ne2o_net_add_neuron(net, cx, py, pz, NE2O_EXC);
            if (members) members[m] = id;
            ++m;
        }
    }
    return m;
}

/* builders.rs:88-131 (create_3d_grid: member k = (z*w + x)*h + y) */
uint32_t ne2o_create_3d_grid(ne2o_net *net, uint32_t w, uint32_t h, uint32_t d, float dist, float cx,
                             float cy, float cz, uint32_t *members) {
    uint32_t m = 0;
    for (uint32_t z = 0; z < d; ++z) {
        for (uint32_t x = 0; x < w; ++x) {
            for (uint32_t y = 0; y < h; ++y) {
                float px = cx + ((float)x - (float)w / 2.0f) * dist;
                float py = cy + ((float)y - (float)h / 2.0f) * dist;
                float pz = cz + ((float)z - (float)d / 2.0f) * dist;
                uint32_t id = ne2o_net_add_neuron(net, px, py, pz, NE2O_EXC);
                if (members) members[m] = id;
                ++m;
            }
        }
    }
    return m;
}

static double pair_prob(const ne2o_net *net, uint32_t a, uint32_t b, double scaling, double lambda) {
    const float *pa = net->pos + 3 * (size_t)a, *pb = net->pos + 3 * (size_t)b;
    float dx = pa[0] - pb[0], dy = pa[1] - pb[1], dz = pa[2] - pb[2];
    double dist = (double)sqrtf(dx * dx + dy * dy + dz * dz);
    double q = dist / lambda;
    return scaling * exp(-(q * q));
}

/* builders.rs:136-181 (every ordered pair n1 != n2, one f64 draw per pair) */
void ne2o_create_connections(ne2o_net *net, const uint32_t *members, uint32_t m, double scaling,
                             double lambda, float weight, ne2o_rng *rng) {
    for (uint32_t i = 0; i < m; ++i) {
        uint32_t n1 = members[i];
        for (uint32_t j = 0; j < m; ++j) {
            uint32_t n2 = members[j];
            if (n1 == n2) continue;
            double p = pair_prob(net, n1, n2, scaling, lambda);
            if (ne2o_rng_f64(rng) < p) ne2o_net_connect(net, n1, n2, weight);
        }
    }
}

/* builders.rs:262-277 */
void ne2o_set_exc_inh(ne2o_net *net, const uint32_t *members, uint32_t m, double inh_fraction,
                      ne2o_rng *rng) {
    for (uint32_t i = 0; i < m; ++i) {
        int kind = ne2o_rng_f64(rng) < inh_fraction ? NE2O_INH : NE2O_EXC;
        ne2o_net_set_kind(net, members[i], kind);
    }
}

/* builders.rs:280-295 */
void ne2o_set_exc_inh_exact(ne2o_net *net, const uint32_t *members, uint32_t m, uint32_t n_inh,
                            ne2o_rng *rng) {
    uint32_t *v = XMALLOC(uint32_t, m);
    memcpy(v, members, sizeof(uint32_t) * m);
    ne2o_rng_shuffle_u32(rng, v, m);
    for (uint32_t i = 0; i < m; ++i) ne2o_net_set_kind(net, v[i], i < n_inh ? NE2O_INH : NE2O_EXC);
    free(v);
}

/* sim/src/bench.rs:10-52 */
ne2o_net *ne2o_bench_net(uint32_t n, uint32_t k, uint64_t seed, float w_scale, float w_inh) {
    ne2o_rng rng;
    ne2o_rng_seed(&rng, seed);
    ne2o_net *net = ne2o_net_new();
    net->conduction_speed = 1000.0f;
    uint64_t n_exc = (uint64_t)n * 4 / 5;
    for (uint32_t i = 0; i < n; ++i) {
        float x = (float)ne2o_rng_uniform(&rng, -500.0, 500.0);
        float y = (float)ne2o_rng_uniform(&rng, -500.0, 500.0);
        float z = (float)ne2o_rng_uniform(&rng, -500.0, 500.0);
        ne2o_net_add_neuron(net, x, y, z, i < n_exc ? NE2O_EXC : NE2O_INH);
    }
    for (uint32_t src = 0; src < n; ++src) {
        int exc = src < n_exc;
        float w = exc ? 6.0f * w_scale : w_inh;
        for (uint32_t j = 0; j < k; ++j) {
            uint32_t tgt = (uint32_t)ne2o_rng_below(&rng, n);
            float delay = exc ? (float)ne2o_rng_uniform(&rng, 1.0, 21.0) : 1.0f;
            ne2o_net_push_synapse(net, src, tgt, w, delay, 0.0f);
        }
    }
    return net;
}

/* Random K-out net of the measured 10k/100k/1M workloads (project
 * definition, bench.rs:10-52 with the workload's weight/delay rules):
 *   neurons: positions U(-500,500)^3 um drawn x,y,z per neuron; index <
 *     0.8n excitatory RS, the rest inhibitory FS;
 *   per source, K synapses in draw order: tgt = below(n);
 *     |w| = f32(f64() * hi) * w_scale (hi = exc_hi or inh_hi; Dale's law
 *     signs it at CSR build); delay = distance / 100 um/ms, floor 1e-3,
 *     capped at delay_cap_ms. */
ne2o_net *ne2o_gen_random_kout(uint32_t n, uint32_t k, uint64_t seed, float w_scale, float exc_hi,
                               float inh_hi, float delay_cap_ms) {
    ne2o_rng rng;
    ne2o_rng_seed(&rng, seed);
    ne2o_net *net = ne2o_net_new();
    uint64_t n_exc = (uint64_t)n * 4 / 5;
    for (uint32_t i = 0; i < n; ++i) {
        float x = (float)ne2o_rng_uniform(&rng, -500.0, 500.0);
        float y = (float)ne2o_rng_uniform(&rng, -500.0, 500.0);
        float z = (float)ne2o_rng_uniform(&rng, -500.0, 500.0);
        ne2o_net_add_neuron(net, x, y, z, i < n_exc ? NE2O_EXC : NE2O_INH);
    }
    for (uint32_t src = 0; src < n; ++src) {
        double hi = src < n_exc ? (double)exc_hi : (double)inh_hi;
        for (uint32_t j = 0; j < k; ++j) {
            uint32_t tgt = (uint32_t)ne2o_rng_below(&rng, n);
            float w = (float)(ne2o_rng_f64(&rng) * hi) * w_scale;
            float delay = ne2o_net_conduction_delay_ms(net, src, tgt);
            if (delay > delay_cap_ms) delay = delay_cap_ms;
            ne2o_net_push_synapse(net, src, tgt, w, delay, 0.0f);
        }
    }
    return net;
}

/* AdEx stock rows, sim/src/model/adex.rs:22-26 (TONIC exc, NONADAP inh) */
static const float ADEX_TONIC[10] = {281.0f, 30.0f, -70.6f, -50.4f, 2.0f, 4.0f, 144.0f, 80.5f, -70.6f, 20.0f};
static const float ADEX_NONADAP[10] = {281.0f, 30.0f, -70.6f, -50.4f, 2.0f, 0.0f, 144.0f, 0.0f, -70.6f, 20.0f};

/* Local 3-D liquid of the batched/served workloads (project definition):
 *   create_3d_grid(side^3, spacing 60 um) -> set_exc_inh(0.2) with
 *   Rng(seed) -> for AdEx liquids every neuron takes the AdEx kind default
 *   row (model/adex.rs:193-198) -> neighbourhood-limited
 *   create_connections: for each n1 in member order, each n2 in member
 *   order with lattice offset |o|^2 <= radius^2 and n2 != n1, draw f64() <
 *   exp(-(d/lambda)^2) (builders.rs:176-178 with scaling 1, lambda =
 *   lambda_units*60 um) -> connect(n1, n2, w_rec) with the distance delay
 *   -> n_inputs inputs, each with `targets_per_input` targets drawn on the
 *   x = 0 face (y = below(side), z = below(side)) at weight w_in.
 *   AdEx liquids multiply w_rec and w_in by C = 281 pF (the model's noise
 *   gain), so a weight moves v by the same mV as in an izh liquid. */
ne2o_net *ne2o_gen_liquid(uint32_t side, uint64_t seed, double lambda_units, int radius_units,
                          float w_rec, uint32_t n_inputs, uint32_t targets_per_input, float w_in,
                          int model) {
    ne2o_rng rng;
    ne2o_rng_seed(&rng, seed);
    ne2o_net *net = ne2o_net_new();
    const float spacing = 60.0f;
    uint32_t m = side * side * side;
    uint32_t *members = XMALLOC(uint32_t, m);
    ne2o_create_3d_grid(net, side, side, side, spacing, 0.0f, 0.0f, 0.0f, members);
    ne2o_set_exc_inh(net, members, m, 0.2, &rng);
    float gain = 1.0f;
    if (model == NE2O_MODEL_ADEX) {
        for (uint32_t i = 0; i < m; ++i)
            set_row(net, members[i], NE2O_MODEL_ADEX, net->kind[members[i]] == NE2O_INH ? ADEX_NONADAP : ADEX_TONIC, 10);
        gain = 281.0f;
    }
    float wr = w_rec * gain, wi = w_in * gain;
    double lambda = lambda_units * (double)spacing;
    int R = radius_units;
    for (uint32_t k1 = 0; k1 < m; ++k1) {
        int y1 = (int)(k1 % side), x1 = (int)((k1 / side) % side), z1 = (int)(k1 / side / side);
        for (int dz = -R; dz <= R; ++dz) {
            int z2 = z1 + dz;
            if (z2 < 0 || z2 >= (int)side) continue;
            for (int dx = -R; dx <= R; ++dx) {
                int x2 = x1 + dx;
                if (x2 < 0 || x2 >= (int)side) continue;
                for (int dy = -R; dy <= R; ++dy) {
                    int y2 = y1 + dy;
                    if (y2 < 0 || y2 >= (int)side) continue;
                    if (dx * dx + dy * dy + dz * dz > R * R) continue;
                    uint32_t k2 = ((uint32_t)z2 * side + (uint32_t)x2) * side + (uint32_t)y2;
                    if (k2 == k1) continue;
                    double p = pair_prob(net, members[k1], members[k2], 1.0, lambda);
                    if (ne2o_rng_f64(&rng) < p) ne2o_net_connect(net, members[k1], members[k2], wr);
                }
            }
        }
    }
    uint32_t *tg = XMALLOC(uint32_t, targets_per_input);
    float *tw = XMALLOC(float, targets_per_input);
    for (uint32_t k = 0; k < n_inputs; ++k) {
        for (uint32_t j = 0; j < targets_per_input; ++j) {
            uint32_t y = (uint32_t)ne2o_rng_below(&rng, side);
            uint32_t z = (uint32_t)ne2o_rng_below(&rng, side);
            tg[j] = members[(z * side + 0) * side + y];
            tw[j] = wi;
        }
        ne2o_net_add_input(net, tg, tw, targets_per_input);
    }
    free(tg);
    free(tw);
    free(members);
    return net;
}

/* ================================================================= CSR */
/* net-format/src/network.rs:654-692: stable sort by source, Dale's law sign
 * from the source kind, steps = max(1, round(delay/dt)), u16 overflow is an
 * error. */
int ne2o_synapse_csr(const ne2o_net *net, float dt_ms, ne2o_csr *out, char *err, size_t errlen) {
    uint32_t n = net->n;
    uint64_t e = net->ns;
    memset(out, 0, sizeof *out);
    out->n = n;
    out->e = e;
    out->src_ptr = XMALLOC(uint32_t, (uint64_t)n + 1);
    out->tgt = XMALLOC(uint32_t, e);
    out->w = XMALLOC(float, e);
    out->delay = XMALLOC(uint16_t, e);
    out->tau = XMALLOC(float, e);
    /* counting sort by src == stable sort_by_key */
    uint64_t *cnt = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
    for (uint64_t j = 0; j < e; ++j) cnt[net->s_src[j] + 1]++;
    for (uint32_t i = 0; i < n; ++i) cnt[i + 1] += cnt[i];
    for (uint32_t i = 0; i <= n; ++i) out->src_ptr[i] = (uint32_t)cnt[i];
    for (uint64_t j = 0; j < e; ++j) {
        uint32_t s = net->s_src[j];
        uint64_t pos = cnt[s]++;
        float w = fabsf(net->s_w[j]);
        out->tgt[pos] = net->s_tgt[j];
        out->w[pos] = net->kind[s] == NE2O_INH ? -w : w;
        out->tau[pos] = net->s_tau[j];
        float steps = roundf(net->s_delay[j] / dt_ms);
        if (steps < 1.0f) steps = 1.0f;
        if (!(steps <= 65535.0f)) {
            if (err)
                snprintf(err, errlen,
                         "synapse %u -> %u: delay %g ms = %g steps at dt %g ms exceeds the 65535-step ring",
                         s, net->s_tgt[j], (double)net->s_delay[j], (double)steps, (double)dt_ms);
            free(cnt);
            ne2o_csr_free(out);
            return -1;
        }
        out->delay[pos] = (uint16_t)steps;
    }
    free(cnt);
    return 0;
}

void ne2o_csr_free(ne2o_csr *c) {
    free(c->src_ptr); free(c->tgt); free(c->w); free(c->delay); free(c->tau);
    memset(c, 0, sizeof *c);
}

/* =============================================================== noise */
static inline uint64_t mix64(uint64_t h) {
    h ^= h >> 30;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 27;
    h *= 0x94D049BB133111EBull;
    h ^= h >> 31;
    return h;
}
static inline uint64_t noise_base(uint32_t i, uint64_t t, uint64_t seed) {
    return (uint64_t)i * 0x9E3779B97F4A7C15ull + t * 0xBF58476D1CE4E5B9ull + seed * 0x94D049BB133111EBull;
}
/* sim/src/state.rs:284-295 */
uint32_t ne2o_noise_hash(uint32_t i, uint64_t t, uint64_t seed) {
    return (uint32_t)(mix64(noise_base(i, t, seed)) >> 32);
}
/* state.rs:299-301 */
int ne2o_noise_fires(uint32_t i, uint64_t t, uint64_t seed, float p) {
    return (float)ne2o_noise_hash(i, t, seed) * 2.3283064e-10f < p;
}
/* Gaussian current noise (project definition, not in the reference): the
 * step part of the noise base, st = t*0xBF58476D1CE4E5B9 + seed*0x94D049BB133111EB
 * (noise_base without the neuron term), and the neuron index give one 32-bit
 * hash: x = i ^ lo32(st) through the lowbias32 mixer (x ^= x>>16;
 * x *= 0x7feb352d; x ^= x>>15; x *= 0x846ca68b; x ^= x>>16; C. Wellons'
 * hash-prospector), then x ^= hi32(st); x *= 0x9e3779b1; x ^= x>>16.  Its
 * four bytes are uniforms on [0, 255]; their sum S is Irwin-Hall(4) with
 * mean 510 and variance 4*(256^2-1)/12, so (S - 510) * sqrt(3)/256 has mean 0
 * and variance 1 - 2^-16.  Integer-exact on CPU and GPU; tails end at
 * +-510*sqrt(3)/256 = 3.45 sd. */
int64_t ne2o_gauss_numer(uint32_t i, uint64_t t, uint64_t seed) {
    const uint64_t st = t * 0xBF58476D1CE4E5B9ull + seed * 0x94D049BB133111EBull;
    uint32_t x = i ^ (uint32_t)st;
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    x ^= (uint32_t)(st >> 32);
    x *= 0x9e3779b1u;
    x ^= x >> 16;
    const int64_t s = (int64_t)(x & 0xff) + (int64_t)((x >> 8) & 0xff) + (int64_t)((x >> 16) & 0xff) +
                      (int64_t)(x >> 24);
    return s - 510;
}
float ne2o_gauss_scale(float sd) {
    return (float)((double)sd * 1.7320508075688772 / 256.0);
}

/* ===================================================== deterministic exp */
/* exp(x) in single precision by Cody-Waite reduction x = k*ln2 + r (fdlibm's
 * split of ln2: a 15-bit head 0x1.62e4p-1, so k*head is exact for |k| <= 150,
 * and a tail 0x1.7f7d1cp-20), the degree-7 Taylor polynomial of e^r
 * (coefficients 1/i! rounded to float) evaluated by Horner with fmaf, and
 * the scale 2^k applied as two exact powers of two, k = k1 + k2 with
 * k1 = k/2, so that neither factor underflows before the last rounding.
 * Every step is a rounded IEEE-754 single operation, so the device kernels
 * reproduce it bit-for-bit; it is within 2 ulp of the correctly rounded exp
 * on [-104, 88.8]. */
static float det_pow2f(int e) {
    const uint32_t bits = (uint32_t)(e + 127) << 23;
    float f;
    memcpy(&f, &bits, sizeof f);
    return f;
}

float ne2o_det_expf(float x) {
    if (x != x) return x;
    if (x > 88.8f) return INFINITY;
    if (x < -104.0f) return 0.0f;
    const float xl = x * 0x1.715476p+0f;
    const float k = rintf(xl);
    float r = fmaf(-k, 0x1.62e4p-1f, x);
    r = fmaf(-k, 0x1.7f7d1cp-20f, r);
    float p = 0x1.a01a02p-13f;
    p = fmaf(p, r, 0x1.6c16c2p-10f);
    p = fmaf(p, r, 0x1.111112p-7f);
    p = fmaf(p, r, 0x1.555556p-5f);
    p = fmaf(p, r, 0x1.555556p-3f);
    p = fmaf(p, r, 0.5f);
    p = fmaf(p, r, 1.0f);
    p = fmaf(p, r, 1.0f);
    const int ki = (int)k, k1 = ki / 2, k2 = ki - k1;
    p = p * det_pow2f(k1);
    return p * det_pow2f(k2);
}

struct expf_job {
    float (*f)(float);
    uint32_t lo_bits, hi_bits; /* ordered float keys, see expf_key */
    uint32_t stride, first, step;
    uint64_t bad, checked;     /* bad: mismatches, or the largest ulp distance in ulp_mode */
    int ulp_mode;
};
/* total order of float bit patterns as unsigned keys: -x < -0 < +0 < x */
static uint32_t expf_key(float x) {
    uint32_t b;
    memcpy(&b, &x, sizeof b);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
static float expf_unkey(uint32_t k) {
    uint32_t b = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    float x;
    memcpy(&x, &b, sizeof x);
    return x;
}
static void *expf_worker(void *arg) {
    struct expf_job *j = (struct expf_job *)arg;
    for (uint64_t k = (uint64_t)j->lo_bits + (uint64_t)j->first * j->stride; k <= j->hi_bits;
         k += (uint64_t)j->step * j->stride) {
        const float x = expf_unkey((uint32_t)k);
        const float a = j->f(x), b = ne2o_det_expf(x);
        j->checked++;
        if (j->ulp_mode) {
            /* distance in representable floats (both results are >= 0) */
            const uint32_t ka = expf_key(a), kb = expf_key(b);
            const uint64_t d = ka > kb ? ka - kb : kb - ka;
            if (d > j->bad) j->bad = d;
        } else if (memcmp(&a, &b, sizeof a) != 0) {
            j->bad++;
        }
    }
    return NULL;
}
static uint64_t expf_scan(float (*f)(float), float lo, float hi, uint32_t stride, uint32_t threads,
                          uint64_t *checked, int ulp_mode) {
    if (threads < 1) threads = 1;
    if (threads > 64) threads = 64;
    if (stride < 1) stride = 1;
    struct expf_job jobs[64];
    pthread_t th[64];
    for (uint32_t i = 0; i < threads; ++i) {
        jobs[i] = (struct expf_job){f, expf_key(lo), expf_key(hi), stride, i, threads, 0, 0, ulp_mode};
        pthread_create(&th[i], NULL, expf_worker, &jobs[i]);
    }
    uint64_t bad = 0, n = 0;
    for (uint32_t i = 0; i < threads; ++i) {
        pthread_join(th[i], NULL);
        if (ulp_mode) bad = jobs[i].bad > bad ? jobs[i].bad : bad;
        else bad += jobs[i].bad;
        n += jobs[i].checked;
    }
    if (checked) *checked = n;
    return bad;
}
uint64_t ne2o_expf_mismatches(float (*f)(float), float lo, float hi, uint32_t stride, uint32_t threads,
                              uint64_t *checked) {
    return expf_scan(f, lo, hi, stride, threads, checked, 0);
}
uint64_t ne2o_expf_max_ulp(float (*f)(float), float lo, float hi, uint32_t stride, uint32_t threads,
                           uint64_t *checked) {
    return expf_scan(f, lo, hi, stride, threads, checked, 1);
}
/* exp in double, rounded once to float: the correctly rounded exp except
 * where exp(x) falls within a double ulp of a float midpoint */
float ne2o_expf_ref(float x) {
    return (float)exp((double)x);
}

/* ============================================================ readout */
/* sim/src/readout.rs:144-188: L L^T = a, then L z = b, L^T w = z */
int ne2o_cholesky_solve(const double *a, const double *b, uint32_t n, double *w) {
    double *l = (double *)calloc((size_t)n * n, sizeof(double));
    double *z = (double *)calloc(n ? n : 1, sizeof(double));
    int ok = 1;
    for (uint32_t i = 0; i < n && ok; ++i)
        for (uint32_t j = 0; j <= i; ++j) {
            double sum = a[(size_t)i * n + j];
            for (uint32_t k = 0; k < j; ++k) sum -= l[(size_t)i * n + k] * l[(size_t)j * n + k];
            if (i == j) {
                if (sum <= 0.0) {
                    ok = 0;
                    break;
                }
                l[(size_t)i * n + j] = sqrt(sum);
            } else {
                l[(size_t)i * n + j] = sum / l[(size_t)j * n + j];
            }
        }
    if (ok) {
        for (uint32_t i = 0; i < n; ++i) {
            double sum = b[i];
            for (uint32_t k = 0; k < i; ++k) sum -= l[(size_t)i * n + k] * z[k];
            z[i] = sum / l[(size_t)i * n + i];
        }
        for (uint32_t i = n; i-- > 0;) {
            double sum = z[i];
            for (uint32_t k = i + 1; k < n; ++k) sum -= l[(size_t)k * n + i] * w[k];
            w[i] = sum / l[(size_t)i * n + i];
        }
    }
    free(l);
    free(z);
    return ok;
}

/* sim/src/readout.rs:103-141: a[i][j] (i <= j) and b accumulated row by row,
 * the bias column, symmetrised, lambda on the diagonal and taken off the
 * bias again; not positive definite: 1e-3 + lambda more on the diagonal,
 * then zeros */
void ne2o_fit_ridge(const float *x, uint32_t t, uint32_t f, const float *y, float lambda, double *w_out) {
    const uint32_t nf = f + 1;
    double *a = (double *)calloc((size_t)nf * nf, sizeof(double));
    double *b = (double *)calloc(nf, sizeof(double));
    for (uint32_t r = 0; r < t; ++r) {
        const float *row = x + (size_t)r * f;
        for (uint32_t i = 0; i < f; ++i) {
            const double xi = (double)row[i];
            b[i] += xi * (double)y[r];
            for (uint32_t j = i; j < f; ++j) a[(size_t)i * nf + j] += xi * (double)row[j];
        }
        b[f] += (double)y[r];
        for (uint32_t j = 0; j < f; ++j) a[(size_t)j * nf + f] += (double)row[j];
        a[(size_t)f * nf + f] += 1.0;
    }
    for (uint32_t i = 0; i < nf; ++i) {
        for (uint32_t j = 0; j < i; ++j) a[(size_t)i * nf + j] = a[(size_t)j * nf + i];
        a[(size_t)i * nf + i] += (double)lambda;
    }
    a[(size_t)f * nf + f] -= (double)lambda;
    if (!ne2o_cholesky_solve(a, b, nf, w_out)) {
        for (uint32_t i = 0; i < nf; ++i) a[(size_t)i * nf + i] += 1e-3 + (double)lambda;
        if (!ne2o_cholesky_solve(a, b, nf, w_out))
            for (uint32_t i = 0; i < nf; ++i) w_out[i] = 0.0;
    }
    free(a);
    free(b);
}

/* sim/src/readout.rs:190-252: centre the columns, Gram G = Xc Xc^T + lambda I
 * (four accumulators per dot as the reference sums), one Cholesky solve per
 * class against the centred one-hot targets, w = Xc^T a, bias = ybar - w.mu */
void ne2o_fit_ridge_multi(const float *x, uint32_t t, uint32_t f, const uint32_t *labels, uint32_t k, double lambda,
                          double *w_out) {
    double *mu = (double *)calloc(f ? f : 1, sizeof(double));
    double *xc = (double *)malloc(sizeof(double) * ((size_t)t * f + 1));
    double *ybar = (double *)calloc(k ? k : 1, sizeof(double));
    double *g = (double *)malloc(sizeof(double) * ((size_t)t * t + 1));
    double *yc = (double *)malloc(sizeof(double) * (t + 1));
    double *a = (double *)malloc(sizeof(double) * (t + 1));
    for (uint32_t r = 0; r < t; ++r)
        for (uint32_t c = 0; c < f; ++c) mu[c] += (double)x[(size_t)r * f + c];
    for (uint32_t c = 0; c < f; ++c) mu[c] /= (double)t;
    for (size_t i = 0; i < (size_t)t * f; ++i) xc[i] = (double)x[i] - mu[i % f];
    for (uint32_t r = 0; r < t; ++r) ybar[labels[r]] += 1.0 / (double)t;
    for (uint32_t i = 0; i < t; ++i) {
        const double *ri = xc + (size_t)i * f;
        for (uint32_t j = 0; j <= i; ++j) {
            const double *rj = xc + (size_t)j * f;
            double acc[4] = {0.0, 0.0, 0.0, 0.0};
            const uint32_t f4 = f / 4 * 4;
            for (uint32_t c = 0; c < f4; c += 4)
                for (int q = 0; q < 4; ++q) acc[q] += ri[c + q] * rj[c + q];
            double s = 0.0;
            for (uint32_t c = f4; c < f; ++c) s += ri[c] * rj[c];
            s += ((acc[0] + acc[1]) + acc[2]) + acc[3];
            g[(size_t)i * t + j] = s;
            g[(size_t)j * t + i] = s;
        }
        g[(size_t)i * t + i] += lambda;
    }
    for (uint32_t c = 0; c < k; ++c) {
        for (uint32_t r = 0; r < t; ++r) yc[r] = (labels[r] == c ? 1.0 : 0.0) - ybar[c];
        if (!ne2o_cholesky_solve(g, yc, t, a))
            for (uint32_t r = 0; r < t; ++r) a[r] = 0.0;
        double *w = w_out + (size_t)c * (f + 1);
        for (uint32_t q = 0; q <= f; ++q) w[q] = 0.0;
        for (uint32_t r = 0; r < t; ++r)
            for (uint32_t q = 0; q < f; ++q) w[q] += a[r] * xc[(size_t)r * f + q];
        double dot = 0.0;
        for (uint32_t q = 0; q < f; ++q) dot += w[q] * mu[q];
        w[f] = ybar[c] - dot;
    }
    free(mu);
    free(xc);
    free(ybar);
    free(g);
    free(yc);
    free(a);
}

/* ================================================================ sim */
/* sim/src/state.rs:35-49 defaults, net-format/src/lib.rs:26-39 */
void ne2o_cfg_default(ne2o_cfg *c) {
    c->dt_ms = 0.1f;
    c->synapse_tau_ms = 2.0f;
    c->readout_tau_ms = 2.0f;
    c->noise_rate_hz = 0.0f;
    c->noise_kick_mv = 20.0f;
    c->seed = 1;
    c->record_spikes = 0;
    c->spike_record_steps = 512;
    c->int_weights = 0;
    c->gauss_sd = 0.0f;
    c->exp_mode = 0;
}

typedef struct {
    float *series;
    uint64_t len;
    uint64_t start;
    int looped;
} stim_series;

struct ne2o_sim {
    uint32_t n;
    ne2o_cfg cfg;
    /* params: model registry id and padded rows (state.rs:58-74) */
    uint8_t *model;
    float *p;  /* n * NE2O_PMAX */
    float *x0; /* n * 2 */
    ne2o_csr csr;
    int32_t *wq; /* fixed-point weights lrintf(w*4096) */
    uint32_t d;
    /* custom-tau synapses (state.rs:231-275) */
    uint32_t *xsyn_map;
    uint32_t nx;
    float *xdecay, *xw, *xsyn;
    uint32_t *xt_ptr, *xt_idx;
    uint32_t **xring; uint32_t *xring_len, *xring_cap;
    /* stimulus (stim.rs:9-58, 102-127) */
    uint32_t ninputs;
    uint32_t *st_ptr, *st_in;
    float *st_w;
    float *constants;
    stim_series *series;
    /* state */
    float *x, *s, *trace, *ext;
    float *ring;
    int32_t *iring;
    uint64_t *spike_bits;
    uint32_t *spike_counts;
    uint32_t rec_rows;
    uint64_t *pn_total;
    uint32_t words;
    uint64_t t, spikes_total;
    uint32_t *spiked;
    uint32_t nspiked;
    /* editor watches (cpu.rs:63-95): per-step state of watched neurons,
     * the last NE2O_V_HIST_CAP samples kept (a ring, oldest at hist_head),
     * and per grid group the last spike step of every texel */
    uint32_t nwatch;
    uint32_t *v_watch;
    float *x_hist;  /* [2][nwatch][NE2O_V_HIST_CAP] */
    uint32_t hist_head, hist_len;
    uint32_t ngw;
    uint32_t *gw_ptr;     /* [ngw+1] member ranges */
    uint32_t *gw_members; /* texel order */
    int32_t *gw_map;      /* [ngw][n] texel of neuron, -1 if none */
    uint32_t *gw_ls;      /* [gw_ptr[ngw]] last spike step, UINT32_MAX never */
};

static void sim_free_parts(ne2o_sim *s) {
    free(s->model); free(s->p); free(s->x0); ne2o_csr_free(&s->csr); free(s->wq);
    free(s->xsyn_map); free(s->xdecay); free(s->xw); free(s->xsyn); free(s->xt_ptr); free(s->xt_idx);
    if (s->xring) for (uint32_t k = 0; k < s->d; ++k) free(s->xring[k]);
    free(s->xring); free(s->xring_len); free(s->xring_cap);
    free(s->st_ptr); free(s->st_in); free(s->st_w); free(s->constants);
    if (s->series) for (uint32_t k = 0; k < s->ninputs; ++k) free(s->series[k].series);
    free(s->series);
    free(s->x); free(s->s); free(s->trace); free(s->ext); free(s->ring); free(s->iring);
    free(s->spike_bits); free(s->spike_counts); free(s->pn_total); free(s->spiked);
    free(s->v_watch); free(s->x_hist); free(s->gw_ptr); free(s->gw_members); free(s->gw_map); free(s->gw_ls);
}

void ne2o_sim_free(ne2o_sim *s) {
    if (!s) return;
    sim_free_parts(s);
    free(s);
}

/* model inits: izh.rs:175-178 (v=-65, u=b*v); adex.rs:149-152 (v=EL, w=0) */
static void model_init(int model, const float *p, float *x) {
    if (model == NE2O_MODEL_ADEX) { x[0] = p[2]; x[1] = 0.0f; }
    else { x[0] = -65.0f; x[1] = p[1] * x[0]; }
}

/* sim/src/cpu.rs:100-150 (CpuSim::with_params) */
ne2o_sim *ne2o_sim_new(const ne2o_net *net, const ne2o_cfg *cfg, char *err, size_t errlen) {
    ne2o_sim *s = (ne2o_sim *)calloc(1, sizeof(ne2o_sim));
    if (!s) abort();
    s->n = net->n;
    s->cfg = *cfg;
    uint32_t n = s->n;
    if (ne2o_synapse_csr(net, cfg->dt_ms, &s->csr, err, errlen) != 0) {
        free(s);
        return NULL;
    }
    s->model = XMALLOC(uint8_t, n);
    s->p = XMALLOC(float, (uint64_t)n * NE2O_PMAX);
    s->x0 = XMALLOC(float, (uint64_t)n * 2);
    memcpy(s->model, net->model, n);
    memcpy(s->p, net->params, sizeof(float) * NE2O_PMAX * (size_t)n);
    for (uint32_t i = 0; i < n; ++i) model_init(s->model[i], s->p + (size_t)i * NE2O_PMAX, s->x0 + 2 * (size_t)i);
    /* ring_depth, state.rs:221-224 */
    uint32_t maxd = 1;
    for (uint64_t j = 0; j < s->csr.e; ++j) if (s->csr.delay[j] > maxd) maxd = s->csr.delay[j];
    if (s->csr.e == 0) maxd = 1;
    s->d = maxd + 1 < 2 ? 2 : maxd + 1;
    /* fixed-point weights, kernels.rs:60-61 rt_put */
    s->wq = XMALLOC(int32_t, s->csr.e);
    for (uint64_t j = 0; j < s->csr.e; ++j) s->wq[j] = (int32_t)lrintf(s->csr.w[j] * 4096.0f);
    /* XSyn::build, state.rs:245-274 */
    s->xsyn_map = XMALLOC(uint32_t, s->csr.e);
    uint32_t nx = 0;
    for (uint64_t j = 0; j < s->csr.e; ++j) s->xsyn_map[j] = (s->csr.tau[j] > 0.0f) ? nx++ : 0xFFFFFFFFu;
    s->nx = nx;
    s->xdecay = XMALLOC(float, nx);
    s->xw = XMALLOC(float, nx);
    s->xsyn = (float *)calloc(nx ? nx : 1, sizeof(float));
    s->xt_ptr = (uint32_t *)calloc((size_t)n + 1, sizeof(uint32_t));
    s->xt_idx = XMALLOC(uint32_t, nx);
    for (uint64_t j = 0; j < s->csr.e; ++j) {
        uint32_t k = s->xsyn_map[j];
        if (k == 0xFFFFFFFFu) continue;
        float tau = s->csr.tau[j] > 1e-6f ? s->csr.tau[j] : 1e-6f;
        s->xdecay[k] = expf(-cfg->dt_ms / tau);
        /* the CPU integrates w directly; in fixed-point mode the arrival is
         * rt_get(rt_put(w)) as the CUDA xsyn path (kernels.rs:198, 213) */
        s->xw[k] = cfg->int_weights ? (float)s->wq[j] / 4096.0f : s->csr.w[j];
        s->xt_ptr[s->csr.tgt[j] + 1]++;
    }
    for (uint32_t i = 0; i < n; ++i) s->xt_ptr[i + 1] += s->xt_ptr[i];
    {
        uint32_t *fill = XMALLOC(uint32_t, (uint64_t)n + 1);
        memcpy(fill, s->xt_ptr, sizeof(uint32_t) * ((size_t)n + 1));
        for (uint64_t j = 0; j < s->csr.e; ++j) {
            uint32_t k = s->xsyn_map[j];
            if (k != 0xFFFFFFFFu) s->xt_idx[fill[s->csr.tgt[j]]++] = k;
        }
        free(fill);
    }
    s->xring = (uint32_t **)calloc(s->d, sizeof(uint32_t *));
    s->xring_len = (uint32_t *)calloc(s->d, sizeof(uint32_t));
    s->xring_cap = (uint32_t *)calloc(s->d, sizeof(uint32_t));
    /* StimMap::from_network, stim.rs:26-48 */
    s->ninputs = net->ninputs;
    s->st_ptr = (uint32_t *)calloc((size_t)n + 1, sizeof(uint32_t));
    for (uint32_t k = 0; k < net->ninputs; ++k)
        for (uint32_t j = net->in_ptr[k]; j < net->in_ptr[k + 1]; ++j)
            if (net->in_tgt[j] < n) s->st_ptr[net->in_tgt[j] + 1]++;
    for (uint32_t i = 0; i < n; ++i) s->st_ptr[i + 1] += s->st_ptr[i];
    uint32_t ne = s->st_ptr[n];
    s->st_in = XMALLOC(uint32_t, ne);
    s->st_w = XMALLOC(float, ne);
    {
        uint32_t *fill = XMALLOC(uint32_t, (uint64_t)n + 1);
        memcpy(fill, s->st_ptr, sizeof(uint32_t) * ((size_t)n + 1));
        for (uint32_t k = 0; k < net->ninputs; ++k)
            for (uint32_t j = net->in_ptr[k]; j < net->in_ptr[k + 1]; ++j) {
                uint32_t tg = net->in_tgt[j];
                if (tg >= n) continue;
                uint32_t pos = fill[tg]++;
                s->st_in[pos] = k;
                s->st_w[pos] = net->in_w[j];
            }
        free(fill);
    }
    s->constants = (float *)calloc(s->ninputs ? s->ninputs : 1, sizeof(float));
    s->series = (stim_series *)calloc(s->ninputs ? s->ninputs : 1, sizeof(stim_series));
    /* state */
    s->x = XMALLOC(float, (uint64_t)n * 2);
    s->s = XMALLOC(float, n);
    s->trace = XMALLOC(float, n);
    s->ext = (float *)calloc(n ? n : 1, sizeof(float));
    if (cfg->int_weights) s->iring = XMALLOC(int32_t, (uint64_t)s->d * n);
    else s->ring = XMALLOC(float, (uint64_t)s->d * n);
    s->words = (n + 63) / 64;
    s->rec_rows = cfg->record_spikes ? (cfg->spike_record_steps < 2 ? 2 : cfg->spike_record_steps) : 0;
    s->spike_bits = XMALLOC(uint64_t, (uint64_t)s->rec_rows * s->words);
    s->spike_counts = XMALLOC(uint32_t, s->rec_rows);
    s->pn_total = XMALLOC(uint64_t, n);
    s->spiked = XMALLOC(uint32_t, n);
    ne2o_sim_reset_state(s);
    return s;
}

/* cpu.rs:158-183 */
void ne2o_sim_reset_state(ne2o_sim *s) {
    uint32_t n = s->n;
    memcpy(s->x, s->x0, sizeof(float) * 2 * (size_t)n);
    memset(s->s, 0, sizeof(float) * n);
    memset(s->trace, 0, sizeof(float) * n);
    if (s->ring) memset(s->ring, 0, sizeof(float) * (size_t)s->d * n);
    if (s->iring) memset(s->iring, 0, sizeof(int32_t) * (size_t)s->d * n);
    if (s->nx) memset(s->xsyn, 0, sizeof(float) * s->nx);
    for (uint32_t k = 0; k < s->d; ++k) s->xring_len[k] = 0;
    memset(s->spike_bits, 0, sizeof(uint64_t) * (size_t)s->rec_rows * s->words);
    memset(s->spike_counts, 0, sizeof(uint32_t) * s->rec_rows);
    memset(s->pn_total, 0, sizeof(uint64_t) * n);
    s->hist_head = s->hist_len = 0; /* cpu.rs:176-183 */
    if (s->ngw) for (uint32_t k = 0; k < s->gw_ptr[s->ngw]; ++k) s->gw_ls[k] = 0xFFFFFFFFu;
    s->t = 0;
    s->spikes_total = 0;
    s->nspiked = 0;
}

/* stim.rs:102-115 (Stimulus::value) */
float ne2o_sim_stim_value(const ne2o_sim *s, uint32_t k, uint64_t t) {
    if (k >= s->ninputs) return 0.0f;
    const stim_series *se = &s->series[k];
    if (se->len > 0) {
        if (se->looped) {
            int64_t d = (int64_t)t - (int64_t)se->start;
            int64_t m = (int64_t)se->len;
            int64_t idx = ((d % m) + m) % m;
            return se->series[idx];
        }
        uint64_t idx = t - se->start; /* wrapping_sub */
        return idx < se->len ? se->series[idx] : 0.0f;
    }
    return s->constants[k];
}

/* Izhikevich step, sim/src/model/izh.rs:184-192 */
static inline int izh_step(const float *p, float *x, float input, float dt) {
    if (x[0] >= 30.0f) {
        x[0] = p[2];
        x[1] += p[3];
    }
    x[0] += dt * (0.04f * x[0] * x[0] + 5.0f * x[0] + 140.0f - x[1] + input);
    x[1] += dt * p[0] * (p[1] * x[0] - x[1]);
    return x[0] >= 30.0f;
}

/* AdEx step, sim/src/model/adex.rs:163-176 */
static inline int adex_step(const float *p, float *x, float input, float dt, int exp_mode) {
    if (x[0] >= p[9]) {
        x[0] = p[8];
        x[1] += p[7];
    }
    float arg = fminf((x[0] - p[3]) / p[4], 10.0f);
    float ex = exp_mode ? ne2o_det_expf(arg) : expf(arg);
    x[0] += dt * (-p[1] * (x[0] - p[2]) + p[1] * p[4] * ex - x[1] + input) / p[0];
    x[1] += dt * (p[5] * (x[0] - p[2]) - x[1]) / p[6];
    int spiked = x[0] >= p[9];
    if (x[0] > p[9]) x[0] = p[9];
    return spiked;
}

/* One dt step: sim/src/cpu.rs:192-306 (CpuSim::step) */
void ne2o_sim_step(ne2o_sim *s) {
    const uint32_t n = s->n;
    const float dt = s->cfg.dt_ms;
    const uint64_t t = s->t;
    const uint32_t slot = (uint32_t)(t % s->d);
    const float p_kick = s->cfg.noise_rate_hz * dt / 1000.0f;
    const float kick = s->cfg.noise_kick_mv != 0.0f ? s->cfg.noise_kick_mv / dt : 0.0f;
    const float tau_s = s->cfg.synapse_tau_ms > 1e-6f ? s->cfg.synapse_tau_ms : 1e-6f;
    const float tau_t = s->cfg.readout_tau_ms > 1e-6f ? s->cfg.readout_tau_ms : 1e-6f;
    const float decay_s = expf(-dt / tau_s);
    const float decay_t = expf(-dt / tau_t);
    const float gk = s->cfg.gauss_sd != 0.0f ? ne2o_gauss_scale(s->cfg.gauss_sd) : 0.0f;

    /* custom-tau arrivals (cpu.rs:206-210) */
    for (uint32_t a = 0; a < s->xring_len[slot]; ++a) {
        uint32_t k = s->xring[slot][a];
        s->xsyn[k] += s->xw[k];
    }
    s->xring_len[slot] = 0;

    const size_t slot_base = (size_t)slot * n;
    s->nspiked = 0;
    for (uint32_t i = 0; i < n; ++i) {
        float arr;
        if (s->iring) {
            arr = (float)s->iring[slot_base + i] / 4096.0f; /* kernels.rs:60 rt_get */
            s->iring[slot_base + i] = 0;
        } else {
            arr = s->ring[slot_base + i];
            s->ring[slot_base + i] = 0.0f;
        }
        s->s[i] += arr;
        float input = s->s[i] + s->ext[i];
        for (uint32_t j = s->xt_ptr[i]; j < s->xt_ptr[i + 1]; ++j) {
            uint32_t k = s->xt_idx[j];
            input += s->xsyn[k];
            s->xsyn[k] *= s->xdecay[k];
        }
        for (uint32_t j = s->st_ptr[i]; j < s->st_ptr[i + 1]; ++j)
            input += s->st_w[j] * ne2o_sim_stim_value(s, s->st_in[j], t);
        const float *p = s->p + (size_t)i * NE2O_PMAX;
        const int model = s->model[i];
        const float gain = model == NE2O_MODEL_ADEX ? p[0] : 1.0f; /* model/mod.rs:104-106, adex.rs:189-191 */
        if (p_kick > 0.0f && ne2o_noise_fires(i, t, s->cfg.seed, p_kick)) input += kick * gain;
        if (gk != 0.0f) input += (float)ne2o_gauss_numer(i, t, s->cfg.seed) * (gk * gain);
        float *x = s->x + 2 * (size_t)i;
        int sp = model == NE2O_MODEL_ADEX ? adex_step(p, x, input, dt, s->cfg.exp_mode)
                                          : izh_step(p, x, input, dt);
        if (sp) {
            s->spiked[s->nspiked++] = i;
            s->trace[i] = 1.0f;
        } else {
            s->trace[i] *= decay_t;
        }
        s->s[i] *= decay_s;
    }

    /* propagation through the source-sorted CSR (cpu.rs:264-278) */
    for (uint32_t a = 0; a < s->nspiked; ++a) {
        uint32_t i = s->spiked[a];
        for (uint32_t j = s->csr.src_ptr[i]; j < s->csr.src_ptr[i + 1]; ++j) {
            uint32_t dst = (uint32_t)((t + s->csr.delay[j]) % s->d);
            uint32_t xid = s->xsyn_map[j];
            if (xid != 0xFFFFFFFFu) {
                if (s->xring_len[dst] == s->xring_cap[dst]) {
                    s->xring_cap[dst] = s->xring_cap[dst] ? 2 * s->xring_cap[dst] : 16;
                    s->xring[dst] = (uint32_t *)xrealloc(s->xring[dst], sizeof(uint32_t) * s->xring_cap[dst]);
                }
                s->xring[dst][s->xring_len[dst]++] = xid;
            } else if (s->iring) {
                /* int atomicAdd wraps two's complement (kernels.rs:200) */
                int32_t *cell = &s->iring[(size_t)dst * n + s->csr.tgt[j]];
                *cell = (int32_t)((uint32_t)*cell + (uint32_t)s->wq[j]);
            } else {
                s->ring[(size_t)dst * n + s->csr.tgt[j]] += s->csr.w[j];
            }
        }
    }

    /* spike record (cpu.rs:280-292) */
    if (s->rec_rows) {
        uint32_t row = (uint32_t)(t % s->rec_rows);
        s->spike_counts[row] = s->nspiked;
        uint64_t *bits = s->spike_bits + (size_t)row * s->words;
        memset(bits, 0, sizeof(uint64_t) * s->words);
        for (uint32_t a = 0; a < s->nspiked; ++a) bits[s->spiked[a] / 64] |= 1ull << (s->spiked[a] % 64);
    }
    for (uint32_t a = 0; a < s->nspiked; ++a) s->pn_total[s->spiked[a]] += 1;
    /* grid watches (cpu.rs:293-304) */
    if (s->ngw) {
        const uint32_t t32 = (uint32_t)(t < 0xFFFFFFFEull ? t : 0xFFFFFFFEull);
        for (uint32_t a = 0; a < s->nspiked; ++a)
            for (uint32_t g = 0; g < s->ngw; ++g) {
                const int32_t k = s->gw_map[(size_t)g * n + s->spiked[a]];
                if (k >= 0) s->gw_ls[s->gw_ptr[g] + (uint32_t)k] = t32;
            }
    }
    s->spikes_total += s->nspiked;
    s->t += 1;
}

/* v-watch recording after each step (cpu.rs:308-326): state slot 0/1 of
 * every watched id (0 for ids beyond n), capped at NE2O_V_HIST_CAP */
static void record_watches(ne2o_sim *s) {
    if (!s->nwatch) return;
    uint32_t pos;
    if (s->hist_len < NE2O_V_HIST_CAP) {
        pos = (s->hist_head + s->hist_len) % NE2O_V_HIST_CAP;
        s->hist_len++;
    } else {
        pos = s->hist_head;
        s->hist_head = (s->hist_head + 1) % NE2O_V_HIST_CAP;
    }
    for (uint32_t slot = 0; slot < 2; ++slot)
        for (uint32_t k = 0; k < s->nwatch; ++k) {
            const uint32_t i = s->v_watch[k];
            s->x_hist[((size_t)slot * s->nwatch + k) * NE2O_V_HIST_CAP + pos] =
                i < s->n ? s->x[2 * (size_t)i + slot] : 0.0f;
        }
}

/* cpu.rs:330-338: a new list resets the history; the same list is a no-op */
void ne2o_sim_set_v_watch(ne2o_sim *s, const uint32_t *ids, uint32_t count) {
    if (count == s->nwatch && (count == 0 || memcmp(ids, s->v_watch, 4 * (size_t)count) == 0)) return;
    free(s->v_watch);
    free(s->x_hist);
    s->nwatch = count;
    s->v_watch = XMALLOC(uint32_t, count ? count : 1);
    if (count) memcpy(s->v_watch, ids, 4 * (size_t)count);
    s->x_hist = XMALLOC(float, 2 * (size_t)(count ? count : 1) * NE2O_V_HIST_CAP);
    s->hist_head = s->hist_len = 0;
}

/* cpu.rs:350-357 drain_state for both slots: out[slot][watch][c], oldest
 * first; returns c and empties the history */
uint32_t ne2o_sim_drain_watch(ne2o_sim *s, float *out) {
    const uint32_t c = s->hist_len;
    for (uint32_t slot = 0; slot < 2; ++slot)
        for (uint32_t k = 0; k < s->nwatch; ++k)
            for (uint32_t j = 0; j < c; ++j)
                out[((size_t)slot * s->nwatch + k) * c + j] =
                    s->x_hist[((size_t)slot * s->nwatch + k) * NE2O_V_HIST_CAP + (s->hist_head + j) % NE2O_V_HIST_CAP];
    s->hist_head = s->hist_len = 0;
    return c;
}

/* cpu.rs:361-387: member lists in texel order; the same lists are a no-op */
void ne2o_sim_set_grid_watches(ne2o_sim *s, const uint32_t *members, const uint32_t *group_ptr, uint32_t ngroups) {
    if (ngroups == s->ngw && (ngroups == 0 || (memcmp(group_ptr, s->gw_ptr, 4 * ((size_t)ngroups + 1)) == 0 &&
                                               memcmp(members, s->gw_members, 4 * (size_t)group_ptr[ngroups]) == 0)))
        return;
    free(s->gw_ptr); free(s->gw_members); free(s->gw_map); free(s->gw_ls);
    const uint32_t total = ngroups ? group_ptr[ngroups] : 0;
    s->ngw = ngroups;
    s->gw_ptr = XMALLOC(uint32_t, (size_t)ngroups + 1);
    memcpy(s->gw_ptr, group_ptr, 4 * ((size_t)ngroups + 1));
    s->gw_members = XMALLOC(uint32_t, total ? total : 1);
    if (total) memcpy(s->gw_members, members, 4 * (size_t)total);
    s->gw_map = XMALLOC(int32_t, (size_t)(ngroups ? ngroups : 1) * (s->n ? s->n : 1));
    for (size_t j = 0; j < (size_t)ngroups * s->n; ++j) s->gw_map[j] = -1;
    for (uint32_t g = 0; g < ngroups; ++g)
        for (uint32_t k = group_ptr[g]; k < group_ptr[g + 1]; ++k)
            if (members[k] < s->n) s->gw_map[(size_t)g * s->n + members[k]] = (int32_t)(k - group_ptr[g]);
    s->gw_ls = XMALLOC(uint32_t, total ? total : 1);
    for (uint32_t k = 0; k < total; ++k) s->gw_ls[k] = 0xFFFFFFFFu;
}

/* cpu.rs:391-407: exp(-(t - last) * dt / tau) per texel, 0 if never */
void ne2o_sim_grid_traces(const ne2o_sim *s, float tau_ms, float *out) {
    const float k = s->cfg.dt_ms / (tau_ms > 1e-6f ? tau_ms : 1e-6f);
    const uint32_t total = s->ngw ? s->gw_ptr[s->ngw] : 0;
    for (uint32_t j = 0; j < total; ++j) {
        const uint32_t l = s->gw_ls[j];
        out[j] = l == 0xFFFFFFFFu ? 0.0f : expf(-(float)(s->t > l ? s->t - l : 0) * k);
    }
}

/* cpu.rs:308-326 */
void ne2o_sim_run_steps(ne2o_sim *s, uint64_t steps) {
    for (uint64_t k = 0; k < steps; ++k) {
        ne2o_sim_step(s);
        record_watches(s);
    }
}

uint64_t ne2o_sim_t(const ne2o_sim *s) { return s->t; }
uint32_t ne2o_sim_n(const ne2o_sim *s) { return s->n; }
uint32_t ne2o_sim_ring_depth(const ne2o_sim *s) { return s->d; }
uint64_t ne2o_sim_spikes_total(const ne2o_sim *s) { return s->spikes_total; }

/* cpu.rs:389-396 */
double ne2o_sim_mean_rate_hz(const ne2o_sim *s) {
    if (s->t == 0) return 0.0;
    double n = s->n ? (double)s->n : 1.0;
    return (double)s->spikes_total / n / ((double)s->t * (double)s->cfg.dt_ms / 1000.0);
}

/* cpu.rs:345-352 */
int ne2o_sim_state(const ne2o_sim *s, uint32_t slot, float *out) {
    if (slot >= 2) return -1;
    for (uint32_t i = 0; i < s->n; ++i) out[i] = s->x[2 * (size_t)i + slot];
    return 0;
}
void ne2o_sim_syn_current(const ne2o_sim *s, float *out) { memcpy(out, s->s, sizeof(float) * s->n); }
void ne2o_sim_trace(const ne2o_sim *s, float *out) { memcpy(out, s->trace, sizeof(float) * s->n); }
void ne2o_sim_pn_total(const ne2o_sim *s, uint64_t *out) { memcpy(out, s->pn_total, sizeof(uint64_t) * s->n); }

/* cpu.rs:399-411 */
uint32_t ne2o_sim_spike_row(const ne2o_sim *s, uint32_t back, uint64_t *out) {
    if (!s->rec_rows || s->t == 0 || back >= s->t || back >= s->rec_rows) return 0;
    uint64_t t = s->t - 1 - back;
    uint32_t row = (uint32_t)(t % s->rec_rows);
    memcpy(out, s->spike_bits + (size_t)row * s->words, sizeof(uint64_t) * s->words);
    return s->words;
}

/* cpu.rs:424-458 */
int ne2o_sim_spike_counts(const ne2o_sim *s, uint64_t rows, uint32_t *out, char *err, size_t errlen) {
    memset(out, 0, sizeof(uint32_t) * s->n);
    if (!s->rec_rows || s->t == 0) return 0;
    if (rows >= s->t) {
        for (uint32_t i = 0; i < s->n; ++i) out[i] = s->pn_total[i] > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)s->pn_total[i];
        return 0;
    }
    if (rows > s->rec_rows) {
        if (err) snprintf(err, errlen, "spike_counts window %llu exceeds the recorded %u steps",
                          (unsigned long long)rows, s->rec_rows);
        return -1;
    }
    for (uint64_t back = 0; back < rows; ++back) {
        uint64_t t = s->t - 1 - back;
        const uint64_t *row = s->spike_bits + (size_t)(t % s->rec_rows) * s->words;
        for (uint32_t wi = 0; wi < s->words; ++wi) {
            uint64_t w = row[wi];
            while (w) {
                int b = __builtin_ctzll(w);
                w &= w - 1;
                uint32_t i = wi * 64 + (uint32_t)b;
                if (i < s->n) out[i]++;
            }
        }
    }
    return 0;
}

uint32_t ne2o_sim_last_step_spikes(const ne2o_sim *s, uint32_t *out) {
    memcpy(out, s->spiked, sizeof(uint32_t) * s->nspiked);
    return s->nspiked;
}

/* cpu.rs:506-508 */
void ne2o_sim_set_external(ne2o_sim *s, uint32_t i, float amps) {
    if (i < s->n) s->ext[i] = amps;
}
/* cpu.rs:498-500 */
void ne2o_sim_set_input_constant(ne2o_sim *s, uint32_t k, float v) {
    if (k < s->ninputs) s->constants[k] = v;
}
/* stim.rs:71-85 (play: per-input playhead at the current step) */
void ne2o_sim_play_input(ne2o_sim *s, uint32_t k, const float *series, uint64_t len) {
    if (k >= s->ninputs) return;
    stim_series *se = &s->series[k];
    free(se->series);
    se->series = XMALLOC(float, len);
    memcpy(se->series, series, sizeof(float) * (size_t)len);
    se->len = len;
    se->start = s->t;
    se->looped = 0;
}
/* stim.rs:90-96 */
void ne2o_sim_loop_input(ne2o_sim *s, uint32_t k, const float *series, uint64_t len) {
    ne2o_sim_play_input(s, k, series, len);
    if (k < s->ninputs) s->series[k].looped = 1;
}
/* sim/src/lib.rs:183, cpu.rs:597-600 */
void ne2o_sim_set_noise(ne2o_sim *s, float rate_hz, float kick_mv) {
    s->cfg.noise_rate_hz = rate_hz;
    s->cfg.noise_kick_mv = kick_mv;
}

/* sim/tests/cpu_ref.rs:230-243: FNV-1a over `rows` record rows (newest
 * first), then the bits of every v */
uint64_t ne2o_sim_fingerprint(const ne2o_sim *s, uint32_t rows) {
    uint64_t h = 0xcbf29ce484222325ull;
    uint64_t *row = XMALLOC(uint64_t, s->words);
    for (uint32_t back = 0; back < rows; ++back) {
        uint32_t nw = ne2o_sim_spike_row(s, back, row);
        for (uint32_t k = 0; k < nw; ++k) { h ^= row[k]; h *= 0x00000100000001B3ull; }
    }
    free(row);
    for (uint32_t i = 0; i < s->n; ++i) {
        uint32_t b;
        memcpy(&b, &s->x[2 * (size_t)i], 4);
        h ^= (uint64_t)b;
        h *= 0x00000100000001B3ull;
    }
    return h;
}

/* ---------------------------------------------------- flattened views */
uint32_t ne2o_net_n(const ne2o_net *net) { return net->n; }
uint64_t ne2o_net_ns(const ne2o_net *net) { return net->ns; }
void ne2o_net_models(const ne2o_net *net, uint8_t *model, float *params_padded10) {
    memcpy(model, net->model, net->n);
    memcpy(params_padded10, net->params, sizeof(float) * NE2O_PMAX * (size_t)net->n);
}
void ne2o_net_kinds(const ne2o_net *net, uint8_t *kind) { memcpy(kind, net->kind, net->n); }
uint32_t ne2o_net_ninputs(const ne2o_net *net) { return net->ninputs; }
uint32_t ne2o_net_input_entries(const ne2o_net *net) { return net->nin_entries; }
void ne2o_net_inputs(const ne2o_net *net, uint32_t *in_ptr, uint32_t *in_tgt, float *in_w) {
    memcpy(in_ptr, net->in_ptr, sizeof(uint32_t) * ((size_t)net->ninputs + 1));
    memcpy(in_tgt, net->in_tgt, sizeof(uint32_t) * net->nin_entries);
    memcpy(in_w, net->in_w, sizeof(float) * net->nin_entries);
}
void ne2o_net_synapses(const ne2o_net *net, uint32_t *src, uint32_t *tgt, float *w, float *delay_ms,
                       float *tau_ms) {
    size_t e = (size_t)net->ns;
    memcpy(src, net->s_src, 4 * e);
    memcpy(tgt, net->s_tgt, 4 * e);
    memcpy(w, net->s_w, 4 * e);
    memcpy(delay_ms, net->s_delay, 4 * e);
    memcpy(tau_ms, net->s_tau, 4 * e);
}
void ne2o_net_positions(const ne2o_net *net, float *pos) { memcpy(pos, net->pos, sizeof(float) * 3 * (size_t)net->n); }
