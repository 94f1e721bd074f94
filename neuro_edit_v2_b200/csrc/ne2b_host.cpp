// ne2b_host.cpp — host-side network building for the C ABI: the source-major
// CSR build of Network::synapse_csr, the workload generators, and the host
// copy of the deterministic exp.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <new>
#include <thread>
#include <vector>

#include "../../include/ne2b.h"
#include "ne2b_net.h"

namespace ne2b {
ne2b_status set_error(ne2b_status st, const char *fmt, ...);
}
using ne2b::set_error;

namespace {

constexpr uint32_t kStride = 10;
// net-format/src/network.rs:53-54
const float kIzhRS[4] = {0.02f, 0.2f, -65.0f, 8.0f};
const float kIzhFS[4] = {0.1f, 0.2f, -65.0f, 2.0f};
// sim/src/model/adex.rs:22-26
const float kAdexTonic[10] = {281.0f, 30.0f, -70.6f, -50.4f, 2.0f, 4.0f, 144.0f, 80.5f, -70.6f, 20.0f};
const float kAdexNonadap[10] = {281.0f, 30.0f, -70.6f, -50.4f, 2.0f, 0.0f, 144.0f, 0.0f, -70.6f, 20.0f};

// xoshiro256** seeded by splitmix64 — the reference's `Rng`
// (net-format/src/rng.rs:16-62).
struct Xoshiro {
    uint64_t s[4];
    explicit Xoshiro(uint64_t seed) {
        uint64_t z = seed;
        for (int k = 0; k < 4; ++k) {
            z += 0x9E3779B97F4A7C15ull;
            uint64_t x = z;
            x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
            x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
            s[k] = x ^ (x >> 31);
        }
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
        const uint64_t r = rotl(s[1] * 5, 7) * 9;
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    double f64() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
    double uniform(double lo, double hi) { return lo + (hi - lo) * f64(); }
    uint64_t below(uint64_t n) { return next() % (n ? n : 1); }
};

void set_row(ne2b_net &net, uint32_t i, uint8_t model, const float *p, uint32_t np) {
    net.model[i] = model;
    for (uint32_t k = 0; k < kStride; ++k) net.params[(size_t)i * kStride + k] = k < np ? p[k] : 0.0f;
}

void add_neuron(ne2b_net &net, float x, float y, float z, uint8_t kind) {
    const uint32_t i = net.n++;
    net.pos.push_back(x);
    net.pos.push_back(y);
    net.pos.push_back(z);
    net.kind.push_back(kind);
    net.model.push_back(0);
    net.params.resize((size_t)net.n * kStride, 0.0f);
    set_row(net, i, NE2B_MODEL_IZH, kind == 1 ? kIzhFS : kIzhRS, 4);
}

// network.rs:530-541: stock izh rows follow the kind.
void set_kind(ne2b_net &net, uint32_t i, uint8_t kind) {
    const float *row = &net.params[(size_t)i * kStride];
    const bool stock = net.model[i] == NE2B_MODEL_IZH &&
                       (memcmp(row, kIzhRS, sizeof kIzhRS) == 0 || memcmp(row, kIzhFS, sizeof kIzhFS) == 0) &&
                       row[4] == 0.0f;
    net.kind[i] = kind;
    if (stock) set_row(net, i, NE2B_MODEL_IZH, kind == 1 ? kIzhFS : kIzhRS, 4);
}

// network.rs:596-601 (f32 throughout, floor 1e-3 ms)
float delay_ms(const ne2b_net &net, uint32_t a, uint32_t b, float speed) {
    const float *pa = &net.pos[3 * (size_t)a], *pb = &net.pos[3 * (size_t)b];
    const float dx = pa[0] - pb[0], dy = pa[1] - pb[1], dz = pa[2] - pb[2];
    const float d = sqrtf(dx * dx + dy * dy + dz * dz);
    const float ms = d / speed;
    return ms > 1e-3f ? ms : 1e-3f;
}

// network.rs:674-685: steps = max(1, round(delay/dt)); > u16 is an error
}  // namespace

namespace ne2b_hostnet {

bool delay_steps(float ms, float dt, uint16_t *out) {
    float st = roundf(ms / dt);
    if (st < 1.0f) st = 1.0f;
    if (!(st <= 65535.0f)) return false;
    *out = (uint16_t)st;
    return true;
}

void build_stim(ne2b_net &net, const std::vector<std::vector<std::pair<uint32_t, float>>> &inputs) {
    // StimMap::from_network (sim/src/stim.rs:26-48): neuron-major rows in
    // input order, then target-list order
    net.n_inputs = (uint32_t)inputs.size();
    net.stim_ptr.assign((size_t)net.n + 1, 0);
    for (const auto &in : inputs)
        for (const auto &tw : in)
            if (tw.first < net.n) net.stim_ptr[tw.first + 1]++;
    for (uint32_t i = 0; i < net.n; ++i) net.stim_ptr[i + 1] += net.stim_ptr[i];
    net.stim_input.assign(net.stim_ptr[net.n], 0);
    net.stim_w.assign(net.stim_ptr[net.n], 0.0f);
    std::vector<uint32_t> fill(net.stim_ptr.begin(), net.stim_ptr.end() - 1);
    for (uint32_t k = 0; k < inputs.size(); ++k)
        for (const auto &tw : inputs[k]) {
            if (tw.first >= net.n) continue;
            const uint32_t p = fill[tw.first]++;
            net.stim_input[p] = k;
            net.stim_w[p] = tw.second;
        }
}

}  // namespace ne2b_hostnet

namespace {
using ne2b_hostnet::build_stim;
using ne2b_hostnet::delay_steps;

}  // namespace

extern "C" {

ne2b_status ne2b_net_from_synapses(uint32_t n, const uint8_t *model, const float *params, uint32_t param_stride,
                                   const uint8_t *kind, uint64_t n_syn, const uint32_t *src, const uint32_t *tgt,
                                   const float *w, const float *dly, const float *tau_ms, float dt_ms,
                                   ne2b_net **out) {
    if (!out) return set_error(NE2B_EINVAL, "null out");
    *out = nullptr;
    if (n && (!model || !params || !kind)) return set_error(NE2B_EINVAL, "model, params and kind are required");
    if (n_syn && (!src || !tgt || !w || !dly)) return set_error(NE2B_EINVAL, "synapse arrays are required");
    if (n_syn > 0xffffffffull) return set_error(NE2B_UNSUPPORTED, "more than 2^32-1 synapses");
    try {
        ne2b_net *net = new ne2b_net();
        net->n = n;
        net->model.assign(model, model + n);
        net->kind.assign(kind, kind + n);
        net->params.assign((size_t)n * kStride, 0.0f);
        for (uint32_t i = 0; i < n; ++i)
            for (uint32_t k = 0; k < kStride && k < param_stride; ++k)
                net->params[(size_t)i * kStride + k] = params[(size_t)i * param_stride + k];
        net->pos.assign((size_t)n * 3, 0.0f);
        // stable counting sort by source (== sort_by_key, network.rs:656-657),
        // over T chunks of the synapse list in parallel: each chunk counts
        // its sources, the chunk offsets of a source follow the chunk order,
        // and each chunk scatters its synapses in order, so the result is the
        // stable order of the whole list
        const unsigned hw = std::thread::hardware_concurrency();
        unsigned T = n_syn >= (1u << 20) ? std::min(8u, hw ? hw : 1u) : 1u;
        if ((uint64_t)T * n > 4ull * n_syn + (1u << 20)) T = 1;  // per-chunk counts would outweigh the list
        std::vector<uint32_t> cnt((size_t)T * n, 0);
        std::vector<uint64_t> bad_ref(T, ~0ull), bad_delay(T, ~0ull);
        auto chunk = [&](unsigned c, uint64_t *lo, uint64_t *hi) {
            *lo = n_syn * c / T;
            *hi = n_syn * (c + 1) / T;
        };
        auto run = [&](auto f) {
            if (T == 1) {
                f(0u);
                return;
            }
            std::vector<std::thread> th;
            for (unsigned c = 0; c < T; ++c) th.emplace_back(f, c);
            for (auto &x : th) x.join();
        };
        run([&](unsigned c) {
            uint64_t lo, hi;
            chunk(c, &lo, &hi);
            uint32_t *cc = cnt.data() + (size_t)c * n;
            for (uint64_t j = lo; j < hi; ++j) {
                if (src[j] >= n || tgt[j] >= n) {
                    bad_ref[c] = j;
                    return;
                }
                cc[src[j]]++;
            }
        });
        const uint64_t first_bad = *std::min_element(bad_ref.begin(), bad_ref.end());
        if (first_bad != ~0ull) {
            delete net;
            return set_error(NE2B_EINVAL, "synapse %llu references %u -> %u but only %u neurons exist",
                             (unsigned long long)first_bad, src[first_bad], tgt[first_bad], n);
        }
        net->src_ptr.assign((size_t)n + 1, 0);
        {
            uint32_t base = 0;
            for (uint32_t i = 0; i < n; ++i) {
                net->src_ptr[i] = base;
                for (unsigned c = 0; c < T; ++c) {  // counts become chunk offsets
                    const uint32_t k = cnt[(size_t)c * n + i];
                    cnt[(size_t)c * n + i] = base;
                    base += k;
                }
            }
            net->src_ptr[n] = base;
        }
        net->tgt.resize(n_syn);
        net->w.resize(n_syn);
        net->delay.resize(n_syn);
        bool any_tau = false;
        for (uint64_t j = 0; tau_ms && j < n_syn && !any_tau; ++j) any_tau = tau_ms[j] > 0.0f;
        if (any_tau) net->tau.resize(n_syn);
        run([&](unsigned c) {
            uint64_t lo, hi;
            chunk(c, &lo, &hi);
            uint32_t *fill = cnt.data() + (size_t)c * n;
            for (uint64_t j = lo; j < hi; ++j) {
                const uint32_t p = fill[src[j]]++;
                if (any_tau) net->tau[p] = tau_ms[j];  // network.rs:673 (tau travels with its synapse)
                net->tgt[p] = tgt[j];
                const float m = fabsf(w[j]);
                net->w[p] = kind[src[j]] == 1 ? -m : m;  // Dale's law, network.rs:668-672
                if (!delay_steps(dly[j], dt_ms, &net->delay[p]) && bad_delay[c] == ~0ull) bad_delay[c] = j;
            }
        });
        const uint64_t first_long = *std::min_element(bad_delay.begin(), bad_delay.end());
        if (first_long != ~0ull) {
            const uint64_t j = first_long;
            delete net;
            return set_error(NE2B_EINVAL, "synapse %u -> %u: delay %g ms at dt %g ms exceeds the 65535-step ring",
                             src[j], tgt[j], (double)dly[j], (double)dt_ms);
        }
        net->stim_ptr.assign((size_t)n + 1, 0);
        *out = net;
        return NE2B_OK;
    } catch (const std::bad_alloc &) {
        return set_error(NE2B_ENOMEM, "host allocation failed");
    }
}

// Random K-out workload net (project definition; bench_net of
// sim/src/bench.rs:10-52 with the workload's weight and delay rules):
// positions U(-500,500)^3 drawn x,y,z per neuron, index < 0.8n excitatory
// RS else inhibitory FS; per source K draws of (tgt = below(n), |w| =
// f32(f64()*hi)*w_scale); delay = distance/100 um/ms capped at
// delay_cap_ms; Dale's law signs inhibitory sources.
ne2b_status ne2b_gen_random_kout(uint32_t n, uint32_t k, uint64_t seed, float w_scale, float exc_hi, float inh_hi,
                                 float delay_cap_ms, float dt_ms, ne2b_net **out) {
    if (!out) return set_error(NE2B_EINVAL, "null out");
    *out = nullptr;
    if ((uint64_t)n * k > 0xffffffffull) return set_error(NE2B_UNSUPPORTED, "n*k exceeds 2^32-1 synapses");
    try {
        ne2b_net *net = new ne2b_net();
        Xoshiro rng(seed);
        const uint64_t n_exc = (uint64_t)n * 4 / 5;
        net->pos.reserve((size_t)n * 3);
        for (uint32_t i = 0; i < n; ++i) {
            const float x = (float)rng.uniform(-500.0, 500.0);
            const float y = (float)rng.uniform(-500.0, 500.0);
            const float z = (float)rng.uniform(-500.0, 500.0);
            add_neuron(*net, x, y, z, i < n_exc ? 0 : 1);
        }
        const uint64_t e = (uint64_t)n * k;
        net->src_ptr.resize((size_t)n + 1);
        net->tgt.resize(e);
        net->w.resize(e);
        net->delay.resize(e);
        uint64_t j = 0;
        for (uint32_t src = 0; src < n; ++src) {
            net->src_ptr[src] = (uint32_t)j;
            const bool exc = src < n_exc;
            const double hi = exc ? (double)exc_hi : (double)inh_hi;
            for (uint32_t q = 0; q < k; ++q, ++j) {
                const uint32_t tg = (uint32_t)rng.below(n);
                const float m = fabsf((float)(rng.f64() * hi) * w_scale);
                float d = delay_ms(*net, src, tg, 100.0f);
                if (d > delay_cap_ms) d = delay_cap_ms;
                net->tgt[j] = tg;
                net->w[j] = exc ? m : -m;
                if (!delay_steps(d, dt_ms, &net->delay[j])) {
                    delete net;
                    return set_error(NE2B_EINVAL, "delay exceeds the 65535-step ring");
                }
            }
        }
        net->src_ptr[n] = (uint32_t)j;
        net->stim_ptr.assign((size_t)n + 1, 0);
        *out = net;
        return NE2B_OK;
    } catch (const std::bad_alloc &) {
        return set_error(NE2B_ENOMEM, "host allocation failed");
    }
}

// Local 3-D liquid workload net (project definition): create_3d_grid
// (builders.rs:88-131, spacing 60 um), set_exc_inh(0.2) (builders.rs:262-277),
// AdEx kind defaults for AdEx liquids (weights scaled by C = 281 pF),
// create_connections (builders.rs:136-181, scaling 1, lambda = lambda_units *
// 60 um) restricted to lattice offsets |o|^2 <= radius^2 in member order,
// connect() with the 100 um/ms distance delay, and n_inputs inputs whose
// targets are drawn on the x = 0 face.
ne2b_status ne2b_gen_liquid(uint32_t side, uint64_t seed, double lambda_units, int32_t radius_units, float w_rec,
                            uint32_t n_inputs, uint32_t targets_per_input, float w_in, int32_t model, float dt_ms,
                            ne2b_net **out) {
    if (!out) return set_error(NE2B_EINVAL, "null out");
    *out = nullptr;
    if (side == 0 || side > 400) return set_error(NE2B_EINVAL, "side %u out of range", side);
    if (radius_units < 0 || radius_units > 32) return set_error(NE2B_EINVAL, "radius %d out of range", radius_units);
    try {
        ne2b_net *net = new ne2b_net();
        Xoshiro rng(seed);
        const float spacing = 60.0f;
        const uint32_t m = side * side * side;
        for (uint32_t z = 0; z < side; ++z)
            for (uint32_t x = 0; x < side; ++x)
                for (uint32_t y = 0; y < side; ++y) {
                    const float h = (float)side / 2.0f;
                    add_neuron(*net, 0.0f + ((float)x - h) * spacing, 0.0f + ((float)y - h) * spacing,
                               0.0f + ((float)z - h) * spacing, 0);
                }
        for (uint32_t i = 0; i < m; ++i) set_kind(*net, i, rng.f64() < 0.2 ? 1 : 0);
        float gain = 1.0f;
        if (model == NE2B_MODEL_ADEX) {
            for (uint32_t i = 0; i < m; ++i)
                set_row(*net, i, NE2B_MODEL_ADEX, net->kind[i] == 1 ? kAdexNonadap : kAdexTonic, 10);
            gain = 281.0f;
        } else if (model != NE2B_MODEL_IZH) {
            delete net;
            return set_error(NE2B_EINVAL, "unknown model %d", model);
        }
        const float wr = w_rec * gain, wi = w_in * gain;
        const double lambda = lambda_units * (double)spacing;
        const int R = radius_units, S = (int)side;
        // connection probability and delay per lattice offset: positions are
        // exact multiples of spacing/2, so distance depends on the offset only
        const int W = 2 * R + 1;
        std::vector<double> prob((size_t)W * W * W, 0.0);
        std::vector<uint16_t> dsteps((size_t)W * W * W, 1);
        for (int dz = -R; dz <= R; ++dz)
            for (int dx = -R; dx <= R; ++dx)
                for (int dy = -R; dy <= R; ++dy) {
                    const float fx = (float)dx * spacing, fy = (float)dy * spacing, fz = (float)dz * spacing;
                    const float d = sqrtf(fx * fx + fy * fy + fz * fz);
                    const double q = (double)d / lambda;
                    const size_t o = ((size_t)(dz + R) * W + (size_t)(dx + R)) * W + (size_t)(dy + R);
                    prob[o] = 1.0 * exp(-(q * q));
                    float ms = d / 100.0f;
                    if (ms < 1e-3f) ms = 1e-3f;
                    delay_steps(ms, dt_ms, &dsteps[o]);
                }
        net->src_ptr.assign((size_t)m + 1, 0);
        for (uint32_t k1 = 0; k1 < m; ++k1) {
            net->src_ptr[k1] = (uint32_t)net->tgt.size();
            const int y1 = (int)(k1 % side), x1 = (int)((k1 / side) % side), z1 = (int)(k1 / side / side);
            const bool inh = net->kind[k1] == 1;
            for (int dz = -R; dz <= R; ++dz) {
                const int z2 = z1 + dz;
                if (z2 < 0 || z2 >= S) continue;
                for (int dx = -R; dx <= R; ++dx) {
                    const int x2 = x1 + dx;
                    if (x2 < 0 || x2 >= S) continue;
                    for (int dy = -R; dy <= R; ++dy) {
                        const int y2 = y1 + dy;
                        if (y2 < 0 || y2 >= S) continue;
                        if (dx * dx + dy * dy + dz * dz > R * R) continue;
                        const uint32_t k2 = ((uint32_t)z2 * side + (uint32_t)x2) * side + (uint32_t)y2;
                        if (k2 == k1) continue;
                        const size_t o = ((size_t)(dz + R) * W + (size_t)(dx + R)) * W + (size_t)(dy + R);
                        if (rng.f64() < prob[o]) {
                            net->tgt.push_back(k2);
                            const float mag = fabsf(wr);
                            net->w.push_back(inh ? -mag : mag);
                            net->delay.push_back(dsteps[o]);
                        }
                    }
                }
            }
        }
        net->src_ptr[m] = (uint32_t)net->tgt.size();
        std::vector<std::vector<std::pair<uint32_t, float>>> inputs(n_inputs);
        for (uint32_t k = 0; k < n_inputs; ++k)
            for (uint32_t j = 0; j < targets_per_input; ++j) {
                const uint32_t y = (uint32_t)rng.below(side);
                const uint32_t z = (uint32_t)rng.below(side);
                inputs[k].push_back({(z * side + 0) * side + y, wi});
            }
        build_stim(*net, inputs);
        *out = net;
        return NE2B_OK;
    } catch (const std::bad_alloc &) {
        return set_error(NE2B_ENOMEM, "host allocation failed");
    }
}

ne2b_status ne2b_net_set_model_all(ne2b_net *net, int32_t model, const float *exc_row, const float *inh_row,
                                   uint32_t row_len) {
    if (!net || !exc_row || !inh_row) return set_error(NE2B_EINVAL, "null argument");
    if (model != NE2B_MODEL_IZH && model != NE2B_MODEL_ADEX) return set_error(NE2B_EINVAL, "unknown model %d", model);
    for (uint32_t i = 0; i < net->n; ++i)
        set_row(*net, i, (uint8_t)model, net->kind[i] == 1 ? inh_row : exc_row, std::min<uint32_t>(row_len, kStride));
    return NE2B_OK;
}

ne2b_status ne2b_net_desc_of(const ne2b_net *net, ne2b_net_desc *d) {
    if (!net || !d) return set_error(NE2B_EINVAL, "null argument");
    memset(d, 0, sizeof *d);
    d->n = net->n;
    d->model = net->model.data();
    d->params = net->params.data();
    d->param_stride = kStride;
    d->x0 = nullptr;
    d->n_syn = net->tgt.size();
    d->src_ptr = net->src_ptr.data();
    d->tgt = net->tgt.data();
    d->w = net->w.data();
    d->delay_steps = net->delay.data();
    d->tau_ms = net->tau.empty() ? nullptr : net->tau.data();
    d->n_inputs = net->n_inputs;
    d->stim_ptr = net->n_inputs ? net->stim_ptr.data() : nullptr;
    d->stim_input = net->stim_input.data();
    d->stim_w = net->stim_w.data();
    return NE2B_OK;
}

ne2b_status ne2b_net_kinds(const ne2b_net *net, uint8_t *kind) {
    if (!net || !kind) return set_error(NE2B_EINVAL, "null argument");
    memcpy(kind, net->kind.data(), net->n);
    return NE2B_OK;
}

ne2b_status ne2b_net_free(ne2b_net *net) {
    delete net;
    return NE2B_OK;
}

// Host copy of the device det_expf (ne2b_device.cuh): the same rounded IEEE
// single operations (fmaf is the fused multiply-add, rounded once), so host
// and device agree bit for bit.
static float pow2f(int e) {
    const uint32_t bits = (uint32_t)(e + 127) << 23;
    float f;
    memcpy(&f, &bits, sizeof f);
    return f;
}
float ne2b_expf(float x) {
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
    p = p * pow2f(k1);
    return p * pow2f(k2);
}

}  // extern "C"
