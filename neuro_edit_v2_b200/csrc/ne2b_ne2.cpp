// ne2b_ne2.cpp — loader of the reference's `.ne2` network files
// (net-format/src/io.rs): the magic "NE2\0", a little-endian u32 format
// version (1..7), then the `Network` struct in bincode 1.x's default
// encoding (little-endian fixed-width integers, u64 lengths for strings,
// vectors and boxed slices, u32 enum variant indices, a u8 tag for Option).
//
// Every version's field order is decoded (io.rs:140-400 lifts v1-v6 to the
// v7 shape), the result is checked with the rules of Network::validate
// (network.rs:1007-1236), and the neurons, synapses and inputs become a
// library net exactly as Sim::new sees them: NeuronParams::from_network
// (sim/src/state.rs:98-153) for the model rows, Network::synapse_csr for the
// CSR at the file's dt, StimMap::from_network for the stimulus routing.
// Readouts, samples, scripts and groups are decoded and validated but not
// kept: the simulator does not read them.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <array>
#include <map>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include "../../include/ne2b.h"
#include "ne2b_net.h"

namespace ne2b {
ne2b_status set_error(ne2b_status st, const char *fmt, ...);
}
using ne2b::set_error;

namespace {

struct DecodeError {
    std::string what;
};

// Bounds-checked little-endian reader over the file bytes.
class Reader {
  public:
    Reader(const uint8_t *p, uint64_t n) : p_(p), n_(n) {}
    uint64_t left() const { return n_ - at_; }
    void need(uint64_t k, const char *what) {
        if (k > left()) throw DecodeError{std::string("unexpected end of file in ") + what};
    }
    uint8_t u8(const char *what) {
        need(1, what);
        return p_[at_++];
    }
    uint16_t u16(const char *what) {
        need(2, what);
        uint16_t v;
        memcpy(&v, p_ + at_, 2);
        at_ += 2;
        return v;
    }
    uint32_t u32(const char *what) {
        need(4, what);
        uint32_t v;
        memcpy(&v, p_ + at_, 4);
        at_ += 4;
        return v;
    }
    uint64_t u64(const char *what) {
        need(8, what);
        uint64_t v;
        memcpy(&v, p_ + at_, 8);
        at_ += 8;
        return v;
    }
    float f32(const char *what) {
        const uint32_t b = u32(what);
        float f;
        memcpy(&f, &b, 4);
        return f;
    }
    // A sequence length whose elements take at least `min_bytes` each: a
    // corrupt length fails here instead of allocating.
    uint64_t len(uint64_t min_bytes, const char *what) {
        const uint64_t k = u64(what);
        if (min_bytes && k > left() / min_bytes) throw DecodeError{std::string("length out of range in ") + what};
        return k;
    }
    std::string str(const char *what) {
        const uint64_t k = len(1, what);
        std::string s((const char *)p_ + at_, (size_t)k);
        at_ += k;
        if (!utf8_ok(s)) throw DecodeError{std::string("invalid UTF-8 in ") + what};
        return s;
    }
    std::vector<float> f32s(const char *what) {
        const uint64_t k = len(4, what);
        std::vector<float> v((size_t)k);
        if (k) memcpy(v.data(), p_ + at_, 4 * (size_t)k);
        at_ += 4 * k;
        return v;
    }
    std::vector<uint32_t> u32s(const char *what) {
        const uint64_t k = len(4, what);
        std::vector<uint32_t> v((size_t)k);
        if (k) memcpy(v.data(), p_ + at_, 4 * (size_t)k);
        at_ += 4 * k;
        return v;
    }
    bool option(const char *what) {
        const uint8_t t = u8(what);
        if (t > 1) throw DecodeError{std::string("invalid Option tag in ") + what};
        return t == 1;
    }
    uint32_t variant(uint32_t count, const char *what) {
        const uint32_t v = u32(what);
        if (v >= count) throw DecodeError{std::string("invalid enum variant in ") + what};
        return v;
    }
    void f32x3(float *out, const char *what) {
        for (int k = 0; k < 3; ++k) out[k] = f32(what);
    }

  private:
    static bool utf8_ok(const std::string &s) {
        const unsigned char *c = (const unsigned char *)s.data();
        size_t i = 0, n = s.size();
        while (i < n) {
            const unsigned char b = c[i];
            size_t k;
            uint32_t cp;
            if (b < 0x80) { i += 1; continue; }
            if ((b & 0xE0) == 0xC0) { k = 1; cp = b & 0x1F; }
            else if ((b & 0xF0) == 0xE0) { k = 2; cp = b & 0x0F; }
            else if ((b & 0xF8) == 0xF0) { k = 3; cp = b & 0x07; }
            else return false;
            if (i + k >= n) return false;  // truncated sequence
            for (size_t j = 1; j <= k; ++j) {
                if ((c[i + j] & 0xC0) != 0x80) return false;
                cp = (cp << 6) | (c[i + j] & 0x3F);
            }
            if ((k == 1 && cp < 0x80) || (k == 2 && cp < 0x800) || (k == 3 && cp < 0x10000) || cp > 0x10FFFF ||
                (cp >= 0xD800 && cp <= 0xDFFF))
                return false;
            i += k + 1;
        }
        return true;
    }
    const uint8_t *p_;
    uint64_t n_, at_ = 0;
};

// The parts of `Network` (network.rs:381-440) in their v7 shape.
struct Type {
    std::string name, model;
    std::vector<float> params;
    uint32_t kind = 0;  // 0 excitatory, 1 inhibitory, 2 regular
};
struct Neuron {
    float pos[3];
    uint16_t ty = 0;
    bool has_params = false;
    std::vector<float> params;
};
struct Synapse {
    uint32_t src, tgt;
    float w, delay_ms, tau_ms;
};
struct Grid {
    uint32_t dims[3];
    float origin[3];
    float spacing;
    uint8_t axes[3];
};
struct Group {
    std::vector<uint32_t> members;
    bool has_grid = false;
    Grid grid;
};
struct Input {
    std::string name;
    std::vector<std::pair<uint32_t, float>> targets;
};
struct Samples {
    std::string name;
    std::vector<float> times, values;
};
struct Mlp {
    std::vector<uint32_t> sizes;
    std::vector<std::vector<float>> w;
    std::vector<float> mu, sd;
    uint32_t head = 0;  // 0 score, 1 softmax
};
struct Readout {
    std::string name;
    std::vector<uint32_t> units;
    std::vector<float> weights;
    float tau_ms = 0.0f;
    bool has_mlp = false;
    Mlp mlp;
    std::vector<uint32_t> mlp_layers;
};
struct Meta {
    float dt_ms, conduction_speed, synapse_tau_ms, readout_tau_ms, noise_rate_hz, noise_kick_mv;
    uint64_t seed;
};
struct Network {
    std::vector<Type> types;
    std::vector<Neuron> neurons;
    std::vector<Synapse> synapses;
    std::vector<Group> groups;
    std::vector<Input> inputs;
    std::vector<Samples> samples;
    std::vector<Readout> readouts;
    uint64_t n_scripts = 0;
    Meta meta;
};

const float kIzhRS[4] = {0.02f, 0.2f, -65.0f, 8.0f};  // network.rs:54
const float kIzhFS[4] = {0.1f, 0.2f, -65.0f, 2.0f};   // network.rs:55

// Pre-v4 neurons carry an izh model and a kind inline; each distinct
// (params bits, kind) becomes one type, named as io.rs:116-160 does.
void lift_inline_neurons(Reader &r, Network &net) {
    const uint64_t k = r.len(4 * 3 + 4 + 16 + 4 + 8, "neurons");
    std::map<std::pair<std::array<uint32_t, 4>, uint32_t>, uint16_t> lut;
    for (uint64_t i = 0; i < k; ++i) {
        r.str("neuron name");
        Neuron nv;
        r.f32x3(nv.pos, "neuron pos");
        r.variant(1, "NeuronModel");  // Izhikevich { a, b, c, d }
        float p[4];
        for (int j = 0; j < 4; ++j) p[j] = r.f32("NeuronModel");
        const uint32_t kind = r.variant(3, "NeuronKind");
        std::array<uint32_t, 4> bits;
        memcpy(bits.data(), p, 16);
        auto key = std::make_pair(bits, kind);
        auto it = lut.find(key);
        if (it == lut.end()) {
            std::string name;
            if (!memcmp(p, kIzhRS, 16) && kind == 0) name = "exc";
            else if (!memcmp(p, kIzhFS, 16) && kind == 1) name = "inh";
            else if (!memcmp(p, kIzhRS, 16) && kind == 2) name = "regular";
            else {
                uint64_t h = 0xcbf29ce484222325ull;  // FNV-1a over the param bits, then the kind
                for (int j = 0; j < 4; ++j)
                    for (int b = 0; b < 4; ++b) h = (h ^ ((bits[j] >> (8 * b)) & 0xffu)) * 0x100000001b3ull;
                h = (h ^ kind) * 0x100000001b3ull;
                char buf[16];
                snprintf(buf, sizeof buf, "izh#%04x", (unsigned)(h & 0xffff));
                name = buf;
            }
            std::string base = name;
            for (uint32_t s = 2;; ++s) {
                bool used = false;
                for (const Type &t : net.types) used |= t.name == name;
                if (!used) break;
                name = base + std::to_string(s);
            }
            Type t;
            t.name = name;
            t.model = "izh";
            t.params.assign(p, p + 4);
            t.kind = kind;
            net.types.push_back(t);
            it = lut.emplace(key, (uint16_t)(net.types.size() - 1)).first;
        }
        nv.ty = it->second;
        net.neurons.push_back(nv);
    }
}

void read_types(Reader &r, Network &net, bool with_color) {
    const uint64_t k = r.len(8 + 8 + 8 + 4, "types");
    for (uint64_t i = 0; i < k; ++i) {
        Type t;
        t.name = r.str("type name");
        t.model = r.str("type model");
        t.params = r.f32s("type params");
        t.kind = r.variant(3, "NeuronKind");
        if (with_color && r.option("type color")) {
            float c[3];
            r.f32x3(c, "type color");
        }
        net.types.push_back(std::move(t));
    }
}

void read_neurons(Reader &r, Network &net) {
    const uint64_t k = r.len(8 + 12 + 2 + 1, "neurons");
    net.neurons.reserve((size_t)k);
    for (uint64_t i = 0; i < k; ++i) {
        r.str("neuron name");
        Neuron nv;
        r.f32x3(nv.pos, "neuron pos");
        nv.ty = r.u16("neuron ty");
        nv.has_params = r.option("neuron params");
        if (nv.has_params) nv.params = r.f32s("neuron params");
        net.neurons.push_back(std::move(nv));
    }
}

void read_synapses(Reader &r, Network &net, bool with_tau) {
    const uint64_t k = r.len(with_tau ? 20 : 16, "synapses");
    net.synapses.resize((size_t)k);
    for (uint64_t i = 0; i < k; ++i) {
        Synapse &s = net.synapses[(size_t)i];
        s.src = r.u32("synapse");
        s.tgt = r.u32("synapse");
        s.w = r.f32("synapse");
        s.delay_ms = r.f32("synapse");
        s.tau_ms = with_tau ? r.f32("synapse") : 0.0f;  // v1/v2: the merged path (io.rs:196-207)
    }
}

void read_groups(Reader &r, Network &net, bool with_grid) {
    const uint64_t k = r.len(16, "groups");
    for (uint64_t i = 0; i < k; ++i) {
        Group g;
        r.str("group name");
        g.members = r.u32s("group members");
        if (with_grid && r.option("group grid")) {
            g.has_grid = true;
            for (int j = 0; j < 3; ++j) g.grid.dims[j] = r.u32("grid");
            r.f32x3(g.grid.origin, "grid");
            g.grid.spacing = r.f32("grid");
            for (int j = 0; j < 3; ++j) g.grid.axes[j] = r.u8("grid");
        }
        net.groups.push_back(std::move(g));
    }
}

void read_inputs(Reader &r, Network &net) {
    const uint64_t k = r.len(8 + 8 + 12, "inputs");
    for (uint64_t i = 0; i < k; ++i) {
        Input in;
        in.name = r.str("input name");
        const uint64_t m = r.len(8, "input targets");
        in.targets.resize((size_t)m);
        for (uint64_t j = 0; j < m; ++j) {
            in.targets[(size_t)j].first = r.u32("input target");
            in.targets[(size_t)j].second = r.f32("input target");
        }
        float pos[3];
        r.f32x3(pos, "input pos");
        net.inputs.push_back(std::move(in));
    }
}

void read_samples(Reader &r, Network &net) {
    const uint64_t k = r.len(24, "samples");
    for (uint64_t i = 0; i < k; ++i) {
        Samples s;
        s.name = r.str("samples name");
        s.times = r.f32s("samples times");
        s.values = r.f32s("samples values");
        net.samples.push_back(std::move(s));
    }
}

// Readout rows: v1-v5 without `mlp`, v6 with the tanh/score MLP, v7 with
// the MLP's activation and head and the `mlp_layers` config.
void read_readouts(Reader &r, Network &net, int shape) {
    const uint64_t k = r.len(8 + 8 + 8 + 12 + 12, "readouts");
    for (uint64_t i = 0; i < k; ++i) {
        Readout ro;
        ro.name = r.str("readout name");
        ro.units = r.u32s("readout units");
        ro.weights = r.f32s("readout weights");
        r.f32("readout bias");
        r.f32("readout bias_weight");
        ro.tau_ms = r.f32("readout tau_ms");
        float pos[3];
        r.f32x3(pos, "readout pos");
        if (shape >= 6 && r.option("readout mlp")) {
            ro.has_mlp = true;
            ro.mlp.sizes = r.u32s("mlp sizes");
            const uint64_t layers = r.len(8, "mlp w");
            for (uint64_t l = 0; l < layers; ++l) ro.mlp.w.push_back(r.f32s("mlp w"));
            ro.mlp.mu = r.f32s("mlp mu");
            ro.mlp.sd = r.f32s("mlp sd");
            if (shape >= 7) {
                r.variant(2, "MlpAct");
                ro.mlp.head = r.variant(2, "MlpHead");
            }
        }
        if (shape >= 7) ro.mlp_layers = r.u32s("readout mlp_layers");
        net.readouts.push_back(std::move(ro));
    }
}

void read_tail(Reader &r, Network &net, int readout_shape) {
    read_inputs(r, net);
    read_samples(r, net);
    read_readouts(r, net, readout_shape);
    net.n_scripts = r.len(16, "scripts");
    for (uint64_t i = 0; i < net.n_scripts; ++i) {
        r.str("script name");
        r.str("script text");
    }
    Meta &m = net.meta;
    m.dt_ms = r.f32("meta");
    m.seed = r.u64("meta");
    m.conduction_speed = r.f32("meta");
    m.synapse_tau_ms = r.f32("meta");
    m.readout_tau_ms = r.f32("meta");
    m.noise_rate_hz = r.f32("meta");
    m.noise_kick_mv = r.f32("meta");
}

// io.rs:427-467 load: version dispatch.
void decode(Reader &r, uint32_t version, Network &net) {
    switch (version) {
        case 1:
        case 2:
        case 3:
            lift_inline_neurons(r, net);
            read_synapses(r, net, version >= 3);
            read_groups(r, net, version >= 2);
            read_tail(r, net, 5);
            break;
        case 4:
        case 5:
        case 6:
        case 7:
            read_types(r, net, version >= 5);
            read_neurons(r, net);
            read_synapses(r, net, true);
            read_groups(r, net, true);
            read_tail(r, net, version >= 7 ? 7 : (version == 6 ? 6 : 5));
            break;
        default:
            throw DecodeError{"unsupported .ne2 version " + std::to_string(version)};
    }
}

bool finite(float x) { return isfinite(x) != 0; }

// Network::validate (network.rs:1007-1236); the message of the first rule
// that fails.
std::string validate(const Network &net) {
    char buf[256];
    const uint32_t n = (uint32_t)net.neurons.size();
    const Meta &m = net.meta;
    if (!(finite(m.dt_ms) && m.dt_ms > 0.0f)) return "meta.dt_ms must be positive and finite";
    if (!(finite(m.conduction_speed) && m.conduction_speed > 0.0f))
        return "meta.conduction_speed must be positive and finite";
    const std::pair<const char *, float> nonneg[] = {{"synapse_tau_ms", m.synapse_tau_ms},
                                                     {"readout_tau_ms", m.readout_tau_ms},
                                                     {"noise_rate_hz", m.noise_rate_hz},
                                                     {"noise_kick_mv", m.noise_kick_mv}};
    for (const auto &kv : nonneg)
        if (!(finite(kv.second) && kv.second >= 0.0f)) return std::string("meta.") + kv.first + " must be finite and >= 0";
    for (size_t i = 0; i < net.types.size(); ++i) {
        const Type &t = net.types[i];
        bool dup = t.name.empty();
        for (size_t j = 0; j < i && !dup; ++j) dup = net.types[j].name == t.name;
        if (dup) return "type " + std::to_string(i) + " \"" + t.name + "\" has a missing/duplicate name";
        if (t.model.empty()) return "type \"" + t.name + "\" has an empty model id";
        bool ok = !t.params.empty();
        for (float p : t.params) ok &= finite(p);
        if (!ok) return "type \"" + t.name + "\" has bad params";
    }
    if (net.types.size() > 65536) return "types exceed the u16 ty index";
    for (uint32_t i = 0; i < n; ++i) {
        const Neuron &nv = net.neurons[i];
        if (!(finite(nv.pos[0]) && finite(nv.pos[1]) && finite(nv.pos[2])))
            return "neuron " + std::to_string(i) + " has non-finite pos";
        if (nv.ty >= net.types.size()) {
            snprintf(buf, sizeof buf, "neuron %u has ty %u but only %zu types exist", i, nv.ty, net.types.size());
            return buf;
        }
        if (nv.has_params) {
            bool ok = nv.params.size() == net.types[nv.ty].params.size();
            for (float p : nv.params) ok &= finite(p);
            if (!ok) return "neuron " + std::to_string(i) + " has a bad param override";
        }
    }
    for (size_t i = 0; i < net.synapses.size(); ++i) {
        const Synapse &s = net.synapses[i];
        if (s.src >= n || s.tgt >= n) {
            snprintf(buf, sizeof buf, "synapse %zu references %u -> %u but only %u neurons exist", i, s.src, s.tgt, n);
            return buf;
        }
        if (!(s.tau_ms >= 0.0f && finite(s.tau_ms))) return "synapse " + std::to_string(i) + " has bad tau_ms";
        if (!finite(s.w)) return "synapse " + std::to_string(i) + " has non-finite weight";
        if (!(s.delay_ms >= 0.0f && finite(s.delay_ms))) return "synapse " + std::to_string(i) + " has bad delay_ms";
    }
    for (const Group &g : net.groups) {
        for (uint32_t mm : g.members)
            if (mm >= n) return "a group references neuron " + std::to_string(mm);
        if (g.has_grid) {
            bool seen[3] = {false, false, false};
            for (int k = 0; k < 3; ++k) {
                const uint8_t a = g.grid.axes[k];
                if (a >= 3 || seen[a]) return "a group grid has invalid axes";
                seen[a] = true;
            }
            if (!(finite(g.grid.spacing) && g.grid.spacing != 0.0f)) return "a group grid spacing must be finite and non-zero";
            for (int k = 0; k < 3; ++k)
                if (g.grid.dims[k] == 0) return "a group grid has a zero dim";
        }
    }
    for (const Input &in : net.inputs)
        for (const auto &tw : in.targets) {
            if (tw.first >= n) return "input '" + in.name + "' targets neuron " + std::to_string(tw.first);
            if (!finite(tw.second)) return "input '" + in.name + "' has a non-finite weight";
        }
    for (const Readout &ro : net.readouts) {
        for (uint32_t u : ro.units)
            if (u >= n) return "readout '" + ro.name + "' references unit " + std::to_string(u);
        if (!ro.weights.empty() && ro.weights.size() != ro.units.size())
            return "readout '" + ro.name + "' has weights that do not match its units";
        if (!(finite(ro.tau_ms) && ro.tau_ms > 0.0f)) return "readout '" + ro.name + "' tau_ms must be positive and finite";
        if (ro.mlp_layers.size() > 8) return "readout '" + ro.name + "' has bad mlp layer config";
        for (uint32_t s : ro.mlp_layers)
            if (s == 0 || s > 4096) return "readout '" + ro.name + "' has bad mlp layer config";
        if (ro.has_mlp) {
            const Mlp &mp = ro.mlp;
            const bool out_ok = mp.head == 0 ? (!mp.sizes.empty() && mp.sizes.back() == 1)
                                             : (!mp.sizes.empty() && mp.sizes.back() >= 2);
            bool zero = false;
            for (uint32_t s : mp.sizes) zero |= s == 0;
            if (mp.sizes.size() < 2 || !out_ok || zero) return "readout '" + ro.name + "' has malformed mlp sizes";
            if (mp.w.size() + 1 != mp.sizes.size()) return "readout '" + ro.name + "' mlp weight matrices do not match";
            for (size_t l = 0; l < mp.w.size(); ++l) {
                const uint64_t want = (uint64_t)mp.sizes[l + 1] * ((uint64_t)mp.sizes[l] + 1);
                bool ok = mp.w[l].size() == want;
                for (float v : mp.w[l]) ok &= finite(v);
                if (!ok) return "readout '" + ro.name + "' mlp layer " + std::to_string(l) + " has bad weights";
            }
            if (mp.mu.size() != mp.sizes[0] || mp.sd.size() != mp.sizes[0])
                return "readout '" + ro.name + "' mlp standardization doesn't match its inputs";
        }
    }
    for (const Samples &s : net.samples) {
        if (s.times.size() != s.values.size()) return "samples '" + s.name + "' has mismatched times and values";
        bool ok = true;
        for (float v : s.times) ok &= finite(v);
        for (float v : s.values) ok &= finite(v);
        if (!ok) return "samples '" + s.name + "' has non-finite data";
    }
    return "";
}

ne2b_status build(const Network &net, uint32_t version, ne2b_net **out, ne2b_ne2_meta *meta) {
    const uint32_t n = (uint32_t)net.neurons.size();
    // NeuronParams::from_network (state.rs:98-153): the effective row is the
    // neuron's override or its type's; the model id picks the registry entry
    std::vector<uint8_t> model(n), kind(n);
    std::vector<float> params((size_t)n * 10, 0.0f);
    for (uint32_t i = 0; i < n; ++i) {
        const Neuron &nv = net.neurons[i];
        const Type &t = net.types[nv.ty];
        uint32_t width;
        if (t.model == "izh") {
            model[i] = NE2B_MODEL_IZH;
            width = 4;
        } else if (t.model == "adex") {
            model[i] = NE2B_MODEL_ADEX;
            width = 10;
        } else {
            return set_error(NE2B_UNSUPPORTED, "neuron %u: unknown model \"%s\"", i, t.model.c_str());
        }
        const std::vector<float> &p = nv.has_params ? nv.params : t.params;
        if (p.size() != width)
            return set_error(NE2B_EINVAL, "neuron %u: %zu params, model %s wants %u", i, p.size(), t.model.c_str(),
                             width);
        std::copy(p.begin(), p.end(), params.begin() + (size_t)i * 10);
        kind[i] = (uint8_t)t.kind;
    }
    const size_t e = net.synapses.size();
    std::vector<uint32_t> src(e), tgt(e);
    std::vector<float> w(e), dly(e), tau(e);
    for (size_t j = 0; j < e; ++j) {
        src[j] = net.synapses[j].src;
        tgt[j] = net.synapses[j].tgt;
        w[j] = net.synapses[j].w;
        dly[j] = net.synapses[j].delay_ms;
        tau[j] = net.synapses[j].tau_ms;
    }
    ne2b_net *built = nullptr;
    ne2b_status st = ne2b_net_from_synapses(n, model.data(), params.data(), 10, kind.data(), e, src.data(),
                                            tgt.data(), w.data(), dly.data(), tau.data(), net.meta.dt_ms, &built);
    if (st != NE2B_OK) return st;
    for (uint32_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) built->pos[3 * (size_t)i + k] = net.neurons[i].pos[k];
    std::vector<std::vector<std::pair<uint32_t, float>>> inputs;
    inputs.reserve(net.inputs.size());
    for (const Input &in : net.inputs) inputs.push_back(in.targets);
    ne2b_hostnet::build_stim(*built, inputs);
    if (meta) {
        memset(meta, 0, sizeof *meta);
        meta->version = version;
        meta->dt_ms = net.meta.dt_ms;
        meta->seed = net.meta.seed;
        meta->conduction_speed = net.meta.conduction_speed;
        meta->synapse_tau_ms = net.meta.synapse_tau_ms;
        meta->readout_tau_ms = net.meta.readout_tau_ms;
        meta->noise_rate_hz = net.meta.noise_rate_hz;
        meta->noise_kick_mv = net.meta.noise_kick_mv;
        meta->n_types = (uint32_t)net.types.size();
        meta->n_groups = (uint32_t)net.groups.size();
        meta->n_samples = (uint32_t)net.samples.size();
        meta->n_readouts = (uint32_t)net.readouts.size();
        meta->n_scripts = (uint32_t)net.n_scripts;
    }
    *out = built;
    return NE2B_OK;
}

}  // namespace

extern "C" {

ne2b_status ne2b_net_from_ne2(const uint8_t *bytes, uint64_t len, ne2b_net **out, ne2b_ne2_meta *meta) {
    if (!out) return set_error(NE2B_EINVAL, "null out");
    *out = nullptr;
    if (!bytes && len) return set_error(NE2B_EINVAL, "null bytes");
    try {
        Reader r(bytes, len);
        if (len < 4 || memcmp(bytes, "NE2\0", 4) != 0) return set_error(NE2B_EINVAL, "not a .ne2 file (bad magic)");
        r.u32("magic");
        const uint32_t version = r.u32("version");
        if (version < 1 || version > 7) return set_error(NE2B_UNSUPPORTED, "unsupported .ne2 version %u", version);
        Network net;
        decode(r, version, net);
        const std::string bad = validate(net);
        if (!bad.empty()) return set_error(NE2B_EINVAL, "decode error: %s", bad.c_str());
        return build(net, version, out, meta);
    } catch (const DecodeError &e) {
        return set_error(NE2B_EINVAL, "decode error: %s", e.what.c_str());
    } catch (const std::bad_alloc &) {
        return set_error(NE2B_ENOMEM, "host allocation failed");
    }
}

ne2b_status ne2b_net_load_ne2(const char *path, ne2b_net **out, ne2b_ne2_meta *meta) {
    if (!path || !out) return set_error(NE2B_EINVAL, "null argument");
    *out = nullptr;
    FILE *f = fopen(path, "rb");
    if (!f) return set_error(NE2B_EINVAL, "io error: cannot open %s", path);
    std::vector<uint8_t> bytes;
    uint8_t buf[1 << 16];
    size_t k;
    while ((k = fread(buf, 1, sizeof buf, f)) > 0) bytes.insert(bytes.end(), buf, buf + k);
    const bool err = ferror(f) != 0;
    fclose(f);
    if (err) return set_error(NE2B_EINVAL, "io error: reading %s", path);
    return ne2b_net_from_ne2(bytes.data(), bytes.size(), out, meta);
}

}  // extern "C"
