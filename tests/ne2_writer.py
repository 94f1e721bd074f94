"""Test infrastructure: writes `.ne2` network files (net-format/src/io.rs)
from a plain description, in any format version 1-7, so the library's
loader can be checked on every field order and on nets the oracle also
builds.  The layout is the reference's `Network` (network.rs:381-440)
serialized by bincode 1.x's default options: little-endian fixed-width
integers, u64 lengths for strings and sequences, u32 enum variant indices,
a u8 tag for Option; older versions drop or reshape fields as io.rs:14-400
describes (v1-v3 neurons carry an izh model and a kind inline, v1/v2
synapses have no tau, v1 groups no grid, v4 types no colour, v1-v5 readouts
no MLP, v6 MLPs no activation/head and no layer config)."""
from __future__ import annotations

import struct

import numpy as np

KINDS = {"exc": 0, "inh": 1, "regular": 2}


def _u8(x):
    return struct.pack("<B", x)


def _u16(x):
    return struct.pack("<H", x)


def _u32(x):
    return struct.pack("<I", x)


def _u64(x):
    return struct.pack("<Q", x)


def _f32(x):
    return struct.pack("<f", x)


def _str(s: str):
    b = s.encode("utf-8")
    return _u64(len(b)) + b


def _f32s(v):
    v = list(v)
    return _u64(len(v)) + b"".join(_f32(x) for x in v)


def _u32s(v):
    v = list(v)
    return _u64(len(v)) + b"".join(_u32(x) for x in v)


def _opt(x, enc):
    return _u8(0) if x is None else _u8(1) + enc(x)


def encode(net: dict, version: int = 7) -> bytes:
    """`net` keys: types [(name, model, params, kind, color|None)],
    neurons [(name, pos3, ty, override|None)], synapses [(src, tgt, w,
    delay_ms, tau_ms)], groups [(name, members, grid|None)], inputs [(name,
    [(tgt, w)], pos3)], samples [(name, times, values)], readouts [dict],
    scripts [(name, text)], meta dict.  For version <= 3 every type must be
    an izh type with 4 params (the neurons are written inline)."""
    out = [b"NE2\0", _u32(version)]
    types = net["types"]
    if version <= 3:
        out.append(_u64(len(net["neurons"])))
        for name, pos, ty, override in net["neurons"]:
            tname, model, params, kind, _ = types[ty]
            assert model == "izh" and len(params) == 4 and override is None
            out.append(_str(name) + b"".join(_f32(p) for p in pos) + _u32(0) +
                       b"".join(_f32(p) for p in params) + _u32(KINDS[kind]))
    else:
        out.append(_u64(len(types)))
        for name, model, params, kind, color in types:
            out.append(_str(name) + _str(model) + _f32s(params) + _u32(KINDS[kind]))
            if version >= 5:
                out.append(_opt(color, lambda c: b"".join(_f32(x) for x in c)))
        out.append(_u64(len(net["neurons"])))
        for name, pos, ty, override in net["neurons"]:
            out.append(_str(name) + b"".join(_f32(p) for p in pos) + _u16(ty) + _opt(override, _f32s))
    out.append(_u64(len(net["synapses"])))
    for src, tgt, w, d, tau in net["synapses"]:
        out.append(_u32(src) + _u32(tgt) + _f32(w) + _f32(d))
        if version >= 3:
            out.append(_f32(tau))
        else:
            assert tau == 0.0
    out.append(_u64(len(net["groups"])))
    for name, members, grid in net["groups"]:
        out.append(_str(name) + _u32s(members))
        if version >= 2:
            out.append(_opt(grid, lambda g: b"".join(_u32(x) for x in g["dims"]) +
                            b"".join(_f32(x) for x in g["origin"]) + _f32(g["spacing"]) +
                            b"".join(_u8(x) for x in g["axes"])))
    out.append(_u64(len(net["inputs"])))
    for name, targets, pos in net["inputs"]:
        out.append(_str(name) + _u64(len(targets)) + b"".join(_u32(t) + _f32(w) for t, w in targets) +
                   b"".join(_f32(p) for p in pos))
    out.append(_u64(len(net["samples"])))
    for name, times, values in net["samples"]:
        out.append(_str(name) + _f32s(times) + _f32s(values))
    out.append(_u64(len(net["readouts"])))
    for r in net["readouts"]:
        out.append(_str(r["name"]) + _u32s(r["units"]) + _f32s(r["weights"]) + _f32(r["bias"]) +
                   _f32(r["bias_weight"]) + _f32(r["tau_ms"]) + b"".join(_f32(p) for p in r["pos"]))
        if version >= 6:
            def mlp(m):
                b = _u32s(m["sizes"]) + _u64(len(m["w"])) + b"".join(_f32s(w) for w in m["w"])
                b += _f32s(m["mu"]) + _f32s(m["sd"])
                if version >= 7:
                    b += _u32(m.get("act", 0)) + _u32(m.get("head", 0))
                return b
            out.append(_opt(r.get("mlp"), mlp))
        if version >= 7:
            out.append(_u32s(r.get("mlp_layers", [])))
    out.append(_u64(len(net["scripts"])))
    for name, text in net["scripts"]:
        out.append(_str(name) + _str(text))
    m = net["meta"]
    out.append(_f32(m["dt_ms"]) + _u64(m["seed"]) + _f32(m["conduction_speed"]) + _f32(m["synapse_tau_ms"]) +
               _f32(m["readout_tau_ms"]) + _f32(m["noise_rate_hz"]) + _f32(m["noise_kick_mv"]))
    return b"".join(out)


DEFAULT_META = dict(dt_ms=0.1, seed=7, conduction_speed=100.0, synapse_tau_ms=2.0, readout_tau_ms=2.0,
                    noise_rate_hz=0.0, noise_kick_mv=20.0)


def from_onet(onet, inputs=(), meta=None, izh_only=False) -> dict:
    """A description of an oracle net: one type per distinct (model, row,
    kind), neurons at the origin, the synapses in insertion order, and the
    given inputs [(name, [(tgt, w)])]."""
    model, params = onet.models()
    kinds = onet.kinds()
    src, tgt, w, d, tau = onet.synapses()
    names = {0: "exc", 1: "inh", 2: "regular"}
    types, index, neurons = [], {}, []
    for i in range(len(model)):
        width = 4 if model[i] == 0 else 10
        row = tuple(float(x) for x in np.asarray(params[i][:width], np.float32))
        key = (int(model[i]), row, int(kinds[i]))
        if key not in index:
            assert not izh_only or model[i] == 0
            index[key] = len(types)
            types.append((f"t{len(types)}", "izh" if model[i] == 0 else "adex", list(row), names[int(kinds[i])],
                          None))
        neurons.append((f"n{i}", (0.0, 0.0, 0.0), index[key], None))
    syn = [(int(a), int(b), float(abs(c)), float(e), float(t)) for a, b, c, e, t in zip(src, tgt, w, d, tau)]
    return dict(types=types, neurons=neurons, synapses=syn, groups=[], inputs=[(nm, list(t), (0.0, 0.0, 0.0))
                                                                             for nm, t in inputs],
                samples=[], readouts=[], scripts=[], meta=dict(meta or DEFAULT_META))
