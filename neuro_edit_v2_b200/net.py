"""Networks in the flat layout the B200 backend consumes.

A network reaches the backend as `ne2b_net_desc`: the per-neuron model ids
and parameter rows of `NeuronParams::from_network` (sim/src/state.rs:98-153),
the source-major CSR of `Network::synapse_csr`
(net-format/src/network.rs:654-692) and the stimulus map of
`StimMap::from_network` (sim/src/stim.rs:26-48).

`FlatNet` keeps the numpy arrays alive for as long as the descriptor is used;
`NativeNet` wraps a network built inside the library (the workload
generators and the CSR build).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from ._abi import check, lib, ptr


@dataclass
class FlatNet:
    model: np.ndarray                      # u8[n]
    params: np.ndarray                     # f32[n, stride]
    src_ptr: np.ndarray                    # u32[n+1]
    tgt: np.ndarray                        # u32[E]
    w: np.ndarray                          # f32[E], Dale-signed
    delay_steps: np.ndarray                # u16[E]
    n_inputs: int = 0
    stim_ptr: np.ndarray | None = None     # u32[n+1]
    stim_input: np.ndarray | None = None   # u32[entries]
    stim_w: np.ndarray | None = None       # f32[entries]
    x0: np.ndarray | None = None           # f32[n, 2]
    kind: np.ndarray | None = None         # u8[n] (0 exc, 1 inh, 2 regular)
    tau_ms: np.ndarray | None = None       # f32[E]: > 0 gives the synapse its own current (XSyn)
    _desc: _abi.NetDesc | None = field(default=None, repr=False)

    def __post_init__(self):
        self.model = np.ascontiguousarray(self.model, dtype=np.uint8)
        self.params = np.ascontiguousarray(self.params, dtype=np.float32)
        if self.params.ndim == 1:
            self.params = self.params.reshape(len(self.model), -1)
        self.src_ptr = np.ascontiguousarray(self.src_ptr, dtype=np.uint32)
        self.tgt = np.ascontiguousarray(self.tgt, dtype=np.uint32)
        self.w = np.ascontiguousarray(self.w, dtype=np.float32)
        self.delay_steps = np.ascontiguousarray(self.delay_steps, dtype=np.uint16)
        for name, dt in (("stim_ptr", np.uint32), ("stim_input", np.uint32), ("stim_w", np.float32),
                         ("x0", np.float32), ("kind", np.uint8), ("tau_ms", np.float32)):
            v = getattr(self, name)
            if v is not None:
                setattr(self, name, np.ascontiguousarray(v, dtype=dt))

    @property
    def n(self) -> int:
        return int(self.model.shape[0])

    @property
    def n_syn(self) -> int:
        return int(self.tgt.shape[0])

    def desc(self) -> _abi.NetDesc:
        d = _abi.NetDesc()
        d.n = self.n
        d.model = ptr(self.model)
        d.params = ptr(self.params)
        d.param_stride = self.params.shape[1] if self.params.ndim == 2 else 0
        d.x0 = ptr(self.x0)
        d.n_syn = self.n_syn
        d.src_ptr = ptr(self.src_ptr)
        d.tgt = ptr(self.tgt)
        d.w = ptr(self.w)
        d.delay_steps = ptr(self.delay_steps)
        d.tau_ms = ptr(self.tau_ms) if self.tau_ms is not None else None
        d.n_inputs = self.n_inputs
        d.stim_ptr = ptr(self.stim_ptr) if self.n_inputs else None
        d.stim_input = ptr(self.stim_input) if self.n_inputs else None
        d.stim_w = ptr(self.stim_w) if self.n_inputs else None
        self._desc = d
        return d

    def ring_depth(self) -> int:
        """`ring_depth` (sim/src/state.rs:221-224)."""
        m = int(self.delay_steps.max()) if self.n_syn else 1
        return max(m + 1, 2)


class NativeNet:
    """A network owned by the library (generators / CSR build)."""

    def __init__(self, handle: C.c_void_p):
        self._h = handle
        self._desc = _abi.NetDesc()
        check(lib.ne2b_net_desc_of(self._h, C.byref(self._desc)))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib.ne2b_net_free(h)
            self._h = None

    @property
    def n(self) -> int:
        return int(self._desc.n)

    @property
    def n_syn(self) -> int:
        return int(self._desc.n_syn)

    @property
    def n_inputs(self) -> int:
        return int(self._desc.n_inputs)

    def desc(self) -> _abi.NetDesc:
        return self._desc

    def kinds(self) -> np.ndarray:
        k = np.zeros(self.n, dtype=np.uint8)
        check(lib.ne2b_net_kinds(self._h, ptr(k)))
        return k

    def arrays(self) -> FlatNet:
        """Copy the network out into numpy arrays."""
        d = self._desc
        n, e = int(d.n), int(d.n_syn)

        def arr(p, count, ct, dt):
            if count == 0 or not p:
                return np.zeros(0, dtype=dt)
            return np.ctypeslib.as_array(C.cast(p, C.POINTER(ct)), shape=(count,)).astype(dt, copy=True)

        stride = int(d.param_stride)
        ni = int(d.n_inputs)
        sp = arr(d.stim_ptr, n + 1, C.c_uint32, np.uint32) if ni else None
        ne = int(sp[-1]) if sp is not None and n else 0
        return FlatNet(
            model=arr(d.model, n, C.c_uint8, np.uint8),
            params=arr(d.params, n * stride, C.c_float, np.float32).reshape(n, stride),
            src_ptr=arr(d.src_ptr, n + 1, C.c_uint32, np.uint32),
            tgt=arr(d.tgt, e, C.c_uint32, np.uint32),
            w=arr(d.w, e, C.c_float, np.float32),
            delay_steps=arr(d.delay_steps, e, C.c_uint16, np.uint16),
            tau_ms=arr(d.tau_ms, e, C.c_float, np.float32) if d.tau_ms else None,
            n_inputs=ni,
            stim_ptr=sp,
            stim_input=arr(d.stim_input, ne, C.c_uint32, np.uint32) if ni else None,
            stim_w=arr(d.stim_w, ne, C.c_float, np.float32) if ni else None,
            kind=self.kinds(),
        )


def from_synapses(model, params, kind, src, tgt, w, delay_ms, dt_ms=0.1, tau_ms=None) -> NativeNet:
    """`Network::synapse_csr` (net-format/src/network.rs:654-692) in the library."""
    model = np.ascontiguousarray(model, dtype=np.uint8)
    params = np.ascontiguousarray(params, dtype=np.float32)
    kind = np.ascontiguousarray(kind, dtype=np.uint8)
    src = np.ascontiguousarray(src, dtype=np.uint32)
    tgt = np.ascontiguousarray(tgt, dtype=np.uint32)
    w = np.ascontiguousarray(w, dtype=np.float32)
    delay_ms = np.ascontiguousarray(delay_ms, dtype=np.float32)
    tau = None if tau_ms is None else np.ascontiguousarray(tau_ms, dtype=np.float32)
    n = len(model)
    stride = params.shape[1] if params.ndim == 2 else (params.size // max(n, 1))
    h = C.c_void_p()
    check(lib.ne2b_net_from_synapses(n, ptr(model), ptr(params), stride, ptr(kind), len(src), ptr(src), ptr(tgt),
                                     ptr(w), ptr(delay_ms), ptr(tau), dt_ms, C.byref(h)))
    return NativeNet(h)


def random_kout(n: int, k: int = 100, seed: int = 1, w_scale: float = 0.7, exc_hi: float = 0.5,
                inh_hi: float = 1.0, delay_cap_ms: float = 20.0, dt_ms: float = 0.1) -> NativeNet:
    """Random K-out net of the 10k / 100k / 1M workloads (80/20 izh RS/FS)."""
    h = C.c_void_p()
    check(lib.ne2b_gen_random_kout(n, k, seed, w_scale, exc_hi, inh_hi, delay_cap_ms, dt_ms, C.byref(h)))
    return NativeNet(h)


def liquid(side: int, seed: int = 1, lambda_units: float = 2.0, radius_units: int = 6, w_rec: float = 3.0,
           n_inputs: int = 8, targets_per_input: int = 24, w_in: float = 12.0, model: int = _abi.MODEL_IZH,
           dt_ms: float = 0.1) -> NativeNet:
    """Local 3-D liquid of the batched / served workloads."""
    h = C.c_void_p()
    check(lib.ne2b_gen_liquid(side, seed, lambda_units, radius_units, w_rec, n_inputs, targets_per_input, w_in,
                              model, dt_ms, C.byref(h)))
    return NativeNet(h)


def _meta_dict(m: _abi.Ne2Meta) -> dict:
    return {f: getattr(m, f) for f, _ in m._fields_}


def load_ne2(path) -> tuple[NativeNet, dict]:
    """A reference `.ne2` network file (versions 1-7) as a library net, and
    the file's version and Meta (dt_ms, seed, conduction_speed,
    synapse_tau_ms, readout_tau_ms, noise_rate_hz, noise_kick_mv)."""
    h = C.c_void_p()
    m = _abi.Ne2Meta()
    check(lib.ne2b_net_load_ne2(os.fsencode(path), C.byref(h), C.byref(m)))
    return NativeNet(h), _meta_dict(m)


def from_ne2_bytes(data: bytes) -> tuple[NativeNet, dict]:
    """`load_ne2` from the file's bytes."""
    buf = (C.c_uint8 * len(data)).from_buffer_copy(data) if data else None
    h = C.c_void_p()
    m = _abi.Ne2Meta()
    check(lib.ne2b_net_from_ne2(buf, len(data), C.byref(h), C.byref(m)))
    return NativeNet(h), _meta_dict(m)


def config_from_meta(meta: dict, **overrides) -> _abi.Config:
    """The sim config a `.ne2` file asks for (its Meta), as Sim::new builds it."""
    kw = dict(dt_ms=meta["dt_ms"], synapse_tau_ms=meta["synapse_tau_ms"], readout_tau_ms=meta["readout_tau_ms"],
              noise_rate_hz=meta["noise_rate_hz"], noise_kick_mv=meta["noise_kick_mv"], seed=meta["seed"])
    kw.update(overrides)
    return _abi.default_config(**kw)


ADEX_TONIC = np.array([281.0, 30.0, -70.6, -50.4, 2.0, 4.0, 144.0, 80.5, -70.6, 20.0], dtype=np.float32)
ADEX_NONADAP = np.array([281.0, 30.0, -70.6, -50.4, 2.0, 0.0, 144.0, 0.0, -70.6, 20.0], dtype=np.float32)


def to_adex(net: NativeNet, exc_row=ADEX_TONIC, inh_row=ADEX_NONADAP) -> NativeNet:
    """Turn every neuron of a library net into AdEx (kind default rows)."""
    e = np.ascontiguousarray(exc_row, dtype=np.float32)
    i = np.ascontiguousarray(inh_row, dtype=np.float32)
    check(lib.ne2b_net_set_model_all(net._h, _abi.MODEL_ADEX, ptr(e), ptr(i), len(e)))
    check(lib.ne2b_net_desc_of(net._h, C.byref(net._desc)))
    return net
