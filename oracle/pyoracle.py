"""ctypes wrapper of the C parity oracle (oracle/ne2_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
the CPU-baseline leg of bench.py, never by the neuro_edit_v2_b200 package.
The oracle restates the reference CPU step (sim/src/cpu.rs:192-306) and the
net-format builders; see ne2_oracle.h for the parity pins.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libne2oracle.so")

EXC, INH, REGULAR = 0, 1, 2
IZH, ADEX = 0, 1
PMAX = 10


def build(force: bool = False) -> str:
    src = [os.path.join(HERE, f) for f in ("ne2_oracle.c", "ne2_oracle.h", "Makefile")]
    if force or not os.path.exists(LIB_PATH) or any(os.path.getmtime(s) > os.path.getmtime(LIB_PATH) for s in src):
        subprocess.run(["make", "-C", HERE, "-s"], check=True)
    return LIB_PATH


class Cfg(C.Structure):
    _fields_ = [
        ("dt_ms", C.c_float), ("synapse_tau_ms", C.c_float), ("readout_tau_ms", C.c_float),
        ("noise_rate_hz", C.c_float), ("noise_kick_mv", C.c_float), ("seed", C.c_uint64),
        ("record_spikes", C.c_int), ("spike_record_steps", C.c_uint32), ("int_weights", C.c_int),
        ("gauss_sd", C.c_float), ("exp_mode", C.c_int),
    ]


class Rng(C.Structure):
    _fields_ = [("s", C.c_uint64 * 4)]


class Csr(C.Structure):
    _fields_ = [("n", C.c_uint32), ("e", C.c_uint64), ("src_ptr", C.c_void_p), ("tgt", C.c_void_p),
                ("w", C.c_void_p), ("delay", C.c_void_p), ("tau", C.c_void_p)]


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        vp, u32, u64, f32, f64, i32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_float, C.c_double, C.c_int
        sigs = {
            "ne2o_rng_seed": (None, [vp, u64]), "ne2o_rng_next_u64": (u64, [vp]), "ne2o_rng_f64": (f64, [vp]),
            "ne2o_rng_below": (u64, [vp, u64]),
            "ne2o_net_new": (vp, []), "ne2o_net_free": (None, [vp]),
            "ne2o_net_add_neuron": (u32, [vp, f32, f32, f32, i32]),
            "ne2o_net_set_model": (None, [vp, u32, i32, vp, i32]),
            "ne2o_net_set_kind": (None, [vp, u32, i32]),
            "ne2o_net_connect": (u64, [vp, u32, u32, f32]),
            "ne2o_net_push_synapse": (None, [vp, u32, u32, f32, f32, f32]),
            "ne2o_net_add_input": (u32, [vp, vp, vp, u32]),
            "ne2o_create_2d_grid": (u32, [vp, u32, u32, f32, f32, f32, f32, vp]),
            "ne2o_create_3d_grid": (u32, [vp, u32, u32, u32, f32, f32, f32, f32, vp]),
            "ne2o_create_connections": (None, [vp, vp, u32, f64, f64, f32, vp]),
            "ne2o_set_exc_inh": (None, [vp, vp, u32, f64, vp]),
            "ne2o_set_exc_inh_exact": (None, [vp, vp, u32, u32, vp]),
            "ne2o_bench_net": (vp, [u32, u32, u64, f32, f32]),
            "ne2o_gen_random_kout": (vp, [u32, u32, u64, f32, f32, f32, f32]),
            "ne2o_gen_liquid": (vp, [u32, u64, f64, i32, f32, u32, u32, f32, i32]),
            "ne2o_synapse_csr": (i32, [vp, f32, vp, C.c_char_p, C.c_size_t]),
            "ne2o_csr_free": (None, [vp]),
            "ne2o_noise_hash": (u32, [u32, u64, u64]),
            "ne2o_noise_fires": (i32, [u32, u64, u64, f32]),
            "ne2o_gauss_numer": (C.c_int64, [u32, u64, u64]),
            "ne2o_gauss_scale": (f32, [f32]),
            "ne2o_det_expf": (f32, [f32]),
            "ne2o_expf_mismatches": (u64, [vp, f32, f32, u32, u32, vp]),
            "ne2o_expf_max_ulp": (u64, [vp, f32, f32, u32, u32, vp]),
            "ne2o_expf_ref": (f32, [f32]),
            "ne2o_fit_ridge_multi": (None, [vp, u32, u32, vp, u32, f64, vp]),
            "ne2o_fit_ridge": (None, [vp, u32, u32, vp, f32, vp]),
            "ne2o_cholesky_solve": (i32, [vp, vp, u32, vp]),
            "ne2o_cfg_default": (None, [vp]),
            "ne2o_sim_new": (vp, [vp, vp, C.c_char_p, C.c_size_t]),
            "ne2o_sim_free": (None, [vp]), "ne2o_sim_step": (None, [vp]),
            "ne2o_sim_run_steps": (None, [vp, u64]), "ne2o_sim_reset_state": (None, [vp]),
            "ne2o_sim_t": (u64, [vp]), "ne2o_sim_n": (u32, [vp]), "ne2o_sim_ring_depth": (u32, [vp]),
            "ne2o_sim_spikes_total": (u64, [vp]), "ne2o_sim_mean_rate_hz": (f64, [vp]),
            "ne2o_sim_state": (i32, [vp, u32, vp]), "ne2o_sim_syn_current": (None, [vp, vp]),
            "ne2o_sim_trace": (None, [vp, vp]), "ne2o_sim_pn_total": (None, [vp, vp]),
            "ne2o_sim_spike_row": (u32, [vp, u32, vp]),
            "ne2o_sim_spike_counts": (i32, [vp, u64, vp, C.c_char_p, C.c_size_t]),
            "ne2o_sim_set_v_watch": (None, [vp, vp, u32]),
            "ne2o_sim_drain_watch": (u32, [vp, vp]),
            "ne2o_sim_set_grid_watches": (None, [vp, vp, vp, u32]),
            "ne2o_sim_grid_traces": (None, [vp, C.c_float, vp]),
            "ne2o_sim_last_step_spikes": (u32, [vp, vp]),
            "ne2o_sim_set_external": (None, [vp, u32, f32]),
            "ne2o_sim_set_input_constant": (None, [vp, u32, f32]),
            "ne2o_sim_play_input": (None, [vp, u32, vp, u64]),
            "ne2o_sim_loop_input": (None, [vp, u32, vp, u64]),
            "ne2o_sim_set_noise": (None, [vp, f32, f32]),
            "ne2o_sim_stim_value": (f32, [vp, u32, u64]),
            "ne2o_sim_fingerprint": (u64, [vp, u32]),
            "ne2o_net_n": (u32, [vp]), "ne2o_net_ns": (u64, [vp]),
            "ne2o_net_models": (None, [vp, vp, vp]), "ne2o_net_kinds": (None, [vp, vp]),
            "ne2o_net_ninputs": (u32, [vp]), "ne2o_net_input_entries": (u32, [vp]),
            "ne2o_net_inputs": (None, [vp, vp, vp, vp]),
            "ne2o_net_synapses": (None, [vp, vp, vp, vp, vp, vp]),
            "ne2o_net_positions": (None, [vp, vp]),
        }
        for name, (res, args) in sigs.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data if a is not None else None


def rng(seed: int) -> Rng:
    r = Rng()
    lib().ne2o_rng_seed(C.byref(r), seed)
    return r


def cfg(**kw) -> Cfg:
    c = Cfg()
    lib().ne2o_cfg_default(C.byref(c))
    for k, v in kw.items():
        setattr(c, k, v)
    return c


class ONet:
    """An oracle `Network` (net-format/src/network.rs) with the builders."""

    def __init__(self, handle=None):
        self.h = handle if handle is not None else lib().ne2o_net_new()

    def __del__(self):
        if getattr(self, "h", None):
            lib().ne2o_net_free(self.h)
            self.h = None

    @classmethod
    def bench_net(cls, n, k, seed, w_scale=0.7, w_inh=5.0):
        return cls(lib().ne2o_bench_net(n, k, seed, w_scale, w_inh))

    @classmethod
    def random_kout(cls, n, k=100, seed=1, w_scale=0.7, exc_hi=0.5, inh_hi=1.0, delay_cap_ms=20.0):
        return cls(lib().ne2o_gen_random_kout(n, k, seed, w_scale, exc_hi, inh_hi, delay_cap_ms))

    @classmethod
    def liquid(cls, side, seed=1, lambda_units=2.0, radius_units=6, w_rec=3.0, n_inputs=8, targets_per_input=24,
               w_in=12.0, model=IZH):
        return cls(lib().ne2o_gen_liquid(side, seed, lambda_units, radius_units, w_rec, n_inputs,
                                         targets_per_input, w_in, model))

    @property
    def n(self) -> int:
        return int(lib().ne2o_net_n(self.h))

    @property
    def ns(self) -> int:
        return int(lib().ne2o_net_ns(self.h))

    def add_neuron(self, x, y, z, kind=EXC) -> int:
        return int(lib().ne2o_net_add_neuron(self.h, x, y, z, kind))

    def set_model(self, i, model, params):
        p = np.ascontiguousarray(params, dtype=np.float32)
        lib().ne2o_net_set_model(self.h, i, model, _p(p), len(p))

    def set_kind(self, i, kind):
        lib().ne2o_net_set_kind(self.h, i, kind)

    def connect(self, a, b, w) -> int:
        return int(lib().ne2o_net_connect(self.h, a, b, w))

    def push_synapse(self, a, b, w, delay_ms, tau_ms=0.0):
        lib().ne2o_net_push_synapse(self.h, a, b, w, delay_ms, tau_ms)

    def add_input(self, targets) -> int:
        t = np.ascontiguousarray([x[0] for x in targets], dtype=np.uint32)
        w = np.ascontiguousarray([x[1] for x in targets], dtype=np.float32)
        return int(lib().ne2o_net_add_input(self.h, _p(t), _p(w), len(t)))

    def create_2d_grid(self, w, h, dist, center=(0.0, 0.0, 0.0)) -> np.ndarray:
        m = np.zeros(w * h, dtype=np.uint32)
        lib().ne2o_create_2d_grid(self.h, w, h, dist, *center, _p(m))
        return m

    def create_3d_grid(self, w, h, d, dist, center=(0.0, 0.0, 0.0)) -> np.ndarray:
        m = np.zeros(w * h * d, dtype=np.uint32)
        lib().ne2o_create_3d_grid(self.h, w, h, d, dist, *center, _p(m))
        return m

    def create_connections(self, members, scaling, lam, weight, r: Rng):
        m = np.ascontiguousarray(members, dtype=np.uint32)
        lib().ne2o_create_connections(self.h, _p(m), len(m), scaling, lam, weight, C.byref(r))

    def set_exc_inh(self, members, frac, r: Rng):
        m = np.ascontiguousarray(members, dtype=np.uint32)
        lib().ne2o_set_exc_inh(self.h, _p(m), len(m), frac, C.byref(r))

    def set_exc_inh_exact(self, members, n_inh, r: Rng):
        m = np.ascontiguousarray(members, dtype=np.uint32)
        lib().ne2o_set_exc_inh_exact(self.h, _p(m), len(m), n_inh, C.byref(r))

    def synapses(self):
        e = self.ns
        src = np.zeros(e, np.uint32); tgt = np.zeros(e, np.uint32); w = np.zeros(e, np.float32)
        d = np.zeros(e, np.float32); tau = np.zeros(e, np.float32)
        lib().ne2o_net_synapses(self.h, _p(src), _p(tgt), _p(w), _p(d), _p(tau))
        return src, tgt, w, d, tau

    def models(self):
        n = self.n
        model = np.zeros(n, np.uint8)
        params = np.zeros((n, PMAX), np.float32)
        lib().ne2o_net_models(self.h, _p(model), _p(params))
        return model, params

    def kinds(self) -> np.ndarray:
        k = np.zeros(self.n, np.uint8)
        lib().ne2o_net_kinds(self.h, _p(k))
        return k

    def csr(self, dt_ms=0.1):
        """`Network::synapse_csr` (network.rs:654-692) -> numpy arrays."""
        c = Csr()
        err = C.create_string_buffer(512)
        if lib().ne2o_synapse_csr(self.h, dt_ms, C.byref(c), err, 512) != 0:
            raise ValueError(err.value.decode())
        n, e = c.n, c.e

        def cp(p, count, ct, dt):
            if count == 0:
                return np.zeros(0, dt)
            return np.ctypeslib.as_array(C.cast(p, C.POINTER(ct)), shape=(count,)).astype(dt, copy=True)

        out = dict(src_ptr=cp(c.src_ptr, n + 1, C.c_uint32, np.uint32), tgt=cp(c.tgt, e, C.c_uint32, np.uint32),
                   w=cp(c.w, e, C.c_float, np.float32), delay=cp(c.delay, e, C.c_uint16, np.uint16),
                   tau=cp(c.tau, e, C.c_float, np.float32))
        lib().ne2o_csr_free(C.byref(c))
        return out

    def stim_map(self):
        """`StimMap::from_network` (sim/src/stim.rs:26-48)."""
        L = lib()
        ni = int(L.ne2o_net_ninputs(self.h))
        ne = int(L.ne2o_net_input_entries(self.h))
        in_ptr = np.zeros(ni + 1, np.uint32); in_tgt = np.zeros(ne, np.uint32); in_w = np.zeros(ne, np.float32)
        if ni:
            L.ne2o_net_inputs(self.h, _p(in_ptr), _p(in_tgt), _p(in_w))
        n = self.n
        per = [[] for _ in range(n)]
        for k in range(ni):
            for j in range(in_ptr[k], in_ptr[k + 1]):
                if in_tgt[j] < n:
                    per[in_tgt[j]].append((k, in_w[j]))
        ptr = np.zeros(n + 1, np.uint32)
        for i in range(n):
            ptr[i + 1] = ptr[i] + len(per[i])
        inp = np.array([k for row in per for k, _ in row], dtype=np.uint32)
        w = np.array([x for row in per for _, x in row], dtype=np.float32)
        return ni, ptr, inp, w

    def flat(self, dt_ms=0.1):
        """The flat arrays the product's C ABI takes (ne2b_net_desc)."""
        from neuro_edit_v2_b200.net import FlatNet  # the product's descriptor type, not its compute

        c = self.csr(dt_ms)
        model, params = self.models()
        ni, ptr, inp, w = self.stim_map()
        tau = c["tau"] if c["tau"] is not None and np.any(c["tau"] > 0) else None
        return FlatNet(model=model, params=params, src_ptr=c["src_ptr"], tgt=c["tgt"], w=c["w"],
                       delay_steps=c["delay"], n_inputs=ni, stim_ptr=ptr if ni else None,
                       stim_input=inp if ni else None, stim_w=w if ni else None, kind=self.kinds(), tau_ms=tau)


class OSim:
    """The oracle `CpuSim` (sim/src/cpu.rs)."""

    def __init__(self, net: ONet, c: Cfg):
        err = C.create_string_buffer(512)
        self.h = lib().ne2o_sim_new(net.h, C.byref(c), err, 512)
        if not self.h:
            raise ValueError(err.value.decode())
        self.n = int(lib().ne2o_sim_n(self.h))

    def __del__(self):
        if getattr(self, "h", None):
            lib().ne2o_sim_free(self.h)
            self.h = None

    def run_steps(self, k):
        lib().ne2o_sim_run_steps(self.h, k)

    def step(self):
        lib().ne2o_sim_step(self.h)

    def reset_state(self):
        lib().ne2o_sim_reset_state(self.h)

    @property
    def t(self) -> int:
        return int(lib().ne2o_sim_t(self.h))

    def ring_depth(self) -> int:
        return int(lib().ne2o_sim_ring_depth(self.h))

    def spikes_total(self) -> int:
        return int(lib().ne2o_sim_spikes_total(self.h))

    def mean_rate_hz(self) -> float:
        return float(lib().ne2o_sim_mean_rate_hz(self.h))

    def state(self, slot) -> np.ndarray:
        out = np.zeros(self.n, np.float32)
        lib().ne2o_sim_state(self.h, slot, _p(out))
        return out

    def syn_current(self) -> np.ndarray:
        out = np.zeros(self.n, np.float32)
        lib().ne2o_sim_syn_current(self.h, _p(out))
        return out

    def trace(self) -> np.ndarray:
        out = np.zeros(self.n, np.float32)
        lib().ne2o_sim_trace(self.h, _p(out))
        return out

    def pn_total(self) -> np.ndarray:
        out = np.zeros(self.n, np.uint64)
        lib().ne2o_sim_pn_total(self.h, _p(out))
        return out

    def spike_row(self, back) -> np.ndarray | None:
        out = np.zeros((self.n + 63) // 64 or 1, np.uint64)
        k = lib().ne2o_sim_spike_row(self.h, back, _p(out))
        return out[:k] if k else None

    def spike_counts(self, rows) -> np.ndarray:
        out = np.zeros(max(self.n, 1), np.uint32)
        err = C.create_string_buffer(512)
        if lib().ne2o_sim_spike_counts(self.h, rows, _p(out), err, 512) != 0:
            raise ValueError(err.value.decode())
        return out[: self.n]

    def last_step_spikes(self) -> np.ndarray:
        out = np.zeros(max(self.n, 1), np.uint32)
        k = lib().ne2o_sim_last_step_spikes(self.h, _p(out))
        return out[:k]

    def set_external(self, i, amps):
        lib().ne2o_sim_set_external(self.h, i, amps)

    def set_input_constant(self, k, v):
        lib().ne2o_sim_set_input_constant(self.h, k, v)

    def play_input(self, k, series):
        s = np.ascontiguousarray(series, dtype=np.float32)
        lib().ne2o_sim_play_input(self.h, k, _p(s), len(s))

    def loop_input(self, k, series):
        s = np.ascontiguousarray(series, dtype=np.float32)
        lib().ne2o_sim_loop_input(self.h, k, _p(s), len(s))

    def set_noise(self, rate, kick):
        lib().ne2o_sim_set_noise(self.h, rate, kick)

    def stim_value(self, k, t) -> float:
        return float(lib().ne2o_sim_stim_value(self.h, k, t))

    def fingerprint(self, rows) -> int:
        return int(lib().ne2o_sim_fingerprint(self.h, rows))

    # editor watches (cpu.rs:308-407)
    def set_v_watch(self, ids):
        self._watch = np.ascontiguousarray(ids, dtype=np.uint32)
        lib().ne2o_sim_set_v_watch(self.h, _p(self._watch), len(self._watch))

    def drain_watch(self) -> np.ndarray:
        """[state slot][watch][samples oldest first]"""
        w = len(getattr(self, "_watch", ()))
        out = np.zeros(max(2 * w * 4096, 1), np.float32)
        c = lib().ne2o_sim_drain_watch(self.h, _p(out))
        return out[: 2 * w * c].reshape(2, w, c)

    def set_grid_watches(self, groups):
        ptr = np.zeros(len(groups) + 1, np.uint32)
        ptr[1:] = np.cumsum([len(g) for g in groups])
        members = np.ascontiguousarray(np.concatenate([np.asarray(g, np.uint32) for g in groups])
                                       if groups else np.zeros(0, np.uint32), dtype=np.uint32)
        self._gw = (members, ptr)
        lib().ne2o_sim_set_grid_watches(self.h, _p(members), _p(ptr), len(groups))

    def grid_traces(self, tau_ms) -> list:
        members, ptr = getattr(self, "_gw", (np.zeros(0, np.uint32), np.zeros(1, np.uint32)))
        out = np.zeros(max(int(ptr[-1]), 1), np.float32)
        lib().ne2o_sim_grid_traces(self.h, tau_ms, _p(out))
        return [out[ptr[g]:ptr[g + 1]].copy() for g in range(len(ptr) - 1)]


def noise_hash(i, t, seed) -> int:
    return int(lib().ne2o_noise_hash(i, t, seed))


def gauss_numer(i, t, seed) -> int:
    return int(lib().ne2o_gauss_numer(i, t, seed))


def det_expf(x) -> float:
    return float(lib().ne2o_det_expf(x))


def fit_ridge_multi(x, labels, k: int, lam: float) -> np.ndarray:
    """sim/src/readout.rs:190-252 on a [T x F] design: [k x (F + 1)] weights, bias last."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    lab = np.ascontiguousarray(labels, dtype=np.uint32)
    t, f = x.shape
    w = np.zeros((k, f + 1), np.float64)
    lib().ne2o_fit_ridge_multi(_p(x), t, f, _p(lab), k, float(lam), _p(w))
    return w


def fit_ridge(x, y, lam: float) -> np.ndarray:
    """sim/src/readout.rs:103-141 on a [T x F] design: F + 1 weights, bias last."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    y = np.ascontiguousarray(y, dtype=np.float32)
    t, f = x.shape
    w = np.zeros(f + 1, np.float64)
    lib().ne2o_fit_ridge(_p(x), t, f, _p(y), float(lam), _p(w))
    return w
