"""Python mirror of the reference `sim::Backend` trait (sim/src/lib.rs:119-184)
over the B200 C ABI.

`B200Sim` exposes the same methods, argument meanings and error behaviour as
`CpuSim` / `CudaSim` (sim/src/cpu.rs, sim/src/cuda.rs): stepping is
asynchronous, every read synchronises, `spike_counts` raises on a window that
the record ring can no longer answer.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import Ne2bError, check, lib, ptr


class SpikeWindowError(Ne2bError):
    """`spike_counts` window between the record depth and t (cpu.rs:437-442)."""


def _cfg(cfg: _abi.Config | None, **kw) -> _abi.Config:
    if cfg is None:
        return _abi.default_config(**kw)
    for k, v in kw.items():
        setattr(cfg, k, v)
    return cfg


def _list_array(a, dtype):
    """(length, pointer, keep-alive) of a 1-D synapse-list column: a numpy array (made
    contiguous in `dtype`) or a contiguous device array of that dtype (any
    object with __cuda_array_interface__, e.g. a CUDA torch tensor), whose
    pointer is passed as it is."""
    cai = getattr(a, "__cuda_array_interface__", None)
    if cai is not None:
        if np.dtype(cai["typestr"]) != np.dtype(dtype) or len(cai["shape"]) != 1:
            raise ValueError(f"a device list column must be 1-D {np.dtype(dtype).name}")
        if cai.get("strides") not in (None, (np.dtype(dtype).itemsize,)):
            raise ValueError("a device list column must be contiguous")
        return int(cai["shape"][0]), int(cai["data"][0]), a
    a = np.ascontiguousarray(a, dtype=dtype).reshape(-1)
    return len(a), a.ctypes.data, a


class B200Sim:
    """One network on one B200: `Backend` with kind B200."""

    def __init__(self, net, cfg: _abi.Config | None = None, device: int = 0, **cfg_kw):
        self._net = net  # keeps the arrays behind the descriptor alive during create
        self.cfg = _cfg(cfg, **cfg_kw)
        h = C.c_void_p()
        check(lib.ne2b_create(C.byref(net.desc()), C.byref(self.cfg), device, C.byref(h)))
        self._h = h
        n = C.c_uint32()
        check(lib.ne2b_n(self._h, C.byref(n)))
        self._n = int(n.value)
        self.n_inputs = int(net.n_inputs)

    @classmethod
    def from_synapses(cls, model, params, kind, src, tgt, w, delay_ms, cfg: _abi.Config | None = None,
                      device: int = 0, x0=None, **cfg_kw) -> "B200Sim":
        """A sim whose synapse CSR is built on the GPU from a plain synapse
        list (`Network::synapse_csr`, net-format/src/network.rs:654-692):
        equal to `B200Sim(from_synapses(...))` bit for bit."""
        self = cls.__new__(cls)
        self.cfg = _cfg(cfg, **cfg_kw)
        model = np.ascontiguousarray(model, dtype=np.uint8)
        params = np.ascontiguousarray(params, dtype=np.float32)
        cols = [_list_array(a, t) for a, t in ((kind, np.uint8), (src, np.uint32), (tgt, np.uint32),
                                               (w, np.float32), (delay_ms, np.float32))]
        (nk, pk, _), (e, ps, _), (nt, pt, _), (nw, pw, _), (nd, pd, _) = cols
        x0 = None if x0 is None else np.ascontiguousarray(x0, dtype=np.float32)
        n = len(model)
        if nk != n or not nt == nw == nd == e:
            raise ValueError("one kind per neuron and equal-length src, tgt, w, delay_ms")
        d = _abi.NetDesc()
        d.n = n
        d.model, d.params = model.ctypes.data, params.ctypes.data
        d.param_stride = params.shape[1] if params.ndim == 2 else (params.size // max(n, 1))
        d.x0 = None if x0 is None else x0.ctypes.data
        h = C.c_void_p()
        check(lib.ne2b_create_from_synapses(C.byref(d), pk, e, ps, pt, pw, pd, C.byref(self.cfg), device,
                                            C.byref(h)))
        self._h = h
        self._net = None
        self._n = n
        self.n_inputs = 0
        return self

    def syn_count(self) -> int:
        e = C.c_uint64()
        check(lib.ne2b_syn_count(self._h, C.byref(e)))
        return int(e.value)

    def read_csr(self):
        """The device CSR: (rowptr u32[n+1], tgt u32[E], weight bits u32[E]
        (int32 fixed point with the int ring, else f32 bits), delay steps
        u16[E])."""
        e = self.syn_count()
        rowptr = np.empty(self._n + 1, np.uint32)
        tgt = np.empty(e, np.uint32)
        wb = np.empty(e, np.uint32)
        dl = np.empty(e, np.uint16)
        check(lib.ne2b_read_csr(self._h, rowptr.ctypes.data, tgt.ctypes.data, wb.ctypes.data, dl.ctypes.data))
        return rowptr, tgt, wb, dl

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib.ne2b_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # --- Backend (sim/src/lib.rs:119-184) -------------------------------
    def kind(self) -> str:
        return "B200"

    def n(self) -> int:
        return self._n

    def step_count(self) -> int:
        t = C.c_uint64()
        check(lib.ne2b_step_count(self._h, C.byref(t)))
        return int(t.value)

    def time_ms(self) -> float:
        v = C.c_double()
        check(lib.ne2b_time_ms(self._h, C.byref(v)))
        return float(v.value)

    def ring_depth(self) -> int:
        d = C.c_uint32()
        check(lib.ne2b_ring_depth(self._h, C.byref(d)))
        return int(d.value)

    def run_steps(self, n: int) -> None:
        check(lib.ne2b_run_steps(self._h, int(n)))

    def run_ms(self, ms: float) -> None:
        check(lib.ne2b_run_ms(self._h, float(ms)))

    def reset_state(self) -> None:
        check(lib.ne2b_reset_state(self._h))

    def synchronize(self) -> None:
        check(lib.ne2b_synchronize(self._h))

    def dev_mem_bytes(self) -> int:
        b = C.c_uint64()
        check(lib.ne2b_dev_mem_bytes(self._h, C.byref(b)))
        return int(b.value)

    def trace(self) -> np.ndarray:
        out = np.empty(self._n, dtype=np.float32)
        check(lib.ne2b_read_trace(self._h, ptr(out)))
        return out

    def state(self, slot: int) -> np.ndarray:
        if slot >= 2:
            return np.zeros(0, dtype=np.float32)  # cpu.rs:346-349: empty for unknown slots
        out = np.empty(self._n, dtype=np.float32)
        check(lib.ne2b_read_state(self._h, slot, ptr(out)))
        return out

    def v(self) -> np.ndarray:
        return self.state(0)

    def syn_current(self) -> np.ndarray:
        out = np.empty(self._n, dtype=np.float32)
        check(lib.ne2b_read_syn_current(self._h, ptr(out)))
        return out

    def last_spikes(self) -> np.ndarray:
        cnt = C.c_uint32()
        check(lib.ne2b_last_spikes(self._h, None, 0, C.byref(cnt)))
        out = np.empty(max(cnt.value, 1), dtype=np.uint32)
        check(lib.ne2b_last_spikes(self._h, ptr(out), cnt.value, C.byref(cnt)))
        return out[: cnt.value]

    def spike_counts(self, rows: int) -> np.ndarray:
        out = np.empty(self._n, dtype=np.uint32)
        st = lib.ne2b_spike_counts(self._h, min(int(rows), 2**64 - 1), ptr(out))
        if st == _abi.NE2B_EWINDOW:
            raise SpikeWindowError(st, lib.ne2b_last_error().decode())
        check(st)
        return out

    def spike_counts_noalloc(self, rows: int) -> np.ndarray:
        """spike_counts that allocates no device memory (fixed 1,048,576-neuron
        scratch compiled into the library; overlapping calls race)."""
        out = np.empty(self._n, dtype=np.uint32)
        st = lib.ne2b_spike_counts_noalloc(self._h, min(int(rows), 2**64 - 1), ptr(out))
        if st == _abi.NE2B_EWINDOW:
            raise SpikeWindowError(st, lib.ne2b_last_error().decode())
        check(st)
        return out

    def spike_row(self, back: int) -> np.ndarray | None:
        out = np.empty((self._n + 63) // 64, dtype=np.uint64)
        st = lib.ne2b_spike_row(self._h, int(back), ptr(out))
        if st == _abi.NE2B_ENODATA:
            return None
        check(st)
        return out

    def spikes_total(self) -> int:
        v = C.c_uint64()
        check(lib.ne2b_spikes_total(self._h, C.byref(v)))
        return int(v.value)

    def mean_rate_hz(self) -> float:
        v = C.c_double()
        check(lib.ne2b_mean_rate_hz(self._h, C.byref(v)))
        return float(v.value)

    def set_input_constant(self, input: int, value: float) -> None:
        check(lib.ne2b_set_input_constant(self._h, input, value))

    def input_values(self) -> np.ndarray:
        out = np.empty(max(self.n_inputs, 1), dtype=np.float32)
        check(lib.ne2b_input_values(self._h, ptr(out)))
        return out[: self.n_inputs]

    def play_input(self, input: int, series) -> None:
        s = np.ascontiguousarray(series, dtype=np.float32)
        check(lib.ne2b_play_input(self._h, input, ptr(s), len(s)))

    def loop_input(self, input: int, series) -> None:
        s = np.ascontiguousarray(series, dtype=np.float32)
        check(lib.ne2b_loop_input(self._h, input, ptr(s), len(s)))

    def external(self) -> np.ndarray:
        out = np.empty(self._n, dtype=np.float32)
        check(lib.ne2b_external(self._h, ptr(out)))
        return out

    def set_external(self, neuron: int, amps: float) -> None:
        check(lib.ne2b_set_external(self._h, neuron, amps))

    def set_external_all(self, ext) -> None:
        e = np.ascontiguousarray(ext, dtype=np.float32)
        check(lib.ne2b_set_external_all(self._h, ptr(e), len(e)))

    def set_noise(self, rate_hz: float, kick_mv: float) -> None:
        check(lib.ne2b_set_noise(self._h, rate_hz, kick_mv))

    def set_gauss_noise(self, sd: float) -> None:
        check(lib.ne2b_set_gauss_noise(self._h, sd))

    # --- editor observability (lib.rs:164-176) --------------------------
    def set_v_watch(self, ids) -> None:
        a = np.ascontiguousarray(ids, dtype=np.uint32)
        check(lib.ne2b_set_v_watch(self._h, ptr(a), len(a)))

    def drain_watch(self) -> np.ndarray:
        """[state slot][watch][samples oldest first] since the last drain."""
        w, c = C.c_uint32(), C.c_uint32()
        check(lib.ne2b_watch_count(self._h, C.byref(w), C.byref(c)))
        out = np.zeros(max(2 * w.value * c.value, 1), np.float32)
        got = C.c_uint32()
        check(lib.ne2b_drain_watch(self._h, ptr(out), C.byref(got)))
        return out[: 2 * w.value * got.value].reshape(2, w.value, got.value)

    def set_grid_watches(self, groups) -> None:
        gp = np.zeros(len(groups) + 1, np.uint32)
        gp[1:] = np.cumsum([len(g) for g in groups])
        members = np.ascontiguousarray(np.concatenate([np.asarray(g, np.uint32) for g in groups])
                                       if groups else np.zeros(0, np.uint32), dtype=np.uint32)
        check(lib.ne2b_set_grid_watches(self._h, ptr(members), ptr(gp), len(groups)))
        self._gw_ptr = gp

    def grid_traces(self, tau_ms: float) -> list:
        gp = getattr(self, "_gw_ptr", np.zeros(1, np.uint32))
        out = np.zeros(max(int(gp[-1]), 1), np.float32)
        check(lib.ne2b_grid_traces(self._h, tau_ms, ptr(out)))
        return [out[gp[g]:gp[g + 1]].copy() for g in range(len(gp) - 1)]

    # --- kernel selection (new) -----------------------------------------
    def set_kernel_mode(self, mode: int) -> None:
        """_abi.KERNEL_AUTO / KERNEL_STREAM / KERNEL_RESIDENT."""
        check(lib.ne2b_set_kernel_mode(self._h, mode))

    def kernel_mode(self) -> tuple[int, bool]:
        m, r = C.c_int32(), C.c_int32()
        check(lib.ne2b_kernel_mode(self._h, C.byref(m), C.byref(r)))
        return int(m.value), bool(r.value)

    def autotune(self, steps_per_trial: int = 128) -> dict:
        """Pick the fastest kernel and tile shape for this net (state kept)."""
        check(lib.ne2b_autotune(self._h, steps_per_trial))
        return self.tiling()

    def set_tile_shape(self, block: int, neurons_per_thread: int, blocks_per_sm: int = 0) -> None:
        check(lib.ne2b_set_tile_shape(self._h, block, neurons_per_thread, blocks_per_sm))

    def set_delivery_warps(self, on: bool) -> None:
        """Separate delivery warps in the streaming step kernel (one-net sims;
        tile blocks of 128, 256 or 512 threads); results are unchanged."""
        check(lib.ne2b_set_delivery_warps(self._h, 1 if on else 0))

    def delivery_warps(self) -> tuple[bool, bool]:
        """(requested, used by the kernel that runs)."""
        a, b = C.c_int32(), C.c_int32()
        check(lib.ne2b_delivery_warps(self._h, C.byref(a), C.byref(b)))
        return bool(a.value), bool(b.value)

    def tiling(self) -> dict:
        a, b, c = C.c_uint32(), C.c_uint32(), C.c_uint32()
        check(lib.ne2b_tile_shape(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return {"kernel": "resident" if self.kernel_mode()[1] else "stream", "block": int(a.value),
                "neurons_per_thread": int(b.value), "blocks_per_sm": int(c.value),
                "delivery_warps": self.delivery_warps()[1]}

    # --- instrumentation (new) ------------------------------------------
    def stream_handle(self) -> int:
        """The cudaStream_t this sim launches on (for CUDA-event timing)."""
        p = C.c_void_p()
        check(lib.ne2b_stream(self._h, C.byref(p)))
        return int(p.value or 0)

    def kernel_launches(self) -> int:
        v = C.c_uint64()
        check(lib.ne2b_kernel_launches(self._h, C.byref(v)))
        return int(v.value)

    # --- on-device window counts (new) ---------------------------------
    def windows_done(self) -> int:
        c = C.c_uint32()
        check(lib.ne2b_windows_done(self._h, C.byref(c)))
        return int(c.value)

    def window_counts(self, window: int) -> np.ndarray:
        out = np.empty(self._n, dtype=np.uint16)
        check(lib.ne2b_window_counts(self._h, window, ptr(out)))
        return out


class Batch:
    """Many independent networks stepped together in one kernel per step."""

    def __init__(self, nets, cfgs, device: int = 0):
        self._nets = list(nets)
        descs = (_abi.NetDesc * len(self._nets))(*[n.desc() for n in self._nets])
        cfg_arr = (_abi.Config * len(cfgs))(*cfgs)
        h = C.c_void_p()
        check(lib.ne2b_batch_create(descs, cfg_arr, len(self._nets), device, C.byref(h)))
        self._h = h
        self.sizes = [int(n.n) for n in self._nets]

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib.ne2b_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def play_input(self, net: int, input: int, series) -> None:
        s = np.ascontiguousarray(series, dtype=np.float32)
        check(lib.ne2b_batch_play_input(self._h, net, input, ptr(s), len(s)))

    def set_input_matrix(self, net: int, inputs) -> None:
        """Device-resident [steps x n_inputs] inputs of one net from its current step."""
        x = np.ascontiguousarray(inputs, dtype=np.float32)
        check(lib.ne2b_batch_set_input_matrix(self._h, net, ptr(x), x.shape[0]))

    def run_steps(self, n: int) -> None:
        check(lib.ne2b_batch_run_steps(self._h, int(n)))

    def reset_state(self) -> None:
        check(lib.ne2b_batch_reset_state(self._h))

    def synchronize(self) -> None:
        check(lib.ne2b_batch_synchronize(self._h))

    def window_counts(self, net: int, window: int) -> np.ndarray:
        out = np.empty(self.sizes[net], dtype=np.uint16)
        check(lib.ne2b_batch_window_counts(self._h, net, window, ptr(out)))
        return out

    def fit_ridge_multi(self, nets, windows: int, labels, k: int, lam: float) -> np.ndarray:
        """Ridge readout (readout.rs:190-252) trained on the device from the
        window counts of `nets` (one trial each, features [windows][n]):
        [k x (windows * n + 1)] weights, bias last."""
        ns = np.ascontiguousarray(nets, dtype=np.uint32)
        lab = np.ascontiguousarray(labels, dtype=np.uint32)
        if lab.shape != ns.shape:
            raise ValueError("one label per trial")
        n = self.sizes[int(ns[0])]
        w = np.zeros((k, windows * n + 1), np.float64)
        nf = C.c_uint32()
        check(lib.ne2b_batch_fit_ridge_multi(self._h, ptr(ns), len(ns), windows, ptr(lab), k, float(lam),
                                             C.byref(nf), ptr(w)))
        return w

    def fit_ridge(self, nets, windows: int, y, lam: float) -> np.ndarray:
        """Binary ridge readout (readout.rs:103-141) trained on the device
        from the window counts of `nets`: windows * n + 1 weights, bias last."""
        ns = np.ascontiguousarray(nets, dtype=np.uint32)
        yy = np.ascontiguousarray(y, dtype=np.float32)
        if yy.shape != ns.shape:
            raise ValueError("one target per trial")
        n = self.sizes[int(ns[0])]
        w = np.zeros(windows * n + 1, np.float64)
        nf = C.c_uint32()
        check(lib.ne2b_batch_fit_ridge(self._h, ptr(ns), len(ns), windows, ptr(yy), float(lam), C.byref(nf), ptr(w)))
        return w

    def spikes_total(self, net: int) -> int:
        v = C.c_uint64()
        check(lib.ne2b_batch_spikes_total(self._h, net, C.byref(v)))
        return int(v.value)

    def state(self, net: int, slot: int) -> np.ndarray:
        out = np.empty(self.sizes[net], dtype=np.float32)
        check(lib.ne2b_batch_read_state(self._h, net, slot, ptr(out)))
        return out

    def autotune(self, steps_per_trial: int = 128) -> tuple[int, int, int]:
        check(lib.ne2b_batch_autotune(self._h, steps_per_trial))
        return self.tile_shape()

    def tile_shape(self) -> tuple[int, int, int]:
        a, b, c = C.c_uint32(), C.c_uint32(), C.c_uint32()
        check(lib.ne2b_batch_tile_shape(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return int(a.value), int(b.value), int(c.value)

    def set_tile_shape(self, block: int, npt: int, blocks_per_sm: int = 0) -> None:
        check(lib.ne2b_batch_set_tile_shape(self._h, block, npt, blocks_per_sm))

    def dev_mem_bytes(self) -> int:
        b = C.c_uint64()
        check(lib.ne2b_batch_dev_mem_bytes(self._h, C.byref(b)))
        return int(b.value)

    def stream_handle(self) -> int:
        p = C.c_void_p()
        check(lib.ne2b_batch_stream(self._h, C.byref(p)))
        return int(p.value or 0)

    def set_kernel_mode(self, mode: int) -> None:
        check(lib.ne2b_batch_set_kernel_mode(self._h, mode))

    def kernel_mode(self) -> tuple[int, bool]:
        m, r = C.c_int32(), C.c_int32()
        check(lib.ne2b_batch_kernel_mode(self._h, C.byref(m), C.byref(r)))
        return int(m.value), bool(r.value)

    def kernel_launches(self) -> int:
        v = C.c_uint64()
        check(lib.ne2b_batch_kernel_launches(self._h, C.byref(v)))
        return int(v.value)


class Server:
    """Continuous-batching trial server (admission by device footprint).

    admission_threads = 0: `submit` builds the request on the device before
    it returns.  k > 0: k library threads build requests while the device
    steps; the request joins at a later `step`, and the server keeps the
    net and the input matrix alive until the result is taken."""

    def __init__(self, neuron_capacity: int, synapse_capacity: int, ring_capacity: int, max_requests: int = 256,
                 steps_per_launch: int = 100, int_weights: bool = True, device: int = 0,
                 admission_threads: int = 0):
        c = _abi.ServerConfig(neuron_capacity, synapse_capacity, ring_capacity, max_requests, steps_per_launch,
                              1 if int_weights else 0, admission_threads)
        h = C.c_void_p()
        check(lib.ne2b_server_create(C.byref(c), device, C.byref(h)))
        self._h = h
        self.int_weights = int_weights
        self._keep = {}  # request id -> arrays a builder thread may still read

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib.ne2b_server_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def submit(self, net, cfg: _abi.Config, inputs: np.ndarray, steps: int) -> int | None:
        """Admit a request; None when it does not fit right now."""
        x = np.ascontiguousarray(inputs, dtype=np.float32)
        rid = C.c_uint64()
        st = lib.ne2b_server_submit(self._h, C.byref(net.desc()), C.byref(cfg), ptr(x), int(steps), C.byref(rid))
        if st == _abi.NE2B_EFULL:
            return None
        check(st)
        self._keep[int(rid.value)] = (net, x)
        return int(rid.value)

    def step(self) -> tuple[int, int]:
        a, f = C.c_uint32(), C.c_uint32()
        check(lib.ne2b_server_step(self._h, C.byref(a), C.byref(f)))
        return int(a.value), int(f.value)

    def synchronize(self) -> None:
        check(lib.ne2b_server_synchronize(self._h))

    def set_tile_shape(self, block: int, npt: int, blocks_per_sm: int = 0) -> None:
        check(lib.ne2b_server_set_tile_shape(self._h, block, npt, blocks_per_sm))

    def finished(self) -> list[int]:
        """Finished requests whose results are ready to take."""
        cnt = C.c_uint32()
        check(lib.ne2b_server_finished_ids(self._h, None, 0, C.byref(cnt)))
        cap = cnt.value
        if cap == 0:
            return []
        ids = np.zeros(cap, dtype=np.uint64)
        # more requests may become ready between the two calls: only the
        # first min(cap, count) entries are filled
        check(lib.ne2b_server_finished_ids(self._h, ptr(ids), cap, C.byref(cnt)))
        return [int(x) for x in ids[: min(cap, cnt.value)]]

    def take(self, rid: int) -> tuple[np.ndarray, int]:
        n, w = C.c_uint32(), C.c_uint32()
        check(lib.ne2b_server_result_shape(self._h, rid, C.byref(n), C.byref(w)))
        out = np.zeros((w.value, n.value), dtype=np.uint16)
        tot = C.c_uint64()
        st = lib.ne2b_server_take_result(self._h, rid, ptr(out), C.byref(tot))
        if st != _abi.NE2B_ENODATA:
            self._keep.pop(rid, None)
        check(st)
        return out, int(tot.value)

    def stream_handle(self) -> int:
        p = C.c_void_p()
        check(lib.ne2b_server_stream(self._h, C.byref(p)))
        return int(p.value or 0)

    def kernel_launches(self) -> int:
        v = C.c_uint64()
        check(lib.ne2b_server_kernel_launches(self._h, C.byref(v)))
        return int(v.value)

    def stats(self) -> dict:
        a, r, act, nu, su = C.c_uint64(), C.c_uint64(), C.c_uint32(), C.c_uint64(), C.c_uint64()
        check(lib.ne2b_server_stats(self._h, C.byref(a), C.byref(r), C.byref(act), C.byref(nu), C.byref(su)))
        return {"admitted": a.value, "retired": r.value, "active": act.value, "neurons_used": nu.value,
                "synapses_used": su.value}


def footprint(net, cfg: _abi.Config) -> tuple[int, int, int]:
    a, b, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
    check(lib.ne2b_request_footprint(C.byref(net.desc()), C.byref(cfg), C.byref(a), C.byref(b), C.byref(c)))
    return int(a.value), int(b.value), int(c.value)
