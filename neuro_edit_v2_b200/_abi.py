"""ctypes binding of include/ne2b.h (the C ABI of the B200 simulation core).

The shared library is loaded from neuro_edit_v2_b200/_lib/libne2b.so.  There
is no fallback: if the library is missing or fails to load, importing the
package raises, so a run without the CUDA path can never pass silently.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libne2b.so")

NE2B_OK = 0
NE2B_EINVAL = 1
NE2B_ENOMEM = 2
NE2B_ECUDA = 3
NE2B_EWINDOW = 4
NE2B_UNSUPPORTED = 5
NE2B_EFULL = 6
NE2B_ENODATA = 7
STATUS_NAMES = {0: "OK", 1: "EINVAL", 2: "ENOMEM", 3: "ECUDA", 4: "EWINDOW", 5: "UNSUPPORTED", 6: "EFULL",
                7: "ENODATA"}

MODEL_IZH = 0
MODEL_ADEX = 1

KERNEL_AUTO = 0
KERNEL_STREAM = 1
KERNEL_RESIDENT = 2


class Ne2Meta(C.Structure):
    """ne2b_ne2_meta: a .ne2 file's version and Meta (network.rs:381-392)."""
    _fields_ = [
        ("version", C.c_uint32),
        ("dt_ms", C.c_float),
        ("seed", C.c_uint64),
        ("conduction_speed", C.c_float),
        ("synapse_tau_ms", C.c_float),
        ("readout_tau_ms", C.c_float),
        ("noise_rate_hz", C.c_float),
        ("noise_kick_mv", C.c_float),
        ("n_types", C.c_uint32),
        ("n_groups", C.c_uint32),
        ("n_samples", C.c_uint32),
        ("n_readouts", C.c_uint32),
        ("n_scripts", C.c_uint32),
    ]


class NetDesc(C.Structure):
    _fields_ = [
        ("n", C.c_uint32),
        ("model", C.c_void_p),
        ("params", C.c_void_p),
        ("param_stride", C.c_uint32),
        ("x0", C.c_void_p),
        ("n_syn", C.c_uint64),
        ("src_ptr", C.c_void_p),
        ("tgt", C.c_void_p),
        ("w", C.c_void_p),
        ("delay_steps", C.c_void_p),
        ("tau_ms", C.c_void_p),
        ("n_inputs", C.c_uint32),
        ("stim_ptr", C.c_void_p),
        ("stim_input", C.c_void_p),
        ("stim_w", C.c_void_p),
    ]


class Config(C.Structure):
    _fields_ = [
        ("dt_ms", C.c_float),
        ("synapse_tau_ms", C.c_float),
        ("readout_tau_ms", C.c_float),
        ("noise_rate_hz", C.c_float),
        ("noise_kick_mv", C.c_float),
        ("seed", C.c_uint64),
        ("record_spikes", C.c_int32),
        ("spike_record_steps", C.c_uint32),
        ("int_weights", C.c_int32),
        ("gauss_sd", C.c_float),
        ("window_steps", C.c_uint32),
        ("max_windows", C.c_uint32),
    ]


class ServerConfig(C.Structure):
    _fields_ = [
        ("neuron_capacity", C.c_uint64),
        ("synapse_capacity", C.c_uint64),
        ("ring_capacity", C.c_uint64),
        ("max_requests", C.c_uint32),
        ("steps_per_launch", C.c_uint32),
        ("int_weights", C.c_int32),
        ("admission_threads", C.c_uint32),
    ]


class Ne2bError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"ne2b {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python neuro_edit_v2_b200/build.py` "
            "(the B200 backend has no CPU fallback)")
    return C.CDLL(LIB_PATH)


lib = _load()

_p = C.c_void_p
_u32 = C.c_uint32
_u64 = C.c_uint64
_i32 = C.c_int32
_f32 = C.c_float
_f64 = C.c_double
_pu32 = C.POINTER(C.c_uint32)
_pu64 = C.POINTER(C.c_uint64)
_pf32 = C.POINTER(C.c_float)
_pf64 = C.POINTER(C.c_double)

_SIGS = {
    "ne2b_config_default": (None, [C.POINTER(Config)]),
    "ne2b_last_error": (C.c_char_p, []),
    "ne2b_version": (C.c_char_p, []),
    "ne2b_create": (C.c_int, [C.POINTER(NetDesc), C.POINTER(Config), C.c_int, C.POINTER(_p)]),
    "ne2b_destroy": (C.c_int, [_p]),
    "ne2b_create_from_synapses": (C.c_int, [C.POINTER(NetDesc), _p, _u64, _p, _p, _p, _p, C.POINTER(Config), C.c_int,
                                            C.POINTER(_p)]),
    "ne2b_syn_count": (C.c_int, [_p, _pu64]),
    "ne2b_fit_ridge_multi": (C.c_int, [_p, _u32, _u32, _p, _u32, _f64, C.c_int, _p]),
    "ne2b_batch_fit_ridge_multi": (C.c_int, [_p, _p, _u32, _u32, _p, _u32, _f64, _pu32, _p]),
    "ne2b_fit_ridge": (C.c_int, [_p, _u32, _u32, _p, _f32, C.c_int, _p]),
    "ne2b_batch_fit_ridge": (C.c_int, [_p, _p, _u32, _u32, _p, _f32, _pu32, _p]),
    "ne2b_read_csr": (C.c_int, [_p, _p, _p, _p, _p]),
    "ne2b_n": (C.c_int, [_p, _pu32]),
    "ne2b_step_count": (C.c_int, [_p, _pu64]),
    "ne2b_time_ms": (C.c_int, [_p, _pf64]),
    "ne2b_ring_depth": (C.c_int, [_p, _pu32]),
    "ne2b_run_steps": (C.c_int, [_p, _u64]),
    "ne2b_run_ms": (C.c_int, [_p, _f32]),
    "ne2b_reset_state": (C.c_int, [_p]),
    "ne2b_synchronize": (C.c_int, [_p]),
    "ne2b_dev_mem_bytes": (C.c_int, [_p, _pu64]),
    "ne2b_read_trace": (C.c_int, [_p, _p]),
    "ne2b_read_state": (C.c_int, [_p, _u32, _p]),
    "ne2b_read_syn_current": (C.c_int, [_p, _p]),
    "ne2b_last_spikes": (C.c_int, [_p, _p, _u32, _pu32]),
    "ne2b_spike_counts": (C.c_int, [_p, _u64, _p]),
    "ne2b_spike_row": (C.c_int, [_p, _u32, _p]),
    "ne2b_spike_counts_noalloc": (C.c_int, [_p, _u64, _p]),
    "ne2b_spikes_total": (C.c_int, [_p, _pu64]),
    "ne2b_mean_rate_hz": (C.c_int, [_p, _pf64]),
    "ne2b_window_counts": (C.c_int, [_p, _u32, _p]),
    "ne2b_windows_done": (C.c_int, [_p, _pu32]),
    "ne2b_set_input_constant": (C.c_int, [_p, _u32, _f32]),
    "ne2b_input_values": (C.c_int, [_p, _p]),
    "ne2b_play_input": (C.c_int, [_p, _u32, _p, _u64]),
    "ne2b_loop_input": (C.c_int, [_p, _u32, _p, _u64]),
    "ne2b_set_external": (C.c_int, [_p, _u32, _f32]),
    "ne2b_set_external_all": (C.c_int, [_p, _p, _u32]),
    "ne2b_external": (C.c_int, [_p, _p]),
    "ne2b_set_noise": (C.c_int, [_p, _f32, _f32]),
    "ne2b_set_gauss_noise": (C.c_int, [_p, _f32]),
    "ne2b_set_kernel_mode": (C.c_int, [_p, _i32]),
    "ne2b_kernel_mode": (C.c_int, [_p, C.POINTER(_i32), C.POINTER(_i32)]),
    "ne2b_batch_set_kernel_mode": (C.c_int, [_p, _i32]),
    "ne2b_batch_kernel_mode": (C.c_int, [_p, C.POINTER(_i32), C.POINTER(_i32)]),
    "ne2b_autotune": (C.c_int, [_p, _u32]),
    "ne2b_tile_shape": (C.c_int, [_p, _pu32, _pu32, _pu32]),
    "ne2b_set_tile_shape": (C.c_int, [_p, _u32, _u32, _u32]),
    "ne2b_set_delivery_warps": (C.c_int, [_p, C.c_int32]),
    "ne2b_delivery_warps": (C.c_int, [_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "ne2b_stream": (C.c_int, [_p, C.POINTER(_p)]),
    "ne2b_kernel_launches": (C.c_int, [_p, _pu64]),
    "ne2b_batch_stream": (C.c_int, [_p, C.POINTER(_p)]),
    "ne2b_batch_kernel_launches": (C.c_int, [_p, _pu64]),
    "ne2b_server_stream": (C.c_int, [_p, C.POINTER(_p)]),
    "ne2b_server_synchronize": (C.c_int, [_p]),
    "ne2b_selftest_barrier_timeout": (C.c_int, [C.c_int, _u32, C.POINTER(C.c_int32)]),
    "ne2b_server_set_tile_shape": (C.c_int, [_p, _u32, _u32, _u32]),
    "ne2b_server_kernel_launches": (C.c_int, [_p, _pu64]),
    "ne2b_set_v_watch": (C.c_int, [_p, _p, _u32]),
    "ne2b_set_grid_watches": (C.c_int, [_p, _p, _p, _u32]),
    "ne2b_watch_count": (C.c_int, [_p, C.POINTER(_u32), C.POINTER(_u32)]),
    "ne2b_drain_watch": (C.c_int, [_p, _p, C.POINTER(_u32)]),
    "ne2b_grid_traces": (C.c_int, [_p, _f32, _p]),
    "ne2b_batch_create": (C.c_int, [C.POINTER(NetDesc), C.POINTER(Config), _u32, C.c_int, C.POINTER(_p)]),
    "ne2b_batch_destroy": (C.c_int, [_p]),
    "ne2b_batch_play_input": (C.c_int, [_p, _u32, _u32, _p, _u64]),
    "ne2b_batch_set_input_matrix": (C.c_int, [_p, _u32, _p, _u64]),
    "ne2b_batch_run_steps": (C.c_int, [_p, _u64]),
    "ne2b_batch_reset_state": (C.c_int, [_p]),
    "ne2b_batch_synchronize": (C.c_int, [_p]),
    "ne2b_batch_window_counts": (C.c_int, [_p, _u32, _u32, _p]),
    "ne2b_batch_spikes_total": (C.c_int, [_p, _u32, _pu64]),
    "ne2b_batch_read_state": (C.c_int, [_p, _u32, _u32, _p]),
    "ne2b_batch_autotune": (C.c_int, [_p, _u32]),
    "ne2b_batch_tile_shape": (C.c_int, [_p, _pu32, _pu32, _pu32]),
    "ne2b_batch_set_tile_shape": (C.c_int, [_p, _u32, _u32, _u32]),
    "ne2b_batch_dev_mem_bytes": (C.c_int, [_p, _pu64]),
    "ne2b_batch_last_step_ms": (C.c_int, [_p, _pf32]),
    "ne2b_request_footprint": (C.c_int, [C.POINTER(NetDesc), C.POINTER(Config), _pu64, _pu64, _pu64]),
    "ne2b_server_create": (C.c_int, [C.POINTER(ServerConfig), C.c_int, C.POINTER(_p)]),
    "ne2b_server_destroy": (C.c_int, [_p]),
    "ne2b_server_submit": (C.c_int, [_p, C.POINTER(NetDesc), C.POINTER(Config), _p, _u64, _pu64]),
    "ne2b_server_step": (C.c_int, [_p, _pu32, _pu32]),
    "ne2b_server_result_shape": (C.c_int, [_p, _u64, _pu32, _pu32]),
    "ne2b_server_take_result": (C.c_int, [_p, _u64, _p, _pu64]),
    "ne2b_server_finished_ids": (C.c_int, [_p, _p, _u32, _pu32]),
    "ne2b_server_stats": (C.c_int, [_p, _pu64, _pu64, _pu32, _pu64, _pu64]),
    "ne2b_net_from_synapses": (C.c_int, [_u32, _p, _p, _u32, _p, _u64, _p, _p, _p, _p, _p, _f32, C.POINTER(_p)]),
    "ne2b_gen_random_kout": (C.c_int, [_u32, _u32, _u64, _f32, _f32, _f32, _f32, _f32, C.POINTER(_p)]),
    "ne2b_net_load_ne2": (C.c_int, [C.c_char_p, C.POINTER(_p), _p]),
    "ne2b_net_from_ne2": (C.c_int, [_p, _u64, C.POINTER(_p), _p]),
    "ne2b_gen_liquid": (C.c_int, [_u32, _u64, _f64, _i32, _f32, _u32, _u32, _f32, _i32, _f32, C.POINTER(_p)]),
    "ne2b_net_set_model_all": (C.c_int, [_p, _i32, _p, _p, _u32]),
    "ne2b_net_desc_of": (C.c_int, [_p, C.POINTER(NetDesc)]),
    "ne2b_net_kinds": (C.c_int, [_p, _p]),
    "ne2b_net_free": (C.c_int, [_p]),
    "ne2b_expf": (C.c_float, [C.c_float]),
}

for _name, (_res, _args) in _SIGS.items():
    _fn = getattr(lib, _name)
    _fn.restype = _res
    _fn.argtypes = _args

EXPORTED = sorted(_SIGS)


def check(status: int) -> None:
    if status != NE2B_OK:
        raise Ne2bError(status, lib.ne2b_last_error().decode(errors="replace"))


def ptr(a: np.ndarray | None) -> int | None:
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays passed to ne2b must be C-contiguous"
    return a.ctypes.data


def default_config(**kw) -> Config:
    c = Config()
    lib.ne2b_config_default(C.byref(c))
    for k, v in kw.items():
        if not hasattr(c, k):
            raise AttributeError(f"ne2b_config has no field {k!r}")
        setattr(c, k, v)
    return c
