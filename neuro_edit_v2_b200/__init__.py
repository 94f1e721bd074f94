"""neuro_edit_v2_b200 — B200-native simulation core for neuro_edit v2 networks.

The step loop of the reference `sim` crate (Izhikevich/AdEx update, spike
compaction, delivery into the per-delay synaptic ring in fp32 or int32 fixed
point, current decay, noise, stimulus and spike-count readout) as
ahead-of-time sm_100a CUDA kernels behind the C ABI of include/ne2b.h.  This
package is the Python mirror of that ABI; importing it loads the library and
fails loudly if it is missing.
"""
from . import _abi
from ._abi import (KERNEL_AUTO, KERNEL_RESIDENT, KERNEL_STREAM, MODEL_ADEX, MODEL_IZH, Config, Ne2bError,
                   default_config)
from .net import (FlatNet, NativeNet, config_from_meta, from_ne2_bytes, from_synapses, liquid, load_ne2, random_kout,
                  to_adex)
from .readout import fit_ridge, fit_ridge_multi, ridge_predict
from .sim import B200Sim, Batch, Server, SpikeWindowError, footprint

__all__ = [
    "B200Sim", "Batch", "Server", "SpikeWindowError", "footprint", "FlatNet", "NativeNet", "from_synapses",
    "liquid", "random_kout", "to_adex", "load_ne2", "from_ne2_bytes", "config_from_meta", "Config", "default_config", "Ne2bError", "MODEL_IZH", "MODEL_ADEX",
    "KERNEL_AUTO", "KERNEL_STREAM", "KERNEL_RESIDENT",
    "expf", "selftest_barrier_timeout", "fit_ridge", "fit_ridge_multi", "ridge_predict",
]


def selftest_barrier_timeout(limit_ms: int = 50, device: int = 0) -> bool:
    """Run the bounded grid-barrier self-test (one cooperative block never
    arrives); True when the waiting blocks gave up and flagged it."""
    import ctypes

    t = ctypes.c_int32()
    _abi.check(_abi.lib.ne2b_selftest_barrier_timeout(device, limit_ms, ctypes.byref(t)))
    return bool(t.value)


def expf(x: float) -> float:
    """The deterministic exp of the AdEx step (host copy of the device code)."""
    return float(_abi.lib.ne2b_expf(float(x)))
