"""Readout training on the GPU: `fit_ridge_multi` of the reference
(sim/src/readout.rs:190-252) through `ne2b_fit_ridge_multi`, with the
reference's f64 arithmetic in its order (bit-equal weights)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._abi import check, lib


def _design_pointer(x):
    """(pointer, T, F, keep-alive) of a [T x F] float32 design in host
    memory (numpy) or device memory (any object with __cuda_array_interface__,
    e.g. a CUDA torch tensor)."""
    cai = getattr(x, "__cuda_array_interface__", None)
    if cai is not None:
        if np.dtype(cai["typestr"]) != np.float32 or len(cai["shape"]) != 2:
            raise ValueError("a device design must be a 2-D float32 array")
        t, f = cai["shape"]
        if cai.get("strides") not in (None, (4 * f, 4)):
            raise ValueError("a device design must be C-contiguous")
        return int(cai["data"][0]), int(t), int(f), x
    a = np.ascontiguousarray(x, dtype=np.float32)
    if a.ndim != 2:
        raise ValueError("the design must be 2-D [trials x features]")
    return a.ctypes.data, a.shape[0], a.shape[1], a


def fit_ridge_multi(x, labels, k: int, lam: float, device: int = 0) -> np.ndarray:
    """[k x (F + 1)] ridge weights (bias last) of the centred design x
    [T x F] for labels in 0..k-1."""
    p, t, f, keep = _design_pointer(x)
    lab = np.ascontiguousarray(labels, dtype=np.uint32)
    if lab.shape != (t,):
        raise ValueError("one label per row")
    w = np.zeros((k, f + 1), np.float64)
    check(lib.ne2b_fit_ridge_multi(p, t, f, lab.ctypes.data, k, float(lam), device, w.ctypes.data))
    del keep
    return w


def fit_ridge(x, y, lam: float, device: int = 0) -> np.ndarray:
    """F + 1 ridge weights (bias last) of the design x [T x F] for the
    targets y (e.g. 0/1 or +-1)."""
    p, t, f, keep = _design_pointer(x)
    yy = np.ascontiguousarray(y, dtype=np.float32)
    if yy.shape != (t,):
        raise ValueError("one target per row")
    w = np.zeros(f + 1, np.float64)
    check(lib.ne2b_fit_ridge(p, t, f, yy.ctypes.data, float(lam), device, w.ctypes.data))
    del keep
    return w


def ridge_predict(w: np.ndarray, x) -> np.ndarray:
    """Argmax class per row (the reference's ridge_predict): x @ w[:, :F].T + bias."""
    x = np.asarray(x, dtype=np.float64)
    return np.argmax(x @ w[:, :-1].T + w[:, -1], axis=1)
