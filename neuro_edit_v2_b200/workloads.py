"""Synthetic trial workloads: the batched-liquid set and the served request
stream.

Definitions (seeded, so a run is reproducible):
  * batched liquids: 256 local 3-D liquids, neuron counts log-uniform in
    [1000, 27000] -> cube side round(cbrt(N)) in [10, 30]; wiring
    p = exp(-(d/lambda)^2), lambda = 2 lattice units (120 um), Dale's law
    with a 20% inhibitory split; 8 Bernoulli bit streams (p = 0.05 per ms,
    each bit held 10 steps = 1 ms at dt 0.1 ms) into the x = 0 face;
    1000 ms trials, per-neuron spike counts per 50 ms window.
  * served requests: Poisson arrivals (mean 200/s); neurons log-uniform in
    [2000, 50000]; Izhikevich or AdEx 50/50; random K=100 or local wiring
    50/50; duration U(200, 2000) ms; 8 input streams whose bits are made
    coincident in labelled windows (the RngStream::window pattern of
    sim/src/script.rs:2849-2895: in an event window each listed pair shares
    one Bernoulli(p) bit per ms with probability `strength`); 50 ms windows.
The stream values come from numpy's seeded PCG64 (not the reference Rng):
they are inputs, and the same arrays feed every backend that is compared.
"""
from __future__ import annotations

import math
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass

import numpy as np

from . import _abi
from .net import FlatNet, liquid, random_kout

DT_MS = 0.1
SPB = 10          # steps per ms
WINDOW_STEPS = 500  # 50 ms
PAIRS = [(0, 1), (2, 3), (4, 5), (6, 7)]
ADEX_GAIN = 281.0  # AdEx C (pF): weights in pA move v by the same mV as in izh


def bit_streams(rng: np.random.Generator, ms: int, n_src: int = 8, p: float = 0.05) -> np.ndarray:
    bits = (rng.random((ms, n_src)) < p).astype(np.float32)
    return np.repeat(bits, SPB, axis=0)


def coincident_streams(rng: np.random.Generator, ms: int, n_src: int = 8, p: float = 0.05,
                       window_ms: int = 50, strength: float = 1.0):
    """Streams with one labelled pair coincident per event window
    (script.rs:2867-2894); returns (inputs [ms*SPB x n_src], labels per window)."""
    bits = np.zeros((ms, n_src), np.float32)
    labels = []
    for w0 in range(0, ms, window_ms):
        label = int(rng.integers(-1, len(PAIRS)))  # -1 = no event window
        labels.append(label)
        for t in range(w0, min(ms, w0 + window_ms)):
            bits[t] = rng.random(n_src) < p
            if label >= 0 and rng.random() < strength:
                b = float(rng.random() < p)
                i, j = PAIRS[label]
                bits[t, i] = b
                bits[t, j] = b
    return np.repeat(bits, SPB, axis=0), labels


def batched_liquid_sizes(count: int = 256, seed: int = 4) -> list[int]:
    rng = np.random.default_rng(seed)
    n = np.exp(rng.uniform(math.log(1000), math.log(27000), count))
    return [int(min(30, max(10, round(x ** (1.0 / 3.0))))) for x in n]


def batched_liquids(count: int = 256, seed: int = 4, threads: int = 8):
    """The 256-liquid set: (nets, input matrices [10000 x 8])."""
    sides = batched_liquid_sizes(count, seed)
    with ThreadPoolExecutor(threads) as ex:
        nets = list(ex.map(lambda k: liquid(sides[k], seed=1000 + k), range(count)))
    rng = np.random.default_rng(seed + 1)
    inputs = [bit_streams(rng, 1000) for _ in range(count)]
    return nets, inputs


def with_inputs(net, n_inputs: int, targets: int, w_in: float, rng: np.random.Generator) -> FlatNet:
    """A library net copied out with `n_inputs` inputs on random targets."""
    f = net.arrays()
    n = f.n
    per = [[] for _ in range(n)]
    for k in range(n_inputs):
        for tg in rng.integers(0, n, targets):
            per[int(tg)].append((k, w_in))
    ptr = np.zeros(n + 1, np.uint32)
    ptr[1:] = np.cumsum([len(r) for r in per])
    f.n_inputs = n_inputs
    f.stim_ptr = ptr
    f.stim_input = np.array([k for r in per for k, _ in r], np.uint32)
    f.stim_w = np.array([w for r in per for _, w in r], np.float32)
    return f


@dataclass
class Request:
    arrival_s: float
    n: int
    model: int
    wiring: str
    steps: int
    net: object
    inputs: np.ndarray
    labels: list


def request_stream(count: int, rate_hz: float = 200.0, seed: int = 7, threads: int = 8) -> list[Request]:
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate_hz, count)
    arrivals = np.cumsum(gaps) - gaps[0]
    specs = []
    for r in range(count):
        n = int(round(math.exp(rng.uniform(math.log(2000), math.log(50000)))))
        model = _abi.MODEL_IZH if rng.random() < 0.5 else _abi.MODEL_ADEX
        wiring = "random" if rng.random() < 0.5 else "local"
        ms = int(round(rng.uniform(200.0, 2000.0)))
        inputs, labels = coincident_streams(rng, ms)
        specs.append((float(arrivals[r]), n, model, wiring, ms * SPB, inputs, labels, 5000 + r))

    def build(sp):
        arrival, n, model, wiring, steps, inputs, labels, seed_r = sp
        gain = ADEX_GAIN if model == _abi.MODEL_ADEX else 1.0
        if wiring == "local":
            side = max(2, int(round(n ** (1.0 / 3.0))))
            net = liquid(side, seed=seed_r, model=model)
            n = side ** 3
        else:
            base = random_kout(n, 100, seed_r, w_scale=0.7 * gain)
            if model == _abi.MODEL_ADEX:
                from .net import to_adex

                to_adex(base)
            net = with_inputs(base, 8, 24, 12.0 * gain, np.random.default_rng(seed_r))
        return Request(arrival, n, model, wiring, steps, net, inputs, labels)

    with ThreadPoolExecutor(threads) as ex:
        return list(ex.map(build, specs))


def request_config(req: Request, seed: int) -> _abi.Config:
    return _abi.default_config(int_weights=1, window_steps=WINDOW_STEPS,
                               max_windows=(req.steps + WINDOW_STEPS - 1) // WINDOW_STEPS, seed=seed)


def outdegree(net) -> np.ndarray:
    d = net.desc()
    n = int(d.n)
    import ctypes as C

    sp = np.ctypeslib.as_array(C.cast(d.src_ptr, C.POINTER(C.c_uint32)), shape=(n + 1,))
    return np.diff(sp.astype(np.int64))
