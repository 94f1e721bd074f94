"""The C ABI without a GPU: the library loads, exports every symbol
include/ne2b.h declares, and its host-side net building (the CSR build of
Network::synapse_csr and the workload generators) matches the oracle
bit-for-bit.  No kernel is launched here."""
import ctypes
import os
import re
import struct

import numpy as np
import pytest

import pyoracle as O
import neuro_edit_v2_b200 as nb
from neuro_edit_v2_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    text = open(os.path.join(ROOT, "include", "ne2b.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ne2b_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    syms = header_symbols()
    assert len(syms) > 60
    lib = ctypes.CDLL(_abi.LIB_PATH)
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    # and the Python binding covers the whole header
    assert sorted(set(syms) - set(_abi.EXPORTED)) == []


def test_config_default_matches_simconfig_default():
    """sim/src/state.rs:35-49"""
    c = nb.default_config()
    assert (c.dt_ms, c.synapse_tau_ms, c.readout_tau_ms) == (pytest.approx(0.1), 2.0, 2.0)
    assert (c.noise_rate_hz, c.noise_kick_mv, c.seed) == (0.0, 20.0, 1)
    assert (c.record_spikes, c.spike_record_steps, c.int_weights) == (0, 512, 0)


def _same_flat(a, b):
    assert np.array_equal(a.src_ptr, b.src_ptr)
    assert np.array_equal(a.tgt, b.tgt)
    assert np.array_equal(a.w.view(np.uint32), b.w.view(np.uint32))
    assert np.array_equal(a.delay_steps, b.delay_steps)
    assert np.array_equal(a.model, b.model)
    assert np.array_equal(a.params[:, :10].view(np.uint32), b.params[:, :10].view(np.uint32))
    assert a.n_inputs == b.n_inputs
    assert (a.tau_ms is None) == (b.tau_ms is None)
    if a.tau_ms is not None:
        assert np.array_equal(a.tau_ms.view(np.uint32), b.tau_ms.view(np.uint32))
    if a.n_inputs:
        assert np.array_equal(a.stim_ptr, b.stim_ptr)
        assert np.array_equal(a.stim_input, b.stim_input)
        assert np.array_equal(a.stim_w.view(np.uint32), b.stim_w.view(np.uint32))


@pytest.mark.parametrize("n,k,seed", [(1000, 100, 1), (2500, 37, 9)])
def test_random_kout_generator_matches_oracle(n, k, seed):
    prod = nb.random_kout(n, k, seed).arrays()
    ora = O.ONet.random_kout(n, k, seed).flat()
    _same_flat(prod, ora)
    assert np.array_equal(prod.kind, ora.kind)


@pytest.mark.parametrize("side,seed,model", [(6, 3, O.IZH), (9, 11, O.IZH), (7, 5, O.ADEX)])
def test_liquid_generator_matches_oracle(side, seed, model):
    prod = nb.liquid(side, seed, model=model).arrays()
    ora = O.ONet.liquid(side, seed, model=model).flat()
    _same_flat(prod, ora)


def test_csr_build_matches_oracle():
    """Network::synapse_csr (network.rs:654-692) in the library vs the oracle,
    on the fingerprint net of cpu_ref.rs:208-244 plus an inhibitory twist."""
    net = O.ONet()
    r = O.rng(3)
    m = net.create_2d_grid(8, 8, 30.0)
    net.set_exc_inh(m, 0.3, r)
    net.create_connections(m, 0.35, 80.0, 6.0, r)
    src, tgt, w, d, tau = net.synapses()
    model, params = net.models()
    prod = nb.from_synapses(model, params, net.kinds(), src, tgt, w, d, 0.1).arrays()
    _same_flat(prod, net.flat())


def test_csr_build_keeps_per_synapse_tau_in_csr_order():
    """tau travels with its synapse through the stable sort (network.rs:673)."""
    net = O.ONet()
    r = O.rng(5)
    m = net.create_2d_grid(6, 6, 30.0)
    net.set_exc_inh(m, 0.3, r)
    net.create_connections(m, 0.35, 80.0, 6.0, r)
    rng = np.random.default_rng(1)
    for _ in range(200):
        net.push_synapse(int(rng.integers(36)), int(rng.integers(36)), 2.0, float(rng.uniform(0.1, 5.0)),
                         float(rng.uniform(1.0, 20.0)))
    src, tgt, w, d, tau = net.synapses()
    model, params = net.models()
    prod = nb.from_synapses(model, params, net.kinds(), src, tgt, w, d, 0.1, tau_ms=tau).arrays()
    flat = net.flat()
    assert flat.tau_ms is not None
    _same_flat(prod, flat)


def test_csr_build_rejects_delay_overflow():
    """cpu_ref.rs:447-462"""
    with pytest.raises(nb.Ne2bError, match="exceeds"):
        nb.from_synapses([0, 0], np.zeros((2, 4), np.float32), [0, 0], [0], [1], [1.0], [7000.0], 0.1)


def test_csr_build_rejects_bad_index():
    with pytest.raises(nb.Ne2bError, match="only 2 neurons"):
        nb.from_synapses([0, 0], np.zeros((2, 4), np.float32), [0, 0], [0], [5], [1.0], [1.0], 0.1)


def test_host_expf_matches_oracle_det_expf():
    xs = np.linspace(-110.0, 95.0, 40001, dtype=np.float32)
    for x in xs[::7]:
        a = struct.pack("<f", nb.expf(float(x)))
        b = struct.pack("<f", O.det_expf(float(x)))
        assert a == b, x


def test_host_expf_equals_oracle_on_a_stride_of_all_floats():
    """The library's host copy of the device exp equals the oracle's on every
    64th float of [-104, 88.8] (every float with NE2B_EXHAUSTIVE_EXP=1:
    2,239,863,196 values)."""
    key = lambda x: (lambda b: (~b & 0xFFFFFFFF) if b >> 31 else b | 0x80000000)(
        struct.unpack("<I", struct.pack("<f", x))[0])
    n = key(88.8) - key(-104.0) + 1
    assert n == 2_239_863_196
    stride = 1 if os.environ.get("NE2B_EXHAUSTIVE_EXP") == "1" else 64
    fn = ctypes.cast(nb._abi.lib.ne2b_expf, ctypes.c_void_p)
    checked = ctypes.c_uint64()
    bad = O.lib().ne2o_expf_mismatches(fn, -104.0, 88.8, stride, os.cpu_count() or 1, ctypes.byref(checked))
    assert checked.value == (n + stride - 1) // stride
    assert bad == 0


@pytest.mark.parametrize("first, second, want", [(0, 2, []), (1, 3, [7]), (2, 2, [7, 8])])
def test_server_finished_lists_only_the_ids_it_received(monkeypatch, first, second, want):
    """ne2b_server_finished_ids is called for the count, then for the ids; a
    request that becomes ready between the two calls raises the second count
    above the buffer, and only the filled entries are ids."""
    from neuro_edit_v2_b200 import sim as S

    calls = []

    def fake(h, ids, cap, cnt):
        calls.append(cap)
        if ids:
            arr = (ctypes.c_uint64 * cap).from_address(ids)
            for i in range(min(cap, second)):
                arr[i] = 7 + i
        cnt._obj.value = first if len(calls) == 1 else second
        return 0

    monkeypatch.setattr(S.lib, "ne2b_server_finished_ids", fake)
    srv = S.Server.__new__(S.Server)
    srv._h = None
    assert srv.finished() == want


def test_request_footprint_needs_no_gpu():
    net = nb.liquid(10, 1)
    cfg = nb.default_config(int_weights=1, window_steps=500)
    neurons, syn, ring = nb.footprint(net, cfg)
    assert neurons == 1024 and syn == net.n_syn
    assert ring == neurons * net.arrays().ring_depth()


def test_parallel_csr_build_is_the_stable_order():
    """Above 2^20 synapses the CSR build sorts in parallel chunks; the result
    must still be the stable order by source (network.rs:656-657), with
    Dale's sign, delay steps and per-synapse tau carried along."""
    rng = np.random.default_rng(7)
    n, e = 5000, 1_500_000
    src = rng.integers(0, n, e).astype(np.uint32)
    tgt = rng.integers(0, n, e).astype(np.uint32)
    w = rng.random(e).astype(np.float32)
    d = (rng.random(e) * 20).astype(np.float32)
    tau = np.where(rng.random(e) < 0.1, rng.uniform(1, 20, e), 0).astype(np.float32)
    kind = (rng.random(n) < 0.2).astype(np.uint8)
    model = np.zeros(n, np.uint8)
    params = np.tile(np.array([0.02, 0.2, -65, 8], np.float32), (n, 1))
    a = nb.from_synapses(model, params, kind, src, tgt, w, d, 0.1, tau_ms=tau).arrays()
    order = np.argsort(src, kind="stable")
    assert np.array_equal(a.src_ptr, np.concatenate([[0], np.cumsum(np.bincount(src, minlength=n))]))
    assert np.array_equal(a.tgt, tgt[order])
    sign = np.where(kind[src[order]] == 1, -1.0, 1.0).astype(np.float32)
    assert np.array_equal(a.w, sign * w[order])
    assert np.array_equal(a.tau_ms, tau[order])
    q = (d[order] / np.float32(0.1)).astype(np.float64)  # f32 quotient; roundf rounds half away from zero
    steps = np.maximum(1, np.floor(q + 0.5)).astype(np.uint16)
    assert np.array_equal(a.delay_steps, steps)


def test_deterministic_exp_within_two_ulp():
    """The deterministic exp (single precision, shared by kernel, library and
    oracle) lies within 2 ulp of exp computed in double and rounded to float,
    on every 64th float of [-104, 88.8] (every float with
    NE2B_EXHAUSTIVE_EXP=1), subnormal results included."""
    stride = 1 if os.environ.get("NE2B_EXHAUSTIVE_EXP") == "1" else 64
    fn = ctypes.cast(O.lib().ne2o_expf_ref, ctypes.c_void_p)
    checked = ctypes.c_uint64()
    worst = O.lib().ne2o_expf_max_ulp(fn, -104.0, 88.8, stride, os.cpu_count() or 1, ctypes.byref(checked))
    assert checked.value == (2_239_863_196 + stride - 1) // stride
    assert worst <= 2, worst
