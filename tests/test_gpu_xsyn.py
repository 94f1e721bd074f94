"""Synapses with their own tau (sim/src/state.rs:231-275, cpu.rs:206-228,
kernels.rs:208-215): the B200 kernels against the C oracle.

With the int ring every raster row and every state bit must equal the
oracle's (the custom currents are per synapse, each arrives at most once
per step, and the input sums them in the oracle's target-major order).  The
fp32 ring keeps the float-atomic order caveat of the merged ring."""
import numpy as np
import pytest

import pyoracle as O
import neuro_edit_v2_b200 as nb
from helpers import FP32_COUNT_RTOL, assert_state_bits_equal, lockstep

pytestmark = pytest.mark.gpu

MODES = pytest.mark.parametrize("mode", [nb.KERNEL_STREAM, nb.KERNEL_RESIDENT], ids=["stream", "resident"])


def mixed_tau_net(n, k, seed, frac, tau_lo=1.0, tau_hi=30.0):
    """bench_net (sim/src/bench.rs:10-52) plus extra synapses of which a
    fraction `frac` carry their own tau (the rest a merged-ring weight)."""
    net = O.ONet.bench_net(n, k, seed, 0.7, 5.0)
    rng = np.random.default_rng(seed)
    extra = n * 10
    src = rng.integers(0, n, extra)
    tgt = rng.integers(0, n, extra)
    w = rng.uniform(0.5, 4.0, extra)
    d = rng.uniform(0.1, 15.0, extra)
    tau = np.where(rng.random(extra) < frac, rng.uniform(tau_lo, tau_hi, extra), 0.0)
    for a, b, ww, dd, tt in zip(src, tgt, w, d, tau):
        net.push_synapse(int(a), int(b), float(ww), float(dd), float(tt))
    return net


@MODES
def test_custom_tau_net_int_ring_bit_exact(mode):
    onet = mixed_tau_net(3000, 40, 11, 0.5)
    flat = onet.flat()
    assert flat.tau_ms is not None and int((flat.tau_ms > 0).sum()) > 10000
    g, o, first = lockstep(onet, 1500, int_weights=True, chunk=100, noise_rate_hz=500.0, noise_kick_mv=20.0,
                           seed=5, mode=mode, flat=flat)
    assert first < 0, f"raster diverged at step {first}"
    assert o.mean_rate_hz() > 5.0
    assert_state_bits_equal(g, o)


def test_all_synapses_custom_tau_int_ring_bit_exact():
    """Every synapse on its own current: the merged ring carries nothing."""
    net2 = O.ONet.bench_net(2000, 30, 12, 0.7, 5.0)
    src, tgt, w, d, _ = net2.synapses()
    allx = O.ONet()
    for i in range(2000):
        allx.add_neuron(0.0, 0.0, 0.0, O.EXC if i < 1600 else O.INH)
    rng = np.random.default_rng(3)
    for a, b, ww, dd in zip(src, tgt, w, d):
        allx.push_synapse(int(a), int(b), float(abs(ww)), float(dd), float(rng.uniform(0.5, 40.0)))
    g, o, first = lockstep(allx, 1000, int_weights=True, chunk=100, noise_rate_hz=500.0, noise_kick_mv=20.0,
                           seed=6)
    assert first < 0, f"raster diverged at step {first}"
    assert o.spikes_total() > 0
    assert np.all(g.syn_current() == 0.0)  # the merged current stays empty
    assert_state_bits_equal(g, o)


def test_custom_tau_fp32_ring_counts():
    onet = mixed_tau_net(3000, 40, 13, 0.5)
    g, o, first = lockstep(onet, 1500, int_weights=False, chunk=100, noise_rate_hz=500.0, noise_kick_mv=20.0,
                           seed=7)
    a, b = g.spikes_total(), o.spikes_total()
    assert b > 0 and abs(a - b) <= FP32_COUNT_RTOL * b, (a, b, first)


def test_custom_tau_arrives_then_decays_on_gpu():
    """sim/tests/cpu_ref.rs:116-165: a custom-tau synapse delivers into its
    own current, not the merged one, and decays with its own tau."""
    net = O.ONet()
    net.add_neuron(0, 0, 0, O.EXC)
    net.add_neuron(10, 0, 0, O.EXC)
    net.push_synapse(0, 1, 30.0, 0.2, 20.0)
    g, o, first = lockstep(net, 400, int_weights=True, chunk=50,
                           drive=lambda s: s.set_external(0, 30.0))
    assert first < 0
    assert np.all(g.syn_current() == 0.0)
    assert_state_bits_equal(g, o)
    assert g.spikes_total() == o.spikes_total() > 0


def test_tau_below_dt_decays_safely_on_gpu():
    """sim/tests/cpu_ref.rs:467-498: tau below dt is clamped and stays finite."""
    net = O.ONet()
    net.add_neuron(0, 0, 0, O.EXC)
    net.add_neuron(10, 0, 0, O.EXC)
    net.push_synapse(0, 1, 5.0, 1.0, 0.05)
    g, o, first = lockstep(net, 300, int_weights=True, chunk=50, drive=lambda s: s.set_external(0, 30.0))
    assert first < 0
    assert np.all(np.isfinite(g.state(1)))
    assert_state_bits_equal(g, o)


def test_custom_tau_reset_and_autotune_keep_results():
    """reset clears the custom currents and pending arrivals; autotuning
    restores them from its snapshot."""
    onet = mixed_tau_net(2500, 30, 14, 0.5)
    flat = onet.flat()
    cfg = dict(int_weights=1, record_spikes=1, noise_rate_hz=500.0, noise_kick_mv=20.0, seed=9)
    a = nb.B200Sim(flat, **cfg)
    b = nb.B200Sim(flat, **cfg)
    a.run_steps(400)
    a.reset_state()
    a.run_steps(300)
    b.run_steps(300)
    a.autotune(64)
    a.run_steps(400)
    b.run_steps(400)
    assert a.spikes_total() == b.spikes_total() > 0
    assert np.array_equal(a.v().view(np.uint32), b.v().view(np.uint32))
