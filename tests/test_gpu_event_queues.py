"""Event-queue delivery (nets whose ring does not fit in L2): arrivals with
delay >= 2 are appended per arrival step and added into the ring slot the
step before it is read.  Integer sums commute, so with the int ring every
raster row and state bit must equal the oracle's, as with direct adds.

NE2B_EVQ=1 turns the queues on for every net built while it is set, so
these tests run them on nets small enough for the oracle; the 1M-neuron
configuration (tests/test_gpu_long_runs.py) uses them by size."""
import os

import numpy as np
import pytest

import pyoracle as O
import neuro_edit_v2_b200 as nb
from helpers import FP32_COUNT_RTOL, assert_state_bits_equal, lockstep, set_ext

pytestmark = pytest.mark.gpu

MODES = pytest.mark.parametrize("mode", [nb.KERNEL_STREAM, nb.KERNEL_RESIDENT], ids=["stream", "resident"])


@pytest.fixture
def queues():
    old = os.environ.get("NE2B_EVQ")
    os.environ["NE2B_EVQ"] = "1"
    yield
    if old is None:
        del os.environ["NE2B_EVQ"]
    else:
        os.environ["NE2B_EVQ"] = old


@MODES
def test_bench_net_event_heavy_bit_exact(queues, mode):
    onet = O.ONet.bench_net(4000, 100, 5, 0.7, 5.0)
    g, o, first = lockstep(onet, 1500, int_weights=True, chunk=100, noise_rate_hz=500.0, noise_kick_mv=20.0,
                           seed=3, mode=mode)
    assert first < 0, f"raster diverged at step {first}"
    assert o.mean_rate_hz() > 5.0
    assert_state_bits_equal(g, o)


@MODES
def test_100k_active_regime_bit_exact(queues, mode):
    """The 100k configuration with Poisson kicks (~23 Hz, ~2e4 events per
    step, including its 239 delay-1 synapses, which bypass the queues)."""
    onet = O.ONet.random_kout(100_000, 100, 1)
    g, o, first = lockstep(onet, 1500, int_weights=True, chunk=250, gauss_sd=1.0, synapse_tau_ms=5.0,
                           noise_rate_hz=100.0, noise_kick_mv=20.0, seed=1, mode=mode)
    assert first < 0, f"raster diverged at step {first}"
    assert_state_bits_equal(g, o)


def constant_delay_net(n, k, delay_ms, seed):
    """n neurons, k random targets each, every synapse the same delay: a
    synchronous volley puts all n * k arrivals into one bucket, past its
    cap of n_pad events (the overflow adds into the ring directly)."""
    rng = np.random.default_rng(seed)
    net = O.ONet()
    for i in range(n):
        net.add_neuron(float(i), 0.0, 0.0, O.EXC if i % 5 else O.INH)
    tg = rng.integers(0, n, (n, k))
    w = rng.uniform(0.0, 0.6, (n, k)).astype(np.float32)
    for i in range(n):
        for j in range(k):
            net.push_synapse(i, int(tg[i, j]), float(w[i, j]), delay_ms)
    return net


@MODES
def test_bucket_overflow_bit_exact(queues, mode):
    n = 3000
    onet = constant_delay_net(n, 40, 1.5, 11)

    def drive(s):
        set_ext(s, n, range(n), 30.0)  # every neuron fires every few steps, nearly together

    g, o, first = lockstep(onet, 400, int_weights=True, chunk=50, drive=drive, mode=mode)
    assert first < 0, f"raster diverged at step {first}"
    # some steps had far more than n arrivals due at once
    assert g.spikes_total() > 5 * n
    assert_state_bits_equal(g, o)


def test_reset_and_autotune_keep_results(queues):
    onet = O.ONet.bench_net(6000, 40, 9, 0.7, 5.0)
    a = nb.B200Sim(onet.flat(), int_weights=1, record_spikes=1, noise_rate_hz=300.0)
    b = nb.B200Sim(onet.flat(), int_weights=1, record_spikes=1, noise_rate_hz=300.0)
    a.run_steps(300)
    b.run_steps(300)
    a.autotune(64)
    a.run_steps(700)
    b.run_steps(700)
    assert a.spikes_total() == b.spikes_total() > 0
    assert np.array_equal(a.v().view(np.uint32), b.v().view(np.uint32))
    # a reset empties the queues: the run repeats itself exactly
    a.reset_state()
    a.run_steps(1000)
    assert a.spikes_total() == b.spikes_total()
    assert np.array_equal(a.v().view(np.uint32), b.v().view(np.uint32))


def test_batch_with_queues_equals_alone(queues):
    nets = [O.ONet.bench_net(n, 50, 20 + k, 0.7, 5.0).flat() for k, n in enumerate((1500, 4000, 2500))]
    cfgs = [nb.default_config(int_weights=1, record_spikes=1, noise_rate_hz=400.0, seed=k) for k in range(3)]
    b = nb.Batch(nets, cfgs)
    b.run_steps(800)
    for k, net in enumerate(nets):
        alone = nb.B200Sim(net, cfgs[k])
        alone.run_steps(800)
        assert b.spikes_total(k) == alone.spikes_total() > 0
        assert np.array_equal(b.state(k, 0).view(np.uint32), alone.v().view(np.uint32))


def test_fp32_ring_counts(queues):
    onet = O.ONet.bench_net(4000, 100, 5, 0.7, 5.0)
    g, o, first = lockstep(onet, 1500, int_weights=False, chunk=100, noise_rate_hz=500.0, noise_kick_mv=20.0,
                           seed=3)
    a, b = o.spikes_total(), g.spikes_total()
    assert a > 0 and abs(a - b) / a < FP32_COUNT_RTOL
