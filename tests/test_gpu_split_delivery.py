"""Split delivery: the step kernel lists each tile's spiking neurons and a
second kernel per step delivers them (one warp per tile).  The adds are the
fused path's, in another order, so with the int ring every raster row and
state bit must equal the oracle's.

NE2B_SPLIT=1, set while a sim is created, fixes split delivery for it (the
resident kernel always delivers itself, so these tests force streaming)."""
import os

import numpy as np
import pytest

import pyoracle as O
import neuro_edit_v2_b200 as nb
from helpers import FP32_COUNT_RTOL, assert_state_bits_equal, lockstep, set_ext

pytestmark = pytest.mark.gpu


def _env(name, value):
    old = os.environ.get(name)
    os.environ[name] = value
    return old


def _restore(name, old):
    if old is None:
        os.environ.pop(name, None)
    else:
        os.environ[name] = old


@pytest.fixture
def split():
    old = _env("NE2B_SPLIT", "1")
    yield
    _restore("NE2B_SPLIT", old)


@pytest.fixture
def split_and_queues():
    a, b = _env("NE2B_SPLIT", "1"), _env("NE2B_EVQ", "1")
    yield
    _restore("NE2B_SPLIT", a)
    _restore("NE2B_EVQ", b)


def test_bench_net_bit_exact(split):
    onet = O.ONet.bench_net(4000, 100, 5, 0.7, 5.0)
    g, o, first = lockstep(onet, 1500, int_weights=True, chunk=100, noise_rate_hz=500.0, noise_kick_mv=20.0,
                           seed=3, mode=nb.KERNEL_STREAM)
    assert g.split_delivery()
    assert first < 0, f"raster diverged at step {first}"
    assert_state_bits_equal(g, o)


@pytest.mark.parametrize("shape", [(128, 1), (256, 4)], ids=lambda s: f"{s[0]}x{s[1]}")
def test_100k_active_regime_bit_exact(split, shape):
    onet = O.ONet.random_kout(100_000, 100, 1)

    def drive(s):
        if isinstance(s, nb.B200Sim):
            s.set_tile_shape(*shape)

    g, o, first = lockstep(onet, 1000, int_weights=True, chunk=250, gauss_sd=1.0, synapse_tau_ms=5.0,
                           noise_rate_hz=100.0, noise_kick_mv=20.0, seed=1, mode=nb.KERNEL_STREAM, drive=drive)
    assert first < 0, f"raster diverged at step {first}"
    assert_state_bits_equal(g, o)


def test_synchronous_bursts_bit_exact(split_and_queues):
    """Whole tiles spiking together: a warp delivers hundreds of rows per
    tile, and the queues overflow into the ring."""
    n = 20_000
    onet = O.ONet.random_kout(n, 100, 4)

    def drive(s):
        if isinstance(s, nb.B200Sim):
            s.set_tile_shape(256, 2)
        set_ext(s, n, range(n), 40.0)

    g, o, first = lockstep(onet, 200, int_weights=True, chunk=50, gauss_sd=1.0, synapse_tau_ms=5.0, drive=drive,
                           mode=nb.KERNEL_STREAM)
    assert first < 0, f"raster diverged at step {first}"
    assert g.spikes_total() > 5 * n
    assert_state_bits_equal(g, o)


def test_with_event_queues_bit_exact(split_and_queues):
    onet = O.ONet.random_kout(100_000, 100, 2)
    g, o, first = lockstep(onet, 1000, int_weights=True, chunk=250, gauss_sd=1.0, synapse_tau_ms=5.0,
                           noise_rate_hz=100.0, noise_kick_mv=20.0, seed=4, mode=nb.KERNEL_STREAM)
    assert first < 0, f"raster diverged at step {first}"
    assert_state_bits_equal(g, o)


def test_custom_tau_net_keeps_immediate_delivery(split):
    """Synapses with their own tau are delivered by the step kernel even
    when the engine splits; bit-exact against the oracle."""
    from test_gpu_xsyn import mixed_tau_net

    onet = mixed_tau_net(3000, 40, 11, 0.5)
    g, o, first = lockstep(onet, 1500, int_weights=True, chunk=100, noise_rate_hz=400.0, noise_kick_mv=20.0,
                           seed=5, mode=nb.KERNEL_STREAM)
    assert g.split_delivery()
    assert first < 0, f"raster diverged at step {first}"
    assert g.spikes_total() > 0
    assert_state_bits_equal(g, o)


def test_switching_between_launches_and_autotune_keep_results():
    onet = O.ONet.bench_net(6000, 40, 9, 0.7, 5.0)
    a = nb.B200Sim(onet.flat(), int_weights=1, record_spikes=1, noise_rate_hz=300.0)
    b = nb.B200Sim(onet.flat(), int_weights=1, record_spikes=1, noise_rate_hz=300.0)
    for s in (a, b):
        s.set_kernel_mode(nb.KERNEL_STREAM)
    for k in range(6):
        a.set_split_delivery(k % 2 == 0)
        a.run_steps(150)
        b.run_steps(150)
    a.autotune(64)
    a.run_steps(400)
    b.run_steps(400)
    assert a.spikes_total() == b.spikes_total() > 0
    assert np.array_equal(a.v().view(np.uint32), b.v().view(np.uint32))
    assert np.array_equal(a.spike_counts(256), b.spike_counts(256))


def test_batch_with_split_equals_alone(split):
    nets = [O.ONet.bench_net(n, 50, 30 + k, 0.7, 5.0).flat() for k, n in enumerate((1500, 4000, 2500))]
    cfgs = [nb.default_config(int_weights=1, record_spikes=1, noise_rate_hz=400.0, seed=k) for k in range(3)]
    b = nb.Batch(nets, cfgs)
    b.set_kernel_mode(nb.KERNEL_STREAM)
    assert b.split_delivery()
    b.run_steps(800)
    old = _env("NE2B_SPLIT", "0")
    try:
        for k, net in enumerate(nets):
            alone = nb.B200Sim(net, cfgs[k])
            alone.run_steps(800)
            assert b.spikes_total(k) == alone.spikes_total() > 0
            assert np.array_equal(b.state(k, 0).view(np.uint32), alone.v().view(np.uint32))
    finally:
        _restore("NE2B_SPLIT", old)


def test_fp32_ring_counts(split):
    onet = O.ONet.bench_net(4000, 100, 5, 0.7, 5.0)
    g, o, first = lockstep(onet, 1500, int_weights=False, chunk=100, noise_rate_hz=500.0, noise_kick_mv=20.0,
                           seed=3, mode=nb.KERNEL_STREAM)
    a, b = o.spikes_total(), g.spikes_total()
    assert a > 0 and abs(a - b) / a < FP32_COUNT_RTOL
