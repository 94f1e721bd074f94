"""The warp-specialised streaming kernel (separate delivery warps fed by a
shared-memory queue of spiking neurons' CSR rows) against the C oracle.

With the int ring every raster row and every state bit must equal the
oracle's, as for the kernel that delivers with the tile's own threads: the
queue changes only which warp adds an arrival and when within the step, and
integer sums are order-independent.  Bursts fill and wrap the queue many
times within one step; the record-free instance, AdEx rows, custom-tau
synapses and the f32 ring are covered beside the plain int-ring case."""
import numpy as np
import pytest

import pyoracle as O
import neuro_edit_v2_b200 as nb
from helpers import FP32_COUNT_RTOL, assert_state_bits_equal, configs, lockstep, set_ext
from test_gpu_xsyn import mixed_tau_net

pytestmark = pytest.mark.gpu

ADEX_TONIC = [281.0, 30.0, -70.6, -50.4, 2.0, 4.0, 144.0, 80.5, -70.6, 20.0]  # model/adex.rs:22-24

WS_SHAPES = pytest.mark.parametrize("shape", [(128, 1), (256, 2), (512, 4)], ids=lambda s: f"{s[0]}x{s[1]}")


def with_ws(shape, extra=None):
    """A lockstep drive that puts the GPU sim on the delivery-warp kernel in
    `shape` (and applies `extra` to both backends)."""

    def drive(s):
        if isinstance(s, nb.B200Sim):
            s.set_tile_shape(*shape)
            s.set_delivery_warps(True)
            assert s.delivery_warps() == (True, True)
        if extra:
            extra(s)

    return drive


@WS_SHAPES
def test_synchronous_bursts_bit_exact(shape):
    """Whole tiles spiking in the same step: thousands of queued rows per
    block and step, the 256-cell queue wrapping many times."""
    n = 20_000
    onet = O.ONet.random_kout(n, 100, 4)
    g, o, first = lockstep(onet, 200, int_weights=True, chunk=50, gauss_sd=1.0, synapse_tau_ms=5.0,
                           drive=with_ws(shape, lambda s: set_ext(s, n, range(n), 40.0)), mode=nb.KERNEL_STREAM)
    assert first < 0, f"raster diverged at step {first}"
    assert g.spikes_total() > 5 * n
    assert_state_bits_equal(g, o)


@WS_SHAPES
def test_active_random_net_bit_exact(shape):
    """The 100k workload net in its active regime (Poisson kicks 100 Hz x
    20 mV on top of the Gaussian noise, ~23 Hz), rasters and state."""
    onet = O.ONet.random_kout(100_000, 100, 1)
    g, o, first = lockstep(onet, 600, int_weights=True, chunk=100, gauss_sd=1.0, synapse_tau_ms=5.0,
                           noise_rate_hz=100.0, noise_kick_mv=20.0, seed=1, drive=with_ws(shape),
                           mode=nb.KERNEL_STREAM)
    assert first < 0, f"raster diverged at step {first}"
    assert o.mean_rate_hz() > 5.0
    assert_state_bits_equal(g, o)


def test_record_free_instance_bit_exact():
    """No records and no drive: the plain instance of the delivery-warp
    kernel, three full launch groups, spike totals and every state bit after
    each."""
    onet = O.ONet.random_kout(50_000, 100, 2)
    gc, oc = configs(True, 64, 1, gauss_sd=1.0, synapse_tau_ms=5.0, noise_rate_hz=100.0, noise_kick_mv=20.0)
    gc.record_spikes = oc.record_spikes = 0
    g = nb.B200Sim(onet.flat(0.1), gc)
    g.set_kernel_mode(nb.KERNEL_STREAM)
    g.set_tile_shape(256, 2)
    g.set_delivery_warps(True)
    assert g.delivery_warps() == (True, True)
    o = O.OSim(onet, oc)
    for c in range(3):
        g.run_steps(256)
        o.run_steps(256)
        assert g.spikes_total() == o.spikes_total(), f"spike totals differ after launch group {c}"
        assert_state_bits_equal(g, o)
    assert g.spikes_total() > 0


def test_adex_bit_exact():
    onet = O.ONet.random_kout(20_000, 100, 5, w_scale=0.7 * 281.0)
    for i in range(onet.n):
        onet.set_model(i, O.ADEX, ADEX_TONIC)
    g, o, first = lockstep(onet, 800, int_weights=True, chunk=100, gauss_sd=1.0, synapse_tau_ms=5.0,
                           noise_rate_hz=100.0, noise_kick_mv=20.0, seed=2, drive=with_ws((256, 1)),
                           mode=nb.KERNEL_STREAM)
    assert first < 0, f"raster diverged at step {first}"
    assert g.spikes_total() > 0
    assert_state_bits_equal(g, o)


def test_custom_tau_synapses_bit_exact():
    """Delivery warps mark custom-tau arrivals in the bit ring instead of
    adding to the merged ring."""
    onet = mixed_tau_net(3000, 40, 11, 0.5)
    flat = onet.flat()
    g, o, first = lockstep(onet, 1000, int_weights=True, chunk=100, noise_rate_hz=500.0, noise_kick_mv=20.0,
                           seed=5, mode=nb.KERNEL_STREAM, flat=flat, drive=with_ws((128, 2)))
    assert first < 0, f"raster diverged at step {first}"
    assert o.mean_rate_hz() > 5.0
    assert_state_bits_equal(g, o)


def test_f32_ring_counts():
    """f32 ring: float atomics in arbitrary order, so the rasters follow the
    oracle up to a first divergence and the totals stay within the count
    tolerance."""
    onet = O.ONet.bench_net(4000, 100, 5, 0.7, 5.0)
    g, o, first = lockstep(onet, 1000, int_weights=False, chunk=100, noise_rate_hz=500.0, noise_kick_mv=20.0,
                           seed=3, drive=with_ws((128, 4)), mode=nb.KERNEL_STREAM)
    print(f"f32 ring with delivery warps: first divergent step {first}")
    assert first < 0 or first > 5
    a, b = g.spikes_total(), o.spikes_total()
    assert abs(a - b) <= FP32_COUNT_RTOL * b, (a, b)


def test_applies_only_to_streaming_one_net_kernels():
    onet = O.ONet.random_kout(5000, 50, 3)
    g = nb.B200Sim(onet.flat(0.1), nb.default_config(int_weights=1))
    g.set_kernel_mode(nb.KERNEL_RESIDENT)
    g.set_tile_shape(128, 1)
    g.set_delivery_warps(True)
    assert g.delivery_warps() == (True, False)  # the resident kernel delivers with its tile threads
    g.set_kernel_mode(nb.KERNEL_STREAM)
    assert g.delivery_warps() == (True, True)
    g.set_tile_shape(64, 1)  # no delivery-warp instance at 64 threads
    assert g.delivery_warps() == (True, False)
    g.run_steps(10)
    g.set_tile_shape(256, 1)
    g.set_delivery_warps(False)
    assert g.delivery_warps() == (False, False)


def test_autotune_may_choose_delivery_warps_and_keeps_state():
    """Autotune times both kernels on snapshots; whatever it keeps, the run
    continues bit-exact against the oracle."""
    onet = O.ONet.random_kout(30_000, 100, 6)
    gc, oc = configs(True, 100, 1, gauss_sd=1.0, synapse_tau_ms=5.0, noise_rate_hz=100.0, noise_kick_mv=20.0,
                     seed=4)
    g = nb.B200Sim(onet.flat(0.1), gc)
    o = O.OSim(onet, oc)
    g.run_steps(100)
    o.run_steps(100)
    g.set_kernel_mode(nb.KERNEL_STREAM)
    tiling = g.autotune(64)
    print("autotuned:", tiling)
    for _ in range(3):
        g.run_steps(100)
        o.run_steps(100)
    for back in range(100):
        assert np.array_equal(g.spike_row(back), o.spike_row(back)), back
    assert_state_bits_equal(g, o)
