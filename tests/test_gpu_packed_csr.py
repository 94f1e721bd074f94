"""The CSR's packed synapse records on the GPU against the C oracle.

A synapse is one 8-byte record, {target | delay_steps << 24, weight bits},
read with one 64-bit load.  Nets whose delays need more than 8 bits (a ring
deeper than 256 slots) or whose targets need more than 24 bits (more than
2^24 neurons) keep the bare target in the record and the delays in their
own u16 array.  Both layouts must give the oracle's rasters and state bit
for bit with the int ring, through the fused, resident and delivery-warp
kernels."""
import numpy as np
import pytest

import pyoracle as O
import neuro_edit_v2_b200 as nb
from helpers import assert_state_bits_equal, lockstep, lockstep_many

pytestmark = pytest.mark.gpu


def long_delay_net(n, k, seed, max_delay_ms):
    """Random K-out net (80/20 RS/FS) with delays uniform in
    [0.05, max_delay_ms] ms: a ring deeper than 256 slots at dt 0.1."""
    rng = np.random.default_rng(seed)
    net = O.ONet()
    for i in range(n):
        net.add_neuron(0.0, 0.0, 0.0, O.EXC if i < 0.8 * n else O.INH)
    src = np.repeat(np.arange(n), k)
    tgt = rng.integers(0, n, n * k)
    w = rng.uniform(0.5, 6.0, n * k)
    d = rng.uniform(0.05, max_delay_ms, n * k)
    for a, b, ww, dd in zip(src, tgt, w, d):
        net.push_synapse(int(a), int(b), float(ww), float(dd))
    return net


@pytest.mark.parametrize("variant", ["stream", "resident", "delivery_warps"])
def test_long_delays_keep_a_u16_delay_array(variant):
    onet = long_delay_net(3000, 40, 3, 40.0)

    def drive(s):
        if isinstance(s, nb.B200Sim) and variant == "delivery_warps":
            s.set_tile_shape(128, 2)
            s.set_delivery_warps(True)
            assert s.delivery_warps() == (True, True)

    mode = nb.KERNEL_RESIDENT if variant == "resident" else nb.KERNEL_STREAM
    g, o, first = lockstep(onet, 1500, int_weights=True, chunk=100, noise_rate_hz=500.0, noise_kick_mv=20.0, seed=9,
                           mode=mode, drive=drive)
    assert g.ring_depth() > 256
    assert first < 0, f"raster diverged at step {first}"
    assert o.mean_rate_hz() > 5.0
    assert_state_bits_equal(g, o)


@pytest.mark.slow
def test_targets_past_24_bits_keep_bare_targets():
    """2^24 + 4096 neurons, two random targets each (delays capped at 1 ms):
    a third of the spikes land on neurons whose index needs 25 bits.  Poisson
    kicks make every neuron fire; 40 steps, every raster row and state bit,
    with the fused kernel and with delivery warps."""
    n = (1 << 24) + 4096
    onet = O.ONet.random_kout(n, 2, 5, delay_cap_ms=1.0)
    variants = [{"mode": nb.KERNEL_STREAM}, {"mode": nb.KERNEL_STREAM, "ws": (256, 4)}]
    gs, o, firsts = lockstep_many(onet, 40, variants, chunk=20, noise_rate_hz=2000.0, noise_kick_mv=20.0,
                                  seed=4, synapse_tau_ms=5.0)
    src, tgt, _, _, _ = onet.synapses()
    assert int(np.max(tgt)) >= 1 << 24
    for g, f, v in zip(gs, firsts, variants):
        assert f < 0, f"{v}: diverged at step {f}"
        assert g.spikes_total() == o.spikes_total() > 0
        for slot in (0, 1):
            assert np.array_equal(g.state(slot).view(np.uint32), o.state(slot).view(np.uint32)), (v, slot)
        assert np.array_equal(g.syn_current().view(np.uint32), o.syn_current().view(np.uint32)), v
