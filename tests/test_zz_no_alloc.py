"""ne2b_spike_counts_noalloc: spike counts for callers that cannot allocate
device memory (a serving thread on a fixed memory budget, or one that must
not stall on cudaMalloc/cudaFree, which synchronise the device).  Called
through the C ABI and checked against ne2b_spike_counts, exactly (the counts
are integers), on two calls in a row.  This file is collected last so that a
run stopping at the first failure has already run every other test."""
import numpy as np
import pytest

import pyoracle as O
import neuro_edit_v2_b200 as nb
from neuro_edit_v2_b200 import _abi

pytestmark = pytest.mark.gpu


def counts(fn, sim, rows):
    out = np.full(sim.n(), 0xDEADBEEF, dtype=np.uint32)
    st = fn(sim._h, rows, out.ctypes.data)
    assert st == _abi.NE2B_OK, _abi.lib.ne2b_last_error().decode()
    return out


def test_noalloc_spike_counts_match_the_allocating_entry_point():
    onet = O.ONet.bench_net(5000, 50, 4, 0.7, 5.0)
    sim = nb.B200Sim(onet.flat(), int_weights=1, record_spikes=1, spike_record_steps=300, noise_rate_hz=400.0)
    sim.run_steps(700)
    # two calls in a row: a sliding window, then lifetime totals
    a1 = counts(_abi.lib.ne2b_spike_counts_noalloc, sim, 250)
    a2 = counts(_abi.lib.ne2b_spike_counts_noalloc, sim, 10**9)
    b1 = counts(_abi.lib.ne2b_spike_counts, sim, 250)
    b2 = counts(_abi.lib.ne2b_spike_counts, sim, 10**9)
    assert np.array_equal(a1, b1)
    assert np.array_equal(a2, b2)
    assert b2.sum() == sim.spikes_total() > 0 and not np.array_equal(b1, b2)
    # and after more steps the shared scratch holds the new counts, not the old
    sim.run_steps(200)
    assert np.array_equal(counts(_abi.lib.ne2b_spike_counts_noalloc, sim, 300),
                          counts(_abi.lib.ne2b_spike_counts, sim, 300))


def test_noalloc_spike_counts_keep_the_window_rules_and_size_limit():
    onet = O.ONet.bench_net(1000, 20, 2, 0.7, 5.0)
    sim = nb.B200Sim(onet.flat(), int_weights=1, record_spikes=1, spike_record_steps=64, noise_rate_hz=400.0)
    sim.run_steps(200)
    with pytest.raises(nb.SpikeWindowError):
        sim.spike_counts_noalloc(100)
    n = (1 << 20) + 64  # one past the scratch array's 1,048,576 neurons
    big = nb.FlatNet(model=np.zeros(n, np.uint8), params=np.tile(np.float32([0.02, 0.2, -65, 8]), (n, 1)),
                     src_ptr=np.zeros(n + 1, np.uint32), tgt=np.zeros(0, np.uint32), w=np.zeros(0, np.float32),
                     delay_steps=np.zeros(0, np.uint16))
    b = nb.B200Sim(big, record_spikes=1)
    b.run_steps(2)
    with pytest.raises(nb.Ne2bError, match="scratch"):
        b.spike_counts_noalloc(1)
