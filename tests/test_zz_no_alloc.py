"""ne2b_spike_counts_noalloc: spike counts for callers that cannot allocate
device memory (a serving thread on a fixed memory budget, or one that must
not stall on cudaMalloc/cudaFree, which synchronise the device).  Called
through the C ABI and checked against ne2b_spike_counts, exactly (the counts
are integers), on two calls in a row; device free memory must not move
across its calls.  This file is collected last so that a run stopping at the
first failure has already run every other test."""
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


def noalloc(sim, rows):
    return counts(_abi.lib.ne2b_spike_counts_noalloc, sim, rows)


def alloc(sim, rows):
    return counts(_abi.lib.ne2b_spike_counts, sim, rows)


def test_noalloc_spike_counts_match_the_allocating_entry_point():
    onet = O.ONet.bench_net(5000, 50, 4, 0.7, 5.0)
    sim = nb.B200Sim(onet.flat(), int_weights=1, record_spikes=1, spike_record_steps=300, noise_rate_hz=400.0)
    sim.run_steps(700)
    # two calls in a row: a sliding window, then lifetime totals
    a1 = noalloc(sim, 250)
    a2 = noalloc(sim, 10**9)
    b1 = alloc(sim, 250)
    b2 = alloc(sim, 10**9)
    assert np.array_equal(a1, b1)
    assert np.array_equal(a2, b2)
    assert b2.sum() == sim.spikes_total() > 0 and not np.array_equal(b1, b2)
    # and after more steps the shared scratch holds the new counts, not the old
    sim.run_steps(200)
    assert np.array_equal(noalloc(sim, 300), alloc(sim, 300))


def test_noalloc_spike_counts_leave_device_free_memory_unchanged():
    import torch

    onet = O.ONet.bench_net(20_000, 50, 6, 0.7, 5.0)
    sim = nb.B200Sim(onet.flat(), int_weights=1, record_spikes=1, spike_record_steps=200, noise_rate_hz=400.0)
    sim.run_steps(300)
    sim.synchronize()
    noalloc(sim, 100)  # loads the kernels' module if it is not loaded yet
    free0, _ = torch.cuda.mem_get_info(0)
    a1 = noalloc(sim, 100)
    a2 = noalloc(sim, 10**9)
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, f"device free memory moved by {free0 - free1} bytes"
    assert np.array_equal(a1, alloc(sim, 100))
    assert np.array_equal(a2, alloc(sim, 10**9))


def test_noalloc_spike_counts_without_recording_or_steps_are_zeros():
    onet = O.ONet.bench_net(3000, 20, 2, 0.7, 5.0)
    quiet = nb.B200Sim(onet.flat(), int_weights=1, record_spikes=0, noise_rate_hz=400.0)
    quiet.run_steps(100)
    assert quiet.spikes_total() > 0
    assert np.array_equal(noalloc(quiet, 50), alloc(quiet, 50))
    assert not noalloc(quiet, 50).any()
    fresh = nb.B200Sim(onet.flat(), int_weights=1, record_spikes=1, spike_record_steps=64)
    assert not noalloc(fresh, 10).any() and np.array_equal(noalloc(fresh, 10), alloc(fresh, 10))


def test_noalloc_spike_counts_of_a_smaller_sim_after_a_larger_one():
    """The scratch keeps the last call's contents: a smaller sim called after
    a larger one must see only its own n entries."""
    big = nb.B200Sim(O.ONet.bench_net(40_000, 50, 8, 0.7, 5.0).flat(), int_weights=1, record_spikes=1,
                     spike_record_steps=128, noise_rate_hz=800.0)
    small = nb.B200Sim(O.ONet.bench_net(2_000, 20, 9, 0.7, 5.0).flat(), int_weights=1, record_spikes=1,
                       spike_record_steps=128, noise_rate_hz=200.0)
    big.run_steps(300)
    small.run_steps(300)
    assert noalloc(big, 10**9).sum() == big.spikes_total() > 0
    s1 = noalloc(small, 100)
    s2 = noalloc(small, 10**9)
    assert np.array_equal(s1, alloc(small, 100))
    assert np.array_equal(s2, alloc(small, 10**9))
    assert s2.sum() == small.spikes_total()


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
    assert not b.spike_counts_noalloc(1).any()  # t == 0: zeros at any size, as ne2b_spike_counts
    b.run_steps(2)
    with pytest.raises(nb.Ne2bError, match="scratch"):
        b.spike_counts_noalloc(1)
