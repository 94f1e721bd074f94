"""`Backend` semantics of the B200 sim through the C ABI, each against the
reference test it mirrors (and the oracle where a value is compared)."""
import numpy as np
import pytest

import pyoracle as O
import neuro_edit_v2_b200 as nb
from helpers import configs, set_ext

pytestmark = pytest.mark.gpu


def one_neuron(depth=64, **kw):
    net = O.ONet()
    net.add_neuron(0, 0, 0, O.EXC)
    g, o = configs(True, depth, **kw)
    return net, nb.B200Sim(net.flat(), g), O.OSim(net, o)


def test_single_neuron_hand_computed_on_gpu():
    """sim/tests/cpu_ref.rs:16-46"""
    net, g, o = one_neuron()
    g.set_external(0, 10.0)
    g.run_steps(1)
    assert abs(g.state(0)[0] - (-64.3)) < 1e-4
    assert abs(g.state(1)[0] - (-12.99972)) < 1e-4


def test_spike_bits_cleared_on_ring_wrap():
    """sim/tests/spike_ring.rs:61-76"""
    net, g, _ = one_neuron(64)
    g.set_external(0, 40.0)
    g.run_steps(64 * 20)
    g.set_external(0, 0.0)
    g.run_steps(200)
    before = g.spikes_total()
    g.run_steps(64)
    assert g.spike_counts(64)[0] == g.spikes_total() - before


def test_spike_counts_window_semantics():
    """sim/tests/spike_ring.rs:78-91"""
    net, g, o = one_neuron(64)
    for s in (g, o):
        s.set_external(0, 40.0)
        s.run_steps(300)
    direct = g.spike_counts(5000)[0]
    assert direct > 0 and direct == g.spikes_total()
    with pytest.raises(nb.SpikeWindowError):
        g.spike_counts(200)
    for rows in (1, 17, 64, 300, 10**9):
        assert np.array_equal(g.spike_counts(rows), o.spike_counts(rows))


def test_spike_row_and_last_spikes_outside_window():
    net, g, o = one_neuron(8)
    assert g.spike_row(0) is None and len(g.last_spikes()) == 0
    g.set_external(0, 40.0)
    o.set_external(0, 40.0)
    for _ in range(30):
        g.run_steps(1)
        o.run_steps(1)
        assert np.array_equal(g.last_spikes(), o.last_step_spikes())
    assert g.spike_row(8) is None
    assert g.spike_row(7) is not None


def test_reset_clears_state_keeps_drive():
    """sim/tests/cpu_ref.rs:322-334; reset keeps ext and stimulus (cpu.rs:155-157)"""
    net = O.ONet()
    for i in range(4):
        net.add_neuron(i * 50.0, 0, 0, O.EXC)
    net.connect(0, 1, 5.0)
    g = nb.B200Sim(net.flat(), record_spikes=1, int_weights=1)
    g.set_external(0, 30.0)
    g.run_steps(50)
    assert g.spikes_total() > 0
    g.reset_state()
    assert g.step_count() == 0 and g.spikes_total() == 0
    assert np.all(g.state(0) == -65.0)
    assert np.all(g.syn_current() == 0.0)
    assert g.external()[0] == 30.0
    g2 = nb.B200Sim(net.flat(), record_spikes=1, int_weights=1)
    g2.set_external(0, 30.0)
    g.run_steps(50)
    g2.run_steps(50)
    assert np.array_equal(g.v().view(np.uint32), g2.v().view(np.uint32))


def test_stimulus_play_loop_and_constants_match_oracle():
    """stim.rs play/loop/constant semantics through run_steps chunks."""
    net = O.ONet()
    for i in range(3):
        net.add_neuron(i * 50.0, 0, 0, O.EXC)
    net.add_input([(0, 1.0), (2, 2.0)])
    net.add_input([(1, 3.0)])
    gc, oc = configs(True, 64)
    g = nb.B200Sim(net.flat(), gc)
    o = O.OSim(net, oc)
    ramp = np.linspace(0, 20, 37).astype(np.float32)
    for s in (g, o):
        s.set_input_constant(0, 5.0)
        s.loop_input(1, [4.0, 0.0, 9.0])
    for k in (7, 1, 100, 2500):
        g.run_steps(k)
        o.run_steps(k)
    for s in (g, o):
        s.play_input(0, ramp)
    g.run_steps(3000)
    o.run_steps(3000)
    assert np.array_equal(g.v().view(np.uint32), o.state(0).view(np.uint32))
    assert g.spikes_total() == o.spikes_total() > 0


def test_set_noise_on_live_sim():
    """lib.rs:183 set_noise; kernel args follow cfg (cuda.rs:807-810)."""
    onet = O.ONet.random_kout(2000, 20, 3)
    gc, oc = configs(True, 64)
    g = nb.B200Sim(onet.flat(), gc)
    o = O.OSim(onet, oc)
    g.run_steps(100)
    o.run_steps(100)
    g.set_noise(800.0, 20.0)
    o.set_noise(800.0, 20.0)
    g.run_steps(500)
    o.run_steps(500)
    assert g.spikes_total() == o.spikes_total() > 0
    assert np.array_equal(g.v().view(np.uint32), o.state(0).view(np.uint32))


def test_empty_net_advances_clock():
    """sim/tests/bounds.rs: an empty net runs (cuda.rs:585-590)."""
    flat = nb.FlatNet(model=np.zeros(0, np.uint8), params=np.zeros((0, 4), np.float32),
                      src_ptr=np.zeros(1, np.uint32), tgt=np.zeros(0, np.uint32), w=np.zeros(0, np.float32),
                      delay_steps=np.zeros(0, np.uint16))
    g = nb.B200Sim(flat, record_spikes=1)
    g.run_steps(10)
    assert g.step_count() == 10 and g.spikes_total() == 0
    assert len(g.spike_counts(5)) == 0


def test_invalid_calls_are_errors():
    net, g, _ = one_neuron()
    with pytest.raises(nb.Ne2bError, match="EINVAL"):
        g.set_input_constant(3, 1.0)
    bad = net.flat()
    bad.tgt = np.array([5], np.uint32)
    bad.src_ptr = np.array([0, 1], np.uint32)
    bad.w = np.array([1.0], np.float32)
    bad.delay_steps = np.array([1], np.uint16)
    with pytest.raises(nb.Ne2bError, match="EINVAL"):
        nb.B200Sim(bad)


def test_window_counts_equal_sliding_spike_counts():
    """On-device per-window counts equal spike_counts(window) at each window end."""
    onet = O.ONet.bench_net(3000, 50, 2, 0.7, 5.0)
    g = nb.B200Sim(onet.flat(), record_spikes=1, spike_record_steps=250, int_weights=1, noise_rate_hz=500.0,
                   window_steps=250, max_windows=8)
    for w in range(6):
        g.run_steps(250)
        ref = g.spike_counts(250)
        assert np.array_equal(g.window_counts(w).astype(np.uint32), ref)
    assert g.windows_done() == 6


@pytest.mark.parametrize("ws, rec", [(1, 2), (7, 5), (100, 64), (250, 300)])
def test_windows_and_record_rows_wrapping_inside_a_launch_group(ws, rec):
    """Windows and record rings shorter than a launch group (256 steps) wrap
    several times inside one group: each window's count equals the oracle's
    spikes over that window's steps, and the last `rec` record rows equal
    the oracle's."""
    onet = O.ONet.bench_net(2000, 40, 3, 0.7, 5.0)
    steps = 600
    n_win = steps // ws
    g = nb.B200Sim(onet.flat(), record_spikes=1, spike_record_steps=rec, int_weights=1, noise_rate_hz=500.0,
                   window_steps=ws, max_windows=n_win)
    o = O.OSim(onet, O.cfg(record_spikes=1, spike_record_steps=steps, int_weights=1, noise_rate_hz=500.0))
    g.run_steps(37)  # the groups then start mid-window
    g.run_steps(steps - 37)
    o.run_steps(steps)
    assert g.windows_done() == n_win
    n = onet.n
    bits = lambda words: np.unpackbits(words.view(np.uint8), bitorder="little")[:n].astype(np.int64)
    rows = np.stack([bits(o.spike_row(steps - 1 - t)) for t in range(steps)])  # [step, neuron]
    for w in range(n_win):
        ref = rows[w * ws:(w + 1) * ws].sum(axis=0)
        assert np.array_equal(g.window_counts(w).astype(np.int64), np.minimum(ref, 65535)), w
    for back in range(rec):
        assert np.array_equal(g.spike_row(back), o.spike_row(back)), back
    assert g.spikes_total() == o.spikes_total() > 0


def test_sim_autotune_restores_state_and_keeps_results():
    """Autotuning times candidate kernels on device snapshots and restores
    the state: a tuned sim continues bit-identically to an untuned one."""
    onet = O.ONet.bench_net(6000, 40, 9, 0.7, 5.0)
    a = nb.B200Sim(onet.flat(), int_weights=1, record_spikes=1, noise_rate_hz=300.0)
    b = nb.B200Sim(onet.flat(), int_weights=1, record_spikes=1, noise_rate_hz=300.0)
    a.run_steps(300)
    b.run_steps(300)
    tiling = a.autotune(64)
    assert tiling["kernel"] in ("stream", "resident") and tiling["block"] in (64, 128, 256, 512)
    assert a.step_count() == 300
    a.run_steps(700)
    b.run_steps(700)
    assert a.spikes_total() == b.spikes_total() > 0
    assert np.array_equal(a.v().view(np.uint32), b.v().view(np.uint32))
    assert np.array_equal(a.trace().view(np.uint32), b.trace().view(np.uint32))
    assert np.array_equal(a.spike_counts(512), b.spike_counts(512))


def test_ne2_file_runs_bit_exact_against_oracle():
    """A `.ne2` file (written by tests/ne2_writer.py from an oracle net, v7)
    loaded by the library and run on the GPU equals the oracle run of the
    same net, with the file's Meta as the config."""
    import ne2_writer as W
    from helpers import assert_state_bits_equal, lockstep

    onet = O.ONet()
    r = O.rng(8)
    m = onet.create_3d_grid(8, 8, 8, 60.0)
    onet.set_exc_inh(m, 0.2, r)
    onet.create_connections(m, 1.0, 120.0, 3.0, r)
    rng = np.random.default_rng(2)
    for _ in range(300):
        onet.push_synapse(int(rng.integers(512)), int(rng.integers(512)), 3.0, float(rng.uniform(0.1, 9.0)),
                          float(rng.uniform(1.0, 25.0)))
    inputs = [("in0", [(int(t), 12.0) for t in rng.integers(0, 512, 24)])]
    for _, tw in inputs:
        onet.add_input(tw)
    desc = W.from_onet(onet, inputs)
    desc["meta"].update(noise_rate_hz=200.0, noise_kick_mv=15.0, seed=21)
    net, meta = nb.from_ne2_bytes(W.encode(desc, 7))
    cfg = nb.config_from_meta(meta)
    series = (rng.random(1200) < 0.05).astype(np.float32)

    def drive(s):
        s.play_input(0, series)

    g, o, first = lockstep(onet, 1200, int_weights=True, chunk=100, flat=net.arrays(), drive=drive,
                           noise_rate_hz=cfg.noise_rate_hz, noise_kick_mv=cfg.noise_kick_mv, seed=cfg.seed,
                           synapse_tau_ms=cfg.synapse_tau_ms, readout_tau_ms=cfg.readout_tau_ms)
    assert first < 0, f"raster diverged at step {first}"
    assert o.spikes_total() > 0
    assert_state_bits_equal(g, o)


def _nine():
    net = O.ONet()
    for i in range(9):
        net.add_neuron(i * 10.0, 0.0, 0.0, O.EXC)
    return net


def test_v_watch_equals_oracle_and_keeps_reference_rules():
    """sim/tests/v_watch.rs on the device: every step recorded, bit-equal to
    the oracle (int ring), drained once, a changed list restarts, the same
    list keeps its history, ids beyond n record 0, duplicates repeat, and
    only the last 4096 samples are kept."""
    onet = O.ONet.bench_net(500, 20, 3, 0.7, 5.0)
    gc, oc = configs(True, 64, noise_rate_hz=500.0, noise_kick_mv=20.0, seed=4)
    g = nb.B200Sim(onet.flat(), gc)
    o = O.OSim(onet, oc)
    ids = [0, 7, 7, 499, 10_000]
    for s in (g, o):
        s.set_v_watch(ids)
        s.run_steps(300)
    a, b = g.drain_watch(), o.drain_watch()
    assert a.shape == (2, 5, 300) and np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert np.all(a[:, 4] == 0.0) and np.array_equal(a[:, 1], a[:, 2])
    assert g.drain_watch().shape == (2, 5, 0)
    for s in (g, o):
        s.set_v_watch(ids)  # same list: a no-op
        s.run_steps(50)
        s.set_v_watch([3])  # new list: history restarts now
        s.run_steps(5000)  # beyond the 4096-sample cap
    a, b = g.drain_watch(), o.drain_watch()
    assert a.shape == (2, 1, 4096) and np.array_equal(a.view(np.uint32), b.view(np.uint32))
    for s in (g, o):
        s.reset_state()
        s.run_steps(10)
    assert np.array_equal(g.drain_watch().view(np.uint32), o.drain_watch().view(np.uint32))


@pytest.mark.parametrize("mode", [nb.KERNEL_STREAM, nb.KERNEL_RESIDENT], ids=["stream", "resident"])
def test_grid_traces_equal_oracle(mode):
    """sim/tests/grid_trace.rs on the device: texel = member-list position,
    groups independent, exp(-age*dt/tau) equal to the oracle's, reset
    clears, no watches means no traces."""
    onet = O.ONet.bench_net(600, 20, 5, 0.7, 5.0)
    gc, oc = configs(True, 64, noise_rate_hz=300.0, noise_kick_mv=20.0, seed=8)
    g = nb.B200Sim(onet.flat(), gc)
    g.set_kernel_mode(mode)
    o = O.OSim(onet, oc)
    assert g.grid_traces(20.0) == []
    groups = [list(range(0, 600, 3)), [5, 2, 5, 599, 9999], list(range(100))]
    for s in (g, o):
        s.set_grid_watches(groups)
        s.run_steps(777)
    for a, b in zip(g.grid_traces(20.0), o.grid_traces(20.0)):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert any(np.any(x > 0) for x in g.grid_traces(5.0))
    for s in (g, o):
        s.reset_state()
    assert all(np.all(x == 0.0) for x in g.grid_traces(20.0))
    for s in (g, o):
        s.run_steps(123)
    for a, b in zip(g.grid_traces(2.0), o.grid_traces(2.0)):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_grid_trace_single_spike_decays_as_the_reference_asserts():
    """grid_trace.rs:23-50"""
    g = nb.B200Sim(_nine().flat(), dt_ms=0.1)
    g.set_grid_watches([list(range(9))])
    g.set_external(4, 1000.0)
    g.run_steps(1)
    g.set_external(4, 0.0)
    g.run_steps(99)
    tr = g.grid_traces(20.0)[0]
    assert abs(tr[4] - np.exp(-100 * 0.1 / 20.0)) < 1e-5
    assert np.all(np.delete(tr, 4) == 0.0)


def test_bounded_grid_barrier_times_out_and_device_stays_usable():
    """A grid-barrier wait that can never end (one block never arrives) stops
    at its limit with the error flag set, and the device keeps working: a
    sim afterwards still equals the oracle."""
    import time

    t0 = time.perf_counter()
    assert nb.selftest_barrier_timeout(50)
    assert time.perf_counter() - t0 < 10.0
    onet = O.ONet.bench_net(1000, 20, 2, 0.7, 5.0)
    gc, oc = configs(True, 100, noise_rate_hz=500.0, noise_kick_mv=20.0, seed=3)
    g = nb.B200Sim(onet.flat(), gc)
    g.set_kernel_mode(nb.KERNEL_RESIDENT)
    o = O.OSim(onet, oc)
    g.run_steps(500)
    o.run_steps(500)
    assert g.spikes_total() == o.spikes_total() > 0


@pytest.mark.parametrize("tau", [2.0, 1000.0])
def test_trace_equals_oracle_for_short_and_long_readout_tau(tau):
    """The readout trace (cpu.rs:252-260): a step-count table for short
    taus, the f32 trace itself where that table would be too long; both
    equal the oracle's repeated multiply bit for bit."""
    onet = O.ONet.bench_net(1500, 30, 6, 0.7, 5.0)
    gc, oc = configs(True, 100, noise_rate_hz=500.0, noise_kick_mv=20.0, seed=2, readout_tau_ms=tau)
    g = nb.B200Sim(onet.flat(), gc)
    o = O.OSim(onet, oc)
    for _ in range(3):
        g.run_steps(700)
        o.run_steps(700)
        assert np.array_equal(g.trace().view(np.uint32), o.trace().view(np.uint32))
    g.reset_state()
    o.reset_state()
    g.run_steps(50)
    o.run_steps(50)
    assert np.array_equal(g.trace().view(np.uint32), o.trace().view(np.uint32))


def test_adex_noise_gain_drives_lone_neuron_on_gpu():
    """sim/tests/adex.rs:174-243 on the device, equal to the oracle."""
    def rates(rate_hz, kick_mv, steps=200_000):
        net = O.ONet()
        net.add_neuron(0.0, 0.0, 0.0, O.EXC)
        net.set_model(0, 1, [281.0, 30.0, -70.6, -50.4, 2.0, 4.0, 144.0, 80.5, -70.6, 20.0])
        g = nb.B200Sim(net.flat(), noise_rate_hz=rate_hz, noise_kick_mv=kick_mv, seed=5)
        o = O.OSim(net, O.cfg(noise_rate_hz=rate_hz, noise_kick_mv=kick_mv, seed=5, exp_mode=1))
        g.run_steps(steps)
        o.run_steps(steps)
        assert g.spikes_total() == o.spikes_total()
        return g.spikes_total() / 20.0

    assert rates(60.0, 14.0) > 0.5
    assert rates(120.0, 18.0) > 1.5 * rates(30.0, 18.0)
