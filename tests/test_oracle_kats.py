"""The oracle against the reference's own known-answer tests.

Each test restates one test of the reference (cited file:line) against the C
restatement in oracle/.  Passing them pins the oracle to the Rust CPU path:
above all the FNV fingerprint 0x9d792bd233132f5d of sim/tests/cpu_ref.rs:
208-244 covers Rng, create_2d_grid, create_connections, synapse_csr, Poisson
noise and the Izhikevich step bit-for-bit.
"""
import math
import struct

import numpy as np
import pytest

import pyoracle as O


def net_with(n):
    """cpu_ref.rs:8-14"""
    net = O.ONet()
    for i in range(n):
        net.add_neuron(i * 50.0, 0.0, 0.0, O.EXC)
    return net


def f32(x):
    return struct.unpack("f", struct.pack("f", x))[0]


def test_default_tau_fingerprint():
    """cpu_ref.rs:208-244 — the pinned bit-exact fingerprint."""
    net = O.ONet()
    r = O.rng(3)
    m = net.create_2d_grid(8, 8, 30.0)
    net.create_connections(m, 0.35, 80.0, 6.0, r)
    sim = O.OSim(net, O.cfg(record_spikes=1, spike_record_steps=512, noise_rate_hz=20.0, noise_kick_mv=0.8, seed=7))
    sim.run_steps(400)
    assert sim.fingerprint(400) == 0x9D792BD233132F5D


def test_single_neuron_step_matches_hand_computed():
    """cpu_ref.rs:16-46"""
    net = net_with(1)
    sim = O.OSim(net, O.cfg())
    sim.set_external(0, 10.0)
    sim.run_steps(1)
    assert abs(sim.state(0)[0] - (-64.3)) < 1e-4
    assert abs(sim.state(1)[0] - (-12.99972)) < 1e-4
    sim.run_steps(1)
    v2 = -64.3 + 0.1 * (0.04 * 64.3 * 64.3 - 5.0 * 64.3 + 140.0 + 12.99972 + 10.0)
    assert abs(sim.state(0)[0] - v2) < 1e-3


def test_spike_resets_next_step():
    """cpu_ref.rs:48-69"""
    sim = O.OSim(net_with(1), O.cfg())
    sim.set_external(0, 30.0)
    for _ in range(200):
        sim.run_steps(1)
        if sim.trace()[0] > 0.9:
            break
    else:
        pytest.fail("neuron should spike")
    tr = sim.trace()[0]
    sim.run_steps(1)
    assert sim.state(0)[0] < -60.0
    assert sim.trace()[0] < tr


def _fire_once(sim, amps=25.0):
    sim.set_external(0, amps)
    for _ in range(500):
        before = sim.spikes_total()
        sim.run_steps(1)
        if sim.spikes_total() > before:
            return sim.t - 1
    pytest.fail("no spike")


def test_synapse_arrives_after_delay_and_decays():
    """cpu_ref.rs:71-114"""
    net = net_with(2)
    net.push_synapse(0, 1, 30.0, 0.2, 0.0)
    sim = O.OSim(net, O.cfg())
    _fire_once(sim)
    sim.set_external(0, 0.0)
    sim.run_steps(1)
    assert sim.syn_current()[1] == 0.0
    sim.run_steps(1)
    assert abs(sim.syn_current()[1] - 30.0 * math.exp(-0.1 / 2.0)) < 1e-3
    sim.run_steps(1)
    assert abs(sim.syn_current()[1] - 30.0 * math.exp(-0.05) ** 2) < 1e-2


def test_no_self_connection_and_csr_order():
    """cpu_ref.rs:246-255"""
    net = net_with(3)
    net.connect(0, 1, 5.0)
    net.connect(0, 2, 6.0)
    net.connect(2, 0, 7.0)
    c = net.csr(0.1)
    assert list(c["src_ptr"]) == [0, 2, 2, 3]
    assert list(c["tgt"]) == [1, 2, 0]


def test_stimulus_reaches_only_its_targets():
    """cpu_ref.rs:257-275"""
    net = net_with(3)
    net.add_input([(0, 1.0), (2, 2.0)])
    sim = O.OSim(net, O.cfg())
    sim.set_input_constant(0, 5.0)
    s1 = sim.syn_current()[1]
    sim.run_steps(1)
    assert sim.syn_current()[1] == s1
    v = sim.state(0)
    assert abs(v[2] - v[0]) > 0.05
    assert abs(v[0] - -64.8) < 0.2


def test_played_series_is_step_locked():
    """cpu_ref.rs:277-303"""
    net = net_with(1)
    net.add_input([(0, 1.0)])
    sim = O.OSim(net, O.cfg())
    sim.play_input(0, [10.0, 0.0, 0.0])
    sim.run_steps(1)
    assert abs(sim.state(0)[0] - (-64.3)) < 1e-4
    assert sim.stim_value(0, 3) == 0.0
    sim.play_input(0, [25.0] * 20)
    spiked = False
    for _ in range(20):
        sim.run_steps(1)
        spiked |= sim.trace()[0] == 1.0
    assert spiked


def test_noise_is_deterministic_per_seed():
    """cpu_ref.rs:305-320"""
    net = net_with(64)
    a = O.OSim(net, O.cfg(noise_rate_hz=500.0))
    b = O.OSim(net, O.cfg(noise_rate_hz=500.0))
    c = O.OSim(net, O.cfg(noise_rate_hz=500.0, seed=2))
    for s in (a, b, c):
        s.run_steps(100)
    assert np.array_equal(a.state(0), b.state(0))
    assert not np.array_equal(a.state(0), c.state(0))


def test_reset_clears_state():
    """cpu_ref.rs:322-334"""
    net = net_with(4)
    net.connect(0, 1, 5.0)
    sim = O.OSim(net, O.cfg())
    sim.set_external(0, 30.0)
    sim.run_steps(50)
    sim.reset_state()
    assert sim.t == 0
    assert np.all(sim.state(0) == -65.0)
    assert np.all(sim.syn_current() == 0.0)


def test_inhibitory_source_suppresses_target():
    """cpu_ref.rs:339-394"""

    def pair(inh, synapse):
        net = O.ONet()
        net.add_neuron(0, 0, 0, O.INH if inh else O.EXC)
        net.add_neuron(60.0, 0, 0, O.EXC)
        if synapse:
            net.connect(0, 1, 6.0)
        return net

    def run(net):
        sim = O.OSim(net, O.cfg(record_spikes=1))
        sim.set_external(0, 30.0)
        sim.set_external(1, 12.0)
        sim.run_steps(4000)
        return int(sim.spike_counts(2**63)[1])

    free, inh, exc = run(pair(True, False)), run(pair(True, True)), run(pair(False, True))
    assert free > 0 and inh < free and exc > inh
    assert np.all(pair(True, True).csr()["w"] < 0)
    assert np.all(pair(False, True).csr()["w"] > 0)


def test_delay_over_ring_is_an_error():
    """cpu_ref.rs:447-462"""
    net = O.ONet()
    net.add_neuron(0, 0, 0, O.EXC)
    net.add_neuron(10, 0, 0, O.EXC)
    net.push_synapse(0, 1, 1.0, 7000.0, 0.0)
    with pytest.raises(ValueError, match="exceeds"):
        net.csr(0.1)


def test_custom_tau_arrives_then_decays():
    """cpu_ref.rs:116-165"""
    net = net_with(2)
    net.push_synapse(0, 1, 30.0, 0.2, 20.0)
    sim = O.OSim(net, O.cfg())
    _fire_once(sim)
    sim.set_external(0, 0.0)
    sim.run_steps(1)
    assert sim.syn_current()[1] == 0.0
    sim.run_steps(1)
    assert sim.syn_current()[1] == 0.0  # custom synapse must not feed merged s


def test_tau_below_dt_decays_safely():
    """cpu_ref.rs:467-498"""
    net = O.ONet()
    net.add_neuron(0, 0, 0, O.EXC)
    net.add_neuron(10, 0, 0, O.EXC)
    net.push_synapse(0, 1, 5.0, 1.0, 0.05)
    sim = O.OSim(net, O.cfg(record_spikes=1))
    sim.set_external(0, 30.0)
    sim.run_steps(300)
    assert np.all(np.isfinite(sim.state(1)))
    s = sim.syn_current()
    assert np.all(np.isfinite(s)) and np.all(s >= 0.0)


def _splitmix64(x):
    M = (1 << 64) - 1
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & M
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & M
    return x ^ (x >> 31)


def test_noise_hash_is_splitmix64():
    """sim/tests/noise_hash.rs:15-33 (six golden tuples through an independent splitmix64)"""
    M = (1 << 64) - 1
    for i, t, seed in [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (7, 4096, 42),
                       (0xFFFFFFFF, (2**64 - 1) // 2, 0xDEADBEEF)]:
        base = (i * 0x9E3779B97F4A7C15 + t * 0xBF58476D1CE4E5B9 + seed * 0x94D049BB133111EB) & M
        assert O.noise_hash(i, t, seed) == _splitmix64(base) >> 32


def test_noise_streams_are_uncorrelated():
    """sim/tests/noise_hash.rs:37-80 (agreement of p=0.1 streams ~ 0.82)"""
    p = f32(0.1)
    fires = np.zeros((101, 501), bool)
    for i in range(101):
        for t in range(501):
            fires[i, t] = f32(float(O.noise_hash(i, t, 7)) * f32(2.3283064e-10)) < p
    a = fires[:100, :500]
    agree_n = np.mean(a == fires[1:101, :500])
    agree_t = np.mean(a == fires[:100, 1:501])
    assert abs(agree_n - 0.82) < 0.02 and abs(agree_t - 0.82) < 0.02
    assert abs(a.mean() - 0.1) < 0.01


def test_spike_bits_cleared_on_ring_wrap():
    """sim/tests/spike_ring.rs:25-37"""
    net = O.ONet()
    net.add_neuron(0, 0, 0, O.EXC)
    sim = O.OSim(net, O.cfg(record_spikes=1, spike_record_steps=64))
    sim.set_external(0, 40.0)
    sim.run_steps(64 * 20)
    sim.set_external(0, 0.0)
    sim.run_steps(200)
    before = sim.spikes_total()
    sim.run_steps(64)
    assert sim.spike_counts(64)[0] == sim.spikes_total() - before


def test_spike_counts_window_semantics():
    """sim/tests/spike_ring.rs:41-59"""
    net = O.ONet()
    net.add_neuron(0, 0, 0, O.EXC)
    sim = O.OSim(net, O.cfg(record_spikes=1, spike_record_steps=64))
    sim.set_external(0, 40.0)
    sim.run_steps(300)
    direct = int(sim.pn_total()[0])
    assert direct > 0
    assert sim.spike_counts(5000)[0] == direct
    assert sim.spike_counts(64)[0] <= direct
    with pytest.raises(ValueError, match="exceeds"):
        sim.spike_counts(200)


def test_playing_one_input_does_not_restart_others():
    """sim/tests/stim_playhead.rs:9-24"""
    net = O.ONet()
    net.add_neuron(0, 0, 0, O.EXC)
    net.add_input([(0, 1.0)])
    net.add_input([(0, 1.0)])
    sim = O.OSim(net, O.cfg())
    sim.play_input(0, np.arange(100, dtype=np.float32))
    sim.run_steps(50)
    before = sim.stim_value(0, sim.t)
    sim.play_input(1, np.zeros(10, np.float32))
    assert sim.stim_value(0, sim.t) == before == 50.0


def test_looped_series_repeats():
    """sim/src/stim.rs:501-527 (loop_input phase)"""
    net = O.ONet()
    net.add_neuron(0, 0, 0, O.EXC)
    net.add_input([(0, 10.0)])
    net.add_input([(0, 10.0)])
    sim = O.OSim(net, O.cfg())
    sim.loop_input(1, [1.0, 2.0, 3.0])
    assert [sim.stim_value(1, t) for t in range(7)] == [1, 2, 3, 1, 2, 3, 1]
    sim.run_steps(1000)
    assert sim.stim_value(1, sim.t) == 2.0


ADEX_TONIC = [281.0, 30.0, -70.6, -50.4, 2.0, 4.0, 144.0, 80.5, -70.6, 20.0]


def test_adex_mixed_net_fires_on_cpu():
    """sim/tests/adex.rs:296-323"""
    for exp_mode in (0, 1):
        net = net_with(8)
        for i in (1, 3, 6):
            net.set_model(i, O.ADEX, ADEX_TONIC)
        sim = O.OSim(net, O.cfg(record_spikes=1, exp_mode=exp_mode))
        for i in (1, 3, 6):
            sim.set_external(i, 1000.0)
        sim.run_steps(3000)
        c = sim.spike_counts(2**63)
        assert all(c[i] >= 2 for i in (1, 3, 6)), c


def test_adex_v_cut_at_vpeak():
    """sim/tests/adex.rs:251-276 (every per-step v <= Vpeak)"""
    net = O.ONet()
    net.add_neuron(0, 0, 0, O.EXC)
    net.set_model(0, O.ADEX, ADEX_TONIC)
    sim = O.OSim(net, O.cfg(record_spikes=1, exp_mode=1))
    sim.set_external(0, 1000.0)
    vmax = -1e9
    for _ in range(3000):
        sim.step()
        vmax = max(vmax, sim.state(0)[0])
    assert sim.spike_counts(2**63)[0] >= 2
    assert vmax <= 20.0


def test_det_expf_against_libm():
    """The deterministic exp of the AdEx step stays within 1 ulp of glibc expf
    on a sweep spread evenly over its argument range, and equals it on most
    of the points (94% here; over every float of [-104, 10], which crowd near
    0, on 99.6%)."""
    import ctypes

    libm = ctypes.CDLL("libm.so.6")
    libm.expf.restype = ctypes.c_float
    libm.expf.argtypes = [ctypes.c_float]
    xs = np.concatenate([np.linspace(-103.0, 10.0, 20001, dtype=np.float32),
                         np.array([0.0, -0.0, 1e-30, -1e-30, 88.7, 10.0, -87.3], np.float32)])
    worst = 0
    mism = 0
    for x in xs:
        a = O.det_expf(float(x))
        b = libm.expf(float(x))
        ia = struct.unpack("<i", struct.pack("<f", a))[0]
        ib = struct.unpack("<i", struct.pack("<f", b))[0]
        worst = max(worst, abs(ia - ib))
        mism += ia != ib
    assert worst <= 1
    assert mism <= len(xs) // 10


def test_gauss_noise_moments():
    """Project noise definition: mean 0, variance 1 - 2^-16, the kurtosis of
    a sum of four uniforms (3 - 6/20 = 2.7) on a seeded sample, and no
    correlation between neighbouring neurons or steps."""
    z = np.array([[O.gauss_numer(i, t, 5) for t in range(300)] for i in range(300)], dtype=np.float64)
    assert z.min() >= -510 and z.max() <= 510
    z *= math.sqrt(3.0) / 256.0
    assert abs(z.mean()) < 0.01
    assert abs(z.var() - 1.0) < 0.02
    kurt = ((z - z.mean()) ** 4).mean() / z.var() ** 2
    assert abs(kurt - 2.7) < 0.05, kurt
    for a, b in ((z[1:, :], z[:-1, :]), (z[:, 1:], z[:, :-1])):
        assert abs(np.corrcoef(a.ravel(), b.ravel())[0, 1]) < 0.02


def test_gauss_noise_known_answers():
    """The definition written out in Python integers on a few (i, t, seed)."""
    def ref(i, t, seed):
        m = (1 << 64) - 1
        st = (t * 0xBF58476D1CE4E5B9 + seed * 0x94D049BB133111EB) & m
        x = i ^ (st & 0xFFFFFFFF)
        x ^= x >> 16
        x = (x * 0x7FEB352D) & 0xFFFFFFFF
        x ^= x >> 15
        x = (x * 0x846CA68B) & 0xFFFFFFFF
        x ^= x >> 16
        x ^= st >> 32
        x = (x * 0x9E3779B1) & 0xFFFFFFFF
        x ^= x >> 16
        return sum((x >> s) & 0xFF for s in (0, 8, 16, 24)) - 510

    for i, t, seed in ((0, 0, 0), (1, 0, 0), (0, 1, 0), (12345, 678, 9), (2**32 - 1, 2**40 + 3, 2**63 + 5)):
        assert O.gauss_numer(i, t, seed) == ref(i, t, seed), (i, t, seed)


# --- editor watches (sim/tests/v_watch.rs, sim/tests/grid_trace.rs) ---------
def _four():
    net = O.ONet()
    for _ in range(4):
        net.add_neuron(0.0, 0.0, 0.0, O.EXC)
    return net


def test_watched_neurons_record_every_step():
    """v_watch.rs:17-40"""
    sim = O.OSim(_four(), O.cfg())
    sim.set_v_watch([0, 2])
    sim.set_external(0, 40.0)
    sim.run_steps(200)
    h = sim.drain_watch()[0]
    assert h.shape == (2, 200)
    assert np.any(h[0] > 0.0)
    assert np.all(h[1] < -50.0)
    assert sim.drain_watch().shape[2] == 0
    sim.run_steps(30)
    assert sim.drain_watch().shape[2] == 30


def _nine():
    net = O.ONet()
    for i in range(9):
        net.add_neuron(i * 10.0, 0.0, 0.0, O.EXC)
    return net


def test_grid_trace_marks_spiked_member_and_decays():
    """grid_trace.rs:23-50"""
    sim = O.OSim(_nine(), O.cfg())
    sim.set_grid_watches([list(range(9))])
    sim.set_external(4, 1000.0)
    sim.run_steps(1)
    sim.set_external(4, 0.0)
    sim.run_steps(99)
    tr = sim.grid_traces(20.0)[0]
    for k, v in enumerate(tr):
        if k == 4:
            assert abs(v - np.exp(-100 * 0.1 / 20.0)) < 1e-5
        else:
            assert v == 0.0


def test_grid_texel_is_member_list_position_and_groups_are_independent():
    """grid_trace.rs:52-90"""
    sim = O.OSim(_nine(), O.cfg())
    sim.set_grid_watches([[7, 3, 5]])
    sim.set_external(5, 1000.0)
    sim.run_steps(1)
    tr = sim.grid_traces(20.0)[0]
    assert tr[2] > 0.0 and tr[0] == 0.0 and tr[1] == 0.0
    sim = O.OSim(_nine(), O.cfg())
    sim.set_grid_watches([[0, 1, 2], [2, 4]])
    sim.set_external(2, 1000.0)
    sim.run_steps(1)
    a, b = sim.grid_traces(20.0)
    assert a[2] > 0.0 and a[0] == 0.0 and b[0] > 0.0 and b[1] == 0.0
    sim.reset_state()
    assert all(np.all(x == 0.0) for x in sim.grid_traces(20.0))
    assert O.OSim(_nine(), O.cfg()).grid_traces(20.0) == []


def _lone_adex_rate(rate_hz, kick_mv, ms=20000.0):
    net = O.ONet()
    net.add_neuron(0.0, 0.0, 0.0, O.EXC)
    net.set_model(0, 1, [281.0, 30.0, -70.6, -50.4, 2.0, 4.0, 144.0, 80.5, -70.6, 20.0])
    sim = O.OSim(net, O.cfg(noise_rate_hz=rate_hz, noise_kick_mv=kick_mv, seed=5))
    sim.run_steps(int(round(ms / 0.1)))
    return sim.spikes_total() / (ms / 1000.0)


def test_adex_noise_gain_drives_lone_neuron():
    """sim/tests/adex.rs:174-233: the Poisson kick is scaled by the AdEx gain
    (C), so a lone AdEx cell fires at 60 Hz x 14 mV and fires more at a
    higher noise rate."""
    assert _lone_adex_rate(60.0, 14.0) > 0.5
    assert _lone_adex_rate(120.0, 18.0) > 1.5 * _lone_adex_rate(30.0, 18.0)


def test_ridge_multi_oracle_equals_the_dual_solution():
    """readout.rs:190-252 restated: the dual ridge weights equal numpy's
    solve of (Xc Xc^T + lambda I) A = Yc, w = Xc^T A, bias = ybar - w.mu."""
    rng = np.random.default_rng(0)
    t, f, k, lam = 60, 203, 3, 0.5
    x = rng.poisson(2.0, (t, f)).astype(np.float32)
    lab = rng.integers(0, k, t)
    w = O.fit_ridge_multi(x, lab, k, lam)
    xd = x.astype(np.float64)
    mu = xd.mean(0)
    xc = xd - mu
    ybar = np.array([np.mean(lab == c) for c in range(k)])
    yc = np.stack([(lab == c) - ybar[c] for c in range(k)], 1)
    a = np.linalg.solve(xc @ xc.T + lam * np.eye(t), yc)
    ww = (xc.T @ a).T
    ref = np.concatenate([ww, (ybar - ww @ mu)[:, None]], 1)
    assert np.abs(w - ref).max() < 1e-12 * max(1.0, np.abs(ref).max())


def test_cholesky_solve_rejects_a_matrix_that_is_not_positive_definite():
    """readout.rs:153-156: a non-positive pivot ends the factorization."""
    import ctypes

    a = np.array([[1.0, 2.0], [2.0, 1.0]])
    b = np.ones(2)
    w = np.zeros(2)
    assert O.lib().ne2o_cholesky_solve(a.ctypes.data, b.ctypes.data, 2, w.ctypes.data) == 0
    a = np.array([[4.0, 2.0], [2.0, 3.0]])
    assert O.lib().ne2o_cholesky_solve(a.ctypes.data, b.ctypes.data, 2, w.ctypes.data) == 1
    assert np.allclose(a @ w, b)


def test_ridge_oracle_equals_the_normal_equations():
    """readout.rs:103-141 restated: (X1^T X1 + lambda I', bias unregularised) w = X1^T y."""
    rng = np.random.default_rng(1)
    t, f, lam = 80, 31, 0.5
    x = rng.poisson(2.0, (t, f)).astype(np.float32)
    y = (rng.random(t) < 0.5).astype(np.float32)
    w = O.fit_ridge(x, y, lam)
    x1 = np.concatenate([x.astype(np.float64), np.ones((t, 1))], 1)
    a = x1.T @ x1 + lam * np.eye(f + 1)
    a[f, f] -= lam
    ref = np.linalg.solve(a, x1.T @ y.astype(np.float64))
    assert np.abs(w - ref).max() < 1e-11 * max(1.0, np.abs(ref).max())


def reference_ridge_linear_case():
    """The design of sim/src/readout.rs:311-321 (ridge_fits_linear): six
    samples of two features, y = 2 x0 - x1 + 0.5 computed in f32."""
    x = np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0], [1.0, 1.0], [2.0, 1.0], [-1.0, 2.0]], np.float32)
    y = (np.float32(2.0) * x[:, 0] - x[:, 1] + np.float32(0.5)).astype(np.float32)
    return x, y


def reference_ridge_dual_case():
    """The design of sim/src/readout.rs:355-360 (ridge_multi_dual_matches_primal):
    Rng(3), 40 x 7 features uniform in [-1, 1) as f32, labels row % 3."""
    r = O.rng(3)
    t, f, k = 40, 7, 3
    x = np.array([np.float32(-1.0 + 2.0 * O.lib().ne2o_rng_f64(O.C.byref(r))) for _ in range(t * f)],
                 np.float32).reshape(t, f)
    return x, np.arange(t) % k, k


def ridge_output(w, row):
    """sim/src/readout.rs:254-262: bias first, then the features in order, in f64."""
    s = float(w[-1])
    for i in range(len(row)):
        s += float(w[i]) * float(row[i])
    return s


def test_ridge_fits_linear_reference_case():
    """readout.rs:310-326: weights 2, -1 and bias 0.5 within 1e-3 at lambda 1e-9."""
    x, y = reference_ridge_linear_case()
    w = O.fit_ridge(x, y, 1e-9)
    assert abs(w[0] - 2.0) < 1e-3 and abs(w[1] + 1.0) < 1e-3 and abs(w[2] - 0.5) < 1e-3, w


def test_ridge_multi_dual_matches_primal_reference_case():
    """readout.rs:354-375: each class's dual (multi) readout scores every row
    within 1e-4 of the primal binary readout trained on that class."""
    x, lab, k = reference_ridge_dual_case()
    ws = O.fit_ridge_multi(x, lab, k, 0.7)
    for c in range(k):
        wp = O.fit_ridge(x, (lab == c).astype(np.float32), 0.7)
        for r in range(x.shape[0]):
            assert abs(ridge_output(wp, x[r]) - ridge_output(ws[c], x[r])) < 1e-4, (c, r)
