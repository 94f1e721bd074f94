""".ne2 network files (net-format/src/io.rs) through the library's loader.

Pinned on the reference's own fixtures where the reference tree is present
(net-format/tests/format_versions.rs: v1, v2 and v3 files and their
asserted contents; examples/lsm.ne2, a v6 file), and, everywhere, on files
written by tests/ne2_writer.py from oracle nets in every format version: the
loaded net must equal the oracle's own CSR build bit for bit."""
import os

import numpy as np
import pytest

import pyoracle as O
import neuro_edit_v2_b200 as nb
import ne2_writer as W

# The reference's own fixtures are read from the reference tree named by
# NE2_REFERENCE_ROOT; those tests skip when it is unset.
REF = os.environ.get("NE2_REFERENCE_ROOT", "")
FIXTURES = os.path.join(REF, "net-format", "tests", "fixtures") if REF else ""
has_fixtures = pytest.mark.skipif(not (FIXTURES and os.path.isdir(FIXTURES)),
                                  reason="NE2_REFERENCE_ROOT unset or its fixtures absent")


def same_as_oracle(net: nb.NativeNet, onet: O.ONet, dt=0.1):
    a, b = net.arrays(), onet.flat(dt)
    assert np.array_equal(a.src_ptr, b.src_ptr)
    assert np.array_equal(a.tgt, b.tgt)
    assert np.array_equal(a.w.view(np.uint32), b.w.view(np.uint32))
    assert np.array_equal(a.delay_steps, b.delay_steps)
    assert np.array_equal(a.model, b.model)
    for i in range(a.n):
        width = 4 if a.model[i] == 0 else 10
        assert np.array_equal(a.params[i, :width].view(np.uint32), b.params[i, :width].view(np.uint32)), i
    assert np.array_equal(net.kinds(), onet.kinds())
    assert (a.tau_ms is None) == (b.tau_ms is None)
    if a.tau_ms is not None:
        assert np.array_equal(a.tau_ms.view(np.uint32), b.tau_ms.view(np.uint32))
    assert a.n_inputs == b.n_inputs
    if a.n_inputs:
        assert np.array_equal(a.stim_ptr, b.stim_ptr)
        assert np.array_equal(a.stim_input, b.stim_input)
        assert np.array_equal(a.stim_w.view(np.uint32), b.stim_w.view(np.uint32))


@has_fixtures
@pytest.mark.parametrize("version", [1, 2, 3])
def test_reference_fixtures_load_as_the_reference_asserts(version):
    """format_versions.rs:25-80 (check_lifted and the per-version tau)."""
    net, meta = nb.load_ne2(os.path.join(FIXTURES, f"v{version}.ne2"))
    a = net.arrays()
    assert meta["version"] == version
    assert a.n == 4 and a.n_syn == 2
    assert meta["n_types"] == 3 and meta["n_groups"] == 1 and meta["n_scripts"] == 1
    f = lambda *x: np.array(x, np.float32)
    assert np.array_equal(a.params[0, :4], f(0.02, 0.2, -65.0, 8.0))
    assert np.array_equal(a.params[2, :4], f(0.1, 0.2, -65.0, 2.0))
    assert np.array_equal(a.params[3, :4], f(0.03, 0.25, -60.0, 4.0))
    kinds = net.kinds()
    assert kinds[0] == 0 and kinds[2] == 1
    assert a.w.tolist() == [1.5, -2.0]  # Dale's sign at the CSR (format_versions.rs:48-50)
    assert a.n_inputs == 1
    if version < 3:
        assert a.tau_ms is None  # v1/v2 synapses stay on the merged path
    else:
        assert a.tau_ms is not None and float(a.tau_ms[0]) == 7.5


@pytest.mark.skipif(not (REF and os.path.exists(os.path.join(REF, "examples", "lsm.ne2"))),
                    reason="NE2_REFERENCE_ROOT unset or its example absent")
def test_reference_example_lsm_v6_loads_and_runs_config():
    net, meta = nb.load_ne2(os.path.join(REF, "examples", "lsm.ne2"))
    a = net.arrays()
    assert meta["version"] == 6 and meta["n_readouts"] == 1
    assert a.n == 216 and a.n_syn > 0 and a.n_inputs == 8
    cfg = nb.config_from_meta(meta)
    assert abs(cfg.dt_ms - 0.1) < 1e-7 and cfg.seed == meta["seed"]


def oracle_net(seed=4, with_tau=True):
    net = O.ONet()
    r = O.rng(seed)
    m = net.create_3d_grid(5, 5, 4, 60.0)
    net.set_exc_inh(m, 0.2, r)
    net.create_connections(m, 1.0, 120.0, 3.0, r)
    rng = np.random.default_rng(seed)
    if with_tau:
        for _ in range(60):
            net.push_synapse(int(rng.integers(100)), int(rng.integers(100)), 2.5, float(rng.uniform(0.1, 9.0)),
                             float(rng.uniform(1.0, 25.0)))
    return net


@pytest.mark.parametrize("version", [4, 5, 6, 7])
def test_written_files_equal_the_oracle_build(version):
    onet = oracle_net()
    inputs = [("a", [(0, 12.0), (5, 3.0), (7, 12.0)]), ("b", [(5, 1.5), (99, 2.0)])]
    for name, tw in inputs:
        onet.add_input(tw)
    desc = W.from_onet(onet, inputs)
    desc["readouts"] = [dict(name="r", units=[1, 2, 3], weights=[0.5, 0.25, 0.125], bias=0.1, bias_weight=1.0,
                             tau_ms=20.0, pos=(0, 0, 0),
                             mlp=dict(sizes=[3, 2, 1], w=[[0.0] * 8, [0.0] * 3], mu=[0, 0, 0], sd=[1, 1, 1]),
                             mlp_layers=[2])]
    desc["samples"] = [("s", [0.0, 1.0], [2.0, 3.0])]
    desc["scripts"] = [("main", "print(1)")]
    desc["groups"] = [("all", list(range(10)), dict(dims=[2, 5, 1], origin=[0, 0, 0], spacing=60.0, axes=[0, 1, 2]))]
    net, meta = nb.from_ne2_bytes(W.encode(desc, version))
    assert meta["version"] == version and meta["n_readouts"] == 1 and meta["n_samples"] == 1
    same_as_oracle(net, onet)


@pytest.mark.parametrize("version", [1, 2, 3])
def test_written_inline_neuron_files_equal_the_oracle_build(version):
    onet = oracle_net(with_tau=version >= 3)
    desc = W.from_onet(onet, izh_only=True)
    desc["groups"] = [("g", [0, 1], None)]
    net, meta = nb.from_ne2_bytes(W.encode(desc, version))
    same_as_oracle(net, onet)


def test_adex_types_and_param_overrides():
    """Neuron params override the type row (network.rs:549-555)."""
    onet = O.ONet()
    for i in range(6):
        onet.add_neuron(0.0, 0.0, 0.0, O.EXC if i < 4 else O.INH)
    tonic = [281.0, 30.0, -70.6, -50.4, 2.0, 4.0, 144.0, 80.5, -70.6, 20.0]
    onet.set_model(4, 1, tonic)
    onet.set_model(1, 0, [0.03, 0.25, -60.0, 4.0])
    onet.push_synapse(0, 4, 3.0, 1.0, 0.0)
    onet.push_synapse(4, 1, 2.0, 2.0, 5.0)
    desc = W.from_onet(onet)
    # neuron 1 keeps type 0 with an override row instead of its own type
    t0 = desc["neurons"][0][2]
    desc["neurons"][1] = ("n1", (0, 0, 0), t0, [0.03, 0.25, -60.0, 4.0])
    net, _ = nb.from_ne2_bytes(W.encode(desc, 7))
    same_as_oracle(net, onet)


def test_meta_becomes_the_sim_config():
    onet = oracle_net(with_tau=False)
    desc = W.from_onet(onet)
    desc["meta"] = dict(dt_ms=0.05, seed=99, conduction_speed=200.0, synapse_tau_ms=4.0, readout_tau_ms=3.0,
                        noise_rate_hz=10.0, noise_kick_mv=5.0)
    net, meta = nb.from_ne2_bytes(W.encode(desc, 7))
    same_as_oracle(net, onet, dt=0.05)  # delays in steps of the file's dt
    cfg = nb.config_from_meta(meta)
    assert (cfg.dt_ms, cfg.seed, cfg.synapse_tau_ms, cfg.readout_tau_ms, cfg.noise_rate_hz, cfg.noise_kick_mv) == (
        np.float32(0.05), 99, 4.0, 3.0, 10.0, 5.0)


def small_desc():
    return dict(types=[("exc", "izh", [0.02, 0.2, -65.0, 8.0], "exc", None)],
                neurons=[("a", (0, 0, 0), 0, None), ("b", (1, 0, 0), 0, None)],
                synapses=[(0, 1, 1.0, 1.0, 0.0)], groups=[], inputs=[], samples=[], readouts=[], scripts=[],
                meta=dict(W.DEFAULT_META))


@pytest.mark.parametrize("mutate, err", [
    (lambda b: b"XE2\0" + b[4:], "bad magic"),
    (lambda b: b[:4] + b"\x08\0\0\0" + b[8:], "UNSUPPORTED"),
    (lambda b: b[: len(b) - 3], "end of file"),
])
def test_malformed_files_are_errors(mutate, err):
    b = W.encode(small_desc(), 7)
    with pytest.raises(nb.Ne2bError, match=err):
        nb.from_ne2_bytes(mutate(b))


def test_validation_rules_are_errors():
    """Network::validate (network.rs:1007-1236) rejects these."""
    d = small_desc()
    d["synapses"] = [(0, 5, 1.0, 1.0, 0.0)]
    with pytest.raises(nb.Ne2bError, match="only 2 neurons"):
        nb.from_ne2_bytes(W.encode(d, 7))
    d = small_desc()
    d["synapses"] = [(0, 1, 1.0, 1.0, -1.0)]
    with pytest.raises(nb.Ne2bError, match="tau_ms"):
        nb.from_ne2_bytes(W.encode(d, 7))
    d = small_desc()
    d["types"].append(("exc", "izh", [0.1, 0.2, -65.0, 2.0], "inh", None))
    with pytest.raises(nb.Ne2bError, match="duplicate name"):
        nb.from_ne2_bytes(W.encode(d, 7))
    d = small_desc()
    d["meta"]["dt_ms"] = 0.0
    with pytest.raises(nb.Ne2bError, match="dt_ms"):
        nb.from_ne2_bytes(W.encode(d, 7))


def test_unknown_model_is_unsupported():
    d = small_desc()
    d["types"] = [("lif", "lif", [1.0, 2.0, 3.0], "exc", None)]
    with pytest.raises(nb.Ne2bError, match="UNSUPPORTED"):
        nb.from_ne2_bytes(W.encode(d, 7))
