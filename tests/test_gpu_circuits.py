"""GPU checks of the circuit executor (cufhe_circuit_*) and the autotuner.

* a merged uneven workload (random levelised DAGs + ripple-carry adders) at
  each ciphertext level decrypts to its plaintext evaluation on every wire;
* the CUDA-graph run, its replay and the direct run give identical wires;
* the result is bit-identical to evaluating the same waves one by one
  through cufhe_gate_batch (the circuit adds scheduling, not arithmetic);
* gates with scheduling slack move into narrow later waves without adding
  waves;
* the INT8 form runs circuits as a CUDA graph too (bit-identical to the
  direct run) and decrypts correctly, also split into concurrent groups,
  whose new INT8 workspaces are zeroed in stream order while the other
  group's kernels run;
* cufhe_autotune yields a table of lanes-per-CTA choices and gates stay
  correct under it.
"""
import numpy as np
import pytest

from cufhepp_b200 import circuits as CI, client, engine, params as P

pytestmark = pytest.mark.gpu


def words_of(level):
    return P.TLWE1_WORDS if level == engine.LVL1 else P.TLWE0_WORDS


def prepare(sk, net, level, seed):
    rng = np.random.default_rng(seed)
    bits = rng.integers(0, 2, net.inputs.size).astype(np.uint8)
    host = np.zeros((net.num_wires, words_of(level)), np.uint32)
    host[net.inputs] = client.encrypt_bits(sk, bits, 0 if level == engine.LVL02 else level,
                                           seed=seed)
    return bits, host


def check_decrypts(sk, net, level, bits, wires):
    plain = CI.evaluate(net, bits)
    got = client.decrypt_bits(sk, wires[net.out], 0 if level == engine.LVL02 else level)
    assert int(np.count_nonzero(got != plain[net.out])) == 0


def run_circuit(net, level, host):
    d = engine.to_device(host)
    c = engine.Circuit(level, net.num_wires, net.ops, net.in0, net.in1, net.in2, net.out)
    c.run(d, graph=False)
    direct = engine.from_device(d, host.shape)
    c.run(d, graph=True)
    g1 = engine.from_device(d, host.shape)
    c.run(d, graph=True)
    g2 = engine.from_device(d, host.shape)
    info = c.info()
    c.destroy()
    return direct, g1, g2, info


def wave_by_wave(net, level, host):
    """The same circuit evaluated level by level through cufhe_gate_batch_host."""
    ref = host.copy()
    lv = CI.levels(net)
    for w in range(int(lv.max()) + 1):
        gs = np.nonzero(lv == w)[0]
        rows = lambda idx: ref[np.where(idx[gs] >= 0, idx[gs], 0)]  # noqa: E731
        out = engine.gate_batch_host(net.ops[gs], level, rows(net.in0), rows(net.in1),
                                     rows(net.in2))
        engine.synchronize()
        ref[net.out[gs]] = out
    return ref


@pytest.fixture(scope="module")
def lvl1_ctx(keys):
    sk, ek_kb, _ = keys
    engine.initialize(ek_kb)
    engine.set_precision(P.FP64_FFNT)
    yield sk
    engine.cleanup()


@pytest.mark.parametrize("level", [engine.LVL1, engine.LVL0], ids=["lvl1", "lvl0"])
def test_uneven_circuit_matches_plaintext_and_batches(lvl1_ctx, level):
    sk = lvl1_ctx
    net = CI.uneven_workload(11 + level, dags=12, adders=4, dag_gates=(50, 400),
                             adder_width=(8, 24))
    bits, host = prepare(sk, net, level, 40 + level)
    direct, g1, g2, (waves, max_gates, max_lanes) = run_circuit(net, level, host)
    assert waves == int(CI.levels(net).max()) + 1
    assert np.array_equal(direct, g1) and np.array_equal(g1, g2)
    check_decrypts(sk, net, level, bits, direct)
    assert np.array_equal(direct, wave_by_wave(net, level, host))


def test_circuit_with_not_copy_and_nmux(lvl1_ctx):
    sk = lvl1_ctx
    # hand-written: wires 0..3 inputs
    ops = [P.NOT, P.COPY, P.NMUX, P.XNOR, P.MUX, P.NOT]
    i0 = [0, 1, 2, 4, 6, 8]
    i1 = [-1, -1, 3, 5, 4, -1]
    i2 = [-1, -1, 0, -1, 5, -1]
    out = [4, 5, 6, 7, 8, 9]
    net = CI.Netlist(10, np.arange(4, dtype=np.int32), *(np.asarray(x, np.int32)
                     for x in (ops, i0, i1, i2, out)), np.asarray(out, np.int32))
    for trial in range(3):
        bits, host = prepare(sk, net, engine.LVL1, 90 + trial)
        direct, g1, _, (waves, _, _) = run_circuit(net, engine.LVL1, host)
        assert waves == 3 and np.array_equal(direct, g1)
        check_decrypts(sk, net, engine.LVL1, bits, direct)


def test_slack_gates_fill_narrow_waves(lvl1_ctx):
    """A 6-gate chain beside 1400 independent gates: levelised as soon as
    possible, wave 0 would hold 1401 gates and waves 1-5 one each.  Gates
    with slack move into the narrow later waves (none wider than one resident
    round, 4 lanes per SM); the wave count stays the chain length and every
    wire equals the level-by-level evaluation."""
    import torch

    sk = lvl1_ctx
    width, depth = 1400, 6
    ins = np.arange(width + 1, dtype=np.int32)
    chain_out = width + 1 + np.arange(depth, dtype=np.int32)
    side_out = width + 1 + depth + np.arange(width, dtype=np.int32)
    in0 = np.concatenate([[0], chain_out[:-1], ins[:width]]).astype(np.int32)
    in1 = np.concatenate([np.ones(depth, np.int32), ins[1:width + 1]]).astype(np.int32)
    out = np.concatenate([chain_out, side_out]).astype(np.int32)
    ops = np.full(out.size, P.NAND, np.int32)
    net = CI.Netlist(int(out.max()) + 1, ins, ops, in0, in1, np.full(out.size, -1, np.int32),
                     out, out)
    assert int(CI.levels(net).max()) + 1 == depth
    bits, host = prepare(sk, net, engine.LVL1, 61)
    d = engine.to_device(host)
    c = engine.Circuit(engine.LVL1, net.num_wires, net.ops, net.in0, net.in1, net.in2, net.out)
    try:
        waves, _, max_lanes = c.info()
        gates, lanes = c.wave_sizes()
        c.run(d, graph=False)
        wires = engine.from_device(d, host.shape)
    finally:
        c.destroy()
    cap = 4 * torch.cuda.get_device_properties(0).multi_processor_count
    assert waves == depth
    assert int(gates.sum()) == net.gates and int(lanes.sum()) == net.bootstraps()
    assert max_lanes == int(lanes.max()) <= cap
    assert int(lanes[-1]) > 1  # the narrow waves (latest first) took gates
    check_decrypts(sk, net, engine.LVL1, bits, wires)
    assert np.array_equal(wires, wave_by_wave(net, engine.LVL1, host))


@pytest.mark.parametrize("kb", [False, True], ids=["plain", "kb"])
def test_circuit_int8_form(keys, kb):
    sk, ek_kb, ek_nokb = keys
    engine.initialize(ek_kb if kb else ek_nokb)
    engine.set_precision(P.INT8_EXACT)
    try:
        net = CI.uneven_workload(5, dags=2, adders=1, dag_gates=(50, 80), adder_width=(8, 8))
        bits, host = prepare(sk, net, engine.LVL1, 55)
        direct, g1, g2, (waves, _, _) = run_circuit(net, engine.LVL1, host)
        assert np.array_equal(direct, g1) and np.array_equal(g1, g2)
        check_decrypts(sk, net, engine.LVL1, bits, direct)
        # the same circuit as concurrent groups of its components (each group
        # with its own INT8 workspace): the same bits, graph and direct
        c = engine.Circuit(engine.LVL1, net.num_wires, net.ops, net.in0, net.in1, net.in2,
                           net.out, parts=2)
        d = engine.to_device(host)
        for graph in (True, False):
            d.upload(host)
            engine.synchronize()
            c.run(d, graph=graph)
            assert np.array_equal(engine.from_device(d, host.shape), direct), graph
        c.destroy()
    finally:
        engine.set_precision(P.FP64_FFNT)
        engine.initialize(keys[1])  # the KeyBundle key of the module's other tests


def test_circuit_lvl02():
    sk = client.SecretKey.generate(0xC1C)
    engine.initialize_lvl02(client.EvalKey02.generate(sk, keybundle=True))
    try:
        net = CI.uneven_workload(9, dags=4, adders=2, dag_gates=(50, 150), adder_width=(8, 12))
        bits, host = prepare(sk, net, engine.LVL02, 77)
        direct, g1, g2, _ = run_circuit(net, engine.LVL02, host)
        assert np.array_equal(direct, g1) and np.array_equal(g1, g2)
        check_decrypts(sk, net, engine.LVL02, bits, direct)
        # split into two concurrent groups: the same bits, graph and direct
        c = engine.Circuit(engine.LVL02, net.num_wires, net.ops, net.in0, net.in1, net.in2,
                           net.out, parts=2)
        d = engine.to_device(host)
        for graph in (True, False):
            d.upload(host)
            engine.synchronize()
            c.run(d, graph=graph)
            assert np.array_equal(engine.from_device(d, host.shape), direct), graph
        c.destroy()
    finally:
        engine.cleanup_lvl02()


def test_autotune_table_and_gates(lvl1_ctx):
    sk = lvl1_ctx
    table = engine.autotune()
    assert len(table) >= 4
    bounds = [b for b, _ in table]
    assert bounds == sorted(bounds)
    assert all(g in (1, 2, 4) for _, g in table)
    assert engine.autotune_table() == table
    gates = np.array([P.NAND, P.MUX, P.XOR, P.AND] * 300, np.int32)
    rng = np.random.default_rng(4)
    a, b, c = (rng.integers(0, 2, gates.size).astype(np.uint8) for _ in range(3))
    cts = [client.encrypt_bits(sk, x, 1, seed=140 + i) for i, x in enumerate((a, b, c))]
    out = engine.gate_batch_host(gates, engine.LVL1, *cts)
    engine.synchronize()
    exp = np.array([P.TRUTH[g](int(x), int(y), int(z)) for g, x, y, z in zip(gates, a, b, c)])
    assert np.array_equal(client.decrypt_bits(sk, out, 1), exp)


@pytest.mark.parametrize("level,parts", [(engine.LVL1, 2), (engine.LVL1, 3), (engine.LVL0, 2)],
                         ids=["lvl1-2", "lvl1-3", "lvl0-2"])
def test_split_circuit_is_bit_identical(lvl1_ctx, level, parts):
    """cufhe_circuit_create_split: the circuit's connected components packed
    into groups that run concurrently on streams of their own give the same
    wires, bit for bit, as the one-stream circuit (graph and direct runs, on
    the default and on a created stream), with Ctxt<lvl1> wires (IKS then
    blind rotation) and Ctxt<lvl0> wires (blind rotation then IKS)."""
    sk = lvl1_ctx
    net = CI.uneven_workload(23, dags=12, adders=4, dag_gates=(50, 400), adder_width=(8, 24))
    bits, host = prepare(sk, net, level, 61)
    ref, _, _, _ = run_circuit(net, level, host)
    group, n = engine.circuit_split_plan(level, net.num_wires, net.ops, net.in0, net.in1,
                                         net.in2, net.out, parts)
    assert n == parts
    sub_waves = []
    for k in range(n):
        m = np.flatnonzero(group == k)
        sub_waves.append(engine.circuit_plan(level, net.num_wires, net.ops[m], net.in0[m],
                                             net.in1[m], net.in2[m], net.out[m])[1])
    d = engine.to_device(host)
    c = engine.Circuit(level, net.num_wires, net.ops, net.in0, net.in1, net.in2, net.out,
                       parts=parts)
    assert c.info()[0] == max(sub_waves)
    gs, _ = c.wave_sizes()
    assert gs.sum() == net.gates
    st = engine.Stream(0)
    for graph, stream in ((False, None), (True, None), (True, None), (True, st), (False, st)):
        d.upload(host)
        engine.synchronize()
        c.run(d, stream=stream, graph=graph)
        if stream is not None:
            stream.synchronize()  # the download below runs on the default stream
        got = engine.from_device(d, host.shape)
        assert np.array_equal(got, ref), (graph, stream is not None)
    st.destroy()
    c.destroy()
    check_decrypts(sk, net, level, bits, ref)
