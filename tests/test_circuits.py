"""Circuit workload generators and the circuit executor's host-side checks
(no GPU: cufhe_circuit_create validates and levelises before it needs keys,
and cufhe_circuit_plan runs the validation, levelisation and wave balancing on
the host alone)."""
import ctypes as C

import numpy as np
import pytest

from cufhepp_b200 import circuits as CI, engine, params as P


def test_random_dag_is_levelised():
    rng = np.random.default_rng(1)
    for n in (50, 333, 2000):
        net = CI.random_dag(rng, n)
        assert net.gates == n
        assert set(np.unique(net.ops)) <= set(CI.BINARY.tolist())
        w = CI.levels(net)
        # gates are emitted level by level, each level 1..64 wide
        _, counts = np.unique(w, return_counts=True)
        assert counts.max() <= 64 and counts.min() >= 1
        assert np.all(np.diff(w) >= 0)
        # every gate reads a wire of the previous level
        prod = np.full(net.num_wires, -1)
        prod[net.out] = w
        assert np.all(prod[net.in0] == w - 1)


def test_ripple_carry_adder_adds():
    rng = np.random.default_rng(2)
    for width in (8, 23, 64):
        net = CI.ripple_carry_adder(width)
        for _ in range(5):
            x = int.from_bytes(rng.bytes(8), "little") % (1 << width)
            y = int.from_bytes(rng.bytes(8), "little") % (1 << width)
            cin = int(rng.integers(0, 2))
            bits = np.array([(x >> i) & 1 for i in range(width)] +
                            [(y >> i) & 1 for i in range(width)] + [cin], np.uint8)
            v = CI.evaluate(net, bits)
            got = sum(int(v[w]) << i for i, w in enumerate(net.outputs))
            assert got == x + y + cin
        # depth: all XORs of a and b in wave 0, then one carry Mux per wave
        assert CI.levels(net).max() == width


def test_merge_keeps_each_part():
    rng = np.random.default_rng(3)
    parts = [CI.random_dag(rng, 120), CI.ripple_carry_adder(9), CI.random_dag(rng, 77)]
    m = CI.merge(parts)
    assert m.gates == sum(p.gates for p in parts)
    ins = [rng.integers(0, 2, p.inputs.size).astype(np.uint8) for p in parts]
    vm = CI.evaluate(m, np.concatenate(ins))
    off = 0
    for p, x in zip(parts, ins):
        assert np.array_equal(vm[off:off + p.num_wires], CI.evaluate(p, x))
        off += p.num_wires


def test_uneven_workload_shape():
    net = CI.uneven_workload(7, dags=6, adders=3, dag_gates=(50, 200))
    kinds = [k for k, _ in net.parts]
    assert kinds.count("dag") == 6 and kinds.count("adder") == 3
    assert net.bootstraps() == net.gates + int(np.count_nonzero(net.ops == P.MUX))


def create(level, nw, ops, i0, i1, i2, out):
    arr = lambda a: np.ascontiguousarray(a, np.int32)  # noqa: E731
    ops, i0, i1, i2, out = map(arr, (ops, i0, i1, i2, out))
    h = C.c_void_p()
    rc = engine.load().cufhe_circuit_create(C.byref(h), level, nw, ops.size, engine._p(ops),
                                            engine._p(i0), engine._p(i1), engine._p(i2),
                                            engine._p(out), 0)
    return rc, engine.load().cufhe_last_error().decode()


@pytest.mark.parametrize("case,msg", [
    (dict(ops=[P.NAND, P.AND], i0=[0, 2], i1=[1, 3], out=[3, 2]), "cycle"),
    (dict(ops=[P.NAND, P.AND], i0=[0, 0], i1=[1, 1], out=[2, 2]), "written by gates"),
    (dict(ops=[P.NAND], i0=[0], i1=[9], out=[2]), "out of range"),
    (dict(ops=[P.MUX], i0=[0], i1=[1], i2=[-1], out=[2]), "out of range"),
    (dict(ops=[77], i0=[0], i1=[1], out=[2]), "bad gate id"),
    (dict(ops=[P.NAND], i0=[0], i1=[0], out=[0]), "cycle"),
])
def test_circuit_create_rejects_bad_dags(case, msg):
    n = len(case["ops"])
    rc, err = create(1, 4, case["ops"], case["i0"], case["i1"], case.get("i2", [-1] * n),
                     case["out"])
    assert rc == -1 and msg in err, err


def test_valid_circuit_needs_keys_without_a_gpu():
    # a valid DAG passes validation and then needs the level's keys
    rc, err = create(1, 5, [P.NAND, P.XOR, P.NOT], [0, 2, 3], [1, 1, -1], [-1, -1, -1], [2, 3, 4])
    assert rc == -2 and "initialize" in err


def lanes_of(ops):
    ops = np.asarray(ops)
    return np.where((ops == P.NOT) | (ops == P.COPY), 0,
                    np.where((ops == P.MUX) | (ops == P.NMUX), 2, 1))


def check_plan(net, level, sms):
    """cufhe_circuit_plan's waves keep every dependency, use exactly the
    critical path's number of waves, keep the total work, and never push a
    wave above one resident round of lanes unless levelisation already had
    it there (gates only move into waves with room)."""
    asap = CI.levels(net)
    wave, nwaves = engine.circuit_plan(level, net.num_wires, net.ops, net.in0, net.in1, net.in2,
                                       net.out, sms)
    assert nwaves == int(asap.max()) + 1
    assert np.all(wave >= asap) and wave.max() == nwaves - 1
    prod = np.full(net.num_wires, -1)
    prod[net.out] = np.arange(net.gates)
    for x in (net.in0, net.in1, net.in2):
        has = (x >= 0) & (prod[np.where(x >= 0, x, 0)] >= 0)
        src = prod[x[has]]
        assert np.all(wave[src] < wave[has])
    cap = (2 if level == engine.LVL02 else 4) * sms
    lanes = lanes_of(net.ops)
    load_asap = np.bincount(asap, weights=lanes, minlength=nwaves)
    load = np.bincount(wave, weights=lanes, minlength=nwaves)
    assert load.sum() == load_asap.sum()
    assert np.all(load <= np.maximum(cap, load_asap))
    return wave, load, cap


@pytest.mark.parametrize("level", [engine.LVL1, engine.LVL02], ids=["lvl1", "lvl02"])
def test_plan_balances_an_uneven_workload(level):
    net = CI.uneven_workload(21, dags=24, adders=6, dag_gates=(50, 600), adder_width=(8, 32))
    asap_load = np.bincount(CI.levels(net), weights=lanes_of(net.ops))
    for sms in (8, 148):
        _, load, cap = check_plan(net, level, sms)
        # narrow waves (below one round) never become more numerous; with a
        # small round (8 SMs) this workload has gates with slack for all of them
        assert (load < cap).sum() <= (asap_load < cap).sum()
        if sms == 8:
            assert (asap_load < cap).sum() > 0 and (load < cap).sum() == 0


def test_plan_moves_slack_gates_into_the_narrow_tail():
    # a 6-gate chain beside 1400 independent gates (the GPU test's circuit)
    width, depth = 1400, 6
    ins = np.arange(width + 1, dtype=np.int32)
    chain_out = width + 1 + np.arange(depth, dtype=np.int32)
    side_out = width + 1 + depth + np.arange(width, dtype=np.int32)
    in0 = np.concatenate([[0], chain_out[:-1], ins[:width]]).astype(np.int32)
    in1 = np.concatenate([np.ones(depth, np.int32), ins[1:width + 1]]).astype(np.int32)
    out = np.concatenate([chain_out, side_out]).astype(np.int32)
    net = CI.Netlist(int(out.max()) + 1, ins, np.full(out.size, P.NAND, np.int32), in0, in1,
                     np.full(out.size, -1, np.int32), out, out)
    wave, load, cap = check_plan(net, engine.LVL1, 148)
    assert cap == 592 and load.max() <= cap
    # latest waves first: the last wave fills up to the round, then the one before
    assert load[-1] == cap and load[0] == cap
    assert np.all(wave[:depth] == np.arange(depth))  # the chain itself does not move


def test_plan_reports_the_same_errors_as_create():
    with pytest.raises(RuntimeError, match="cycle"):
        engine.circuit_plan(engine.LVL1, 4, [P.NAND, P.NAND], [0, 3], [1, 1], [-1, -1], [2, 3], 148)
    with pytest.raises(RuntimeError, match="written by gates"):
        engine.circuit_plan(engine.LVL1, 4, [P.NAND, P.AND], [0, 0], [1, 1], [-1, -1], [2, 2], 148)


@pytest.mark.parametrize("parts", [1, 2, 3, 8])
def test_split_plan_groups_whole_components(parts):
    """cufhe_circuit_split_plan packs connected components into groups: every
    component lies in one group (so no wire written in one group is read in
    another), every group is used, and the groups' blind-rotation weights are
    within one component's weight of each other."""
    net = CI.uneven_workload(5, dags=20, adders=6, dag_gates=(50, 300), adder_width=(8, 24))
    group, n = engine.circuit_split_plan(engine.LVL1, net.num_wires, net.ops, net.in0, net.in1,
                                         net.in2, net.out, parts)
    assert n == parts and group.min() == 0 and group.max() == n - 1
    writer = np.full(net.num_wires, -1)
    writer[net.out] = group
    for arr in (net.in0, net.in1, net.in2):
        used = arr >= 0
        w = writer[arr[used]]
        assert np.all((w < 0) | (w == group[used]))
    lanes = np.where((net.ops == P.MUX) | (net.ops == P.NMUX), 2,
                     np.where((net.ops == P.NOT) | (net.ops == P.COPY), 0, 1))
    weight = 16 * lanes + 1
    load = np.bincount(group, weights=weight, minlength=n)
    # connected components (union-find over producer -> consumer wires)
    parent = np.arange(net.gates)

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x
    prod = np.full(net.num_wires, -1)
    prod[net.out] = np.arange(net.gates)
    for g in range(net.gates):
        for arr in (net.in0, net.in1, net.in2):
            if arr[g] >= 0 and prod[arr[g]] >= 0:
                a, b = find(g), find(int(prod[arr[g]]))
                if a != b:
                    parent[a] = b
    roots = np.array([find(g) for g in range(net.gates)])
    _, comp = np.unique(roots, return_inverse=True)
    comp_weight = np.bincount(comp, weights=weight)
    assert all(np.unique(group[comp == k]).size == 1 for k in range(comp_weight.size))
    assert load.max() - load.min() <= comp_weight.max()


def test_split_plan_rejects_bad_part_counts():
    net = CI.ripple_carry_adder(4)
    for bad in (0, 65):
        with pytest.raises(engine.CufheError):
            engine.circuit_split_plan(engine.LVL1, net.num_wires, net.ops, net.in0, net.in1,
                                      net.in2, net.out, bad)
    # one component: one group whatever was asked
    group, n = engine.circuit_split_plan(engine.LVL1, net.num_wires, net.ops, net.in0, net.in1,
                                         net.in2, net.out, 4)
    assert n == 1 and not group.any()
