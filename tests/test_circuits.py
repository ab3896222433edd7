"""Circuit workload generators and the circuit executor's host-side checks
(no GPU: cufhe_circuit_create validates and levelises before it needs keys)."""
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
