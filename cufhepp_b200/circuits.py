"""Seeded gate circuits for the circuit executor (cufhe_circuit_*): levelised
random DAGs and ripple-carry adders -- the uneven-depth workload -- their
merge into one wire table, and their plaintext evaluation.

A Netlist lists gates in creation order, which is a topological order; wire
ids are rows of the circuit's wire table.  Wires no gate writes are inputs.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import params as P

BINARY = np.array([P.NAND, P.OR, P.ORYN, P.ORNY, P.AND, P.ANDYN, P.ANDNY, P.NOR, P.XOR, P.XNOR],
                  np.int32)


@dataclass
class Netlist:
    num_wires: int
    inputs: np.ndarray                   # wire ids the caller encrypts
    ops: np.ndarray                      # int32 gate ids
    in0: np.ndarray
    in1: np.ndarray
    in2: np.ndarray                      # -1 unless Mux/NMux
    out: np.ndarray
    outputs: np.ndarray                  # wire ids of the circuit's results
    parts: list = field(default_factory=list)  # (kind, size) of merged circuits

    @property
    def gates(self) -> int:
        return int(self.ops.size)

    def bootstraps(self) -> int:
        return int(np.count_nonzero((self.ops != P.NOT) & (self.ops != P.COPY)) +
                   np.count_nonzero((self.ops == P.MUX) | (self.ops == P.NMUX)))


def operands(op: int) -> int:
    """Number of input wires gate `op` reads (Not/Copy 1, Mux/NMux 3, else 2)."""
    return 1 if op in (P.NOT, P.COPY) else (3 if op in (P.MUX, P.NMUX) else 2)


def _log_uniform_int(rng, lo: int, hi: int) -> int:
    return int(np.clip(np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi + 1)))), lo, hi))


def random_dag(rng, n_gates: int, max_width: int = 64) -> Netlist:
    """Levelised DAG of n_gates fan-in-2 gates, gate types uniform over the ten
    binary gates, level widths log-uniform in [1, max_width].  Every gate of
    level k reads one wire of level k-1 and one wire of any earlier level, so
    its depth is exactly k."""
    w0 = max(2, _log_uniform_int(rng, 1, max_width))
    nxt = w0
    lo, hi = 0, w0                      # wires of the previous level
    ops, a, b, outs = [], [], [], []
    made = 0
    while made < n_gates:
        w = min(_log_uniform_int(rng, 1, max_width), n_gates - made)
        ops.append(rng.choice(BINARY, w).astype(np.int32))
        a.append(rng.integers(lo, hi, w).astype(np.int32))
        b.append(rng.integers(0, hi, w).astype(np.int32))
        outs.append(np.arange(nxt, nxt + w, dtype=np.int32))
        lo, hi = nxt, nxt + w
        nxt += w
        made += w
    ops, a, b, outs = (np.concatenate(x) for x in (ops, a, b, outs))
    return Netlist(nxt, np.arange(w0, dtype=np.int32), ops, a, b, np.full(ops.size, -1, np.int32),
                   outs, np.arange(lo, hi, dtype=np.int32), [("dag", n_gates)])


def ripple_carry_adder(width: int) -> Netlist:
    """a + b + cin over `width` bits: t = a ^ b, s = t ^ c, c' = t ? c : a
    (three gates per bit, the carry through a Mux).  Wires: a[0..w), b[0..w),
    cin = 2w; outputs: the sum bits then the carry out."""
    a0, b0, cin = 0, width, 2 * width
    nxt = 2 * width + 1
    ops, i0, i1, i2, out = [], [], [], [], []
    c = cin
    sums = []
    for i in range(width):
        t, s, cn = nxt, nxt + 1, nxt + 2
        nxt += 3
        ops += [P.XOR, P.XOR, P.MUX]
        i0 += [a0 + i, t, t]
        i1 += [b0 + i, c, c]
        i2 += [-1, -1, a0 + i]
        out += [t, s, cn]
        sums.append(s)
        c = cn
    arr = lambda x: np.asarray(x, np.int32)  # noqa: E731
    return Netlist(nxt, np.arange(2 * width + 1, dtype=np.int32), arr(ops), arr(i0), arr(i1),
                   arr(i2), arr(out), arr(sums + [c]), [("adder", width)])


def merge(nets: list[Netlist]) -> Netlist:
    """Disjoint union of netlists in one wire table."""
    off = 0
    parts = {k: [] for k in ("inputs", "ops", "in0", "in1", "in2", "out", "outputs")}
    kinds = []
    for n in nets:
        sh = lambda x: np.where(x >= 0, x + off, -1).astype(np.int32)  # noqa: E731
        parts["inputs"].append(n.inputs + off)
        parts["ops"].append(n.ops)
        parts["in0"].append(sh(n.in0))
        parts["in1"].append(sh(n.in1))
        parts["in2"].append(sh(n.in2))
        parts["out"].append(n.out + off)
        parts["outputs"].append(n.outputs + off)
        kinds += n.parts
        off += n.num_wires
    cat = {k: np.concatenate(v).astype(np.int32) for k, v in parts.items()}
    return Netlist(off, cat["inputs"], cat["ops"], cat["in0"], cat["in1"], cat["in2"], cat["out"],
                   cat["outputs"], kinds)


def evaluate(net: Netlist, inputs: np.ndarray) -> np.ndarray:
    """Plaintext wire values (uint8 [num_wires]) given the input bits (in the
    order of net.inputs); gates are applied in list order (topological)."""
    v = np.zeros(net.num_wires, np.uint8)
    v[net.inputs] = inputs
    ops, i0, i1, i2, out = net.ops, net.in0, net.in1, net.in2, net.out
    for g in range(ops.size):
        op = int(ops[g])
        a = int(v[i0[g]])
        b = int(v[i1[g]]) if i1[g] >= 0 else 0
        c = int(v[i2[g]]) if i2[g] >= 0 else 0
        v[out[g]] = P.TRUTH[op](a, b, c)
    return v


def uneven_workload(seed: int, dags: int = 256, adders: int = 64, dag_gates=(50, 2000),
                    adder_width=(8, 64), max_width: int = 64) -> Netlist:
    """The uneven-circuit workload: `dags` random levelised DAGs of
    dag_gates[0]..dag_gates[1] gates and `adders` ripple-carry adders of
    random width, merged into one wire table (seeded)."""
    rng = np.random.default_rng(seed)
    nets = [random_dag(rng, int(rng.integers(dag_gates[0], dag_gates[1] + 1)), max_width)
            for _ in range(dags)]
    nets += [ripple_carry_adder(int(rng.integers(adder_width[0], adder_width[1] + 1)))
             for _ in range(adders)]
    return merge(nets)


def levels(net: Netlist) -> np.ndarray:
    """Wave index of every gate (1 + latest wave among its producers), the
    levelisation the engine performs."""
    prod_wave = np.full(net.num_wires, -1, np.int64)
    wave = np.zeros(net.gates, np.int64)
    for g in range(net.gates):
        w = -1
        for x in (net.in0, net.in1, net.in2)[:operands(int(net.ops[g]))]:
            if x[g] >= 0:
                w = max(w, prod_wave[x[g]])
        wave[g] = w + 1
        prod_wave[net.out[g]] = w + 1
    return wave
