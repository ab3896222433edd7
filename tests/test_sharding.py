"""Splitting one batch or one circuit over several GPUs, without a GPU.

* cufhe_batch_shard_plan: contiguous gate ranges with balanced blind-rotation
  lanes;
* cufhe_circuit_shard_plan: the waves of cufhe_circuit_plan, a shard per gate
  with the lanes of every wave balanced; the wires to move between shards
  follow from the plan by the engine's rule (a wire that shard s writes in
  wave w and shard t != s reads is copied s -> t right after wave w), and a
  plaintext run of every shard against its own wire table under that rule
  reproduces the whole circuit;
* world_size-2 gloo process groups: each rank evaluates its shard of a batch
  and of a circuit on ciphertexts with the oracle, exchanging the planned
  wires after every wave; the merged result is bit-identical to one process
  evaluating everything.
"""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from cufhepp_b200 import circuits as CI, engine, params as P

LANES = {P.NOT: 0, P.COPY: 0, P.MUX: 2, P.NMUX: 2}


def lanes_of(ops):
    return np.array([LANES.get(int(o), 1) for o in ops], np.int64)


def copy_rule(net, wave, shard):
    """(writer wave, writer shard, reader shard, wire) of every wire a shard
    reads from another, as the engine derives them."""
    producer = np.full(net.num_wires, -1, np.int64)
    producer[net.out] = np.arange(net.gates)
    ins = (net.in0, net.in1, net.in2)
    moves = set()
    for g in range(net.gates):
        for k in range(CI.operands(int(net.ops[g]))):
            x = int(ins[k][g])
            p = producer[x]
            if p >= 0 and shard[p] != shard[g]:
                moves.add((int(wave[p]), int(shard[p]), int(shard[g]), x))
    return sorted(moves)


def simulate(net, wave, shard, shards, bits):
    """Plaintext run: shard s evaluates its gates of each wave reading only its
    own table; after each wave the planned wires are copied.  Returns the
    merged wire values (every gate output taken from its writer's table)."""
    unknown = 255
    tables = [np.full(net.num_wires, unknown, np.uint8) for _ in range(shards)]
    for t in tables:
        t[net.inputs] = bits
    moves = copy_rule(net, wave, shard)
    ins = (net.in0, net.in1, net.in2)
    for w in range(int(wave.max()) + 1):
        for g in np.flatnonzero(wave == w):
            tab = tables[shard[g]]
            v = [int(tab[ins[k][g]]) for k in range(CI.operands(int(net.ops[g])))]
            assert unknown not in v, f"gate {g} on shard {shard[g]} lacks an operand"
            tab[net.out[g]] = P.TRUTH[int(net.ops[g])](*(v + [0] * (3 - len(v))))
        for (mw, s, t, x) in moves:
            if mw == w:
                tables[t][x] = tables[s][x]
    merged = tables[0].copy()
    merged[net.out] = [tables[shard[g]][net.out[g]] for g in range(net.gates)]
    return merged


def test_batch_shard_plan_balances_lanes():
    rng = np.random.default_rng(5)
    for count in (1, 7, 100, 4096):
        gates = rng.choice([P.NAND, P.MUX, P.XOR, P.NOT, P.AND], count).astype(np.int32)
        lanes = lanes_of(gates)
        for shards in (1, 2, 3, 8):
            b = engine.batch_shard_plan(gates, count, shards)
            assert b[0] == 0 and b[-1] == count and np.all(np.diff(b) >= 0)
            per = [int(lanes[b[k]:b[k + 1]].sum()) for k in range(shards)]
            assert sum(per) == lanes.sum()
            assert max(per) <= -(-lanes.sum() // shards) + 2, (count, shards, per)
    # a batch that does not bootstrap at all splits by count
    b = engine.batch_shard_plan(None, 10, 4, uniform=P.NOT)
    assert list(b) == [0, 2, 5, 7, 10]


@pytest.mark.parametrize("shards", [2, 3, 4])
def test_circuit_shard_plan_is_a_valid_split(shards):
    net = CI.uneven_workload(11, dags=12, adders=6, dag_gates=(50, 300), adder_width=(8, 20))
    args = (1, net.num_wires, net.ops, net.in0, net.in1, net.in2, net.out)
    wave1, nw1 = engine.circuit_plan(*args)
    wave, shard, nwaves, ncopies = engine.circuit_shard_plan(*args, shards=shards)
    # the waves are the single-device plan's; every gate has a shard
    assert nwaves == nw1 and np.array_equal(wave, wave1)
    assert shard.min() >= 0 and shard.max() < shards
    # per wave, no shard holds more than its share of the lanes (+ one Mux)
    lanes = lanes_of(net.ops)
    for w in range(nwaves):
        m = wave == w
        cap = -(-int(lanes[m].sum()) // shards)
        for s in range(shards):
            assert lanes[m & (shard == s)].sum() <= cap + 1, (w, s)
    # the engine's copy rule gives as many copies as the planner counts, and
    # keeps most dependencies inside a shard
    moves = copy_rule(net, wave, shard)
    assert len(moves) == ncopies
    edges = sum(CI.operands(int(o)) for o in net.ops)
    assert ncopies < 0.5 * edges, (ncopies, edges)
    # every shard finds its operands under that rule and the merge is exact
    bits = np.random.default_rng(3).integers(0, 2, net.inputs.size).astype(np.uint8)
    assert np.array_equal(simulate(net, wave, shard, shards, bits), CI.evaluate(net, bits))


def test_one_shard_needs_no_copies():
    net = CI.uneven_workload(4, dags=3, adders=2, dag_gates=(50, 100), adder_width=(8, 10))
    _, shard, _, ncopies = engine.circuit_shard_plan(1, net.num_wires, net.ops, net.in0, net.in1,
                                                     net.in2, net.out, shards=1)
    assert ncopies == 0 and not shard.any()


def test_shard_plan_rejects_bad_counts():
    net = CI.ripple_carry_adder(4)
    for bad in (0, 65):
        with pytest.raises(engine.CufheError):
            engine.circuit_shard_plan(1, net.num_wires, net.ops, net.in0, net.in1, net.in2,
                                      net.out, shards=bad)
        with pytest.raises(engine.CufheError):
            engine.batch_shard_plan(None, 10, bad, uniform=P.NAND)


# ---------------------------------------------------------------- gloo ranks --
SEED = 0x5AD


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _setup():
    from cufhepp_b200 import client
    from oracle import oracle as O
    sk = client.SecretKey.generate(SEED)
    ek = client.EvalKey.generate(sk, keybundle=True)
    fft = O.FFT()
    return sk, ek, fft, O.bk_to_fft(fft, ek.bk)


def _net():
    rng = np.random.default_rng(SEED)
    return CI.merge([CI.random_dag(rng, 40, max_width=8), CI.ripple_carry_adder(5),
                     CI.random_dag(rng, 24, max_width=6)])


def _eval_gates(O, gates_idx, net, table, ek, fft, bkf):
    """Oracle FP64 gates (KeyBundle) of the listed gates on rows of `table`."""
    if len(gates_idx) == 0:
        return np.zeros((0, P.TLWE1_WORDS), np.uint32)
    row = lambda x: table[np.where(x >= 0, x, 0)]  # noqa: E731
    g = np.asarray(gates_idx)
    return O.gate_batch(net.ops[g], 1, row(net.in0[g]), row(net.in1[g]), row(net.in2[g]), bkf,
                        ek.ksk, True, O.FP64, fft)


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), OMP_NUM_THREADS="2")
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from cufhepp_b200 import client
        from oracle import oracle as O
        sk, ek, fft, bkf = _setup()
        # ---- one batch: rank k evaluates gates [bounds[k], bounds[k + 1])
        rng = np.random.default_rng(SEED + 1)
        n = 24
        gates = rng.choice([P.NAND, P.MUX, P.XOR, P.NOT], n).astype(np.int32)
        cts = [client.encrypt_bits(sk, rng.integers(0, 2, n).astype(np.uint8), 1, seed=SEED + i)
               for i in range(3)]
        b = engine.batch_shard_plan(gates, n, world)
        lo, hi = int(b[rank]), int(b[rank + 1])
        part = O.gate_batch(gates[lo:hi], 1, *(c[lo:hi] for c in cts), bkf, ek.ksk, True, O.FP64,
                            fft)
        parts = [None] * world
        dist.all_gather_object(parts, part)
        batch = np.concatenate(parts)
        # ---- one circuit: each wave's gates of this rank, then the planned
        # wires go to the ranks that read them
        net = _net()
        bits = np.random.default_rng(SEED + 2).integers(0, 2, net.inputs.size).astype(np.uint8)
        table = np.zeros((net.num_wires, P.TLWE1_WORDS), np.uint32)
        table[net.inputs] = client.encrypt_bits(sk, bits, 1, seed=SEED + 9)
        wave, shard, nwaves, ncopies = engine.circuit_shard_plan(
            1, net.num_wires, net.ops, net.in0, net.in1, net.in2, net.out, shards=world)
        moves = copy_rule(net, wave, shard)
        sent = 0
        for w in range(nwaves):
            mine = np.flatnonzero((wave == w) & (shard == rank))
            table[net.out[mine]] = _eval_gates(O, mine, net, table, ek, fft, bkf)
            outgoing = [(t, x, table[x].copy()) for (mw, s, t, x) in moves if mw == w and s == rank]
            sent += len(outgoing)
            inbox = [None] * world
            dist.all_gather_object(inbox, outgoing)
            for lst in inbox:
                for (t, x, r) in lst:
                    if t == rank:
                        table[x] = r
        mine = np.flatnonzero(shard == rank)
        outs = [None] * world
        dist.all_gather_object(outs, (net.out[mine], table[net.out[mine]]))
        if rank == 0:
            merged = table.copy()
            for wires, rows in outs:
                merged[wires] = rows
            out["batch"] = batch
            out["circuit"] = merged[net.out]
            out["ncopies"] = ncopies
        out[f"sent{rank}"] = sent
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_match_one_process():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world,
                       start_method="spawn", join=True)
    from cufhepp_b200 import client
    from oracle import oracle as O
    sk, ek, fft, bkf = _setup()
    # one process: the whole batch, and the circuit wave by wave
    rng = np.random.default_rng(SEED + 1)
    n = 24
    gates = rng.choice([P.NAND, P.MUX, P.XOR, P.NOT], n).astype(np.int32)
    cts = [client.encrypt_bits(sk, rng.integers(0, 2, n).astype(np.uint8), 1, seed=SEED + i)
           for i in range(3)]
    whole = O.gate_batch(gates, 1, *cts, bkf, ek.ksk, True, O.FP64, fft)
    assert np.array_equal(out["batch"], whole)
    net = _net()
    bits = np.random.default_rng(SEED + 2).integers(0, 2, net.inputs.size).astype(np.uint8)
    table = np.zeros((net.num_wires, P.TLWE1_WORDS), np.uint32)
    table[net.inputs] = client.encrypt_bits(sk, bits, 1, seed=SEED + 9)
    wave, _ = engine.circuit_plan(1, net.num_wires, net.ops, net.in0, net.in1, net.in2, net.out)
    for w in range(int(wave.max()) + 1):
        g = np.flatnonzero(wave == w)
        table[net.out[g]] = _eval_gates(O, g, net, table, ek, fft, bkf)
    assert np.array_equal(out["circuit"], table[net.out])
    assert out["sent0"] + out["sent1"] == out["ncopies"] > 0
    # and it decrypts to the plaintext evaluation
    assert np.array_equal(client.decrypt_bits(sk, table[net.out], 1), CI.evaluate(net, bits)[net.out])
