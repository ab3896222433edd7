"""One batch or one circuit split over shards, on the GPU, through the C-ABI.

Shard s runs on device s % cufhe_set_gpu_num; with one GPU every shard runs
on it, each with its own engine stream (batch) or its own sub-circuit, wire
table, stream and event (circuit), so the whole sharded path -- per-shard
waves, the wire copies between shard tables after each wave, the event
ordering between shards and the final collection -- runs as it would across
GPUs, with device-local copies in place of peer stores.  Results must be
bit-identical to the unsharded batch and circuit.
"""
import numpy as np
import pytest

from cufhepp_b200 import circuits as CI, client, engine, params as P

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(keys):
    sk, ek_kb, _ = keys
    engine.initialize(ek_kb)
    engine.set_precision(P.FP64_FFNT)
    yield sk
    engine.set_precision(P.FP64_FFNT)
    engine.cleanup()


@pytest.mark.parametrize("form", [P.FP64_FFNT, P.INT8_EXACT], ids=["fp64", "int8"])
@pytest.mark.parametrize("level", [1, 0], ids=["lvl1", "lvl0"])
def test_sharded_batch_matches_one_batch(ctx, form, level):
    sk = ctx
    engine.set_precision(form)
    try:
        rng = np.random.default_rng(40 + level)
        n = 700
        gates = rng.choice([P.NAND, P.MUX, P.XOR, P.NOT, P.AND, P.NMUX], n).astype(np.int32)
        bits = [rng.integers(0, 2, n).astype(np.uint8) for _ in range(3)]
        cts = [client.encrypt_bits(sk, b, level, seed=50 + i) for i, b in enumerate(bits)]
        ref = engine.gate_batch_host(gates, level, *cts)
        engine.synchronize()
        for shards in (2, 3):
            got = engine.gate_batch_sharded_host(gates, level, *cts, shards=shards)
            assert np.array_equal(got, ref), shards
        exp = np.array([P.TRUTH[g](int(x), int(y), int(z)) for g, x, y, z in zip(gates, *bits)])
        assert np.array_equal(client.decrypt_bits(sk, ref, level), exp)
    finally:
        engine.set_precision(P.FP64_FFNT)


@pytest.mark.parametrize("shards", [2, 3])
def test_sharded_circuit_matches_one_device(ctx, shards):
    import torch
    sk = ctx
    net = CI.uneven_workload(77, dags=6, adders=3, dag_gates=(50, 200), adder_width=(8, 16))
    bits = np.random.default_rng(5).integers(0, 2, net.inputs.size).astype(np.uint8)
    host = np.zeros((net.num_wires, P.TLWE1_WORDS), np.uint32)
    host[net.inputs] = client.encrypt_bits(sk, bits, 1, seed=61)
    # one device, one wire table
    single = torch.from_numpy(host.view(np.int32)).cuda()
    c = engine.Circuit(1, net.num_wires, net.ops, net.in0, net.in1, net.in2, net.out)
    c.run(single.data_ptr(), graph=False)
    engine.synchronize()
    ref = single.cpu().numpy().view(np.uint32)
    c.destroy()
    # the same circuit over shards, each with its own table holding the inputs
    sc = engine.ShardedCircuit(1, net.num_wires, net.ops, net.in0, net.in1, net.in2, net.out,
                               shards=shards)
    waves, copies, n = sc.info()
    assert n == shards and copies > 0
    assert all(sc.device(s) == 0 for s in range(shards))
    tables = [torch.from_numpy(host.view(np.int32)).cuda() for _ in range(shards)]
    for rep in range(2):  # a second run reuses the plans, rows and events
        sc.run([t.data_ptr() for t in tables])
        sc.collect([t.data_ptr() for t in tables], 0)
        sc.synchronize()
        got = tables[0].cpu().numpy().view(np.uint32)
        assert np.array_equal(got[net.out], ref[net.out]), rep
    sc.destroy()
    plain = CI.evaluate(net, bits)
    assert np.array_equal(client.decrypt_bits(sk, ref[net.out], 1), plain[net.out])
