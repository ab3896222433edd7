"""GPU parity of the exact INT8 tensor-core path (tcgen05), through the C-ABI.

The external product runs as INT8 Toeplitz GEMMs on byte limbs with INT32
accumulation, so the whole blind rotation -- and with the integer key switch,
the whole gate -- must be bit-identical to the exact schoolbook oracle.  Both
bootstrapping-key forms are covered:

* plain key (TRGSW[636]): one GEMM per CMUX step, acc += Dec(X^a acc - acc) BK_i;
* KeyBundle key (TRGSW[318][3]): one step per pair, three GEMMs against
  bk0, bk1, bk2 whose products enter as (X^e - 1) P with e = a0 + a1, a0, a1,
  plus the gadget recomposition of the digits (the H term).  The oracle forms
  the combined key H + sum_j bk_j (X^e_j - 1) first and multiplies once
  (include/gatebootstrapping_gpu.cuh:895-1033); the GPU splits the product by
  distributivity, which is exact in Z_2^32[X]/(X^N + 1), so the two agree bit
  for bit.
"""
import numpy as np
import pytest

from cufhepp_b200 import client, engine, params as P
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[False, True], ids=["plain", "kb"])
def ctx(keys, request):
    sk, ek_kb, ek_plain = keys
    ek = ek_kb if request.param else ek_plain
    engine.initialize(ek)
    engine.set_precision(P.INT8_EXACT)
    yield sk, ek
    engine.set_precision(P.FP64_FFNT)
    engine.cleanup()


def rotate(x, steps, count):
    d_in = engine.to_device(x)
    d_acc = engine.DeviceBuffer(count * P.TRLWE1_WORDS * 4)
    engine.blind_rotate(d_in, count, P.MU32, steps, acc_out=d_acc)
    return engine.from_device(d_acc, (count, P.TRLWE1_WORDS))


def lvl0(sk, count, seed):
    rng = np.random.default_rng(seed)
    bits = rng.integers(0, 2, count).astype(np.uint8)
    return bits, client.encrypt_bits(sk, bits, 0, seed=seed)


@pytest.mark.parametrize("steps", [1, 2, 7])
def test_int8_steps_bit_exact(ctx, steps):
    """1, 2 and 7 CMUX steps (plain) or KeyBundle pairs (kb)."""
    sk, ek = ctx
    _, x = lvl0(sk, 8, 100 + steps)
    got = rotate(x, steps, 8)
    ref = O.blind_rotate(x, P.MU32, ek.bk, ek.keybundle, O.EXACT, steps=steps)
    assert np.array_equal(got, ref)


def test_int8_two_lane_groups_bit_exact(ctx):
    sk, ek = ctx
    # 300 lanes span two 256-lane MMA groups (the second one partial)
    _, x = lvl0(sk, 300, 7)
    got = rotate(x, 2, 300)
    ref = O.blind_rotate(x, P.MU32, ek.bk, ek.keybundle, O.EXACT, steps=2)
    assert np.array_equal(got, ref)


def test_int8_many_tiles_per_cta_bit_exact(ctx):
    """2600 lanes = 11 digit groups (the last one partial): each CTA of the
    persistent step GEMM walks several tiles, so the accumulator hand-off, the
    drain buffer and the chunk ring carry over between tiles.  Lanes are
    independent, so a spread of 24 lanes is checked against the oracle."""
    sk, ek = ctx
    count = 2600
    _, x = lvl0(sk, count, 77)
    got = rotate(x, 2, count)
    pick = np.unique(np.concatenate([np.arange(0, count, 131), [255, 256, 2559, 2560, count - 1]]))
    ref = O.blind_rotate(x[pick], P.MU32, ek.bk, ek.keybundle, O.EXACT, steps=2)
    assert np.array_equal(got[pick], ref)


def test_int8_peak_probe():
    """The tcgen05 INT8 throughput probe (the exact path's roofline) runs and
    reports a B200-like figure (nominal dense INT8: 4.5 POP/s)."""
    tops = engine.measure_int8_peak()
    assert 1000.0 < tops < 9000.0


def test_int8_full_rotation_bit_exact(ctx):
    sk, ek = ctx
    bits, x = lvl0(sk, 4, 8)
    got = rotate(x, -1, 4)
    ref = O.blind_rotate(x, P.MU32, ek.bk, ek.keybundle, O.EXACT)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("level", [1, 0])
def test_int8_gates_bit_exact(ctx, level):
    sk, ek = ctx
    gates = np.arange(14, dtype=np.int32).repeat(2)  # every gate id, twice
    rng = np.random.default_rng(50 + level)
    a, b, c = (rng.integers(0, 2, gates.size).astype(np.uint8) for _ in range(3))
    cts = [client.encrypt_bits(sk, x, level, seed=60 + i) for i, x in enumerate((a, b, c))]
    out = engine.gate_batch_host(gates, level, *cts)
    engine.synchronize()
    ref = O.gate_batch(gates, level, *cts, ek.bk, ek.ksk, ek.keybundle, O.EXACT)
    assert np.array_equal(out, ref)
    exp = np.array([P.TRUTH[g](int(x), int(y), int(z)) for g, x, y, z in zip(gates, a, b, c)])
    assert np.array_equal(client.decrypt_bits(sk, out, level), exp)


def test_int8_reproduces_golden_digests(ctx):
    """The INT8 engine path matches the committed exact-oracle digests bit for
    bit, for the key form of this parametrisation (tests/golden/gates_exact.json
    holds both)."""
    import json
    import sys
    from pathlib import Path
    golden = Path(__file__).resolve().parent / "golden"
    sys.path.insert(0, str(golden))
    import make_gate_golden as M
    want = json.loads((golden / "gates_exact.json").read_text())
    kb = ctx[1].keybundle
    tag = "kb" if kb else "plain"
    sk = client.SecretKey.generate(M.SEED)
    ek = client.EvalKey.generate(sk, keybundle=kb)
    assert M.digest(ek.bk) == want["keys"][tag]["bk"]
    engine.initialize(ek)  # golden keys (the module fixture's keys are reinstated below)
    try:
        for level in (1, 0):
            _, cts = M.inputs(sk, level)
            out = engine.gate_batch_host(np.array(M.GATES, np.int32), level, *cts)
            engine.synchronize()
            assert M.digest(out) == want["cases"][f"{tag}_lvl{level}"]["outputs"]
        x = client.encrypt_bits(sk, np.array([0, 1, 1, 0], np.uint8), 0, seed=M.SEED + 99)
        assert M.digest(rotate(x, 3, 4)) == want["cases"][f"{tag}_br3"]["outputs"]
        c1 = client.encrypt_bits(sk, np.arange(16, dtype=np.uint8) & 1, 1, seed=M.SEED + 7)
        d_in = engine.to_device(c1)
        d_out = engine.DeviceBuffer(16 * P.TLWE0_WORDS * 4)
        engine.identity_keyswitch(d_in, 16, d_out)
        assert M.digest(engine.from_device(d_out, (16, P.TLWE0_WORDS))) == \
            want["cases"]["iks16"]["outputs"]
    finally:
        engine.initialize(ctx[1])


def test_int8_fresh_streams_run_concurrently(ctx):
    """Gate batches on newly created engine streams, launched back to back so
    that their kernels overlap: each stream's first launch allocates and
    zeroes its INT8 and key-switch workspaces, in stream order, while the
    other stream's kernels run.  Every output equals the same batch run alone
    on the default stream (the exact form does not depend on scheduling)."""
    sk, ek = ctx
    count = 600
    rng = np.random.default_rng(91)
    gates = rng.choice(np.array([P.NAND, P.AND, P.XOR, P.MUX], np.int32), count)
    cts = [client.encrypt_bits(sk, rng.integers(0, 2, count).astype(np.uint8), 1, seed=92 + i)
           for i in range(3)]
    alone = engine.gate_batch_host(gates, engine.LVL1, *cts)
    engine.synchronize()
    d_in = [engine.to_device(c) for c in cts]
    for _ in range(2):
        streams = [engine.Stream(0) for _ in range(2)]
        outs = [engine.DeviceBuffer(count * P.TLWE1_WORDS * 4) for _ in streams]
        for s, o in zip(streams, outs):
            engine.gate_batch(gates, count, engine.LVL1, o, *d_in, stream=s)
        for s in streams:
            s.synchronize()
        for o in outs:
            assert np.array_equal(engine.from_device(o, (count, P.TLWE1_WORDS)), alone)
        for s in streams:
            s.destroy()
