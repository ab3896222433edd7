"""Edge cases of the batched gate path on the GPU, through the C-ABI.

* empty batches are no-ops at every entry point, and an oversized count is
  refused before anything is launched;
* ragged batch sizes: a gate's output does not depend on the batch around it
  or on which kernel shape ran it (cluster form up to 16 lanes, one or two
  lanes per CTA above, 128-gate key-switch tiles, 256-lane INT8 digit groups
  and the K-split tail units).  Prefixes of a 300-gate batch of every size
  around those boundaries must reproduce the full batch's rows bit for bit,
  in both precision forms and both gate orders.
"""
import numpy as np
import pytest

from cufhepp_b200 import client, engine, params as P

pytestmark = pytest.mark.gpu

SIZES = [1, 2, 15, 16, 17, 127, 128, 129, 255, 256, 257]
FULL = 300
GATES = [P.NAND, P.AND, P.OR, P.XOR, P.XNOR, P.MUX, P.NOR, P.ANDNY, P.ORYN, P.NMUX]


@pytest.fixture(scope="module", params=["fp64", "int8", "int8_kb"])
def form(request, keys):
    sk, ek_kb, ek_nokb = keys
    engine.initialize(ek_nokb if request.param == "int8" else ek_kb)
    engine.set_precision(P.FP64_FFNT if request.param == "fp64" else P.INT8_EXACT)
    yield sk, request.param
    engine.set_precision(P.FP64_FFNT)
    engine.cleanup()


def words(level):
    return P.TLWE1_WORDS if level == engine.LVL1 else P.TLWE0_WORDS


def test_empty_batches_are_no_ops(form):
    for level in (engine.LVL1, engine.LVL0):
        w = words(level)
        empty = np.zeros((0, w), np.uint32)
        out = engine.gate_batch_host(np.zeros(0, np.int32), level, empty, empty, empty)
        assert out.shape == (0, w)
        d = engine.DeviceBuffer(16 * w * 4)
        engine.gate_batch(np.zeros(0, np.int32), 0, level, d, d, d, d)
    d0 = engine.DeviceBuffer(16 * P.TLWE0_WORDS * 4)
    d1 = engine.DeviceBuffer(16 * P.TRLWE1_WORDS * 4)
    engine.blind_rotate(d0, 0, P.MU32, -1, acc_out=d1)
    engine.identity_keyswitch(d1, 0, d0)
    engine.synchronize()


def test_oversized_batch_is_refused(form):
    d = engine.DeviceBuffer(16 * P.TLWE1_WORDS * 4)
    with pytest.raises(RuntimeError):  # one gate id for the whole batch: nothing is read
        engine.gate_batch(None, (1 << 24) + 1, engine.LVL1, d, d, d, d, uniform=P.NAND)
    engine.synchronize()


@pytest.mark.parametrize("level", [engine.LVL1, engine.LVL0], ids=["lvl1", "lvl0"])
def test_prefix_batches_reproduce_the_full_batch(form, level):
    sk, _ = form
    rng = np.random.default_rng(100 + level)
    gates = rng.choice(GATES, FULL).astype(np.int32)
    bits = [rng.integers(0, 2, FULL).astype(np.uint8) for _ in range(3)]
    cts = [client.encrypt_bits(sk, b, level, seed=200 + 7 * i + level) for i, b in enumerate(bits)]
    full = engine.gate_batch_host(gates, level, *cts)
    engine.synchronize()
    exp = np.array([P.TRUTH[g](int(x), int(y), int(z)) for g, x, y, z in zip(gates, *bits)])
    assert np.array_equal(client.decrypt_bits(sk, full, level), exp)
    for n in SIZES:
        part = engine.gate_batch_host(gates[:n], level, *(c[:n] for c in cts))
        engine.synchronize()
        assert np.array_equal(part, full[:n]), n


def test_lvl02_prefix_batches_reproduce_the_full_batch():
    """lvl02 gates (Ctxt<lvl0> I/O through lvl2): prefixes across the cluster
    form's limit (one lane per SM) and the key-switch tiles give the same rows
    as a 400-gate batch, and the full batch decrypts to its truth table."""
    sk = client.SecretKey.generate(0xED6E)
    prev = engine.get_precision()
    engine.set_precision(P.FP64_FFNT)  # the cluster form's limits are those of the FP64 form
    engine.initialize_lvl02(client.EvalKey02.generate(sk, keybundle=True))
    try:
        rng = np.random.default_rng(7)
        n_full = 400
        gates = rng.choice(GATES, n_full).astype(np.int32)
        bits = [rng.integers(0, 2, n_full).astype(np.uint8) for _ in range(3)]
        cts = [client.encrypt_bits(sk, b, 0, seed=300 + i) for i, b in enumerate(bits)]
        dev = [engine.to_device(c) for c in cts]
        d_out = engine.DeviceBuffer(n_full * P.TLWE0_WORDS * 4)
        engine.gate_batch(gates, n_full, engine.LVL02, d_out, *dev)
        engine.synchronize()
        full = engine.from_device(d_out, (n_full, P.TLWE0_WORDS))
        exp = np.array([P.TRUTH[g](int(x), int(y), int(z)) for g, x, y, z in zip(gates, *bits)])
        assert np.array_equal(client.decrypt_bits(sk, full, 0), exp)
        for n in (1, 3, 127, 128, 129, 147, 148, 149, 200):
            engine.gate_batch(gates[:n], n, engine.LVL02, d_out, *dev)
            engine.synchronize()
            assert np.array_equal(engine.from_device(d_out, (n, P.TLWE0_WORDS)), full[:n]), n
    finally:
        engine.cleanup_lvl02()
        engine.set_precision(prev)
