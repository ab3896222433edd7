"""GPU parity of the exact INT8 tensor-core path at lvl02 (lvl0 -> lvl2 blind
rotation: N = 2048, l = 4, Bgbit = 10, Torus64; eight key limbs, two digit
limbs), through the C-ABI.

* CMUX steps of the rotation are bit-identical to the exact Torus64
  schoolbook oracle, for a batch inside one 128-lane digit group and for a
  batch of three groups where every CTA of the step GEMM walks several tiles
  (both limb groups of a coefficient block, the key-window ring, the drain
  buffer carried between tiles);
* SampleExtract of the exact accumulator is the oracle's;
* lvl02 gates under the INT8 form decrypt to their truth tables (the lvl20
  key switch is the integer one of the FP64 form);
* the FP64 form's rounding error against the exact form is measured on the
  same inputs after a full rotation (the report of configs' lvl02 case) and
  stays within the FP64 path's phase tolerance.

Every case runs with the plain key (one GEMM per CMUX step) and with the
KeyBundle key (one step per pair: three key GEMMs whose products enter as
(X^e - 1) P, plus the gadget recomposition of the digits; `steps` counts
pairs), against the oracle's Torus64 CMUX and KeyBundle steps.
"""
import numpy as np
import pytest

from cufhepp_b200 import client, engine, params as P
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MU2 = 1 << 61
PHASE_TOL = 2.0 ** 48   # Torus64 units (2^-16 of the torus), FP64 form, full rotation


def signed64(x):
    return np.asarray(x, np.uint64).view(np.int64).astype(np.float64)


@pytest.fixture(scope="module", params=[False, True], ids=["plain", "kb"])
def ctx(request):
    sk = client.SecretKey.generate(0x1802)
    ek = client.EvalKey02.generate(sk, keybundle=request.param)
    engine.initialize_lvl02(ek)
    engine.set_precision(P.INT8_EXACT)
    yield sk, ek
    engine.set_precision(P.FP64_FFNT)
    engine.cleanup_lvl02()


def lvl0(sk, count, seed):
    rng = np.random.default_rng(seed)
    bits = rng.integers(0, 2, count).astype(np.uint8)
    return bits, client.encrypt_bits(sk, bits, 0, seed=seed)


def rotate(x, count, steps):
    d_in = engine.to_device(x)
    d_acc = engine.DeviceBuffer(count * P.TRLWE2_WORDS * 8)
    d_t2 = engine.DeviceBuffer(count * P.TLWE2_WORDS * 8)
    engine.blind_rotate_lvl02(d_in, count, MU2, steps, acc_out=d_acc, tlwe_out=d_t2)
    acc = engine.from_device(d_acc, (count, P.TRLWE2_WORDS), np.uint64)
    t2 = engine.from_device(d_t2, (count, P.TLWE2_WORDS), np.uint64)
    return acc, t2


@pytest.mark.parametrize("steps", [1, 3])
def test_int8_lvl02_steps_bit_exact(ctx, steps):
    sk, ek = ctx
    _, x = lvl0(sk, 6, 200 + steps)
    acc, t2 = rotate(x, 6, steps)
    ref = O.blind_rotate2(x, MU2, ek.bk, ek.keybundle, O.EXACT, steps=steps)
    assert np.array_equal(acc, ref)
    for i in range(6):
        assert np.array_equal(t2[i], O.sample_extract2(ref[i]))


def test_int8_lvl02_many_tiles_per_cta_bit_exact(ctx):
    """300 lanes = three 128-lane digit groups (the last one partial): each
    CTA walks several tiles.  Lanes are independent, so a spread of lanes is
    checked against the oracle."""
    sk, ek = ctx
    count = 300
    _, x = lvl0(sk, count, 77)
    acc, _ = rotate(x, count, 2)
    pick = np.array([0, 1, 63, 127, 128, 200, 255, 256, 280, 299])
    ref = O.blind_rotate2(x[pick], MU2, ek.bk, ek.keybundle, O.EXACT, steps=2)
    assert np.array_equal(acc[pick], ref)


def test_int8_lvl02_gates_decrypt(ctx):
    sk, _ = ctx
    gates = np.tile(np.arange(14, dtype=np.int32), 9)  # every gate id
    rng = np.random.default_rng(5)
    a, b, c = (rng.integers(0, 2, gates.size).astype(np.uint8) for _ in range(3))
    cts = [client.encrypt_bits(sk, v, 0, seed=300 + i) for i, v in enumerate((a, b, c))]
    out = engine.gate_batch_host(gates, engine.LVL02, *cts)
    engine.synchronize()
    exp = np.array([P.TRUTH[g](int(x), int(y), int(z)) for g, x, y, z in zip(gates, a, b, c)])
    assert np.array_equal(client.decrypt_bits(sk, out, 0), exp)


def test_fp64_rounding_error_against_exact(ctx):
    """Full 636-step rotations of the same inputs in both forms.  The FP64
    form's per-step rounding (about 2^27) exceeds the weight of the lowest
    lvl2 digit (2^24), so later decompositions differ and the two masks
    diverge; the error that matters, on the phase, stays within the FP64
    path's tolerance."""
    sk, _ = ctx
    bits, x = lvl0(sk, 16, 9)
    exact, _ = rotate(x, 16, -1)
    engine.set_precision(P.FP64_FFNT)
    try:
        fp64, _ = rotate(x, 16, -1)
    finally:
        engine.set_precision(P.INT8_EXACT)
    err = np.stack([np.abs(signed64(client.trlwe64_phase(sk, fp64[i]) -
                                    client.trlwe64_phase(sk, exact[i]))) for i in range(16)])
    print(f"FP64 vs exact lvl2 rotation, phase error: max 2^{np.log2(max(err.max(), 1)):.1f}, "
          f"median 2^{np.log2(max(np.median(err), 1)):.1f} Torus64 units")
    assert err.max() < PHASE_TOL
    # coefficient 0 of the exact phase is +-mu2: + for bit 1
    for i in range(16):
        ph0 = int(client.trlwe64_phase(sk, exact[i])[0].view(np.int64))
        assert (ph0 > 0) == bool(bits[i])
        assert abs(abs(ph0) - MU2) < 2 ** 56


def test_int8_lvl02_circuit_graph_matches_direct(ctx):
    """A lvl02 circuit in the INT8 form: the CUDA-graph run equals the direct
    run bit for bit and decrypts to the plaintext evaluation."""
    from cufhepp_b200 import circuits as CI
    sk, _ = ctx
    net = CI.uneven_workload(21, dags=2, adders=1, dag_gates=(40, 80), adder_width=(8, 8))
    rng = np.random.default_rng(22)
    bits = rng.integers(0, 2, net.inputs.size).astype(np.uint8)
    host = np.zeros((net.num_wires, P.TLWE0_WORDS), np.uint32)
    host[net.inputs] = client.encrypt_bits(sk, bits, 0, seed=23)
    d = engine.to_device(host)
    c = engine.Circuit(engine.LVL02, net.num_wires, net.ops, net.in0, net.in1, net.in2, net.out)
    try:
        c.run(d, graph=False)
        direct = engine.from_device(d, host.shape)
        c.run(d, graph=True)
        graph = engine.from_device(d, host.shape)
    finally:
        c.destroy()
    engine.synchronize()
    assert np.array_equal(direct, graph)
    plain = CI.evaluate(net, bits)
    got = client.decrypt_bits(sk, direct[net.out], 0)
    assert int(np.count_nonzero(got != plain[net.out])) == 0
