"""GPU parity of the lvl02 path (lvl0 -> lvl2 blind rotation, lvl2 -> lvl0 key
switching: the *_lvl02 gates, src/cufhe_gates_gpu.cu:826-979), through the C-ABI.

* key switching lvl2 -> lvl0: bit-exact against the oracle (integer);
* one blind-rotation step (KeyBundle pair or CMUX): every Torus64 coefficient
  within STEP_TOL of the exact schoolbook step and of the oracle's FP64 step;
* full rotations: the FP64 error of a step (~2^27) exceeds the weight of the
  lowest lvl2 gadget digit (2^24), so later steps pick different digits in
  any two FP64 implementations (the oracle's FP64 form parts from its own
  exact form the same way); parity is therefore on the phase, within
  PHASE_TOL of the oracle's, which is what decryption reads;
* small batches (the cluster form) equal the one-CTA-per-lane form bit for bit;
* gates: every gate id decrypts to the truth table (test/plain.h:1-70), the
  reference's test_gate_gpu_lvl02.cc check, and 65,536 random gates decrypt
  without a failure.
"""
import os

import numpy as np
import pytest

from cufhepp_b200 import client, engine, params as P
from oracle import oracle as O

pytestmark = pytest.mark.gpu

STEP_TOL = 2.0 ** 32    # Torus64 units, one step
PHASE_TOL = 2.0 ** 48   # Torus64 units (2^-16 of the torus), full rotation
MU2 = 1 << 61


def dist64(a, b):
    d = (np.asarray(a, np.uint64) - np.asarray(b, np.uint64)).view(np.int64)
    return np.abs(d.astype(np.float64))


@pytest.fixture(scope="module")
def keys02():
    sk = client.SecretKey.generate(0xC0FFEE)
    return sk, {True: client.EvalKey02.generate(sk, keybundle=True),
                False: client.EvalKey02.generate(sk, keybundle=False)}


@pytest.fixture(scope="module", params=[True, False], ids=["kb", "nokb"])
def ctx(request, keys02):
    sk, eks = keys02
    ek = eks[request.param]
    engine.initialize_lvl02(ek)
    yield sk, ek, request.param
    engine.cleanup_lvl02()


@pytest.fixture(scope="module")
def fft2():
    return O.FFT2()


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


@pytest.mark.parametrize("lanes", [1, 5, 40, 100])
def test_cluster_form_for_small_batches_is_bit_identical(ctx, lanes):
    """Batches of up to one lane per SM rotate one lane per cluster of two CTAs
    (key multiply-accumulate split over two SMs, products gathered through
    distributed shared memory); CUFHE_BR_CLUSTER=0 keeps one CTA per lane.
    Both give the same accumulators and extracted TLWEs bit for bit."""
    sk, _, _ = ctx
    _, x = lvl0(sk, lanes, 70 + lanes)
    got = {}
    for cluster in (False, True):
        if cluster:
            os.environ.pop("CUFHE_BR_CLUSTER", None)
        else:
            os.environ["CUFHE_BR_CLUSTER"] = "0"
        try:
            got[cluster] = rotate(x, lanes, -1)
        finally:
            os.environ.pop("CUFHE_BR_CLUSTER", None)
    assert np.array_equal(got[True][0], got[False][0])
    assert np.array_equal(got[True][1], got[False][1])


def test_keyswitch20_bit_exact(ctx):
    sk, ek, _ = ctx
    rng = np.random.default_rng(11)
    # random TLWE<lvl2> words (the key switch is integer: any input is valid)
    t2 = rng.integers(0, 2**64, (300, P.TLWE2_WORDS), dtype=np.uint64)
    d_in = engine.to_device(t2)
    d_out = engine.DeviceBuffer(300 * P.TLWE0_WORDS * 4)
    engine.identity_keyswitch_lvl20(d_in, 300, d_out)
    got = engine.from_device(d_out, (300, P.TLWE0_WORDS))
    assert np.array_equal(got, O.iks20_batch(t2, ek.ksk))


def test_keyswitch20_decrypts(ctx):
    sk, ek, kb = ctx
    bits, x = lvl0(sk, 6, 12)
    _, t2 = rotate(x, 6, -1)
    d_in = engine.to_device(t2)
    d_out = engine.DeviceBuffer(6 * P.TLWE0_WORDS * 4)
    engine.identity_keyswitch_lvl20(d_in, 6, d_out)
    got = engine.from_device(d_out, (6, P.TLWE0_WORDS))
    assert np.array_equal(got, O.iks20_batch(t2, ek.ksk))
    # a blind rotation of the plain bit with mu2 = +1/8 decrypts to the bit
    assert np.array_equal(client.decrypt_bits(sk, got, 0), bits)


def test_one_step_matches_exact_and_fp64_oracle(ctx, fft2):
    sk, ek, kb = ctx
    _, x = lvl0(sk, 8, 21)
    acc, _ = rotate(x, 8, 1)
    ex = O.blind_rotate2(x, MU2, ek.bk, kb, O.EXACT, steps=1)
    fp = O.blind_rotate2(x, MU2, O.bk2_to_fft(fft2, ek.bk), kb, O.FP64, fft2, steps=1)
    assert dist64(acc, ex).max() < STEP_TOL
    assert dist64(acc, fp).max() < STEP_TOL


def test_zero_steps_is_test_vector(ctx):
    sk, ek, kb = ctx
    _, x = lvl0(sk, 5, 22)
    acc, t2 = rotate(x, 5, 0)
    ref = O.blind_rotate2(x, MU2, ek.bk, kb, O.EXACT, steps=0)
    assert np.array_equal(acc, ref)
    assert np.array_equal(t2, np.stack([O.sample_extract2(a) for a in ref]))


def test_full_rotation_phase_matches_oracle(ctx, fft2):
    sk, ek, kb = ctx
    bits, x = lvl0(sk, 4, 23)
    acc, t2 = rotate(x, 4, -1)
    fp = O.blind_rotate2(x, MU2, O.bk2_to_fft(fft2, ek.bk), kb, O.FP64, fft2)
    for i in range(4):
        pg = client.trlwe64_phase(sk, acc[i])
        po = client.trlwe64_phase(sk, fp[i])
        assert dist64(pg, po).max() < PHASE_TOL
        assert np.array_equal(O.sample_extract2(acc[i]), t2[i])
        # coefficient 0 of the phase is +-mu2: + for bit 1 (the plain test
        # vector rotated by the encrypted +-mu0)
        ph0 = int(pg[0].view(np.int64))
        assert (ph0 > 0) == bool(bits[i])
        assert abs(abs(ph0) - MU2) < 2 ** 56


@pytest.mark.parametrize("gate", range(14), ids=P.GATE_NAMES)
def test_gate_truth_table(ctx, gate):
    sk, ek, _ = ctx
    n = 32
    rng = np.random.default_rng(100 + gate)
    a, b, c = (rng.integers(0, 2, n).astype(np.uint8) for _ in range(3))
    cts = [client.encrypt_bits(sk, v, 0, seed=200 + 3 * gate + i) for i, v in enumerate((a, b, c))]
    out = engine.gate_batch_host(None, engine.LVL02, *cts, uniform=gate)
    engine.synchronize()
    exp = np.array([P.TRUTH[gate](int(x), int(y), int(z)) for x, y, z in zip(a, b, c)])
    assert np.array_equal(client.decrypt_bits(sk, out, 0), exp)


def test_mixed_batch_matches_oracle_phase(ctx, fft2):
    sk, ek, kb = ctx
    gates = np.array([P.NAND, P.AND, P.OR, P.XOR, P.XNOR, P.MUX, P.NMUX, P.NOT, P.COPY, P.NOR],
                     np.int32)
    rng = np.random.default_rng(31)
    a, b, c = (rng.integers(0, 2, gates.size).astype(np.uint8) for _ in range(3))
    cts = [client.encrypt_bits(sk, v, 0, seed=310 + i) for i, v in enumerate((a, b, c))]
    out = engine.gate_batch_host(gates, engine.LVL02, *cts)
    engine.synchronize()
    ref = O.gate2_batch(gates, *cts, O.bk2_to_fft(fft2, ek.bk), ek.ksk, kb, O.FP64, fft2)
    exp = np.array([P.TRUTH[g](int(x), int(y), int(z)) for g, x, y, z in zip(gates, a, b, c)])
    assert np.array_equal(client.decrypt_bits(sk, out, 0), exp)
    assert np.array_equal(client.decrypt_bits(sk, ref, 0), exp)
    # Not/Copy are exact at lvl0
    nc = (gates == P.NOT) | (gates == P.COPY)
    assert np.array_equal(out[nc], ref[nc])


def test_random_gates_no_failure(ctx):
    sk, ek, _ = ctx
    n = 1 << 16
    rng = np.random.default_rng(77)
    pool = np.array([P.NAND, P.AND, P.OR, P.XOR, P.XNOR, P.NOR, P.MUX, P.NMUX, P.ORYN, P.ANDNY],
                    np.int32)
    gates = rng.choice(pool, n).astype(np.int32)
    a, b, c = (rng.integers(0, 2, n).astype(np.uint8) for _ in range(3))
    cts = [client.encrypt_bits(sk, v, 0, seed=700 + i) for i, v in enumerate((a, b, c))]
    out = engine.gate_batch_host(gates, engine.LVL02, *cts)
    engine.synchronize()
    truth = np.empty(n, np.uint8)
    for g in pool:
        m = gates == g
        truth[m] = np.asarray(P.TRUTH[int(g)](a[m].astype(int), b[m].astype(int), c[m].astype(int)))
    assert int((client.decrypt_bits(sk, out, 0) != truth).sum()) == 0
