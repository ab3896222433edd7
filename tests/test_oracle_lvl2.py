"""Pins the lvl2 (N = 2048, Torus64) oracle on the reference's known-answer
tests, which run the same checks for lvl02param as for lvl1:

* test/test_fft_roundtrip.cu:298-319   -- the three FFNT checks at N = 2048
  (mt19937(42) reals round-trip < 1e-6, (1+X+X^2)^2 < 1e-6, mt19937(123)
  ints in [-5, 5] squared < 0.5); inputs from tests/golden/gen_fft_kat_inputs.cpp.
* test/test_accumulate_diag.cu:349-353 -- zero TRGSW identity and noiseless
  TRGSW(1) rotation for lvl02param; tolerance 2^20 for uint64 (:241-243).
Beyond those: the exact Torus64 external product against a Python-integer
schoolbook, decomposition recomposition, and a full lvl02 gate through the
FP64 and exact forms.
"""
from pathlib import Path

import numpy as np
import pytest

from cufhepp_b200 import client, params as P
from oracle import oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden"
MU2 = 1 << 61
M64 = (1 << 64) - 1


def gadget_trgsw2(m: int) -> np.ndarray:
    t = np.zeros((8, 2, O.N2), np.uint64)
    for row in range(8):
        j, d = row // 4, row % 4
        t[row, j, 0] = np.uint64((m << (64 - (d + 1) * 10)) & M64)
    return t.reshape(-1)


def signed64(x):
    return np.asarray(x, np.uint64).view(np.int64)


@pytest.fixture(scope="module")
def fft2():
    return O.FFT2()


def mu_vec():
    acc = np.zeros(O.TRLWE2, np.uint64)
    acc[O.N2:] = MU2
    return acc


def test_zero_trgsw_identity(fft2):
    acc = mu_vec()
    assert np.array_equal(O.cmux2_step_exact(acc, np.zeros(O.TRGSW2, np.uint64), 0), acc)
    bkf = O.bk2_to_fft(fft2, np.zeros(O.TRGSW2, np.uint64))
    assert np.array_equal(O.cmux2_step_fp64(fft2, acc, bkf, 0), acc)
    assert np.array_equal(O.cmux2_step_fp64(fft2, acc, bkf, 5), acc)


@pytest.mark.parametrize("mode", ["exact", "fp64"])
def test_noiseless_trgsw_one_rotates_by_x(fft2, mode):
    acc = mu_vec()
    trgsw = gadget_trgsw2(1)
    if mode == "exact":
        out = O.cmux2_step_exact(acc, trgsw, 1)
    else:
        out = O.cmux2_step_fp64(fft2, acc, O.bk2_to_fft(fft2, trgsw), 1)
    exp = np.zeros(O.TRLWE2, np.uint64)
    exp[O.N2] = np.uint64((-MU2) & M64)
    exp[O.N2 + 1:] = MU2
    diff = (signed64(out).astype(object) - signed64(exp).astype(object))
    assert max(abs(int(v)) for v in diff) <= 1 << 20


def test_fft2_roundtrip_mt19937_42(fft2):
    x = np.fromfile(GOLDEN / "fft2_roundtrip_in.f64")
    assert x.size == O.N2
    # the first 1024 draws are the N = 1024 input
    assert np.array_equal(x[:O.N], np.fromfile(GOLDEN / "fft_roundtrip_in.f64"))
    assert np.abs(O.ffnt2_roundtrip(fft2, x) - x).max() < 1e-6


def negacyclic_np(a, b):
    n = a.size
    full = np.convolve(a, b)
    out = full[:n].copy()
    out[: n - 1] -= full[n:]
    return out


def test_negacyclic2_square_small(fft2):
    x = np.zeros(O.N2)
    x[:3] = 1.0
    ref = negacyclic_np(x, x)
    assert np.allclose(ref[:5], [1, 2, 3, 2, 1])
    assert np.abs(O.ffnt2_square(fft2, x) - ref).max() < 1e-6


def test_negacyclic2_square_random_mt19937_123(fft2):
    x = np.fromfile(GOLDEN / "negacyclic2_random_in.i32", dtype=np.int32).astype(np.float64)
    assert x.size == O.N2 and x.min() >= -5 and x.max() <= 5
    ref = negacyclic_np(x, x)
    assert np.abs(O.ffnt2_square(fft2, x) - ref).max() < 0.5


def test_decompose2_recomposes():
    rng = np.random.default_rng(19)
    p = rng.integers(0, 2**64, O.N2, dtype=np.uint64)
    d = O.decompose2(p)
    assert d.min() >= -512 and d.max() <= 511
    for n in range(0, O.N2, 97):
        rec = sum(int(d[k, n]) << (64 - 10 * (k + 1)) for k in range(4))
        err = (int(p[n]) - rec) % (1 << 64)
        err = err - (1 << 64) if err >= 1 << 63 else err
        assert abs(err) <= 1 << 23


def test_extprod2_exact_matches_bigint_schoolbook():
    rng = np.random.default_rng(23)
    trgsw = rng.integers(0, 2**64, O.TRGSW2, dtype=np.uint64)
    trlwe = rng.integers(0, 2**64, O.TRLWE2, dtype=np.uint64)
    out = O.extprod2_exact(trgsw, trlwe)
    # independent restatement on a few output coefficients with Python ints
    d = O.decompose2(trlwe[:O.N2]).astype(object), O.decompose2(trlwe[O.N2:]).astype(object)
    g = trgsw.reshape(8, 2, O.N2).astype(object)
    for j in (0, 1):
        for n in (0, 1, 777, O.N2 - 1):
            acc = 0
            for r in range(8):
                dig = d[r // 4][r % 4]
                for m in range(O.N2):
                    if dig[m] == 0:
                        continue
                    idx = n - m
                    acc += dig[m] * (g[r, j, idx] if idx >= 0 else -g[r, j, idx + O.N2])
            assert int(out[j * O.N2 + n]) == acc % (1 << 64)


def test_double_to_torus64_truncates():
    """Input is the torus value already scaled by 2^64 (include/utils_gpu.cuh:48-65):
    the fraction is truncated toward zero and the integer wraps mod 2^64."""
    s64 = 2.0 ** 64
    assert O.double_to_torus64(0.0) == 0
    assert O.double_to_torus64(0.25 * s64) == 1 << 62
    assert O.double_to_torus64(-0.25 * s64) == (-(1 << 62)) & M64
    assert O.double_to_torus64(2.5 * s64) == 1 << 63
    assert O.double_to_torus64(3.75) == 3
    assert O.double_to_torus64(-3.75) == (-3) & M64


@pytest.fixture(scope="module")
def keys02():
    sk = client.SecretKey.generate(0x5151)
    return sk, client.EvalKey02.generate(sk, keybundle=True), client.EvalKey02.generate(
        sk, keybundle=False)


@pytest.mark.parametrize("kb", [True, False])
def test_gate2_fp64_matches_truth(fft2, keys02, kb):
    sk, ekkb, ek = keys02
    key = ekkb if kb else ek
    gates = np.array([P.NAND, P.AND, P.XOR, P.MUX, P.NOR, P.NMUX], np.int32)
    rng = np.random.default_rng(3 + kb)
    a, b, c = (rng.integers(0, 2, gates.size).astype(np.uint8) for _ in range(3))
    cts = [client.encrypt_bits(sk, x, 0, seed=70 + i) for i, x in enumerate((a, b, c))]
    bkf = O.bk2_to_fft(fft2, key.bk)
    out = O.gate2_batch(gates, *cts, bkf, key.ksk, kb, O.FP64, fft2)
    exp = np.array([P.TRUTH[g](int(x), int(y), int(z)) for g, x, y, z in zip(gates, a, b, c)])
    assert np.array_equal(client.decrypt_bits(sk, out, 0), exp)


def test_blind_rotate2_fp64_vs_exact(fft2, keys02):
    """One FP64 KeyBundle step stays within 2^32 of the exact one.  Over more
    steps the two forms pick different gadget digits (the FP64 error, ~2^27,
    exceeds the 2^24 weight of the lowest lvl2 digit), so the ciphertexts part
    ways while their phases -- what decryption sees -- stay together."""
    sk, ekkb, _ = keys02
    x = client.encrypt_bits(sk, np.array([1, 0], np.uint8), 0, seed=5)
    bkf = O.bk2_to_fft(fft2, ekkb.bk)
    ex = O.blind_rotate2(x, MU2, ekkb.bk, True, O.EXACT, steps=1)
    fp = O.blind_rotate2(x, MU2, bkf, True, O.FP64, fft2, steps=1)
    assert np.abs((fp - ex).view(np.int64).astype(np.float64)).max() < 2.0 ** 32
    ex = O.blind_rotate2(x, MU2, ekkb.bk, True, O.EXACT)
    fp = O.blind_rotate2(x, MU2, bkf, True, O.FP64, fft2)
    for i in range(2):
        pe = client.trlwe64_phase(sk, ex[i]).view(np.int64).astype(np.float64)
        pf = client.trlwe64_phase(sk, fp[i]).view(np.int64).astype(np.float64)
        assert np.abs(pe - pf).max() < 2.0 ** 48
        assert np.abs(np.abs(pf) - MU2).max() < 2.0 ** 56
