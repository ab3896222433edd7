"""Pins the oracle on the reference's own known-answer tests.

* test/test_accumulate_diag.cu:266-336  -- zero TRGSW, abar = 0: unchanged.
* test/test_accumulate_diag.cu:137-262  -- noiseless TRGSW(1) (gadget rows
  only, :101-134), abar = 1, (a = 0, b = vec(mu)) -> b = (-mu, mu, ..., mu),
  tolerance 1 for Torus32 (:241-243).
* test/test_fft_roundtrip.cu:141-184    -- mt19937(42) reals round-trip < 1e-6.
* test/test_fft_roundtrip.cu:186-243    -- (1+X+X^2)^2 negacyclic < 1e-6.
* test/test_fft_roundtrip.cu:245-295    -- mt19937(123) ints in [-5,5] squared < 0.5.
The seeded inputs are regenerated with the same std::mt19937 engines and
distributions by tests/golden/gen_fft_kat_inputs.cpp.
"""
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden"
MU = 1 << 29


def gadget_trgsw(m: int) -> np.ndarray:
    t = np.zeros((4, 2, O.N), np.uint32)
    for row in range(4):
        j, d = row // 2, row % 2
        t[row, j, 0] = np.uint32((m << (32 - (d + 1) * 8)) & 0xFFFFFFFF)
    return t.reshape(-1)


def signed(x):
    return np.asarray(x, np.uint32).view(np.int32).astype(np.int64)


@pytest.fixture(scope="module")
def fft():
    return O.FFT()


def test_zero_trgsw_identity(fft):
    acc = np.zeros(O.TRLWE, np.uint32)
    acc[O.N:] = MU
    assert np.array_equal(O.cmux_step_exact(acc, np.zeros(O.TRGSW, np.uint32), 0), acc)
    bkf = O.bk_to_fft(fft, np.zeros(O.TRGSW, np.uint32))
    diff = np.zeros(O.TRLWE, np.uint32)
    assert np.array_equal(O.extprod_fp64(fft, bkf, diff), np.zeros(O.TRLWE, np.uint32))


@pytest.mark.parametrize("mode", ["exact", "fp64"])
def test_noiseless_trgsw_one_rotates_by_x(fft, mode):
    acc = np.zeros(O.TRLWE, np.uint32)
    acc[O.N:] = MU
    trgsw = gadget_trgsw(1)
    if mode == "exact":
        out = O.cmux_step_exact(acc, trgsw, 1)
    else:
        x = np.zeros(O.TLWE0, np.uint32)
        # one CMUX step with abar = 1 through the FP64 external product
        rot = np.concatenate([np.zeros(O.N, np.uint32),
                              np.concatenate([[np.uint32(-MU & 0xFFFFFFFF)],
                                              np.full(O.N - 1, MU, np.uint32)])])
        diff = (rot - acc).astype(np.uint32)
        out = (acc + O.extprod_fp64(fft, O.bk_to_fft(fft, trgsw), diff)).astype(np.uint32)
    exp = np.zeros(O.TRLWE, np.uint32)
    exp[O.N] = np.uint32(-MU & 0xFFFFFFFF)
    exp[O.N + 1:] = MU
    assert np.abs(signed(out) - signed(exp)).max() <= 1


def test_fft_roundtrip_mt19937_42(fft):
    x = np.fromfile(GOLDEN / "fft_roundtrip_in.f64")
    assert x.size == O.N
    assert np.abs(O.ffnt_roundtrip(fft, x) - x).max() < 1e-6


def test_negacyclic_square_small(fft):
    x = np.zeros(O.N)
    x[:3] = 1.0
    ref = O.negacyclic_mul_f64(x, x)
    assert np.allclose(ref[:5], [1, 2, 3, 2, 1])
    assert np.abs(O.ffnt_square(fft, x) - ref).max() < 1e-6


def test_negacyclic_square_random_mt19937_123(fft):
    x = np.fromfile(GOLDEN / "negacyclic_random_in.i32", dtype=np.int32).astype(np.float64)
    assert x.size == O.N and x.min() >= -5 and x.max() <= 5
    ref = O.negacyclic_mul_f64(x, x)
    assert np.abs(O.ffnt_square(fft, x) - ref).max() < 0.5


def test_exact_product_matches_bigint_schoolbook():
    rng = np.random.default_rng(5)
    d = rng.integers(-128, 128, O.N).astype(np.int32)
    k = rng.integers(0, 2**32, O.N, dtype=np.uint64).astype(np.uint32)
    out = O.negacyclic_mul_exact(d, k)
    # independent restatement with Python integers and a Toeplitz matrix
    dd = d.astype(object)
    kk = k.astype(object)
    ref = [0] * O.N
    for m in range(O.N):
        if dd[m] == 0:
            continue
        for n in range(O.N):
            idx = n - m
            if idx >= 0:
                ref[n] += dd[m] * kk[idx]
            else:
                ref[n] -= dd[m] * kk[idx + O.N]
    ref = np.array([v % (1 << 32) for v in ref], dtype=np.uint64).astype(np.uint32)
    assert np.array_equal(out, ref)


def test_decompose_recomposes():
    rng = np.random.default_rng(9)
    p = rng.integers(0, 2**32, O.N, dtype=np.uint64).astype(np.uint32)
    d = O.decompose(p)
    assert d.min() >= -128 and d.max() <= 127
    rec = (d[0].astype(np.int64) << 24) + (d[1].astype(np.int64) << 16)
    err = ((p.astype(np.int64) - rec + (1 << 31)) % (1 << 32)) - (1 << 31)
    assert np.abs(err).max() <= 1 << 15


def test_test_vector_special_cases():
    tv = O.test_vector(2 * O.N, MU)
    assert (tv[:O.N] == 0).all() and (tv[O.N:] == MU).all()
    tv = O.test_vector(3, MU)
    assert (signed(tv[O.N:O.N + 3]) == -MU).all() and (tv[O.N + 3:] == MU).all()
    tv = O.test_vector(O.N + 3, MU)
    assert (tv[O.N:O.N + 3] == MU).all() and (signed(tv[O.N + 3:]) == -MU).all()
