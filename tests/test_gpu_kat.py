"""The reference's accumulate known-answer tests, run on the GPU through the
C-ABI in both precision forms (test/test_accumulate_diag.cu:369-605):

* a zero bootstrapping key leaves the accumulator unchanged: after every
  CMUX step the accumulator is still the test polynomial, exactly;
* a noiseless TRGSW(1) as the key of every step, with abar_0 = k and every
  other abar 0, turns a = 0, b = vec(mu) into a = 0, b = X^k vec(mu).  The
  gadget decomposition of mu = 2^29 is exact (l Bgbit = 16 bits), so the FP64
  form must give the exact answer as well, with the plain key and with the
  KeyBundle key (bk0 = TRGSW(s0 s1), bk1 = TRGSW(s0 (1 - s1)),
  bk2 = TRGSW((1 - s0) s1) at s0 = 1, s1 = 0: bk1 = TRGSW(1), bk0 = bk2 = 0).
  The INT8 form runs every case with both key forms as well.
"""
import numpy as np
import pytest

from cufhepp_b200 import client, engine, params as P

pytestmark = pytest.mark.gpu

N = P.LVL1_N
SHIFTS = [0, 1, 5, 511, 1023, 1024, 1027, 2047]  # abar_0 per lane


def trgsw_one() -> np.ndarray:
    """Noiseless TRGSW(1): row (j, d) holds 2^(32 - 8 (d + 1)) at coefficient 0
    of polynomial j, TFHEpp layout [row][poly][N]."""
    t = np.zeros((2 * P.LVL1_L, 2, N), np.uint32)
    for j in range(2):
        for d in range(P.LVL1_L):
            t[j * P.LVL1_L + d, j, 0] = 1 << (32 - P.LVL1_BGBIT * (d + 1))
    return t


def bootstrapping_key(kind: str) -> np.ndarray:
    if kind == "zero":
        return np.zeros(P.BK_WORDS, np.uint32)
    if kind == "zero_kb":
        return np.zeros(P.BKKB_WORDS, np.uint32)
    if kind == "one":
        return np.broadcast_to(trgsw_one(), (P.LVL0_N,) + trgsw_one().shape).ravel().copy()
    # KeyBundle of noiseless keys at s0 = 1, s1 = 0: [pair][bk0, bk1, bk2]
    kb = np.zeros((P.LVL0_N // 2, 3) + trgsw_one().shape, np.uint32)
    kb[:, 1] = trgsw_one()
    return kb.ravel()


def inputs() -> np.ndarray:
    """lvl0 TLWEs with b = 0 (test polynomial vec(mu)), a_0 = k 2^21 so that
    abar_0 = (a_0 + 2^20) >> 21 = k, every other a_i = 0 (abar_i = 0)."""
    x = np.zeros((len(SHIFTS), P.TLWE0_WORDS), np.uint32)
    x[:, 0] = np.asarray(SHIFTS, np.uint64) << 21
    return x


def rotated_test_vector(k: int) -> np.ndarray:
    i = np.arange(N)
    neg = (i < (k & (N - 1))) ^ bool(k >> 10)
    return np.where(neg, (-P.MU32) & 0xFFFFFFFF, P.MU32).astype(np.uint32)


def run(kind: str, form: int, steps: int) -> np.ndarray:
    rng = np.random.default_rng(1)
    ksk = rng.integers(0, 2**32, P.KSK_WORDS, dtype=np.uint64).astype(np.uint32)
    engine.initialize(client.EvalKey(bootstrapping_key(kind), ksk, kind.endswith("_kb")))
    try:
        engine.set_precision(form)
        x = inputs()
        d_in = engine.to_device(x)
        d_acc = engine.DeviceBuffer(len(SHIFTS) * P.TRLWE1_WORDS * 4)
        engine.blind_rotate(d_in, len(SHIFTS), P.MU32, steps, acc_out=d_acc)
        engine.synchronize()
        return engine.from_device(d_acc, (len(SHIFTS), 2, N))
    finally:
        engine.set_precision(P.FP64_FFNT)
        engine.cleanup()


FORMS = [pytest.param(P.FP64_FFNT, id="fp64"), pytest.param(P.INT8_EXACT, id="int8")]


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("kind", ["zero", "zero_kb"], ids=["plain", "kb"])
@pytest.mark.parametrize("steps", [1, 7, -1], ids=["1step", "7steps", "all"])
def test_zero_key_leaves_the_accumulator_unchanged(form, kind, steps):
    """A zero key leaves the accumulator unchanged; with a KeyBundle key the
    pair's result is the gadget recomposition of the digits (the H term),
    which is exact for the test polynomial (mu = 2^29 has no bits below
    2^16)."""
    acc = run(kind, form, steps)
    for lane in range(len(SHIFTS)):
        assert not acc[lane, 0].any()
        assert np.array_equal(acc[lane, 1], rotated_test_vector(0))


@pytest.mark.parametrize("form", FORMS)
def test_trgsw_one_rotates_by_x_to_the_abar(form):
    acc = run("one", form, -1)
    for lane, k in enumerate(SHIFTS):
        assert not acc[lane, 0].any(), k
        assert np.array_equal(acc[lane, 1], rotated_test_vector(k)), k


@pytest.mark.parametrize("form", FORMS)
def test_keybundle_of_noiseless_keys_rotates_by_x_to_the_abar(form):
    acc = run("one_kb", form, -1)
    for lane, k in enumerate(SHIFTS):
        assert not acc[lane, 0].any(), k
        assert np.array_equal(acc[lane, 1], rotated_test_vector(k)), k
