"""Large-sample correctness of every precision form, through the C-ABI.

* >= 10^6 random *bootstrapped* gates per form (gate ids drawn over all 14,
  so NOT/COPY, which do not bootstrap, are drawn too but not counted; both
  ciphertext levels) decrypt to the truth tables of test/plain.h with zero
  failures: the FP64-FFNT form (KeyBundle key), the INT8-exact form with the
  plain key and the INT8-exact form with the KeyBundle key;
* a 1024-gate subset on the INT8 form is bit-identical to the exact
  schoolbook oracle (the whole gate is integer arithmetic there).
"""
import numpy as np
import pytest

from cufhepp_b200 import client, engine, params as P
from oracle import oracle as O

pytestmark = pytest.mark.gpu

CHUNK = 1 << 16
TARGET = 10 ** 6  # bootstrapped gates per form


def run_million(sk, level_split=4):
    """Returns (gates, bootstrapped gates, failures, smallest |phase| margin
    in units of mu); chunks are added until TARGET gates have bootstrapped."""
    rng = np.random.default_rng(2026)
    total = boots = fails = 0
    margin = np.inf
    c = 0
    while boots < TARGET:
        level = 0 if c % level_split == 0 else 1
        gates = rng.integers(0, 14, CHUNK).astype(np.int32)
        a, b, cc = (rng.integers(0, 2, CHUNK).astype(np.uint8) for _ in range(3))
        cts = [client.encrypt_bits(sk, x, level, seed=1000 * c + i, stream0=0)
               for i, x in enumerate((a, b, cc))]
        out = engine.gate_batch_host(gates, level, *cts)
        engine.synchronize()
        exp = np.zeros(CHUNK, np.uint8)
        for g in range(14):
            m = gates == g
            exp[m] = P.TRUTH[g](a[m], b[m], cc[m])
        got = client.decrypt_bits(sk, out, level)
        fails += int(np.count_nonzero(got != exp))
        ph = client.phase(sk, out, level).view(np.int32).astype(np.float64)
        margin = min(margin, float(np.abs(ph).min()) / P.MU32)
        total += CHUNK
        boots += int(np.count_nonzero((gates != P.NOT) & (gates != P.COPY)))
        c += 1
    return total, boots, fails, margin


@pytest.mark.parametrize("form", ["fp64", "int8", "int8_kb"])
def test_one_million_gates_zero_failures(keys, form):
    sk, ek_kb, ek_nokb = keys
    ek = ek_nokb if form == "int8" else ek_kb
    engine.initialize(ek)
    try:
        engine.set_precision(P.FP64_FFNT if form == "fp64" else P.INT8_EXACT)
        total, boots, fails, margin = run_million(sk)
        print(f"{form}: {total} gates ({boots} bootstrapped), {fails} decryption failures, "
              f"min |phase| = {margin:.3f} mu")
        assert boots >= TARGET
        assert fails == 0
        assert margin > 0.5  # outputs sit near +-mu, far from the decision boundary
    finally:
        engine.set_precision(P.FP64_FFNT)
        engine.cleanup()


@pytest.mark.parametrize("kb", [False, True], ids=["plain", "kb"])
def test_int8_1024_gates_bit_exact_vs_oracle(keys, kb):
    sk, ek_kb, ek_nokb = keys
    ek = ek_kb if kb else ek_nokb
    engine.initialize(ek)
    try:
        engine.set_precision(P.INT8_EXACT)
        rng = np.random.default_rng(77)
        gates = rng.choice([P.NAND, P.AND, P.OR, P.XOR, P.XNOR, P.MUX], size=1024).astype(np.int32)
        a, b, c = (rng.integers(0, 2, gates.size).astype(np.uint8) for _ in range(3))
        cts = [client.encrypt_bits(sk, x, 1, seed=90 + i) for i, x in enumerate((a, b, c))]
        out = engine.gate_batch_host(gates, 1, *cts)
        engine.synchronize()
        ref = O.gate_batch(gates, 1, *cts, ek.bk, ek.ksk, ek.keybundle, O.EXACT)
        assert np.array_equal(out, ref)
    finally:
        engine.set_precision(P.FP64_FFNT)
        engine.cleanup()
