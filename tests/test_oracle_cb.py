"""Oracle checks of the circuit-bootstrapping pieces (CPU only).

The reference's circuit bootstrapping is annihilation-based and has no
private key switching, so these pieces restate CGGI17 and are checked on
their defining properties rather than on reference vectors:
* private key switching (basebit 4, t 10) maps a Torus64 TLWE of phase p
  to a TRLWE<lvl1> of phase f(p): p at coefficient 0 for f = x, -p s1(X)
  for f = -x s1 (small source dimension, so the key stays small);
* the generic external product (l = 3, Bgbit = 6) agrees between the exact
  and FP64 forms; CMUX with noiseless TRGSW(0)/(1) selects d0 / d1;
* a CMUX-tree lookup table over encrypted address bits decrypts to the
  table's output bits.
"""
import numpy as np
import pytest

from cufhepp_b200 import client, params as P
from oracle import oracle as O

L, BG = O.CB_L, O.CB_BGBIT


def signed32(x):
    return np.asarray(x, np.uint32).view(np.int32).astype(np.int64)


@pytest.fixture(scope="module")
def sk():
    return client.SecretKey.generate(0xCB0)


@pytest.fixture(scope="module")
def fft():
    return O.FFT()


def small_tlwe64(rng, key, msg64):
    a = rng.integers(0, 2**64, key.size, dtype=np.uint64)
    noise = np.uint64(int(rng.normal(0, 2.0 ** 20)) % (1 << 64))
    with np.errstate(over="ignore"):
        b = (np.sum(a * key.astype(np.uint64), dtype=np.uint64) + np.uint64(msg64) + noise)
    return np.concatenate([a, [b]]).astype(np.uint64)


@pytest.mark.parametrize("func", [0, 1])
def test_private_keyswitch_applies_the_function(sk, func):
    rng = np.random.default_rng(40 + func)
    n_src = 8
    key_src = rng.integers(0, 2, n_src).astype(np.int32)
    ksk = client.privks_key(key_src, sk.lvl1, func, seed=99)
    assert ksk.size == (n_src + 1) * O.PKS_T * O.PKS_NU * O.TRLWE
    for m in (0, 1, 3):
        msg64 = m << 58
        t = small_tlwe64(rng, key_src, msg64)
        out = O.privks(t, ksk, n_src)[0]
        ph = signed32(client.trlwe_phase(sk, out))
        c = m << 26  # the Torus64 phase in Torus32
        if func == 1:
            want = np.zeros(P.LVL1_N, np.int64)
            want[0] = c
        else:
            # -c s1(X): coefficient k is -c s1[k]
            want = -c * sk.lvl1.astype(np.int64)
        d = (ph - want + (1 << 31)) % (1 << 32) - (1 << 31)
        assert np.abs(d).max() < 1 << 16


def test_extprod_exact_vs_fp64_cb_gadget(fft):
    rng = np.random.default_rng(5)
    trgsw = rng.integers(0, 2**32, 2 * L * O.TRLWE, dtype=np.uint64).astype(np.uint32)
    trlwe = rng.integers(0, 2**32, O.TRLWE, dtype=np.uint64).astype(np.uint32)
    ex = O.extprod_g(trgsw, trlwe, L, BG, O.EXACT)
    fp = O.extprod_g(O.polys_to_fft(fft, trgsw), trlwe, L, BG, O.FP64, fft)
    assert np.abs(signed32(fp - ex)).max() <= 1


@pytest.mark.parametrize("mode", ["exact", "fp64"])
def test_cmux_selects_with_noiseless_trgsw(sk, fft, mode):
    rng = np.random.default_rng(6)
    d1, d0 = (rng.integers(0, 2**32, (1, O.TRLWE), dtype=np.uint64).astype(np.uint32)
              for _ in range(2))
    for m in (0, 1):
        t = client.trgsw_encrypt_g(sk, m, seed=1, stream=m, l=L, bgbit=BG, alpha=0.0)
        key = t if mode == "exact" else O.polys_to_fft(fft, t)
        out = O.cmux_batch(key, d1, d0, L, BG, O.EXACT if mode == "exact" else O.FP64, fft)
        want = d1 if m else d0
        # noiseless TRGSW: the only error is the gadget rounding, |err| <= 2^13
        # per coefficient of the selected difference, times the key polynomial
        d = signed32(client.trlwe_phase(sk, out[0])) - signed32(client.trlwe_phase(sk, want[0]))
        d = (d + (1 << 31)) % (1 << 32) - (1 << 31)
        assert np.abs(d).max() < 1 << 24


def test_lut_by_cmux_tree_decrypts(sk, fft):
    rng = np.random.default_rng(7)
    luts = rng.integers(0, 256, (2, 256)).astype(np.uint8)
    addr = rng.integers(0, 256, 2)
    tr = []
    for q in range(2):
        for k in range(8):
            bit = (int(addr[q]) >> k) & 1
            tr.append(client.trgsw_encrypt_g(sk, bit, seed=11, stream=q * 8 + k, l=L, bgbit=BG))
    tf = O.polys_to_fft(fft, np.concatenate(tr))
    out = O.lut_eval(tf, luts, P.MU32, O.FP64, fft)
    for q in range(2):
        bits = client.decrypt_bits(sk, out[q], 1)
        want = [(int(luts[q][addr[q]]) >> b) & 1 for b in range(8)]
        assert list(bits) == want
