"""GPU checks of circuit bootstrapping (CGGI17 form), CMUX and CMUX-tree
lookup tables, through the C-ABI.

* private key switching lvl2 -> lvl1: bit-exact against the oracle, both key
  functions, on random Torus64 inputs;
* circuit bootstrapping: every TRGSW row equals the oracle's private key
  switch of the engine's own lvl2 blind rotation (with the digit's offset
  added to b) bit for bit, and decrypts to m 2^-6(i+1) (rows j = 1) or
  -m 2^-6(i+1) s1 (rows j = 0);
* CMUX, both gadgets: one external product within FP64_TOL of the exact
  oracle and of the oracle's FP64 form;
* lookup tables: 128 random 8-bit tables over 1024 circuit-bootstrapped
  address bits (the circuit-bootstrapping workload) decrypt to the tables'
  output bits.
The reference's circuit bootstrapping is annihilation-based, so the private
key switching and the CB construction are pinned on CGGI17's definitions
rather than on reference outputs.
"""
import numpy as np
import pytest

from cufhepp_b200 import client, engine, params as P
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FP64_TOL = 2   # Torus32 units, one external product
ROW_TOL = 1 << 18


def signed32(x):
    return np.asarray(x, np.uint32).view(np.int32).astype(np.int64)


def wrap(d):
    return (d + (1 << 31)) % (1 << 32) - (1 << 31)


@pytest.fixture(scope="module")
def cb():
    sk = client.SecretKey.generate(0xCB1)
    key = client.CBKey.generate(sk)
    engine.initialize_lvl02(key.ek02)
    engine.initialize_cb(key)
    yield sk, key
    engine.cleanup_cb()
    engine.cleanup_lvl02()


@pytest.fixture(scope="module")
def fft():
    return O.FFT()


@pytest.mark.parametrize("func", [0, 1])
def test_private_keyswitch_bit_exact(cb, func):
    sk, key = cb
    rng = np.random.default_rng(3 + func)
    n = 40
    t2 = rng.integers(0, 2**64, (n, P.TLWE2_WORDS), dtype=np.uint64)
    d_in = engine.to_device(t2)
    d_out = engine.DeviceBuffer(n * P.TRLWE1_WORDS * 4)
    engine.private_keyswitch(d_in, n, func, d_out)
    got = engine.from_device(d_out, (n, P.TRLWE1_WORDS))
    ref = O.privks(t2, key.privks0 if func == 0 else key.privks1)
    assert np.array_equal(got, ref)


def test_circuit_bootstrap_rows(cb):
    sk, key = cb
    rng = np.random.default_rng(9)
    n = 6
    bits = rng.integers(0, 2, n).astype(np.uint8)
    x = client.encrypt_bits(sk, bits, 0, seed=91)
    d_x = engine.to_device(x)
    d_t = engine.DeviceBuffer(n * 6 * P.TRLWE1_WORDS * 4)
    engine.circuit_bootstrap(d_x, n, d_t)
    trgsw = engine.from_device(d_t, (n, 6, P.TRLWE1_WORDS))
    d_t2 = engine.DeviceBuffer(n * P.TLWE2_WORDS * 8)
    for i in range(3):
        mu = 1 << (64 - 6 * (i + 1) - 1)
        engine.blind_rotate_lvl02(d_x, n, mu, -1, tlwe_out=d_t2)
        t2 = engine.from_device(d_t2, (n, P.TLWE2_WORDS), np.uint64).copy()
        t2[:, P.LVL2_N] += np.uint64(mu)
        assert np.array_equal(trgsw[:, 0 * 3 + i], O.privks(t2, key.privks0))
        assert np.array_equal(trgsw[:, 1 * 3 + i], O.privks(t2, key.privks1))
        g = 1 << (32 - 6 * (i + 1))
        for b in range(n):
            m = int(bits[b])
            ph1 = signed32(client.trlwe_phase(sk, trgsw[b, 3 + i]))
            want1 = np.zeros(P.LVL1_N, np.int64)
            want1[0] = m * g
            assert np.abs(wrap(ph1 - want1)).max() < ROW_TOL
            ph0 = signed32(client.trlwe_phase(sk, trgsw[b, i]))
            want0 = -m * g * sk.lvl1.astype(np.int64)
            assert np.abs(wrap(ph0 - want0)).max() < ROW_TOL


@pytest.mark.parametrize("gadget", [engine.GADGET_CB, engine.GADGET_LVL1], ids=["cb", "lvl1"])
def test_cmux_matches_oracle(cb, fft, gadget):
    sk, _ = cb
    L, bg = (3, 6) if gadget == engine.GADGET_CB else (2, 8)
    rng = np.random.default_rng(20 + gadget)
    n = 24
    sel = rng.integers(0, 2, n)
    trgsw = np.stack([client.trgsw_encrypt_g(sk, int(m), seed=5, stream=i, l=L, bgbit=bg)
                      for i, m in enumerate(sel)])
    d1, d0 = (rng.integers(0, 2**32, (n, P.TRLWE1_WORDS), dtype=np.uint64).astype(np.uint32)
              for _ in range(2))
    dt = engine.to_device(trgsw)
    df = engine.DeviceBuffer(n * 2 * L * 2 * 512 * 16)
    engine.trgsw_to_fft(gadget, dt, n, df)
    dd1, dd0 = engine.to_device(d1), engine.to_device(d0)
    dout = engine.DeviceBuffer(n * P.TRLWE1_WORDS * 4)
    engine.cmux(gadget, df, dd1, dd0, dout, n)
    got = engine.from_device(dout, (n, P.TRLWE1_WORDS))
    ex = O.cmux_batch(trgsw, d1, d0, L, bg, O.EXACT)
    fp = O.cmux_batch(O.polys_to_fft(fft, trgsw), d1, d0, L, bg, O.FP64, fft)
    assert np.abs(wrap(signed32(got) - signed32(ex))).max() <= FP64_TOL
    assert np.abs(wrap(signed32(got) - signed32(fp))).max() <= FP64_TOL


def test_lookup_tables_over_circuit_bootstrapped_bits(cb):
    """The circuit-bootstrapping workload: 1024 lvl0 bits -> TRGSW, then 128
    random 8-bit tables addressed by them."""
    sk, _ = cb
    rng = np.random.default_rng(31)
    q = 128
    luts = rng.integers(0, 256, (q, 256)).astype(np.uint8)
    addr = rng.integers(0, 256, q)
    bits = np.array([(int(addr[t]) >> k) & 1 for t in range(q) for k in range(8)], np.uint8)
    x = client.encrypt_bits(sk, bits, 0, seed=131)
    d_x = engine.to_device(x)
    d_t = engine.DeviceBuffer(q * 8 * 6 * P.TRLWE1_WORDS * 4)
    engine.circuit_bootstrap(d_x, q * 8, d_t)
    d_f = engine.DeviceBuffer(q * 8 * 6 * 2 * 512 * 16)
    engine.trgsw_to_fft(engine.GADGET_CB, d_t, q * 8, d_f)
    d_o = engine.DeviceBuffer(q * 8 * P.TLWE1_WORDS * 4)
    engine.lut_eval(luts, d_f, P.MU32, d_o)
    out = engine.from_device(d_o, (q, 8, P.TLWE1_WORDS))
    got = client.decrypt_bits(sk, out.reshape(-1, P.TLWE1_WORDS), 1).reshape(q, 8)
    want = np.array([[(int(luts[t][addr[t]]) >> b) & 1 for b in range(8)] for t in range(q)])
    assert int(np.count_nonzero(got != want)) == 0
    # output margin: every phase within mu/2 of +-mu
    ph = signed32(client.phase(sk, out.reshape(-1, P.TLWE1_WORDS), 1)).astype(np.float64)
    assert np.abs(np.abs(ph) - P.MU32).max() < P.MU32 / 2
