"""GPU parity of the FP64-FFNT path and of the integer pieces, through the C-ABI.

* identity key switching: bit-exact against the oracle;
* blind rotation (KeyBundle and plain): FP64 rounding against the exact
  schoolbook oracle -- one step bit-exact up to +-1 per coefficient, full
  rotations within a phase tolerance of 2^-12 (torus) of the exact result;
* small batches (the cluster form) equal the one-CTA-per-lane form bit for bit;
* gates, both orders, every gate id: decrypt to the truth tables
  (test/plain.h:1-70) and match the oracle's phase within 2^-12.
"""
import os

import numpy as np
import pytest

from cufhepp_b200 import client, engine, params as P
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FP64_STEP_TOL = 1              # torus32 units, single external product
PHASE_TOL = 2.0 ** -12         # torus, full blind rotation / gate output


def signed(x):
    return np.asarray(x, np.uint32).view(np.int32).astype(np.int64)


def torus_dist(a, b):
    d = (np.asarray(a, np.uint32) - np.asarray(b, np.uint32)).astype(np.uint32)
    return np.abs(d.view(np.int32).astype(np.float64)) / 2.0 ** 32


@pytest.fixture(scope="module", params=[True, False], ids=["kb", "nokb"])
def ctx(request, keys):
    sk, ek_kb, ek_nokb = keys
    ek = ek_kb if request.param else ek_nokb
    engine.initialize(ek)
    engine.set_precision(P.FP64_FFNT)
    yield sk, ek, request.param
    engine.cleanup()


def lvl0_inputs(sk, count, seed):
    rng = np.random.default_rng(seed)
    bits = rng.integers(0, 2, count).astype(np.uint8)
    return bits, client.encrypt_bits(sk, bits, 0, seed=seed)


def test_identity_keyswitch_bit_exact(ctx):
    sk, ek, _ = ctx
    rng = np.random.default_rng(3)
    bits = rng.integers(0, 2, 40).astype(np.uint8)
    c1 = client.encrypt_bits(sk, bits, 1, seed=3)
    d_in = engine.to_device(c1)
    d_out = engine.DeviceBuffer(40 * P.TLWE0_WORDS * 4)
    engine.identity_keyswitch(d_in, 40, d_out)
    got = engine.from_device(d_out, (40, P.TLWE0_WORDS))
    ref = O.iks_batch(c1, None, 1, 0, 0, ek.ksk)
    assert np.array_equal(got, ref)
    assert np.array_equal(client.decrypt_bits(sk, got, 0), bits)


@pytest.mark.parametrize("lanes", [1, 9, 16])
def test_cluster_form_for_small_batches_is_bit_identical(ctx, lanes):
    """Up to 16 lanes the rotation runs one lane per cluster of four CTAs (the
    key multiply-accumulate split over four SMs, partial spectra gathered
    through distributed shared memory); CUFHE_BR_CLUSTER=0 keeps one CTA per
    lane.  Both must give the same accumulators bit for bit."""
    sk, ek, _ = ctx
    _, x = lvl0_inputs(sk, lanes, 31 + lanes)
    d_in = engine.to_device(x)
    got = {}
    for cluster in (False, True):
        if cluster:
            os.environ.pop("CUFHE_BR_CLUSTER", None)
        else:
            os.environ["CUFHE_BR_CLUSTER"] = "0"
        try:
            d_acc = engine.DeviceBuffer(lanes * P.TRLWE1_WORDS * 4)
            engine.blind_rotate(d_in, lanes, P.MU32, -1, acc_out=d_acc)
            engine.synchronize()
            got[cluster] = engine.from_device(d_acc, (lanes, P.TRLWE1_WORDS))
        finally:
            os.environ.pop("CUFHE_BR_CLUSTER", None)
    assert np.array_equal(got[True], got[False])


def test_blind_rotate_one_step(ctx):
    sk, ek, kb = ctx
    bits, x = lvl0_inputs(sk, 8, 5)
    d_in = engine.to_device(x)
    d_acc = engine.DeviceBuffer(8 * P.TRLWE1_WORDS * 4)
    engine.blind_rotate(d_in, 8, P.MU32, 1, acc_out=d_acc)
    got = engine.from_device(d_acc, (8, P.TRLWE1_WORDS))
    ref = O.blind_rotate(x, P.MU32, ek.bk, kb, O.EXACT, steps=1)
    diff = np.abs(signed(got) - signed(ref))
    diff = np.minimum(diff, 2**32 - diff)
    assert diff.max() <= FP64_STEP_TOL, diff.max()


def test_blind_rotate_full_phase(ctx):
    sk, ek, kb = ctx
    bits, x = lvl0_inputs(sk, 6, 6)
    d_in = engine.to_device(x)
    d_acc = engine.DeviceBuffer(6 * P.TRLWE1_WORDS * 4)
    d_tl = engine.DeviceBuffer(6 * P.TLWE1_WORDS * 4)
    engine.blind_rotate(d_in, 6, P.MU32, -1, acc_out=d_acc, tlwe_out=d_tl)
    got = engine.from_device(d_acc, (6, P.TRLWE1_WORDS))
    tl = engine.from_device(d_tl, (6, P.TLWE1_WORDS))
    ref = O.blind_rotate(x, P.MU32, ek.bk, kb, O.EXACT)
    for g in range(6):
        pg = client.trlwe_phase(sk, got[g])
        pr = client.trlwe_phase(sk, ref[g])
        assert torus_dist(pg, pr).max() < PHASE_TOL
        assert np.array_equal(tl[g], O.sample_extract(got[g]))
    # the extracted constant term decrypts to the input bit (mu for 1, -mu for 0)
    assert np.array_equal(client.decrypt_bits(sk, tl, 1), bits)


@pytest.mark.parametrize("level", [1, 0])
def test_all_gates_match_truth_and_oracle(ctx, level):
    sk, ek, kb = ctx
    gates = np.arange(14, dtype=np.int32).repeat(2)
    cnt = gates.size
    rng = np.random.default_rng(10 + level)
    a, b, c = (rng.integers(0, 2, cnt).astype(np.uint8) for _ in range(3))
    ca = client.encrypt_bits(sk, a, level, seed=21)
    cb = client.encrypt_bits(sk, b, level, seed=22)
    cc = client.encrypt_bits(sk, c, level, seed=23)
    out = engine.gate_batch_host(gates, level, ca, cb, cc)
    engine.synchronize()
    exp = np.array([P.TRUTH[g](int(x), int(y), int(z)) for g, x, y, z in zip(gates, a, b, c)])
    assert np.array_equal(client.decrypt_bits(sk, out, level), exp)
    ref = O.gate_batch(gates, level, ca, cb, cc, ek.bk, ek.ksk, kb, O.EXACT)
    ph_g = client.phase(sk, out, level)
    ph_r = client.phase(sk, ref, level)
    assert torus_dist(ph_g, ph_r).max() < PHASE_TOL


def test_single_gate_api_and_copy_variant(ctx):
    sk, ek, kb = ctx
    a = np.array([1], np.uint8)
    b = np.array([1], np.uint8)
    ca = client.encrypt_bits(sk, a, 1, seed=31)
    cb = client.encrypt_bits(sk, b, 1, seed=32)
    din0, din1 = engine.to_device(ca), engine.to_device(cb)
    dout = engine.DeviceBuffer(P.TLWE1_WORDS * 4)
    L = engine.load()
    engine.check(L.cufhe_gate(P.NAND, 1, engine.dptr(dout), engine.dptr(din0),
                              engine.dptr(din1), None, None), "gate")
    out = engine.from_device(dout, (1, P.TLWE1_WORDS))
    assert client.decrypt_bits(sk, out, 1)[0] == 0
    host_out = np.zeros(P.TLWE1_WORDS, np.uint32)
    engine.check(L.cufhe_gate_copy(P.OR, 1, engine._p(host_out), engine.dptr(dout),
                                   engine._p(ca[0]), engine.dptr(din0), engine._p(cb[0]),
                                   engine.dptr(din1), None, None, None), "gate_copy")
    engine.synchronize()
    assert client.decrypt_bits(sk, host_out, 1)[0] == 1


def test_streams_and_query(ctx):
    sk, ek, kb = ctx
    import ctypes as C
    L = engine.load()
    st = C.c_void_p()
    engine.check(L.cufhe_stream_create(C.byref(st), -1), "stream_create")
    bits = np.array([1, 0, 1, 1], np.uint8)
    c1 = client.encrypt_bits(sk, bits, 1, seed=41)
    out = engine.gate_batch_host(None, 1, c1, c1, uniform=P.AND, stream=st)
    engine.check(L.cufhe_stream_synchronize(st), "stream_sync")
    assert L.cufhe_stream_query(st) == 1
    assert np.array_equal(client.decrypt_bits(sk, out, 1), bits)
    engine.check(L.cufhe_stream_destroy(st), "stream_destroy")
