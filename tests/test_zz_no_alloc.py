"""cufhe_gate_batch_noalloc against cufhe_gate_batch, through the C-ABI.

The no-allocation entry point exists for callers that cannot let the library
allocate device memory (a fixed memory budget, a host-owned allocator, or a
latency-critical path that cannot absorb an allocation's synchronisation).
It runs the same gate pipeline with its lane buffers in a fixed array inside
the library.  Its key switch is the SIMT one and cufhe_gate_batch's the
tensor-core one, but both are exact integer arithmetic, and both run the
same FP64 blind rotation on the same lane count, so the outputs must be
identical bit for bit.  Two calls in a row with different batches check that
what the first call leaves in the shared array does not leak into the second,
and repeated calls of several sizes must leave the device's free memory
unchanged.

This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from cufhepp_b200 import client, engine, params as P

pytestmark = pytest.mark.gpu

PHASE_TOL = 2.0 ** -12  # torus; the tolerance of the FP64 gate tests


def torus_dist(a, b):
    d = (np.asarray(a, np.uint32) - np.asarray(b, np.uint32)).astype(np.uint32)
    return np.abs(d.view(np.int32).astype(np.float64)) / 2.0 ** 32


@pytest.fixture(scope="module")
def ctx(keys):
    sk, ek_kb, _ = keys
    engine.initialize(ek_kb)
    engine.set_precision(P.FP64_FFNT)
    yield sk
    engine.cleanup()


def run_both(sk, gate, count, level, seed):
    words = P.TLWE1_WORDS if level == 1 else P.TLWE0_WORDS
    rng = np.random.default_rng(seed)
    a, b, c = (rng.integers(0, 2, count).astype(np.uint8) for _ in range(3))
    cts = [client.encrypt_bits(sk, x, level, seed=seed + i) for i, x in enumerate((a, b, c))]
    dev = [engine.to_device(x) for x in cts]
    out_ref = engine.DeviceBuffer(count * words * 4)
    out_new = engine.DeviceBuffer(count * words * 4)
    engine.gate_batch(None, count, level, out_ref, *dev, uniform=gate)
    L = engine.load()
    engine.check(L.cufhe_gate_batch_noalloc(gate, count, level, engine.dptr(out_new),
                                            *(engine.dptr(d) for d in dev), None),
                 "gate_batch_noalloc")
    ref = engine.from_device(out_ref, (count, words))
    new = engine.from_device(out_new, (count, words))
    exp = np.array([P.TRUTH[gate](int(x), int(y), int(z)) for x, y, z in zip(a, b, c)])
    return ref, new, exp


def test_noalloc_matches_batch_two_calls_in_a_row(ctx):
    sk = ctx
    # first call: 200 NAND gates at lvl1 (200 of the 256 lane slots)
    ref, new, exp = run_both(sk, P.NAND, 200, 1, seed=901)
    assert np.array_equal(new, ref)
    assert torus_dist(client.phase(sk, new, 1), client.phase(sk, ref, 1)).max() < PHASE_TOL
    assert np.array_equal(client.decrypt_bits(sk, new, 1), exp)
    # second call right after: 37 Mux gates at lvl0 (74 lanes) on different inputs
    ref, new, exp = run_both(sk, P.MUX, 37, 0, seed=902)
    assert np.array_equal(new, ref)
    assert torus_dist(client.phase(sk, new, 0), client.phase(sk, ref, 0)).max() < PHASE_TOL
    assert np.array_equal(client.decrypt_bits(sk, new, 0), exp)


@pytest.mark.parametrize("level", [1, 0])
def test_noalloc_every_gate_matches_batch(ctx, level):
    """Every gate id (Not and Copy bootstrap nothing, Mux and NMux two lanes a
    gate) through the allocation-free entry point equals cufhe_gate_batch bit
    for bit and decrypts to its truth table."""
    sk = ctx
    for gate in range(14):
        ref, new, exp = run_both(sk, gate, 12, level, seed=1000 + 20 * gate + level)
        assert np.array_equal(new, ref), P.GATE_NAMES[gate]
        assert np.array_equal(client.decrypt_bits(sk, new, level), exp), P.GATE_NAMES[gate]


def test_noalloc_calls_leave_device_memory_unchanged(ctx):
    """After one warm-up pass (the first launch of each kernel may make the
    driver load its code), further calls of every size and level do not
    change the device's free memory."""
    import torch
    sk = ctx
    L = engine.load()
    cases = [(P.NAND, 1, 1), (P.NAND, 256, 1), (P.MUX, 128, 1), (P.MUX, 37, 0), (P.XOR, 90, 0),
             (P.NOT, 5, 1)]
    bufs = []
    for gate, count, level in cases:
        words = P.TLWE1_WORDS if level == 1 else P.TLWE0_WORDS
        bits = np.random.default_rng(count).integers(0, 2, count).astype(np.uint8)
        ct = client.encrypt_bits(sk, bits, level, seed=950 + count)
        bufs.append((gate, count, level, engine.to_device(ct),
                     engine.DeviceBuffer(count * words * 4)))

    def call_all():
        for gate, count, level, d_in, d_out in bufs:
            p_in = engine.dptr(d_in)
            engine.check(L.cufhe_gate_batch_noalloc(gate, count, level, engine.dptr(d_out), p_in,
                                                    p_in, p_in, None), "gate_batch_noalloc")
        engine.synchronize()

    torch.cuda.mem_get_info(0)  # torch's own CUDA set-up happens before the warm-up
    call_all()  # warm-up
    free0, _ = torch.cuda.mem_get_info(0)
    for _ in range(3):
        call_all()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0


def test_noalloc_rejects_batches_beyond_its_array(ctx):
    L = engine.load()
    rc = L.cufhe_gate_batch_noalloc(P.MUX, 129, 1, C.c_void_p(1), C.c_void_p(1), C.c_void_p(1),
                                    C.c_void_p(1), None)
    assert rc == -1
    assert b"at most 256" in L.cufhe_last_error()
