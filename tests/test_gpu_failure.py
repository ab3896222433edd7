"""Failure detection on the GPU without a GPU fault: a kernel whose bounded
mbarrier wait runs out (a barrier nothing arrives at) sets the device error
flag the way the tensor-core kernels do; the engine reports it as
CUFHE_ERR_CUDA at synchronisation, clears it, and the CUDA context stays
usable for gate batches afterwards."""
import numpy as np
import pytest

from cufhepp_b200 import client, engine, params as P

pytestmark = pytest.mark.gpu


def test_bounded_wait_timeout_is_reported_and_context_survives(keys):
    sk, ek_kb, _ = keys
    engine.initialize(ek_kb)
    engine.set_precision(P.FP64_FFNT)
    L = engine.load()
    assert L.cufhe_selftest_wait_timeout() == -3          # CUFHE_ERR_CUDA
    assert "timed out" in L.cufhe_last_error().decode()
    engine.synchronize()                                  # flag cleared: no error now
    gates = np.array([P.NAND, P.XOR, P.MUX, P.AND] * 8, np.int32)
    rng = np.random.default_rng(1)
    a, b, c = (rng.integers(0, 2, gates.size).astype(np.uint8) for _ in range(3))
    cts = [client.encrypt_bits(sk, x, 1, seed=20 + i) for i, x in enumerate((a, b, c))]
    out = engine.gate_batch_host(gates, engine.LVL1, *cts)
    engine.synchronize()
    exp = np.array([P.TRUTH[g](int(x), int(y), int(z)) for g, x, y, z in zip(gates, a, b, c)])
    assert np.array_equal(client.decrypt_bits(sk, out, 1), exp)
