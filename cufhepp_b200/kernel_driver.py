"""Runs one engine stage on seeded synthetic inputs, for profilers.

    python -m cufhepp_b200.kernel_driver br_fp64 LANES [REPS]   # FP64 blind rotation (KeyBundle)
    python -m cufhepp_b200.kernel_driver br_fp64_plain LANES [REPS]  # the same, plain key
    python -m cufhepp_b200.kernel_driver br_int8 LANES [REPS] [STEPS]  # INT8 exact rotation
    python -m cufhepp_b200.kernel_driver br_int8_kb LANES [REPS] [STEPS]  # the same, KeyBundle key
    python -m cufhepp_b200.kernel_driver iks LANES [REPS]       # identity key switching
    python -m cufhepp_b200.kernel_driver gates LANES [REPS]     # full mixed-gate batch (lvl1)
    python -m cufhepp_b200.kernel_driver br2_fp64 LANES [REPS] [STEPS]  # lvl0 -> lvl2 rotation
    python -m cufhepp_b200.kernel_driver br2_int8 LANES [REPS] [STEPS]  # the same, INT8 exact
    python -m cufhepp_b200.kernel_driver br2_int8_kb LANES [REPS] [STEPS]  # INT8, KeyBundle key
    python -m cufhepp_b200.kernel_driver gates02 LANES [REPS]   # mixed *_lvl02 gate batch
    python -m cufhepp_b200.kernel_driver cb BITS [REPS]   # circuit bootstrapping + BITS/8 lookup tables

Each stage is launched REPS times on LANES inputs, so a capture can skip the
first (cold) launch.  Prints one line (with the wall time of the last REPS-1
launches) and exits 0.
"""
from __future__ import annotations

import sys
import time

import numpy as np

from . import client, engine, params as P


def main(argv: list[str]) -> None:
    stage = argv[0]
    lanes = int(argv[1])
    reps = int(argv[2]) if len(argv) > 2 else 2
    sk = client.SecretKey.generate(5)
    lvl02 = stage in ("br2_fp64", "br2_int8", "br2_int8_kb", "gates02", "cb")
    if stage == "cb":
        cbk = client.CBKey.generate(sk)
        engine.initialize_lvl02(cbk.ek02)
        engine.initialize_cb(cbk)
    elif lvl02:
        engine.initialize_lvl02(client.EvalKey02.generate(sk, keybundle=(stage != "br2_int8")))
    else:
        engine.initialize(client.EvalKey.generate(
            sk, keybundle=stage not in ("br_int8", "br_fp64_plain")))
    rng = np.random.default_rng(1)
    bits = rng.integers(0, 2, lanes).astype(np.uint8)
    t0 = None

    def tick(i):
        nonlocal t0
        if i == 0:
            engine.synchronize()
            t0 = time.perf_counter()

    if stage == "cb":
        q = max(1, lanes // 8)
        luts = rng.integers(0, 256, (q, 256)).astype(np.uint8)
        d_x = engine.to_device(client.encrypt_bits(sk, rng.integers(0, 2, 8 * q).astype(np.uint8),
                                                   0, seed=3))
        d_t = engine.DeviceBuffer(8 * q * 6 * P.TRLWE1_WORDS * 4)
        d_f = engine.DeviceBuffer(8 * q * 6 * 2 * 512 * 16)
        d_o = engine.DeviceBuffer(q * 8 * P.TLWE1_WORDS * 4)
        for i in range(reps):
            engine.circuit_bootstrap(d_x, 8 * q, d_t)
            engine.trgsw_to_fft(engine.GADGET_CB, d_t, 8 * q, d_f)
            engine.lut_eval(luts, d_f, P.MU32, d_o)
            tick(i)
    elif stage in ("br2_fp64", "br2_int8", "br2_int8_kb"):
        engine.set_precision(P.FP64_FFNT if stage == "br2_fp64" else P.INT8_EXACT)
        steps = int(argv[3]) if len(argv) > 3 else -1
        d_in = engine.to_device(client.encrypt_bits(sk, bits, 0, seed=3))
        d_out = engine.DeviceBuffer(lanes * P.TLWE2_WORDS * 8)
        for i in range(reps):
            engine.blind_rotate_lvl02(d_in, lanes, P.MU64, steps, tlwe_out=d_out)
            tick(i)
    elif stage == "gates02":
        gates = rng.choice([P.NAND, P.AND, P.OR, P.XOR, P.XNOR, P.MUX], size=lanes).astype(np.int32)
        cts = [engine.to_device(client.encrypt_bits(sk, bits, 0, seed=3 + i)) for i in range(3)]
        d_out = engine.DeviceBuffer(lanes * P.TLWE0_WORDS * 4)
        for i in range(reps):
            engine.gate_batch(gates, lanes, engine.LVL02, d_out, *cts)
            tick(i)
    elif stage in ("br_fp64", "br_fp64_plain", "br_int8", "br_int8_kb"):
        engine.set_precision(P.FP64_FFNT if stage.startswith("br_fp64") else P.INT8_EXACT)
        steps = int(argv[3]) if len(argv) > 3 else -1
        x = client.encrypt_bits(sk, bits, 0, seed=3)
        d_in = engine.to_device(x)
        d_out = engine.DeviceBuffer(lanes * P.TLWE1_WORDS * 4)
        for i in range(reps):
            engine.blind_rotate(d_in, lanes, P.MU32, steps, tlwe_out=d_out)
            tick(i)
    elif stage == "iks":
        x = client.encrypt_bits(sk, bits, 1, seed=3)
        d_in = engine.to_device(x)
        d_out = engine.DeviceBuffer(lanes * P.TLWE0_WORDS * 4)
        for i in range(reps):
            engine.identity_keyswitch(d_in, lanes, d_out)
            tick(i)
    elif stage == "gates":
        gates = rng.choice([P.NAND, P.AND, P.OR, P.XOR, P.XNOR, P.MUX], size=lanes).astype(np.int32)
        cts = [engine.to_device(client.encrypt_bits(sk, bits, 1, seed=3 + i)) for i in range(3)]
        d_out = engine.DeviceBuffer(lanes * P.TLWE1_WORDS * 4)
        for i in range(reps):
            engine.gate_batch(gates, lanes, 1, d_out, *cts)
            tick(i)
    else:
        raise SystemExit(f"unknown stage {stage}")
    engine.synchronize()
    ms = (time.perf_counter() - t0) * 1e3 / (reps - 1) if (t0 is not None and reps > 1) else 0.0
    if stage == "cb":
        engine.cleanup_cb()
    engine.cleanup_lvl02() if lvl02 else engine.cleanup()
    print(f"ok {stage} lanes={lanes} reps={reps} wall_ms_per_rep={ms:.3f}")


if __name__ == "__main__":
    main(sys.argv[1:])
