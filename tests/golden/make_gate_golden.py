"""Regenerates tests/golden/gates_exact.json: SHA-256 digests of the exact
oracle's outputs for seeded keys and inputs (KeyBundle and plain keys, both
ciphertext levels, 12 gate ids), of its identity key switch and of a 3-step
blind rotation, plus digests of the seeded key material.

These pin the client library (key generation, encryption) and the exact
oracle across machines, and the INT8 engine path must reproduce the gate
digests bit for bit.  Run from the repository root:

    python tests/golden/make_gate_golden.py
"""
import hashlib
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from cufhepp_b200 import client, params as P  # noqa: E402
from oracle import oracle as O  # noqa: E402

SEED = 424242
GATES = [P.NAND, P.AND, P.OR, P.XOR, P.XNOR, P.MUX, P.NMUX, P.NOT, P.COPY, P.NOR, P.ANDYN,
         P.ORNY]


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def inputs(sk, level):
    rng = np.random.default_rng(SEED + level)
    bits = [rng.integers(0, 2, len(GATES)).astype(np.uint8) for _ in range(3)]
    cts = [client.encrypt_bits(sk, b, level, seed=SEED + 10 * level + i) for i, b in enumerate(bits)]
    return bits, cts


def build() -> dict:
    sk = client.SecretKey.generate(SEED)
    out = {"seed": SEED, "gates": GATES, "keys": {}, "cases": {}}
    for kb in (True, False):
        ek = client.EvalKey.generate(sk, keybundle=kb)
        tag = "kb" if kb else "plain"
        out["keys"][tag] = {"bk": digest(ek.bk), "ksk": digest(ek.ksk)}
        for level in (1, 0):
            bits, cts = inputs(sk, level)
            res = O.gate_batch(np.array(GATES, np.int32), level, *cts, ek.bk, ek.ksk, kb, O.EXACT)
            dec = client.decrypt_bits(sk, res, level)
            out["cases"][f"{tag}_lvl{level}"] = {
                "inputs": [digest(c) for c in cts], "outputs": digest(res),
                "decrypted": dec.tolist(), "first_words": res[0, :4].tolist()}
        x = client.encrypt_bits(sk, np.array([0, 1, 1, 0], np.uint8), 0, seed=SEED + 99)
        acc = O.blind_rotate(x, P.MU32, ek.bk, kb, O.EXACT, steps=3)
        out["cases"][f"{tag}_br3"] = {"outputs": digest(acc)}
    c1 = client.encrypt_bits(sk, np.arange(16, dtype=np.uint8) & 1, 1, seed=SEED + 7)
    ks = O.iks_batch(c1, None, 1, 0, 0, client.EvalKey.generate(sk, keybundle=False).ksk)
    out["cases"]["iks16"] = {"outputs": digest(ks)}
    return out


if __name__ == "__main__":
    data = build()
    path = Path(__file__).resolve().parent / "gates_exact.json"
    path.write_text(json.dumps(data, indent=1) + "\n")
    print("wrote", path)
