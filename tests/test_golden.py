"""Golden regression pins: the client library and the exact oracle reproduce the
committed digests (tests/golden/gates_exact.json, made by
tests/golden/make_gate_golden.py) on this machine."""
import json
import sys
from pathlib import Path

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))

import make_gate_golden as M  # noqa: E402


def test_client_and_oracle_match_golden_digests():
    want = json.loads((GOLDEN / "gates_exact.json").read_text())
    got = M.build()
    assert got["keys"] == want["keys"]
    for name, case in want["cases"].items():
        assert got["cases"][name] == case, name


def test_golden_decryptions_follow_truth_tables():
    import numpy as np
    from cufhepp_b200 import client, params as P
    want = json.loads((GOLDEN / "gates_exact.json").read_text())
    sk = client.SecretKey.generate(M.SEED)
    for level in (1, 0):
        bits, _ = M.inputs(sk, level)
        exp = [P.TRUTH[g](int(a), int(b), int(c)) for g, a, b, c in zip(M.GATES, *bits)]
        for tag in ("kb", "plain"):
            assert want["cases"][f"{tag}_lvl{level}"]["decrypted"] == exp
