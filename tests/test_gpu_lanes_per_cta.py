"""Every lanes-per-CTA form of the FP64 blind rotation gives the same bits.

k_br_fp64 carries 1, 2 or 4 lanes (gates) per CTA: CUFHE_BR_LANES_PER_CTA
forces one, otherwise the engine picks by batch size or from the
autotuner's table, and the headline batches run two.  Each form is run in a
child process with the variable set (the engine reads it once), on the same
seeded 601-lane batch, so that every form ends on a partly filled CTA.  The
per-bin arithmetic is the same in all forms (the same transforms, the same
order of the multiply-accumulate per bin and output), so after a full
rotation the accumulators must be bit-identical, for both key forms; the
two-lane form's first step is also within one Torus32 unit of the exact
product per coefficient (include/gatebootstrapping_gpu.cuh:69-221, :895-1033).
"""
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from cufhepp_b200 import client, params as P
from oracle import oracle as O

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
LANES = 601
SEED = 77

CHILD = r"""
import sys
import numpy as np
from cufhepp_b200 import client, engine, params as P
kb, steps, lanes, seed, out = sys.argv[1] == "kb", int(sys.argv[2]), int(sys.argv[3]), int(sys.argv[4]), sys.argv[5]
sk = client.SecretKey.generate(seed)
engine.initialize(client.EvalKey.generate(sk, keybundle=kb))
bits = np.random.default_rng(seed + 1).integers(0, 2, lanes).astype(np.uint8)
x = client.encrypt_bits(sk, bits, 0, seed=seed + 2)
d_in = engine.to_device(x)
d_acc = engine.DeviceBuffer(lanes * P.TRLWE1_WORDS * 4)
engine.blind_rotate(d_in, lanes, P.MU32, steps, acc_out=d_acc)
np.save(out, engine.from_device(d_acc, (lanes, P.TRLWE1_WORDS)))
engine.cleanup()
"""


def rotate_in_child(tmp_path, g, kb, steps):
    out = tmp_path / f"g{g}_{'kb' if kb else 'plain'}_{steps}.npy"
    env = dict(os.environ, CUFHE_BR_LANES_PER_CTA=str(g))
    env["PYTHONPATH"] = str(ROOT) + os.pathsep + env.get("PYTHONPATH", "")
    subprocess.run([sys.executable, "-c", CHILD, "kb" if kb else "plain", str(steps), str(LANES),
                    str(SEED), str(out)], env=env, cwd=ROOT, check=True, timeout=900)
    return np.load(out)


@pytest.mark.parametrize("kb", [True, False], ids=["kb", "plain"])
def test_lanes_per_cta_forms_bit_identical(tmp_path, kb):
    acc = {g: rotate_in_child(tmp_path, g, kb, -1) for g in (1, 2, 4)}
    assert np.array_equal(acc[1], acc[2])
    assert np.array_equal(acc[2], acc[4])
    # and the rotation is a real one: the b polynomial is +-mu times a monomial
    # up to the noise, not zeros or a copy of the test vector
    assert np.count_nonzero(acc[2]) > LANES * P.TRLWE1_WORDS // 2


@pytest.mark.parametrize("kb", [True, False], ids=["kb", "plain"])
def test_two_lane_form_one_step_against_exact(tmp_path, kb):
    got = rotate_in_child(tmp_path, 2, kb, 1)
    sk = client.SecretKey.generate(SEED)
    ek = client.EvalKey.generate(sk, keybundle=kb)
    bits = np.random.default_rng(SEED + 1).integers(0, 2, LANES).astype(np.uint8)
    x = client.encrypt_bits(sk, bits, 0, seed=SEED + 2)
    pick = np.array([0, 1, 2, 255, 256, 511, 599, 600])  # first, middle and last CTAs
    ref = O.blind_rotate(x[pick], P.MU32, ek.bk, kb, O.EXACT, steps=1)
    d = (got[pick].astype(np.int64) - ref.astype(np.int64)) % (1 << 32)
    d = np.minimum(d, (1 << 32) - d)
    assert d.max() <= 1, d.max()
