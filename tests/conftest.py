import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")
    config.addinivalue_line("markers", "slow: long-running check")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def keys():
    """Seeded secret keys and both bootstrapping-key forms."""
    from cufhepp_b200 import client
    sk = client.SecretKey.generate(0xC0FFEE)
    ek_kb = client.EvalKey.generate(sk, keybundle=True)
    ek_nokb = client.EvalKey.generate(sk, keybundle=False)
    return sk, ek_kb, ek_nokb
