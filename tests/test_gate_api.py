"""The reference-facing gate API: the C++ shim (include/cufhe_gpu.hpp) and its
Python mirror (cufhepp_b200.gates), exercised the way the reference's
test/test_gate_gpu.cc and test/test_util.h:8-95 drive cuFHEpp."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from cufhepp_b200 import client, gates as G, params as P

ROOT = Path(__file__).resolve().parents[1]
LIB = ROOT / "cufhepp_b200" / "lib"


def build_cpp(tmp_path) -> Path:
    exe = tmp_path / "test_gate_gpu"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", str(ROOT / "include"), "-o", str(exe),
                    str(ROOT / "tests" / "cpp" / "test_gate_gpu.cc"), "-L", str(LIB),
                    "-lcufhe_b200", "-lcufhe_client", f"-Wl,-rpath,{LIB}"],
                   check=True, capture_output=True, text=True)
    return exe


def test_cpp_shim_compiles_and_links(tmp_path):
    assert build_cpp(tmp_path).exists()


@pytest.mark.gpu
def test_cpp_shim_all_gates_both_levels(tmp_path):
    exe = build_cpp(tmp_path)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL TESTS PASSED" in r.stdout


@pytest.mark.gpu
def test_python_mirror_of_the_gate_api(keys):
    sk, ek, _ = keys
    G.Initialize(ek)
    try:
        rng = np.random.default_rng(77)
        st = [G.Stream() for _ in range(4)]
        for s in st:
            s.Create()
        for level in (1, 0):
            n = 8
            pt = rng.integers(0, 2, 4 * n).astype(np.uint8)
            ct = [G.Ctxt(level) for _ in range(4 * n)]
            enc = client.encrypt_bits(sk, pt, level, seed=5 + level)
            for i in range(4 * n):
                ct[i].tlwehost[:] = enc[i]
            for i in range(n):
                s = st[i % 4]
                if i % 3 == 0:
                    G.Nand(ct[i], ct[i + n], ct[i + 2 * n], s)
                elif i % 3 == 1:
                    G.Mux(ct[i], ct[i + n], ct[i + 2 * n], ct[i + 3 * n], s)
                else:
                    G.Xor(ct[i], ct[i + n], ct[i + 2 * n], s)
            G.Synchronize()
            assert all(G.StreamQuery(s) for s in st)
            for i in range(n):
                a, b, c = int(pt[i + n]), int(pt[i + 2 * n]), int(pt[i + 3 * n])
                want = [1 - (a & b), a * b + (1 - a) * c, a ^ b][i % 3]
                got = client.decrypt_bits(sk, ct[i].tlwehost, level)[0]
                assert got == want, (level, i)
        for s in st:
            s.Destroy()
    finally:
        G.CleanUp()
