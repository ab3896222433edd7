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


@pytest.mark.gpu
def test_python_mirror_lvl02_gates():
    """Nand_lvl02 ... NMux_lvl02 on Ctxt<lvl0param> (test/test_gate_gpu_lvl02.cc)."""
    sk = client.SecretKey.generate(0xA11)
    G.Initialize_lvl02(client.EvalKey02.generate(sk, keybundle=True), sk)
    try:
        rng = np.random.default_rng(78)
        st = [G.Stream() for _ in range(3)]
        for s in st:
            s.Create()
        n = 12
        pt = rng.integers(0, 2, 4 * n).astype(np.uint8)
        ct = [G.Ctxt(0) for _ in range(4 * n)]
        enc = client.encrypt_bits(sk, pt, 0, seed=15)
        for i in range(4 * n):
            ct[i].tlwehost[:] = enc[i]
        ops = [(G.Nand_lvl02, lambda a, b, c: 1 - (a & b)), (G.Or_lvl02, lambda a, b, c: a | b),
               (G.AndYN_lvl02, lambda a, b, c: a & (1 - b)), (G.Xnor_lvl02, lambda a, b, c: 1 - (a ^ b)),
               (G.Mux_lvl02, lambda a, b, c: b if a else c), (G.NMux_lvl02, lambda a, b, c: 1 - (b if a else c))]
        for i in range(n):
            f = ops[i % len(ops)][0]
            if f in (G.Mux_lvl02, G.NMux_lvl02):
                f(ct[i], ct[i + n], ct[i + 2 * n], ct[i + 3 * n], st[i % 3])
            else:
                f(ct[i], ct[i + n], ct[i + 2 * n], st[i % 3])
        G.Synchronize()
        for i in range(n):
            a, b, c = int(pt[i + n]), int(pt[i + 2 * n]), int(pt[i + 3 * n])
            want = ops[i % len(ops)][1](a, b, c)
            assert client.decrypt_bits(sk, ct[i].tlwehost, 0)[0] == want, i
        for s in st:
            s.Destroy()
    finally:
        G.CleanUp_lvl02()
