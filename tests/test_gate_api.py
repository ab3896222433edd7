"""The reference-facing gate API: the C++ shim (include/cufhe_gpu.hpp) and its
Python mirror (cufhepp_b200.gates), exercised the way the reference's
test/test_gate_gpu.cc and test/test_util.h:8-95 drive cuFHEpp."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from cufhepp_b200 import client, engine, gates as G, params as P

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


class _View:
    """A Ctxt-shaped view of one row of a device table (the g* gates read only
    the level and the device pointer)."""

    def __init__(self, level, ptr):
        self.level = level
        self.tlwedevices = [engine.DeviceView(ptr)]


@pytest.mark.gpu
def test_intensive_chained_gates_polled_by_stream_query(keys):
    """The reference's intensive test (test/test_intensive.cc:23-134): 1000
    streams, each running a chain of 20 gates in which every gate's output is
    the next gate's input (NAND and MUX alternating), scheduled by a host loop
    that polls StreamQuery and issues a stream's next gate only when the
    stream is idle.  Every chain's last ciphertext decrypts to the chain's
    plaintext evaluation."""
    sk, ek, _ = keys
    streams_n, depth, level = 1000, 20, 1
    words = P.TLWE1_WORDS
    G.Initialize(ek)
    try:
        rng = np.random.default_rng(2024)
        x0 = rng.integers(0, 2, streams_n).astype(np.uint8)
        y = rng.integers(0, 2, (streams_n, depth)).astype(np.uint8)
        z = rng.integers(0, 2, (streams_n, depth)).astype(np.uint8)
        # operand table: rows [0, S) chain starts, then y and z of every step
        ops = np.concatenate([client.encrypt_bits(sk, x0, level, seed=1),
                              client.encrypt_bits(sk, y.ravel(), level, seed=2),
                              client.encrypt_bits(sk, z.ravel(), level, seed=3)])
        d_ops = engine.to_device(ops)
        d_acc = engine.DeviceBuffer(2 * streams_n * words * 4)  # ping-pong per stream
        row = lambda base, r: _View(level, base.ptr + r * words * 4)  # noqa: E731
        yrow = lambda i, k: row(d_ops, streams_n + i * depth + k)  # noqa: E731
        zrow = lambda i, k: row(d_ops, streams_n + streams_n * depth + i * depth + k)  # noqa: E731
        st = [G.Stream() for _ in range(streams_n)]
        for s in st:
            s.Create()
        step = [0] * streams_n
        while True:
            pending = [i for i in range(streams_n) if step[i] < depth]
            if not pending:
                break
            for i in pending:
                if not G.StreamQuery(st[i]):
                    continue
                k = step[i]
                src = row(d_ops, i) if k == 0 else row(d_acc, 2 * i + (k - 1) % 2)
                dst = row(d_acc, 2 * i + k % 2)
                if k % 2 == 0:
                    G.gNand(dst, src, yrow(i, k), st[i])
                else:
                    G.gMux(dst, yrow(i, k), src, zrow(i, k), st[i])
                step[i] += 1
        G.Synchronize()
        assert all(G.StreamQuery(s) for s in st)
        acc = engine.from_device(d_acc, (streams_n, 2, words))[:, (depth - 1) % 2]
        want = x0.astype(np.int64).copy()
        for k in range(depth):
            if k % 2 == 0:
                want = 1 - (want & y[:, k])
            else:
                want = np.where(y[:, k] == 1, want, z[:, k])
        assert np.array_equal(client.decrypt_bits(sk, acc, level), want.astype(np.uint8))
        for s in st:
            s.Destroy()
    finally:
        G.CleanUp()
