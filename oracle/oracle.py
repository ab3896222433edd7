"""ORACLE -- test infrastructure only.

ctypes wrapper of ``oracle/tfhe_oracle.c``, the CPU restatement of
cuFHEpp's lvl1 gate-bootstrapping path (exact schoolbook and FP64 FFNT
forms).  Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline legs
of ``bench.py`` use it, as the checker; the engine never calls it.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIBPATH = HERE / "_build" / "liboracle.so"

EXACT = 0
FP64 = 1
N0, N, HALF = 636, 1024, 512
TLWE0, TLWE1, TRLWE, TRGSW = 637, 1025, 2048, 8192

_lib = None


def build(force: bool = False) -> Path:
    src = HERE / "tfhe_oracle.c"
    if force or not LIBPATH.exists() or LIBPATH.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-C", str(HERE), "-B" if force else "all"], check=True,
                       capture_output=True)
    return LIBPATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIBPATH))
        vp, i, i64, u32, i32 = C.c_void_p, C.c_int, C.c_int64, C.c_uint32, C.c_int32
        sig = {
            "orc_fft_create": ([], vp),
            "orc_fft_destroy": ([vp], None),
            "orc_bk_to_fft": ([vp, vp, i, vp], None),
            "orc_decompose": ([vp, vp], None),
            "orc_extprod_exact": ([vp, vp, vp], None),
            "orc_extprod_fp64": ([vp, vp, vp, vp, i], None),
            "orc_cmux_step_exact": ([vp, vp, u32], None),
            "orc_kb_step_exact": ([vp, vp, u32, u32], None),
            "orc_test_vector": ([u32, u32, vp], None),
            "orc_blind_rotate": ([vp, u32, vp, i, i, vp, i, vp], None),
            "orc_blind_rotate_batch": ([vp, vp, i64, vp, i, i, vp, i, vp], None),
            "orc_sample_extract": ([vp, vp], None),
            "orc_iks_preadd": ([vp, vp, i32, i32, u32, vp, vp], None),
            "orc_iks_batch": ([vp, vp, vp, vp, vp, vp, i64, vp], None),
            "orc_gate_batch": ([vp, i, vp, vp, vp, vp, i64, vp, vp, i, i, vp], None),
            "orc_ffnt_roundtrip": ([vp, vp, vp], None),
            "orc_ffnt_square": ([vp, vp, vp], None),
            "orc_negacyclic_mul_f64": ([vp, vp, vp], None),
            "orc_negacyclic_mul_exact": ([vp, vp, vp], None),
            "orc_fft2_create": ([], vp),
            "orc_fft2_destroy": ([vp], None),
            "orc2_bk_to_fft": ([vp, vp, i, vp], None),
            "orc2_decompose": ([vp, vp], None),
            "orc2_extprod_exact": ([vp, vp, vp], None),
            "orc2_cmux_step_exact": ([vp, vp, u32], None),
            "orc2_cmux_step_fp64": ([vp, vp, vp, u32], None),
            "orc2_blind_rotate_batch": ([vp, C.c_uint64, i64, vp, i, i, vp, i, vp], None),
            "orc2_sample_extract": ([vp, vp], None),
            "orc20_iks_batch": ([vp, vp, i64, vp], None),
            "orc2_gate_batch": ([vp, vp, vp, vp, vp, i64, vp, vp, i, i, vp], None),
            "orc2_ffnt_roundtrip": ([vp, vp, vp], None),
            "orc2_ffnt_square": ([vp, vp, vp], None),
            "orc_double_to_torus64": ([C.c_double], C.c_uint64),
            "orc_privks": ([vp, u32, vp, vp], None),
            "orc_privks_batch": ([vp, i64, u32, vp, vp], None),
            "orc_extprod_exact_g": ([vp, vp, i, i, vp], None),
            "orc_extprod_fp64_g": ([vp, vp, vp, i, i, vp], None),
            "orc_polys_to_fft": ([vp, vp, i64, vp], None),
            "orc_cmux_g": ([vp, vp, vp, i, i, i, vp, vp], None),
            "orc_cmux_batch_g": ([vp, vp, vp, i64, i, i, i, vp, vp], None),
            "orc_circuit_bootstrap_batch": ([vp, i64, vp, i, i, vp, vp, vp, vp], None),
            "orc_lut_eval_batch": ([vp, vp, i64, u32, i, i, i, vp, vp], None),
        }
        for name, (args, res) in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def _p(a):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays passed to the oracle must be contiguous"
    return a.ctypes.data_as(C.c_void_p)


class FFT:
    """FFNT tables (and the X^a - 1 table for KeyBundle), owned on the C side."""

    def __init__(self):
        self.h = lib().orc_fft_create()

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_fft_destroy(self.h)
            self.h = None


def u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def bk_to_fft(fft: FFT, bk: np.ndarray) -> np.ndarray:
    bk = u32(bk)
    ntrgsw = bk.size // TRGSW
    out = np.empty(ntrgsw * 8 * HALF, np.complex128)
    lib().orc_bk_to_fft(fft.h, _p(bk), ntrgsw, _p(out))
    return out


def decompose(poly) -> np.ndarray:
    out = np.empty((2, N), np.int32)
    lib().orc_decompose(_p(u32(poly)), _p(out))
    return out


def extprod_exact(trgsw, trlwe) -> np.ndarray:
    out = np.empty(TRLWE, np.uint32)
    lib().orc_extprod_exact(_p(u32(trgsw)), _p(u32(trlwe)), _p(out))
    return out


def extprod_fp64(fft: FFT, trgsw_f, trlwe) -> np.ndarray:
    out = np.empty(TRLWE, np.uint32)
    lib().orc_extprod_fp64(fft.h, _p(np.ascontiguousarray(trgsw_f, np.complex128)),
                           _p(u32(trlwe)), _p(out), 0)
    return out


def cmux_step_exact(acc, bk_i, abar: int) -> np.ndarray:
    acc = u32(acc).copy()
    lib().orc_cmux_step_exact(_p(acc), _p(u32(bk_i)), abar)
    return acc


def kb_step_exact(acc, bk3, a0: int, a1: int) -> np.ndarray:
    acc = u32(acc).copy()
    lib().orc_kb_step_exact(_p(acc), _p(u32(bk3)), a0, a1)
    return acc


def test_vector(bar: int, mu: int) -> np.ndarray:
    out = np.empty(TRLWE, np.uint32)
    lib().orc_test_vector(bar, mu, _p(out))
    return out


def blind_rotate(x, mu, bk, kb: bool, mode: int, fft: FFT | None = None,
                 steps: int = -1) -> np.ndarray:
    """Blind rotation of lvl0 TLWEs x [count][637] -> TRLWE accumulators."""
    x = u32(x).reshape(-1, TLWE0)
    cnt = x.shape[0]
    mu = np.broadcast_to(np.asarray(mu, np.uint32), (cnt,)).copy()
    bkp = u32(bk) if mode == EXACT else np.ascontiguousarray(bk, np.complex128)
    out = np.empty((cnt, TRLWE), np.uint32)
    lib().orc_blind_rotate_batch(_p(x), _p(mu), cnt, _p(bkp), int(kb), mode,
                                 fft.h if fft else None, steps, _p(out))
    return out


def sample_extract(acc) -> np.ndarray:
    out = np.empty(TLWE1, np.uint32)
    lib().orc_sample_extract(_p(u32(acc)), _p(out))
    return out


def iks_batch(in0, in1, ca, cb, off, ksk) -> np.ndarray:
    in0 = u32(in0).reshape(-1, TLWE1)
    cnt = in0.shape[0]
    in1 = None if in1 is None else u32(in1).reshape(-1, TLWE1)
    ca = np.broadcast_to(np.asarray(ca, np.int32), (cnt,)).copy()
    cb = np.broadcast_to(np.asarray(cb, np.int32), (cnt,)).copy()
    off = np.broadcast_to(np.asarray(off, np.uint32), (cnt,)).copy()
    out = np.empty((cnt, TLWE0), np.uint32)
    lib().orc_iks_batch(_p(in0), _p(in1), _p(ca), _p(cb), _p(off), _p(u32(ksk)), cnt, _p(out))
    return out


def gate_batch(gates, level: int, in0, in1, in2, bk, ksk, kb: bool, mode: int,
               fft: FFT | None = None) -> np.ndarray:
    words = TLWE1 if level == 1 else TLWE0
    gates = np.ascontiguousarray(gates, np.int32)
    cnt = gates.size
    in0 = u32(in0).reshape(cnt, words)
    in1 = None if in1 is None else u32(in1).reshape(cnt, words)
    in2 = None if in2 is None else u32(in2).reshape(cnt, words)
    bkp = u32(bk) if mode == EXACT else np.ascontiguousarray(bk, np.complex128)
    out = np.empty((cnt, words), np.uint32)
    lib().orc_gate_batch(_p(gates), level, _p(in0), _p(in1), _p(in2), _p(out), cnt, _p(bkp),
                         _p(u32(ksk)), int(kb), mode, fft.h if fft else None)
    return out


def ffnt_roundtrip(fft: FFT, x) -> np.ndarray:
    x = np.ascontiguousarray(x, np.float64)
    out = np.empty(N, np.float64)
    lib().orc_ffnt_roundtrip(fft.h, _p(x), _p(out))
    return out


def ffnt_square(fft: FFT, x) -> np.ndarray:
    x = np.ascontiguousarray(x, np.float64)
    out = np.empty(N, np.float64)
    lib().orc_ffnt_square(fft.h, _p(x), _p(out))
    return out


def negacyclic_mul_f64(a, b) -> np.ndarray:
    out = np.empty(N, np.float64)
    lib().orc_negacyclic_mul_f64(_p(np.ascontiguousarray(a, np.float64)),
                                 _p(np.ascontiguousarray(b, np.float64)), _p(out))
    return out


def negacyclic_mul_exact(d, key) -> np.ndarray:
    out = np.empty(N, np.uint32)
    lib().orc_negacyclic_mul_exact(_p(np.ascontiguousarray(d, np.int32)), _p(u32(key)), _p(out))
    return out


# ------------------------------------------------ lvl0 -> lvl2 (Torus64) ---
N2, HALF2, TRLWE2, TRGSW2, TLWE2 = 2048, 1024, 4096, 8 * 4096, 2049


class FFT2:
    """FFNT tables for N = 2048 (1024-point transform)."""

    def __init__(self):
        self.h = lib().orc_fft2_create()

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_fft2_destroy(self.h)
            self.h = None


def u64(a):
    return np.ascontiguousarray(a, dtype=np.uint64)


def bk2_to_fft(fft: FFT2, bk) -> np.ndarray:
    bk = u64(bk)
    ntrgsw = bk.size // TRGSW2
    out = np.empty(ntrgsw * 16 * HALF2, np.complex128)
    lib().orc2_bk_to_fft(fft.h, _p(bk), ntrgsw, _p(out))
    return out


def decompose2(poly) -> np.ndarray:
    out = np.empty((4, N2), np.int32)
    lib().orc2_decompose(_p(u64(poly)), _p(out))
    return out


def extprod2_exact(trgsw, trlwe) -> np.ndarray:
    out = np.empty(TRLWE2, np.uint64)
    lib().orc2_extprod_exact(_p(u64(trgsw)), _p(u64(trlwe)), _p(out))
    return out


def cmux2_step_exact(acc, bk_i, abar: int) -> np.ndarray:
    acc = u64(acc).copy()
    lib().orc2_cmux_step_exact(_p(acc), _p(u64(bk_i)), abar)
    return acc


def cmux2_step_fp64(fft: FFT2, acc, bkf_i, abar: int) -> np.ndarray:
    acc = u64(acc).copy()
    lib().orc2_cmux_step_fp64(fft.h, _p(acc), _p(np.ascontiguousarray(bkf_i, np.complex128)), abar)
    return acc


def blind_rotate2(x, mu: int, bk, kb: bool, mode: int, fft: FFT2 | None = None,
                  steps: int = -1) -> np.ndarray:
    x = u32(x).reshape(-1, TLWE0)
    cnt = x.shape[0]
    bkp = u64(bk) if mode == EXACT else np.ascontiguousarray(bk, np.complex128)
    out = np.empty((cnt, TRLWE2), np.uint64)
    lib().orc2_blind_rotate_batch(_p(x), mu, cnt, _p(bkp), int(kb), mode, fft.h if fft else None,
                                  steps, _p(out))
    return out


def sample_extract2(acc) -> np.ndarray:
    out = np.empty(TLWE2, np.uint64)
    lib().orc2_sample_extract(_p(u64(acc)), _p(out))
    return out


def iks20_batch(tlwe2, ksk) -> np.ndarray:
    tlwe2 = u64(tlwe2).reshape(-1, TLWE2)
    out = np.empty((tlwe2.shape[0], TLWE0), np.uint32)
    lib().orc20_iks_batch(_p(tlwe2), _p(u32(ksk)), tlwe2.shape[0], _p(out))
    return out


def gate2_batch(gates, in0, in1, in2, bk, ksk, kb: bool, mode: int,
                fft: FFT2 | None = None) -> np.ndarray:
    gates = np.ascontiguousarray(gates, np.int32)
    cnt = gates.size
    in0 = u32(in0).reshape(cnt, TLWE0)
    in1 = None if in1 is None else u32(in1).reshape(cnt, TLWE0)
    in2 = None if in2 is None else u32(in2).reshape(cnt, TLWE0)
    bkp = u64(bk) if mode == EXACT else np.ascontiguousarray(bk, np.complex128)
    out = np.empty((cnt, TLWE0), np.uint32)
    lib().orc2_gate_batch(_p(gates), _p(in0), _p(in1), _p(in2), _p(out), cnt, _p(bkp),
                          _p(u32(ksk)), int(kb), mode, fft.h if fft else None)
    return out


def ffnt2_roundtrip(fft: FFT2, x) -> np.ndarray:
    out = np.empty(N2, np.float64)
    lib().orc2_ffnt_roundtrip(fft.h, _p(np.ascontiguousarray(x, np.float64)), _p(out))
    return out


def ffnt2_square(fft: FFT2, x) -> np.ndarray:
    out = np.empty(N2, np.float64)
    lib().orc2_ffnt_square(fft.h, _p(np.ascontiguousarray(x, np.float64)), _p(out))
    return out


def double_to_torus64(d: float) -> int:
    return int(lib().orc_double_to_torus64(d))


# ------------------------------- circuit bootstrapping and CMUX lookup tables ---
CB_L, CB_BGBIT = 3, 6
PKS_BASEBIT, PKS_T, PKS_NU = 4, 10, 15


def privks(tlwe2, key, n_src: int = N2) -> np.ndarray:
    """Exact private key switching of Torus64 TLWEs [count][n_src+1] -> TRLWE<lvl1>."""
    t = u64(tlwe2).reshape(-1, n_src + 1)
    out = np.empty((t.shape[0], TRLWE), np.uint32)
    lib().orc_privks_batch(_p(t), t.shape[0], n_src, _p(u32(key)), _p(out))
    return out


def extprod_g(trgsw, trlwe, L: int, bgbit: int, mode: int, fft: FFT | None = None) -> np.ndarray:
    out = np.empty(TRLWE, np.uint32)
    if mode == EXACT:
        lib().orc_extprod_exact_g(_p(u32(trgsw)), _p(u32(trlwe)), L, bgbit, _p(out))
    else:
        lib().orc_extprod_fp64_g(fft.h, _p(np.ascontiguousarray(trgsw, np.complex128)),
                                 _p(u32(trlwe)), L, bgbit, _p(out))
    return out


def polys_to_fft(fft: FFT, polys) -> np.ndarray:
    polys = u32(polys)
    n = polys.size // N
    out = np.empty(n * HALF, np.complex128)
    lib().orc_polys_to_fft(fft.h, _p(polys), n, _p(out))
    return out


def cmux_batch(trgsw, d1, d0, L: int, bgbit: int, mode: int, fft: FFT | None = None) -> np.ndarray:
    """out[i] = d0[i] + ExtProd(trgsw[i], d1[i] - d0[i]); trgsw raw (EXACT) or Fourier (FP64)."""
    d1 = u32(d1).reshape(-1, TRLWE)
    d0 = u32(d0).reshape(-1, TRLWE)
    t = u32(trgsw) if mode == EXACT else np.ascontiguousarray(trgsw, np.complex128)
    out = np.empty_like(d1)
    lib().orc_cmux_batch_g(_p(t), _p(d1), _p(d0), d1.shape[0], L, bgbit, mode,
                           fft.h if fft else None, _p(out))
    return out


def circuit_bootstrap(x, bk2, kb: bool, mode: int, fft2: FFT2 | None, privks0, privks1) -> np.ndarray:
    """lvl0 TLWEs [count][637] -> TRGSW<lvl1> (l = 3, Bgbit = 6) [count][6][2048]."""
    x = u32(x).reshape(-1, TLWE0)
    bkp = u64(bk2) if mode == EXACT else np.ascontiguousarray(bk2, np.complex128)
    out = np.empty((x.shape[0], 2 * CB_L, TRLWE), np.uint32)
    lib().orc_circuit_bootstrap_batch(_p(x), x.shape[0], _p(bkp), int(kb), mode,
                                      fft2.h if fft2 else None, _p(u32(privks0)),
                                      _p(u32(privks1)), _p(out))
    return out


def lut_eval(trgsw, luts, mu: int, mode: int, fft: FFT | None = None, L: int = CB_L,
             bgbit: int = CB_BGBIT) -> np.ndarray:
    """CMUX-tree lookup tables: luts uint8 [count][256]; trgsw [count][8] TRGSWs
    (raw for EXACT, Fourier for FP64) -> TLWE<lvl1> [count][8][1025]."""
    luts = np.ascontiguousarray(luts, np.uint8).reshape(-1, 256)
    t = u32(trgsw) if mode == EXACT else np.ascontiguousarray(trgsw, np.complex128)
    out = np.empty((luts.shape[0], 8, TLWE1), np.uint32)
    lib().orc_lut_eval_batch(_p(t), _p(luts), luts.shape[0], mu, L, bgbit, mode,
                             fft.h if fft else None, _p(out))
    return out

