"""Client side of the gate API: seeded keys, encryption, decryption.

In the reference this role is TFHEpp's (``TFHEpp::SecretKey``,
``TFHEpp::EvalKey``, ``tlweSymEncrypt``/``tlweSymDecrypt``; see
test/test_gate_gpu.cc:50-58).  The arithmetic lives in
``csrc/client/tfhe_client.c``; this module wraps it with numpy arrays in the
TFHEpp layouts the engine consumes (``include/cufhe_b200.h``).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import params as P
from .build import LIB, build_client

_lib = None


def _load():
    global _lib
    if _lib is None:
        path = LIB / "libcufhe_client.so"
        if not path.exists():
            build_client()
        lib = C.CDLL(str(path))
        u64, u32, i32, dbl, vp, i = C.c_uint64, C.c_uint32, C.c_int32, C.c_double, C.c_void_p, C.c_int
        sigs = {
            "tfhe_keygen_binary": [u64, u64, u32, vp],
            "tfhe_tlwe32_encrypt_bits": [u64, u64, vp, u32, vp, u64, u32, dbl, vp],
            "tfhe_tlwe32_phase_batch": [vp, u32, vp, u64, vp],
            "tfhe_tlwe32_decrypt_bits": [vp, u32, vp, u64, vp],
            "tfhe_trlwe32_encrypt": [u64, u64, vp, u32, vp, dbl, vp],
            "tfhe_trlwe32_phase": [vp, u32, vp, vp],
            "tfhe_trgsw32_encrypt": [u64, u64, vp, u32, u32, u32, i32, dbl, vp],
            "tfhe_bk32_gen": [u64, vp, u32, vp, u32, u32, u32, dbl, i, vp],
            "tfhe_ksk32_gen": [u64, vp, u32, vp, u32, u32, u32, dbl, vp],
            "tfhe_bk64_gen": [u64, vp, u32, vp, u32, u32, u32, dbl, i, vp],
            "tfhe_trlwe64_phase": [vp, u32, vp, vp],
            "tfhe_privks_gen": [u64, vp, u32, vp, u32, u32, u32, dbl, i, vp],
        }
        for name, argt in sigs.items():
            fn = getattr(lib, name)
            fn.argtypes = argt
            fn.restype = None
        lib.tfhe_tlwe32_phase.restype = u32
        lib.tfhe_tlwe64_phase.argtypes = [vp, u32, vp]
        lib.tfhe_tlwe64_phase.restype = u64
        _lib = lib
    return _lib


def _p(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.c_void_p)


@dataclass
class SecretKey:
    """lvl0 (n = 636), lvl1 (N = 1024) and lvl2 (N = 2048) binary keys."""
    lvl0: np.ndarray  # int32 [636]
    lvl1: np.ndarray  # int32 [1024]
    seed: int
    lvl2: np.ndarray | None = None  # int32 [2048]

    @classmethod
    def generate(cls, seed: int) -> "SecretKey":
        lib = _load()
        k0 = np.empty(P.LVL0_N, np.int32)
        k1 = np.empty(P.LVL1_N, np.int32)
        k2 = np.empty(P.LVL2_N, np.int32)
        lib.tfhe_keygen_binary(seed, 0, P.LVL0_N, _p(k0))
        lib.tfhe_keygen_binary(seed, 1, P.LVL1_N, _p(k1))
        lib.tfhe_keygen_binary(seed, 2, P.LVL2_N, _p(k2))
        return cls(k0, k1, seed, k2)


@dataclass
class EvalKey:
    """Bootstrapping key (TRGSW[n0] or, with KeyBundle, TRGSW[n0/2][3]) and
    lvl1->lvl0 key-switching key, in TFHEpp layouts (uint32 words)."""
    bk: np.ndarray
    ksk: np.ndarray
    keybundle: bool

    @classmethod
    def generate(cls, sk: SecretKey, keybundle: bool = True, seed: int | None = None) -> "EvalKey":
        lib = _load()
        seed = sk.seed + 0x5EED if seed is None else seed
        bk = np.empty(P.BKKB_WORDS if keybundle else P.BK_WORDS, np.uint32)
        lib.tfhe_bk32_gen(seed, _p(sk.lvl0), P.LVL0_N, _p(sk.lvl1), P.LVL1_N, P.LVL1_L,
                          P.LVL1_BGBIT, P.LVL1_ALPHA, int(keybundle), _p(bk))
        ksk = np.empty(P.KSK_WORDS, np.uint32)
        lib.tfhe_ksk32_gen(seed + 1, _p(sk.lvl1), P.LVL1_N, _p(sk.lvl0), P.LVL0_N,
                           P.LVL10_BASEBIT, P.LVL10_T, P.LVL0_ALPHA, _p(ksk))
        return cls(bk, ksk, keybundle)


@dataclass
class EvalKey02:
    """lvl0 -> lvl2 bootstrapping key (Torus64 TRGSW<lvl2>[636], or [318][3]
    with KeyBundle) and lvl2 -> lvl0 key-switching key TLWE<lvl0>[2048][7][2]
    (the keys Initialize_lvl02 takes, src/cufhe_gates_gpu.cu:75-90)."""
    bk: np.ndarray   # uint64
    ksk: np.ndarray  # uint32
    keybundle: bool

    @classmethod
    def generate(cls, sk: SecretKey, keybundle: bool = True, seed: int | None = None) -> "EvalKey02":
        lib = _load()
        seed = sk.seed + 0x5EED02 if seed is None else seed
        bk = np.empty(P.BK2KB_WORDS if keybundle else P.BK2_WORDS, np.uint64)
        lib.tfhe_bk64_gen(seed, _p(sk.lvl0), P.LVL0_N, _p(sk.lvl2), P.LVL2_N, P.LVL2_L,
                          P.LVL2_BGBIT, P.LVL2_ALPHA, int(keybundle), _p(bk))
        ksk = np.empty(P.KSK20_WORDS, np.uint32)
        lib.tfhe_ksk32_gen(seed + 1, _p(sk.lvl2), P.LVL2_N, _p(sk.lvl0), P.LVL0_N,
                           P.LVL20_BASEBIT, P.LVL20_T, P.LVL0_ALPHA, _p(ksk))
        return cls(bk, ksk, keybundle)


def privks_key(key_src: np.ndarray, key1: np.ndarray, func: int, seed: int,
               basebit: int = 4, t: int = 10, alpha: float = P.LVL1_ALPHA) -> np.ndarray:
    """Private key-switching key TLWE<src> -> TRLWE<lvl1> for circuit
    bootstrapping: [n_src+1][t][2^basebit-1][2][N] uint32 encrypting
    f(k_i (u+1) 2^-(j+1)basebit), f(x) = -x s1 (func 0) or x (func 1)."""
    lib = _load()
    n_src = int(key_src.size)
    out = np.empty((n_src + 1) * t * ((1 << basebit) - 1) * 2 * P.LVL1_N, np.uint32)
    lib.tfhe_privks_gen(seed, _p(np.ascontiguousarray(key_src, np.int32)), n_src,
                        _p(np.ascontiguousarray(key1, np.int32)), P.LVL1_N, basebit, t, alpha,
                        func, _p(out))
    return out


@dataclass
class CBKey:
    """Keys of circuit bootstrapping lvl0 -> TRGSW<lvl1> (l = 3, Bgbit = 6): the
    lvl02 bootstrapping key (EvalKey02) and the two private key-switching keys
    lvl2 -> lvl1 (basebit 4, t 10) for the a-rows (f = -x s1) and b-rows (f = x)."""
    ek02: EvalKey02
    privks0: np.ndarray
    privks1: np.ndarray

    @classmethod
    def generate(cls, sk: SecretKey, seed: int | None = None, keybundle: bool = True,
                 ek02: EvalKey02 | None = None) -> "CBKey":
        seed = sk.seed + 0xCB if seed is None else seed
        ek02 = ek02 or EvalKey02.generate(sk, keybundle=keybundle)
        return cls(ek02, privks_key(sk.lvl2, sk.lvl1, 0, seed),
                   privks_key(sk.lvl2, sk.lvl1, 1, seed))


def trgsw_encrypt_g(sk: SecretKey, m: int, seed: int, stream: int, l: int, bgbit: int,
                    alpha: float = P.LVL1_ALPHA) -> np.ndarray:
    """TRGSW<lvl1>(m) with l digits of bgbit bits: [2l][2][N] uint32."""
    lib = _load()
    out = np.empty(2 * l * P.TRLWE1_WORDS, np.uint32)
    lib.tfhe_trgsw32_encrypt(seed, stream, _p(sk.lvl1), P.LVL1_N, l, bgbit, m, alpha, _p(out))
    return out


def trlwe64_phase(sk: SecretKey, c: np.ndarray) -> np.ndarray:
    lib = _load()
    c = np.ascontiguousarray(c, dtype=np.uint64)
    out = np.empty(P.LVL2_N, np.uint64)
    lib.tfhe_trlwe64_phase(_p(sk.lvl2), P.LVL2_N, _p(c), _p(out))
    return out


def tlwe64_phase(sk: SecretKey, c: np.ndarray) -> int:
    lib = _load()
    c = np.ascontiguousarray(c, dtype=np.uint64)
    return int(lib.tfhe_tlwe64_phase(_p(sk.lvl2), P.LVL2_N, _p(c)))


def encrypt_bits(sk: SecretKey, bits: np.ndarray, level: int, seed: int,
                 stream0: int = 0, alpha: float | None = None) -> np.ndarray:
    """TLWE encryptions of bits (+mu / -mu) at lvl0 or lvl1: [count][n+1]."""
    lib = _load()
    bits = np.ascontiguousarray(bits, dtype=np.uint8)
    n = P.LVL1_N if level == 1 else P.LVL0_N
    key = sk.lvl1 if level == 1 else sk.lvl0
    if alpha is None:
        alpha = P.LVL1_ALPHA if level == 1 else P.LVL0_ALPHA
    out = np.empty((bits.size, n + 1), np.uint32)
    lib.tfhe_tlwe32_encrypt_bits(seed, stream0, _p(key), n, _p(bits), bits.size, P.MU32,
                                 alpha, _p(out))
    return out


def phase(sk: SecretKey, ct: np.ndarray, level: int) -> np.ndarray:
    lib = _load()
    ct = np.ascontiguousarray(ct, dtype=np.uint32)
    n = P.LVL1_N if level == 1 else P.LVL0_N
    key = sk.lvl1 if level == 1 else sk.lvl0
    cnt = ct.size // (n + 1)
    out = np.empty(cnt, np.uint32)
    lib.tfhe_tlwe32_phase_batch(_p(key), n, _p(ct), cnt, _p(out))
    return out


def decrypt_bits(sk: SecretKey, ct: np.ndarray, level: int) -> np.ndarray:
    lib = _load()
    ct = np.ascontiguousarray(ct, dtype=np.uint32)
    n = P.LVL1_N if level == 1 else P.LVL0_N
    key = sk.lvl1 if level == 1 else sk.lvl0
    cnt = ct.size // (n + 1)
    out = np.empty(cnt, np.uint8)
    lib.tfhe_tlwe32_decrypt_bits(_p(key), n, _p(ct), cnt, _p(out))
    return out


def trlwe_phase(sk: SecretKey, c: np.ndarray) -> np.ndarray:
    lib = _load()
    c = np.ascontiguousarray(c, dtype=np.uint32)
    out = np.empty(P.LVL1_N, np.uint32)
    lib.tfhe_trlwe32_phase(_p(sk.lvl1), P.LVL1_N, _p(c), _p(out))
    return out


def trgsw_encrypt(sk: SecretKey, m: int, seed: int, stream: int = 0,
                  alpha: float = P.LVL1_ALPHA) -> np.ndarray:
    lib = _load()
    out = np.empty(P.TRGSW1_WORDS, np.uint32)
    lib.tfhe_trgsw32_encrypt(seed, stream, _p(sk.lvl1), P.LVL1_N, P.LVL1_L, P.LVL1_BGBIT, m,
                             alpha, _p(out))
    return out


def trlwe_encrypt(sk: SecretKey, msg: np.ndarray | None, seed: int, stream: int = 0,
                  alpha: float = P.LVL1_ALPHA) -> np.ndarray:
    lib = _load()
    out = np.empty(P.TRLWE1_WORDS, np.uint32)
    m = None if msg is None else np.ascontiguousarray(msg, dtype=np.uint32)
    lib.tfhe_trlwe32_encrypt(seed, stream, _p(sk.lvl1), P.LVL1_N,
                             None if m is None else _p(m), alpha, _p(out))
    return out
