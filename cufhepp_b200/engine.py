"""ctypes binding of the engine's C-ABI (``include/cufhe_b200.h``).

Loads the in-tree ``lib/libcufhe_b200.so`` and raises if it is missing or
fails to load: there is no CPU fallback for any engine operation.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import params as P
from .build import LIB

OK = 0
ERR = {-1: "CUFHE_ERR_ARG", -2: "CUFHE_ERR_STATE", -3: "CUFHE_ERR_CUDA", -4: "CUFHE_ERR_NOMEM",
       -5: "CUFHE_ERR_UNSUPPORTED"}

LVL0, LVL1, LVL02 = 0, 1, 2

# every symbol include/cufhe_b200.h declares: (argtypes, restype)
_vp, _sz, _i, _u32, _u64 = C.c_void_p, C.c_size_t, C.c_int, C.c_uint32, C.c_uint64
SIGNATURES = {
    "cufhe_set_gpu_num": ([_i], _i),
    "cufhe_get_gpu_num": ([], _i),
    "cufhe_initialize": ([_vp], _i),
    "cufhe_cleanup": ([], _i),
    "cufhe_synchronize": ([], _i),
    "cufhe_set_precision": ([_i], _i),
    "cufhe_get_precision": ([], _i),
    "cufhe_stream_create": ([_vp, _i], _i),
    "cufhe_stream_destroy": ([_vp], _i),
    "cufhe_stream_query": ([_vp], _i),
    "cufhe_stream_device": ([_vp], _i),
    "cufhe_stream_synchronize": ([_vp], _i),
    "cufhe_stream_cuda": ([_vp, _vp], _i),
    "cufhe_ctxt_alloc": ([_vp, _sz, _i], _i),
    "cufhe_ctxt_free": ([_vp, _i], _i),
    "cufhe_host_register": ([_vp, _sz], _i),
    "cufhe_host_unregister": ([_vp], _i),
    "cufhe_memcpy_h2d": ([_vp, _vp, _sz, _vp], _i),
    "cufhe_memcpy_d2h": ([_vp, _vp, _sz, _vp], _i),
    "cufhe_gate": ([_i, _i, _vp, _vp, _vp, _vp, _vp], _i),
    "cufhe_gate_copy": ([_i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp], _i),
    "cufhe_gate_batch": ([_vp, _i, _sz, _i, _vp, _vp, _vp, _vp, _vp], _i),
    "cufhe_gate_batch_host": ([_vp, _i, _sz, _i, _vp, _vp, _vp, _vp, _vp], _i),
    "cufhe_gate_batch_noalloc": ([_i, _sz, _i, _vp, _vp, _vp, _vp, _vp], _i),
    "cufhe_blind_rotate": ([_vp, _sz, _u32, _i, _vp, _vp, _vp], _i),
    "cufhe_identity_keyswitch": ([_vp, _sz, _vp, _vp], _i),
    "cufhe_last_error": ([], C.c_char_p),
    "cufhe_kernel_launches": ([], _u64),
    "cufhe_device_ok": ([], _i),
    "cufhe_profile_enable": ([_i], _i),
    "cufhe_profile_reset": ([], _i),
    "cufhe_profile_read": ([_i, _vp, _vp], _i),
    "cufhe_measure_fp64_peak": ([_vp], _i),
    "cufhe_measure_int8_peak": ([_vp], _i),
    "cufhe_selftest_wait_timeout": ([], _i),
    "cufhe_initialize_lvl02": ([_vp], _i),
    "cufhe_cleanup_lvl02": ([], _i),
    "cufhe_blind_rotate_lvl02": ([_vp, _sz, _u64, _i, _vp, _vp, _vp], _i),
    "cufhe_identity_keyswitch_lvl20": ([_vp, _sz, _vp, _vp], _i),
    "cufhe_circuit_create": ([_vp, _i, _sz, _sz, _vp, _vp, _vp, _vp, _vp, _i], _i),
    "cufhe_circuit_plan": ([_i, _sz, _sz, _vp, _vp, _vp, _vp, _vp, _i, _vp, _vp], _i),
    "cufhe_circuit_info": ([_vp, _vp, _vp, _vp], _i),
    "cufhe_circuit_wave_sizes": ([_vp, _vp, _vp, _sz], _i),
    "cufhe_circuit_run": ([_vp, _vp, _vp, _i], _i),
    "cufhe_circuit_destroy": ([_vp], _i),
    "cufhe_circuit_create_split": ([_vp, _i, _sz, _sz, _vp, _vp, _vp, _vp, _vp, _i, _i], _i),
    "cufhe_circuit_split_plan": ([_i, _sz, _sz, _vp, _vp, _vp, _vp, _vp, _i, _vp], _i),
    "cufhe_autotune": ([], _i),
    "cufhe_initialize_cb": ([_vp], _i),
    "cufhe_cleanup_cb": ([], _i),
    "cufhe_private_keyswitch": ([_vp, _sz, _i, _vp, _vp], _i),
    "cufhe_circuit_bootstrap": ([_vp, _sz, _vp, _vp], _i),
    "cufhe_trgsw_to_fft": ([_i, _vp, _sz, _vp, _vp], _i),
    "cufhe_cmux": ([_i, _vp, _vp, _vp, _vp, _sz, _vp], _i),
    "cufhe_lut_eval": ([_vp, _sz, _vp, _u32, _vp, _vp], _i),
    "cufhe_autotune_table": ([_vp, _vp, _i], _i),
    "cufhe_batch_shard_plan": ([_vp, _i, _sz, _i, _vp], _i),
    "cufhe_gate_batch_sharded_host": ([_vp, _i, _sz, _i, _vp, _vp, _vp, _vp, _i], _i),
    "cufhe_circuit_shard_plan": ([_i, _sz, _sz, _vp, _vp, _vp, _vp, _vp, _i, _i, _vp, _vp, _vp,
                                  _vp], _i),
    "cufhe_sharded_create": ([_vp, _i, _sz, _sz, _vp, _vp, _vp, _vp, _vp, _i], _i),
    "cufhe_sharded_info": ([_vp, _vp, _vp, _vp], _i),
    "cufhe_sharded_device": ([_vp, _i], _i),
    "cufhe_sharded_run": ([_vp, _vp], _i),
    "cufhe_sharded_collect": ([_vp, _vp, _i], _i),
    "cufhe_sharded_synchronize": ([_vp], _i),
    "cufhe_sharded_destroy": ([_vp], _i),
}

(K_IKS, K_PREADD, K_BR_FP64, K_BR_INT8, K_FINALIZE, K_BR_FP64_LVL02, K_IKS_LVL20, K_PRIVKS,
 K_CMUX) = range(9)
K_NAMES = ["iks", "preadd", "br_fp64", "br_int8", "finalize", "br_fp64_lvl02", "iks_lvl20",
           "privks", "cmux", "br_int8_lvl02"]
GADGET_LVL1, GADGET_CB = 0, 1


class KeyView(C.Structure):
    _fields_ = [("bk", _vp), ("bk_words", _sz), ("ksk", _vp), ("ksk_words", _sz),
                ("keybundle", _i)]


class CBKeyView(C.Structure):
    _fields_ = [("privks0", _vp), ("privks1", _vp), ("words", _sz)]


class CufheError(RuntimeError):
    pass


_lib = None


def lib_path() -> Path:
    return LIB / "libcufhe_b200.so"


def load():
    """Load the engine library (never falls back to anything else)."""
    global _lib
    if _lib is None:
        path = lib_path()
        if not path.exists():
            raise CufheError(f"engine library {path} is not built; run "
                             "`python -m cufhepp_b200.build` (nvcc, sm_100a)")
        L = C.CDLL(str(path))
        for name, (args, res) in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def check(rc: int, what: str = "") -> None:
    if rc != OK:
        msg = load().cufhe_last_error().decode()
        raise CufheError(f"{what}: {ERR.get(rc, rc)}: {msg}")


def _p(a):
    if a is None:
        return None
    if isinstance(a, DeviceBuffer):
        return C.c_void_p(a.ptr)
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.c_void_p)


class DeviceBuffer:
    """A device allocation made through cufhe_ctxt_alloc."""

    def __init__(self, nbytes: int, device: int = 0):
        p = C.c_void_p()
        check(load().cufhe_ctxt_alloc(C.byref(p), max(int(nbytes), 4), device), "ctxt_alloc")
        self.ptr = p.value
        self.nbytes = int(nbytes)
        self.device = device

    def offset(self, nbytes: int) -> "DeviceView":
        return DeviceView(self.ptr + nbytes)

    def upload(self, a: np.ndarray, stream=None) -> None:
        a = np.ascontiguousarray(a)
        assert a.nbytes <= self.nbytes
        check(load().cufhe_memcpy_h2d(C.c_void_p(self.ptr), _p(a), a.nbytes, stream), "h2d")

    def download(self, a: np.ndarray, stream=None) -> np.ndarray:
        assert a.flags["C_CONTIGUOUS"] and a.nbytes <= self.nbytes
        check(load().cufhe_memcpy_d2h(_p(a), C.c_void_p(self.ptr), a.nbytes, stream), "d2h")
        return a

    def free(self):
        if self.ptr:
            load().cufhe_ctxt_free(C.c_void_p(self.ptr), self.device)
            self.ptr = 0

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class DeviceView:
    def __init__(self, ptr: int):
        self.ptr = ptr


def to_device(a: np.ndarray, device: int = 0) -> DeviceBuffer:
    a = np.ascontiguousarray(a)
    d = DeviceBuffer(a.nbytes, device)
    d.upload(a)
    check(load().cufhe_synchronize(), "sync")
    return d


def from_device(d: DeviceBuffer, shape, dtype=np.uint32) -> np.ndarray:
    out = np.empty(shape, dtype)
    d.download(out)
    check(load().cufhe_synchronize(), "sync")
    return out


def dptr(x):
    if x is None:
        return None
    if isinstance(x, (DeviceBuffer, DeviceView)):
        return C.c_void_p(x.ptr)
    if isinstance(x, int):
        return C.c_void_p(x)
    # torch tensors and anything exposing data_ptr()
    return C.c_void_p(x.data_ptr())


def initialize(ek, gpus: int | None = None) -> None:
    L = load()
    if gpus is not None:
        check(L.cufhe_set_gpu_num(gpus), "set_gpu_num")
    bk = np.ascontiguousarray(ek.bk, np.uint32)
    ksk = np.ascontiguousarray(ek.ksk, np.uint32)
    kv = KeyView(bk.ctypes.data, bk.size, ksk.ctypes.data, ksk.size, int(ek.keybundle))
    check(L.cufhe_initialize(C.byref(kv)), "initialize")


def cleanup() -> None:
    check(load().cufhe_cleanup(), "cleanup")


def initialize_lvl02(ek02, gpus: int | None = None) -> None:
    """Initialize_lvl02: uploads a client.EvalKey02 (uint64 BK<lvl2>, lvl20 KSK)."""
    L = load()
    if gpus is not None:
        check(L.cufhe_set_gpu_num(gpus), "set_gpu_num")
    bk = np.ascontiguousarray(ek02.bk, np.uint64)
    ksk = np.ascontiguousarray(ek02.ksk, np.uint32)
    kv = KeyView(bk.ctypes.data, bk.size, ksk.ctypes.data, ksk.size, int(ek02.keybundle))
    check(L.cufhe_initialize_lvl02(C.byref(kv)), "initialize_lvl02")


def cleanup_lvl02() -> None:
    check(load().cufhe_cleanup_lvl02(), "cleanup_lvl02")


def initialize_cb(cbkey) -> None:
    """Circuit bootstrapping: lvl02 keys (if not yet initialised by the caller
    use initialize_lvl02(cbkey.ek02) first) and the private key-switching keys."""
    k0 = np.ascontiguousarray(cbkey.privks0, np.uint32)
    k1 = np.ascontiguousarray(cbkey.privks1, np.uint32)
    assert k0.size == k1.size
    kv = CBKeyView(k0.ctypes.data, k1.ctypes.data, k0.size)
    check(load().cufhe_initialize_cb(C.byref(kv)), "initialize_cb")


def cleanup_cb() -> None:
    check(load().cufhe_cleanup_cb(), "cleanup_cb")


def private_keyswitch(tlwe2, count: int, func: int, out, stream=None) -> None:
    check(load().cufhe_private_keyswitch(dptr(tlwe2), count, func, dptr(out), stream),
          "private_keyswitch")


def circuit_bootstrap(tlwe0, count: int, trgsw_out, stream=None) -> None:
    check(load().cufhe_circuit_bootstrap(dptr(tlwe0), count, dptr(trgsw_out), stream),
          "circuit_bootstrap")


def trgsw_to_fft(gadget: int, trgsw, count: int, out, stream=None) -> None:
    check(load().cufhe_trgsw_to_fft(gadget, dptr(trgsw), count, dptr(out), stream),
          "trgsw_to_fft")


def cmux(gadget: int, trgsw_fft, d1, d0, out, count: int, stream=None) -> None:
    check(load().cufhe_cmux(gadget, dptr(trgsw_fft), dptr(d1), dptr(d0), dptr(out), count,
                            stream), "cmux")


def lut_eval(luts: np.ndarray, trgsw_fft, mu: int, out, stream=None) -> None:
    luts = np.ascontiguousarray(luts, np.uint8).reshape(-1, 256)
    check(load().cufhe_lut_eval(_p(luts), luts.shape[0], dptr(trgsw_fft), mu, dptr(out), stream),
          "lut_eval")


def synchronize() -> None:
    check(load().cufhe_synchronize(), "synchronize")


def set_precision(form: int) -> None:
    check(load().cufhe_set_precision(form), "set_precision")


def get_precision() -> int:
    return int(load().cufhe_get_precision())


def gate_batch(gates, count: int, level: int, out, in0, in1=None, in2=None, stream=None,
               uniform: int = 0) -> None:
    g = None
    if gates is not None:
        g = np.ascontiguousarray(gates, np.int32)
        assert g.size == count
    check(load().cufhe_gate_batch(_p(g), uniform, count, level, dptr(out), dptr(in0), dptr(in1),
                                  dptr(in2), stream), "gate_batch")


def gate_batch_host(gates, level: int, in0: np.ndarray, in1=None, in2=None, stream=None,
                    uniform: int = 0, out: np.ndarray | None = None) -> np.ndarray:
    words = P.TLWE1_WORDS if level == LVL1 else P.TLWE0_WORDS
    in0 = np.ascontiguousarray(in0, np.uint32).reshape(-1, words)
    count = in0.shape[0]
    if out is None:
        out = np.empty((count, words), np.uint32)
    g = None if gates is None else np.ascontiguousarray(gates, np.int32)
    i1 = None if in1 is None else np.ascontiguousarray(in1, np.uint32)
    i2 = None if in2 is None else np.ascontiguousarray(in2, np.uint32)
    check(load().cufhe_gate_batch_host(_p(g), uniform, count, level, _p(out), _p(in0), _p(i1),
                                       _p(i2), stream), "gate_batch_host")
    return out


def blind_rotate(tlwe0, count: int, mu: int, steps: int, acc_out=None, tlwe_out=None,
                 stream=None) -> None:
    check(load().cufhe_blind_rotate(dptr(tlwe0), count, mu, steps, dptr(acc_out),
                                    dptr(tlwe_out), stream), "blind_rotate")


def blind_rotate_lvl02(tlwe0, count: int, mu: int, steps: int, acc_out=None, tlwe_out=None,
                       stream=None) -> None:
    check(load().cufhe_blind_rotate_lvl02(dptr(tlwe0), count, mu, steps, dptr(acc_out),
                                          dptr(tlwe_out), stream), "blind_rotate_lvl02")


def identity_keyswitch_lvl20(tlwe2, count: int, out, stream=None) -> None:
    check(load().cufhe_identity_keyswitch_lvl20(dptr(tlwe2), count, dptr(out), stream),
          "identity_keyswitch_lvl20")


def identity_keyswitch(tlwe1, count: int, out, stream=None) -> None:
    check(load().cufhe_identity_keyswitch(dptr(tlwe1), count, dptr(out), stream),
          "identity_keyswitch")


def circuit_plan(level: int, num_wires: int, ops, in0, in1, in2, out, sms: int = 0):
    """cufhe_circuit_plan: validation, levelisation into waves and balancing on
    the host (no GPU, no keys).  Returns (wave of every gate, number of waves)."""
    ops = np.ascontiguousarray(ops, np.int32)
    arrs = [np.ascontiguousarray(x, np.int32) for x in (in0, in1, in2, out)]
    wave = np.empty(ops.size, np.int32)
    n = C.c_int()
    check(load().cufhe_circuit_plan(level, num_wires, ops.size, _p(ops), *(_p(a) for a in arrs),
                                    sms, _p(wave), C.byref(n)), "circuit_plan")
    return wave, n.value


def circuit_split_plan(level: int, num_wires: int, ops, in0, in1, in2, out, parts: int):
    """cufhe_circuit_split_plan: the group of every gate when the circuit's
    connected components are packed into up to `parts` groups (host only).
    Returns (group of every gate, number of groups)."""
    ops = np.ascontiguousarray(ops, np.int32)
    arrs = [np.ascontiguousarray(x, np.int32) for x in (in0, in1, in2, out)]
    group = np.empty(ops.size, np.int32)
    n = load().cufhe_circuit_split_plan(level, num_wires, ops.size, _p(ops),
                                        *(_p(a) for a in arrs), parts, _p(group))
    check(min(n, 0), "circuit_split_plan")
    return group, n


class Circuit:
    """A DAG of gates over a wire table, levelised into waves by the engine
    (cufhe_circuit_create).  ops/in0/in1/in2/out are per-gate arrays of gate
    ids and wire indices (-1 for an operand the gate does not take).  With
    parts > 1 its connected components are packed into up to `parts` groups
    run concurrently on streams of their own (cufhe_circuit_create_split)."""

    def __init__(self, level: int, num_wires: int, ops, in0, in1, in2, out, device: int = 0,
                 parts: int = 1):
        arr = lambda a: np.ascontiguousarray(a, np.int32)  # noqa: E731
        self.ops, self.in0, self.in1, self.in2, self.out = (arr(x) for x in (ops, in0, in1, in2,
                                                                            out))
        self.level = level
        self.num_wires = int(num_wires)
        self.words = P.TLWE1_WORDS if level == LVL1 else P.TLWE0_WORDS
        h = C.c_void_p()
        check(load().cufhe_circuit_create_split(C.byref(h), level, self.num_wires, self.ops.size,
                                                _p(self.ops), _p(self.in0), _p(self.in1),
                                                _p(self.in2), _p(self.out), device, parts),
              "circuit_create")
        self.h = h

    def info(self) -> tuple[int, int, int]:
        w, g, l = C.c_int(), C.c_int(), C.c_int()
        check(load().cufhe_circuit_info(self.h, C.byref(w), C.byref(g), C.byref(l)), "circuit_info")
        return w.value, g.value, l.value

    def wave_sizes(self) -> tuple[np.ndarray, np.ndarray]:
        n = self.info()[0]
        g = np.zeros(n, np.int32)
        lanes = np.zeros(n, np.int32)
        load().cufhe_circuit_wave_sizes(self.h, _p(g), _p(lanes), n)
        return g, lanes

    def run(self, wires, stream=None, graph: bool = True) -> None:
        check(load().cufhe_circuit_run(self.h, dptr(wires), stream, int(graph)), "circuit_run")

    def destroy(self) -> None:
        if getattr(self, "h", None):
            load().cufhe_circuit_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def batch_shard_plan(gates, count: int, shards: int, uniform: int = 0) -> np.ndarray:
    """cufhe_batch_shard_plan (host only): bounds[0..shards] of the contiguous
    gate ranges of a batch split over `shards` shards with balanced lanes."""
    g = None if gates is None else np.ascontiguousarray(gates, np.int32)
    bounds = np.zeros(shards + 1, np.uint64)
    check(load().cufhe_batch_shard_plan(_p(g), uniform, count, shards, _p(bounds)),
          "batch_shard_plan")
    return bounds.astype(np.int64)


def gate_batch_sharded_host(gates, level: int, in0, in1=None, in2=None, shards: int = 0,
                            uniform: int = 0) -> np.ndarray:
    """cufhe_gate_batch_sharded_host: one host batch split over shards (shard s
    on device s % gpu num); returns when every shard is done."""
    words = P.TLWE1_WORDS if level == LVL1 else P.TLWE0_WORDS
    in0 = np.ascontiguousarray(in0, np.uint32).reshape(-1, words)
    count = in0.shape[0]
    out = np.empty((count, words), np.uint32)
    g = None if gates is None else np.ascontiguousarray(gates, np.int32)
    i1 = None if in1 is None else np.ascontiguousarray(in1, np.uint32)
    i2 = None if in2 is None else np.ascontiguousarray(in2, np.uint32)
    check(load().cufhe_gate_batch_sharded_host(_p(g), uniform, count, level, _p(out), _p(in0),
                                               _p(i1), _p(i2), shards), "gate_batch_sharded_host")
    return out


def circuit_shard_plan(level: int, num_wires: int, ops, in0, in1, in2, out, shards: int,
                       sms: int = 0):
    """cufhe_circuit_shard_plan (host only, no GPU or keys): returns (wave of
    every gate, shard of every gate, number of waves, number of wire copies)."""
    ops = np.ascontiguousarray(ops, np.int32)
    arrs = [np.ascontiguousarray(x, np.int32) for x in (in0, in1, in2, out)]
    wave = np.empty(ops.size, np.int32)
    shard = np.empty(ops.size, np.int32)
    n = C.c_int()
    nc = C.c_size_t()
    check(load().cufhe_circuit_shard_plan(level, num_wires, ops.size, _p(ops),
                                          *(_p(a) for a in arrs), sms, shards, _p(wave),
                                          _p(shard), C.byref(n), C.byref(nc)),
          "circuit_shard_plan")
    return wave, shard, n.value, nc.value


class ShardedCircuit:
    """One circuit split over shards (cufhe_sharded_create): every shard runs
    its part of each wave on device shard % gpu num against its own wire
    table, and wires cross between shards' tables after the wave that writes
    them."""

    def __init__(self, level: int, num_wires: int, ops, in0, in1, in2, out, shards: int = 0):
        arr = lambda a: np.ascontiguousarray(a, np.int32)  # noqa: E731
        self.ops, self.in0, self.in1, self.in2, self.out = (arr(x) for x in (ops, in0, in1, in2,
                                                                            out))
        self.level = level
        self.num_wires = int(num_wires)
        h = C.c_void_p()
        check(load().cufhe_sharded_create(C.byref(h), level, self.num_wires, self.ops.size,
                                          _p(self.ops), _p(self.in0), _p(self.in1),
                                          _p(self.in2), _p(self.out), shards), "sharded_create")
        self.h = h

    def info(self) -> tuple[int, int, int]:
        """(waves, wire copies, shards)"""
        w, c, s = C.c_int(), C.c_size_t(), C.c_int()
        check(load().cufhe_sharded_info(self.h, C.byref(w), C.byref(c), C.byref(s)),
              "sharded_info")
        return w.value, c.value, s.value

    def device(self, shard: int) -> int:
        d = load().cufhe_sharded_device(self.h, shard)
        if d < 0:
            check(d, "sharded_device")
        return d

    @staticmethod
    def _tables(wires) -> C.Array:
        return (C.c_void_p * len(wires))(*[dptr(w).value for w in wires])

    def run(self, wires) -> None:
        check(load().cufhe_sharded_run(self.h, self._tables(wires)), "sharded_run")

    def collect(self, wires, dst: int = 0) -> None:
        check(load().cufhe_sharded_collect(self.h, self._tables(wires), dst), "sharded_collect")

    def synchronize(self) -> None:
        check(load().cufhe_sharded_synchronize(self.h), "sharded_synchronize")

    def destroy(self) -> None:
        if getattr(self, "h", None):
            load().cufhe_sharded_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def autotune() -> list[tuple[int, int]]:
    """Measures the blind rotation's lanes per CTA for a ladder of batch
    sizes on the current device; returns [(max lanes, lanes per CTA)]."""
    L = load()
    check(L.cufhe_autotune(), "autotune")
    return autotune_table()


def autotune_table() -> list[tuple[int, int]]:
    b = np.zeros(32, np.int32)
    g = np.zeros(32, np.int32)
    n = load().cufhe_autotune_table(_p(b), _p(g), 32)
    if n < 0:
        check(n, "autotune_table")
    return [(int(b[i]), int(g[i])) for i in range(n)]


class Stream:
    """An engine stream (cufhe_stream_create) and its CUDA stream handle."""

    def __init__(self, device: int = 0):
        self.h = C.c_void_p()
        check(load().cufhe_stream_create(C.byref(self.h), device), "stream_create")
        self._as_parameter_ = self.h  # pass a Stream wherever the C-ABI takes a cufhe_stream_t
        cs = C.c_void_p()
        check(load().cufhe_stream_cuda(self.h, C.byref(cs)), "stream_cuda")
        self.cuda = cs.value or 0

    def synchronize(self) -> None:
        check(load().cufhe_stream_synchronize(self.h), "stream_synchronize")

    def destroy(self) -> None:
        if self.h:
            load().cufhe_stream_destroy(self.h)
            self.h = None


def profile_enable(on: bool = True) -> None:
    check(load().cufhe_profile_enable(int(on)), "profile_enable")


def profile_reset() -> None:
    check(load().cufhe_profile_reset(), "profile_reset")


def profile_read(cls: int) -> tuple[float, int]:
    ms = C.c_double()
    n = C.c_uint64()
    check(load().cufhe_profile_read(cls, C.byref(ms), C.byref(n)), "profile_read")
    return ms.value, n.value


def measure_fp64_peak() -> float:
    t = C.c_double()
    check(load().cufhe_measure_fp64_peak(C.byref(t)), "measure_fp64_peak")
    return t.value


def measure_int8_peak() -> float:
    """INT8 tcgen05 throughput of the current device in TOP/s."""
    t = C.c_double()
    check(load().cufhe_measure_int8_peak(C.byref(t)), "measure_int8_peak")
    return t.value


def kernel_launches() -> int:
    return int(load().cufhe_kernel_launches())
