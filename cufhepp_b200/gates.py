"""The reference's gate API (include/cufhe_gpu.cuh:42-358) mirrored in Python
over the engine's C-ABI: SetGPUNum, Initialize, CleanUp, Synchronize,
Stream, StreamQuery, Ctxt, and the 14 gates in copying (Nand, ...) and
device-resident (gNand, ...) forms.  Ctxt level 1 is Ctxt<lvl1param>
(key switching, then blind rotation), level 0 is Ctxt<lvl0param>.  The lvl02
path: Initialize_lvl02 / CleanUp_lvl02 and Nand_lvl02 ... NMux_lvl02 on level-0
Ctxts (include/cufhe_gpu.cuh:59-64, :332-358).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import engine, params as P

SetGPUNum = lambda n: engine.check(engine.load().cufhe_set_gpu_num(n), "SetGPUNum")  # noqa: E731


def Initialize(ek) -> None:
    engine.initialize(ek)


def CleanUp() -> None:
    engine.cleanup()


def Initialize_lvl02(ek02, sk=None) -> None:
    """Initialize_lvl02(ek, sk): the secret key is unused, as in the reference."""
    engine.initialize_lvl02(ek02)


def CleanUp_lvl02() -> None:
    engine.cleanup_lvl02()


def Synchronize() -> None:
    engine.synchronize()


class Stream:
    """Round-robin device on construction; Create() makes the CUDA stream."""

    def __init__(self, device_id: int | None = None):
        L = engine.load()
        n = L.cufhe_get_gpu_num()
        Stream._count = getattr(Stream, "_count", 0) + 1
        self._device = (Stream._count - 1) % n if device_id is None else device_id
        self._h = C.c_void_p()

    def Create(self):
        engine.check(engine.load().cufhe_stream_create(C.byref(self._h), self._device),
                     "Stream.Create")

    def Destroy(self):
        engine.check(engine.load().cufhe_stream_destroy(self._h), "Stream.Destroy")
        self._h = C.c_void_p()

    def st(self):
        return self._h

    def device_id(self) -> int:
        return self._device


def StreamQuery(st: Stream) -> bool:
    r = engine.load().cufhe_stream_query(st.st())
    if r < 0:
        engine.check(r, "StreamQuery")
    return r == 1


class Ctxt:
    """TLWE ciphertext with a host copy and one device buffer per GPU."""

    def __init__(self, level: int = 1):
        self.level = level
        words = P.TLWE1_WORDS if level == 1 else P.TLWE0_WORDS
        self.tlwehost = np.zeros(words, np.uint32)
        n = engine.load().cufhe_get_gpu_num()
        self.tlwedevices = [engine.DeviceBuffer(words * 4, d) for d in range(n)]


def _copy(gate, out, a, b=None, c=None, st: Stream | None = None, level: int | None = None):
    d = st.device_id() if st else 0
    h = lambda x: None if x is None else engine._p(x.tlwehost)  # noqa: E731
    v = lambda x: None if x is None else engine.dptr(x.tlwedevices[d])  # noqa: E731
    lv = out.level if level is None else level
    engine.check(engine.load().cufhe_gate_copy(gate, lv, h(out), v(out), h(a), v(a), h(b),
                                               v(b), h(c), v(c), st.st() if st else None),
                 P.GATE_NAMES[gate])


def _dev(gate, out, a, b=None, c=None, st: Stream | None = None):
    d = st.device_id() if st else 0
    v = lambda x: None if x is None else engine.dptr(x.tlwedevices[d])  # noqa: E731
    engine.check(engine.load().cufhe_gate(gate, out.level, v(out), v(a), v(b), v(c),
                                          st.st() if st else None), "g" + P.GATE_NAMES[gate])


def _binary(gid):
    def f(out, in0, in1, st=None):
        _copy(gid, out, in0, in1, None, st)

    def g(out, in0, in1, st=None):
        _dev(gid, out, in0, in1, None, st)
    return f, g


Nand, gNand = _binary(P.NAND)
Or, gOr = _binary(P.OR)
OrYN, gOrYN = _binary(P.ORYN)
OrNY, gOrNY = _binary(P.ORNY)
And, gAnd = _binary(P.AND)
AndYN, gAndYN = _binary(P.ANDYN)
AndNY, gAndNY = _binary(P.ANDNY)
Nor, gNor = _binary(P.NOR)
Xor, gXor = _binary(P.XOR)
Xnor, gXnor = _binary(P.XNOR)


def _binary02(gid):
    def f(out, in0, in1, st=None):
        assert out.level == 0, "the lvl02 gates take Ctxt<lvl0param>"
        _copy(gid, out, in0, in1, None, st, level=engine.LVL02)
    return f


Nand_lvl02 = _binary02(P.NAND)
Or_lvl02 = _binary02(P.OR)
OrYN_lvl02 = _binary02(P.ORYN)
OrNY_lvl02 = _binary02(P.ORNY)
And_lvl02 = _binary02(P.AND)
AndYN_lvl02 = _binary02(P.ANDYN)
AndNY_lvl02 = _binary02(P.ANDNY)
Nor_lvl02 = _binary02(P.NOR)
Xor_lvl02 = _binary02(P.XOR)
Xnor_lvl02 = _binary02(P.XNOR)


def Mux_lvl02(out, inc, in1, in0, st=None):
    _copy(P.MUX, out, inc, in1, in0, st, level=engine.LVL02)


def NMux_lvl02(out, inc, in1, in0, st=None):
    _copy(P.NMUX, out, inc, in1, in0, st, level=engine.LVL02)


def Mux(out, inc, in1, in0, st=None):
    _copy(P.MUX, out, inc, in1, in0, st)


def gMux(out, inc, in1, in0, st=None):
    _dev(P.MUX, out, inc, in1, in0, st)


def NMux(out, inc, in1, in0, st=None):
    _copy(P.NMUX, out, inc, in1, in0, st)


def gNMux(out, inc, in1, in0, st=None):
    _dev(P.NMUX, out, inc, in1, in0, st)


def Not(out, in0, st=None):
    _copy(P.NOT, out, in0, None, None, st)


def gNot(out, in0, st=None):
    _dev(P.NOT, out, in0, None, None, st)


def Copy(out, in0, st=None):
    _copy(P.COPY, out, in0, None, None, st)


def gCopy(out, in0, st=None):
    _dev(P.COPY, out, in0, None, None, st)


def CopyOnHost(out, in0):
    out.tlwehost[:] = in0.tlwehost
