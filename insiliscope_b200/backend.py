"""The named-kernel backend from Python: sim::GpuBackend (WidefieldGpuHost.h:42-77) -- storage buffers of 32-bit
words and the kernels of the reference's GPU hosts dispatched by name (iscu_buffer_*, iscu_dispatch; the kernels and
their parameter blocks are listed in include/iscu.h). The C++ hosts bind the same calls through
include/iscu_gpubackend.hpp."""
from __future__ import annotations

import ctypes as C
import weakref

import numpy as np

from .engine import Engine, check


def f32_bits(x: float) -> int:
    """A float parameter word (the hosts' Bits())."""
    return int(np.array([x], np.float32).view(np.uint32)[0])


class Buffer:
    """A device buffer of the backend (bytes rounded up to 4)."""

    def __init__(self, backend: "GpuBackend", nbytes: int, data=None):
        self.backend = backend
        lib = backend.lib
        h = C.c_void_p()
        src = None if data is None else np.ascontiguousarray(data)
        n = nbytes if src is None else max(nbytes, src.nbytes)
        check(lib.iscu_buffer_create(backend.engine.h, n, None if src is None else src.ctypes.data, C.byref(h)))
        self.h = h
        self.bytes = lib.iscu_buffer_bytes(h)

    def close(self):
        if self.h:
            self.backend.lib.iscu_buffer_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GpuBackend:
    """GpuBackend::Make / Write / Copy / Dispatch / ReadBack / ReadBackLow16 on an Engine's context."""

    def __init__(self, engine: Engine):
        self.engine = engine
        self.lib = engine.lib
        self._buffers = weakref.WeakSet()   # closed before the context is (a buffer must not outlive it)
        engine._plans.add(self)

    def make(self, nbytes: int, data=None) -> Buffer:
        b = Buffer(self, nbytes, data)
        self._buffers.add(b)
        return b

    def write(self, buf: Buffer, offset: int, data):
        src = np.ascontiguousarray(data)
        check(self.lib.iscu_buffer_write(buf.h, offset, src.ctypes.data, src.nbytes))

    def copy(self, dst: Buffer, src: Buffer, nbytes: int):
        check(self.lib.iscu_buffer_copy(dst.h, src.h, nbytes))

    def dispatch(self, kernel: str, params, bufs, x: int, y: int = 1, z: int = 1):
        """params: up to 16 words (ints as uint32, floats as their float32 bits)."""
        words = np.array([f32_bits(p) if isinstance(p, float) else int(p) & 0xFFFFFFFF for p in params], np.uint32)
        hs = (C.c_void_p * max(1, len(bufs)))(*[b.h for b in bufs])
        check(self.lib.iscu_dispatch(self.engine.h, kernel.encode(), words.ctypes.data if len(words) else None,
                                     len(words), hs, len(bufs), x, y, z))

    def read_back(self, buf: Buffer, nbytes: int, dtype=np.uint32) -> np.ndarray:
        out = np.empty(nbytes, np.uint8)
        check(self.lib.iscu_buffer_read(buf.h, nbytes, out.ctypes.data))
        return out.view(dtype)

    def read_back_low16(self, buf: Buffer, words: int) -> np.ndarray:
        out = np.empty(words, np.uint16)
        check(self.lib.iscu_buffer_read_low16(buf.h, words, out.ctypes.data))
        return out

    def close(self):
        for b in list(self._buffers):
            b.close()
