"""ctypes access to ``oracle/_ref/lib<config>.so`` (see build_ref.py, ref_harness.c).

TEST INFRASTRUCTURE ONLY.
"""

from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")


_SINK = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t)


def available(config: str) -> bool:
    return os.path.exists(os.path.join(REF_DIR, "lib%s.so" % config))


class RefOracle:
    """The reference C backend for one grammar configuration."""

    def __init__(self, config: str, path: str = None):
        path = path or os.path.join(REF_DIR, "lib%s.so" % config)
        if not os.path.exists(path):
            raise FileNotFoundError("%s missing: run oracle/build_ref.py %s" % (path, config))
        self.config = config
        self.lib = ctypes.CDLL(path)
        self.lib.ref_run_case.argtypes = [ctypes.c_uint64, ctypes.c_char_p,
                                          ctypes.POINTER(ctypes.POINTER(ctypes.c_uint8)),
                                          ctypes.POINTER(ctypes.c_size_t)]
        self.lib.ref_run_case.restype = ctypes.c_int
        if hasattr(self.lib, "ref_pipeline"):  # combined programs only
            self.lib.ref_pipeline.argtypes = [ctypes.c_uint64, ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64),
                                              ctypes.POINTER(ctypes.c_uint64)]
            self.lib.ref_pipeline.restype = ctypes.c_int
        self.lib.ref_free.argtypes = [ctypes.c_void_p]
        if hasattr(self.lib, "ref_run_case_sink"):
            self.lib.ref_run_case_sink.argtypes = [ctypes.c_uint64, ctypes.c_void_p, _SINK, ctypes.c_void_p]
            self.lib.ref_run_case_sink.restype = ctypes.c_int
        self.lib.ref_layout.argtypes = [ctypes.POINTER(ctypes.c_uint64)]
        self.lib.ref_input_unit.restype = ctypes.c_uint64

    def run_case(self, data: bytes) -> bytes:
        """The exact response record ``run_case`` writes for ``data`` (bytes;
        for a parser-mode program the terminal ids' bytes)."""
        out = ctypes.POINTER(ctypes.c_uint8)()
        n = ctypes.c_size_t()
        count = len(data) // self.lib.ref_input_unit()
        if self.lib.ref_run_case(count, data, ctypes.byref(out), ctypes.byref(n)) != 0:
            raise RuntimeError("open_memstream failed")
        try:
            return ctypes.string_at(out, n.value)
        finally:
            self.lib.ref_free(out)

    def record_digest(self, buf, head: int = 0):
        """(SHA-256 hex, byte count) of the response record ``run_case``
        writes for ``buf`` (a numpy uint8 array or bytes), streamed through a
        callback in 64 MiB pieces: records of several GB are never held.
        With ``head`` > 0 the first ``head`` bytes are left out of the digest
        and returned as a third item (e.g. a record's validity byte and
        count, which a caller streaming its own record learns last)."""
        import hashlib

        import numpy as np
        a = np.frombuffer(buf, dtype=np.uint8) if isinstance(buf, (bytes, bytearray)) else buf
        h = hashlib.sha256()
        size = [0]
        first = bytearray()

        def sink(_user, p, nbytes):
            # a write can be several GB (stdio hands large fwrite calls to the
            # sink whole): hash it in place, without a bytes copy (ctypes'
            # string_at takes a C int size)
            skip = 0
            if len(first) < head:
                skip = min(head - len(first), nbytes)
                first.extend((ctypes.c_char * skip).from_address(p))
            if nbytes > skip:
                h.update((ctypes.c_char * (nbytes - skip)).from_address(p + skip))
            size[0] += nbytes

        cb = _SINK(sink)
        count = len(a) // self.lib.ref_input_unit()
        if self.lib.ref_run_case_sink(count, a.ctypes.data, cb, None) != 0:
            raise RuntimeError("fopencookie failed")
        if head:
            return h.hexdigest(), size[0], bytes(first)
        return h.hexdigest(), size[0]

    def pipeline(self, buf, n=None):
        """lex -> parse -> parents -> compact without serialisation.
        ``buf`` is anything exposing a buffer address (numpy array / bytes)."""
        import numpy as np
        a = np.frombuffer(buf, dtype=np.uint8) if isinstance(buf, (bytes, bytearray)) else buf
        nt = ctypes.c_uint64()
        nn = ctypes.c_uint64()
        ok = self.lib.ref_pipeline(len(a) if n is None else n, a.ctypes.data, ctypes.byref(nt), ctypes.byref(nn))
        return bool(ok), nt.value, nn.value

    def layout(self):
        s = (ctypes.c_uint64 * 4)()
        self.lib.ref_layout(s)
        return tuple(s)
