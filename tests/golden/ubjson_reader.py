"""Minimal Universal Binary JSON (UBJSON draft 12) decoder.

Only what is needed to read the reference's golden ``.ubjson`` data files:
scalars, strings, high-precision numbers, and (optimised) arrays / objects.
Typed numeric arrays are returned as numpy arrays for speed.
"""
import struct

import numpy as np

_FIXED = {
    b"i": (">b", 1), b"U": (">B", 1), b"I": (">h", 2), b"l": (">i", 4),
    b"L": (">q", 8), b"d": (">f", 4), b"D": (">d", 8),
}
_NP = {b"i": ">i1", b"U": ">u1", b"I": ">i2", b"l": ">i4", b"L": ">i8",
       b"d": ">f4", b"D": ">f8"}


class _Reader:
    def __init__(self, buf):
        self.b = buf
        self.p = 0

    def take(self, n):
        out = self.b[self.p:self.p + n]
        self.p += n
        return out

    def marker(self):
        while True:
            m = self.take(1)
            if m != b"N":  # no-op marker
                return m

    def length(self):
        m = self.take(1)
        fmt, n = _FIXED[m]
        return struct.unpack(fmt, self.take(n))[0]

    def value(self, m=None):
        if m is None:
            m = self.marker()
        if m in _FIXED:
            fmt, n = _FIXED[m]
            return struct.unpack(fmt, self.take(n))[0]
        if m == b"Z":
            return None
        if m == b"T":
            return True
        if m == b"F":
            return False
        if m == b"C":
            return self.take(1).decode()
        if m == b"S":
            return self.take(self.length()).decode()
        if m == b"H":
            return float(self.take(self.length()).decode())
        if m == b"[":
            return self.array()
        if m == b"{":
            return self.obj()
        raise ValueError("bad UBJSON marker %r at %d" % (m, self.p - 1))

    def _container_header(self):
        typ, count = None, None
        if self.b[self.p:self.p + 1] == b"$":
            self.p += 1
            typ = self.take(1)
        if self.b[self.p:self.p + 1] == b"#":
            self.p += 1
            count = self.length()
        return typ, count

    def array(self):
        typ, count = self._container_header()
        if count is not None:
            if typ in _NP:
                n = struct.calcsize(_FIXED[typ][0]) * count
                arr = np.frombuffer(self.take(n), dtype=_NP[typ]).astype(
                    np.float64 if typ in (b"d", b"D") else np.int64)
                return arr
            return [self.value(typ) for _ in range(count)]
        out = []
        while True:
            m = self.marker()
            if m == b"]":
                return out
            out.append(self.value(m))

    def obj(self):
        typ, count = self._container_header()
        out = {}
        if count is not None:
            for _ in range(count):
                k = self.take(self.length()).decode()
                out[k] = self.value(typ)
            return out
        while True:
            if self.b[self.p:self.p + 1] == b"}":
                self.p += 1
                return out
            k = self.take(self.length()).decode()
            out[k] = self.value()


def load(path):
    with open(path, "rb") as f:
        return _Reader(f.read()).value()
