"""Minimal reader for R's XDR serialization format (``saveRDS`` version 2/3).

Used only by ``make_golden.py`` to turn the reference's ``.rds`` fixtures into
plain JSON/NPZ golden files.  It understands the subset of the format those
fixtures use: vectors (logical, integer, double, character, list), pairlists,
symbols, attributes, environments (skipped into dicts) and the compact ALTREP
integer/real sequences R writes for ``seq_len`` style vectors.
"""
import gzip
import lzma
import struct

import numpy as np

NILVALUE = 254
GLOBALENV = 253
UNBOUNDVALUE = 252
MISSINGARG = 251
BASENAMESPACE = 250
NAMESPACESXP = 249
PACKAGESXP = 248
PERSISTSXP = 247
EMPTYENV = 242
BASEENV = 241
ATTRLANGSXP = 240
ATTRLISTSXP = 239
ALTREP = 238
REFSXP = 255

NA_INTEGER = -(2 ** 31)


class RObject:
    """A decoded R value: ``value`` plus its attribute dict."""

    def __init__(self, kind, value, attrs=None):
        self.kind = kind
        self.value = value
        self.attrs = attrs or {}

    def attr(self, name, default=None):
        a = self.attrs.get(name)
        return default if a is None else a

    def names(self):
        n = self.attrs.get("names")
        return None if n is None else list(n.value)

    def __getitem__(self, key):
        if isinstance(key, str):
            names = self.names()
            return self.value[names.index(key)]
        return self.value[key]

    def __repr__(self):
        return f"RObject({self.kind}, len={len(self.value) if hasattr(self.value, '__len__') else 1})"


class _Reader:
    def __init__(self, raw):
        self.buf = raw
        self.pos = 0
        self.refs = []

    def read(self, n):
        out = self.buf[self.pos:self.pos + n]
        if len(out) != n:
            raise EOFError("truncated RDS stream")
        self.pos += n
        return out

    def int(self):
        return struct.unpack(">i", self.read(4))[0]

    def length(self):
        n = self.int()
        if n == -1:
            hi = self.int()
            lo = self.int()
            n = (hi << 32) + lo
        return n

    def header(self):
        fmt = self.read(2)
        if fmt != b"X\n":
            raise ValueError(f"unsupported RDS format {fmt!r}")
        version = self.int()
        self.int()
        self.int()
        if version == 3:
            nelen = self.int()
            self.read(nelen)

    def charsxp(self):
        flags = self.int()
        if flags & 0xFF != 9:
            raise ValueError("expected CHARSXP")
        n = self.int()
        if n == -1:
            return None
        return self.read(n).decode("utf-8", errors="replace")

    def item(self):
        flags = self.int()
        t = flags & 0xFF
        has_attr = bool(flags & (1 << 9))
        has_tag = bool(flags & (1 << 10))
        if t == NILVALUE:
            return None
        if t in (GLOBALENV, EMPTYENV, BASEENV, BASENAMESPACE, UNBOUNDVALUE, MISSINGARG):
            return RObject("special", t)
        if t == REFSXP:
            idx = flags >> 8
            if idx == 0:
                idx = self.int()
            return self.refs[idx - 1]
        if t == PERSISTSXP:
            obj = RObject("persist", self.strsxp_body())
            self.refs.append(obj)
            return obj
        if t == 1:  # SYMSXP
            name = self.charsxp()
            obj = RObject("symbol", name)
            self.refs.append(obj)
            return obj
        if t in (NAMESPACESXP, PACKAGESXP):
            self.int()
            obj = RObject("namespace", self.strsxp_items())
            self.refs.append(obj)
            return obj
        if t == 4:  # ENVSXP
            obj = RObject("env", {})
            self.refs.append(obj)
            self.int()  # locked
            self.item()  # enclos
            frame = self.item()
            hashtab = self.item()
            attrs = self.item()
            out = {}
            for src in (frame,):
                if isinstance(src, RObject) and src.kind == "pairlist":
                    out.update(src.value)
            if isinstance(hashtab, RObject) and hashtab.kind == "list":
                for bucket in hashtab.value:
                    if isinstance(bucket, RObject) and bucket.kind == "pairlist":
                        out.update(bucket.value)
            obj.value = out
            if isinstance(attrs, RObject):
                obj.attrs = self.attrs_from_pairlist(attrs)
            return obj
        if t in (2, 6, ATTRLANGSXP, ATTRLISTSXP, 17):  # pairlist-like
            return self.pairlist(flags)
        if t == ALTREP:
            info = self.item()
            state = self.item()
            attr = self.item()
            cls = info.items[0][1].value if isinstance(info, RObject) else None
            obj = self.altrep(cls, state)
            if isinstance(attr, RObject):
                obj.attrs = self.attrs_from_pairlist(attr)
            return obj
        if t in (10, 13):
            n = self.length()
            vals = np.frombuffer(self.read(4 * n), dtype=">i4").astype(np.int64)
            kind = "logical" if t == 10 else "integer"
            obj = RObject(kind, vals)
        elif t == 14:
            n = self.length()
            obj = RObject("double", np.frombuffer(self.read(8 * n), dtype=">f8").astype(np.float64))
        elif t == 15:
            n = self.length()
            obj = RObject("complex", np.frombuffer(self.read(16 * n), dtype=">f8"))
        elif t == 16:
            n = self.length()
            obj = RObject("character", [self.charsxp() for _ in range(n)])
        elif t in (19, 20):
            n = self.length()
            obj = RObject("list", [self.item() for _ in range(n)])
        elif t == 24:
            n = self.length()
            obj = RObject("raw", self.read(n))
        elif t == 9:
            n = self.int()
            obj = RObject("char", None if n == -1 else self.read(n).decode())
        elif t == 25:  # S4
            obj = RObject("s4", None)
        else:
            raise ValueError(f"unsupported SEXP type {t} at byte {self.pos}")
        if has_attr:
            obj.attrs = self.attrs_from_pairlist(self.item())
        return obj

    def strsxp_items(self):
        self.int()  # flags of STRSXP
        return self.strsxp_body()

    def strsxp_body(self):
        n = self.length()
        return [self.charsxp() for _ in range(n)]

    def pairlist(self, flags):
        entries = []
        attrs = None
        while True:
            t = flags & 0xFF
            has_attr = bool(flags & (1 << 9))
            has_tag = bool(flags & (1 << 10))
            if has_attr:
                attrs = self.item()
            tag = self.item() if has_tag else None
            car = self.item()
            entries.append((tag.value if isinstance(tag, RObject) else None, car))
            flags = self.int()
            if flags & 0xFF == NILVALUE:
                break
            if flags & 0xFF not in (2, 6, ATTRLANGSXP, ATTRLISTSXP, 17):
                # cdr is not a pairlist cell: decode it as a value and stop
                self.pos -= 4
                self.item()
                break
        obj = RObject("pairlist", dict((k, v) for k, v in entries if k is not None))
        obj.items = entries
        if attrs is not None:
            obj.attrs = self.attrs_from_pairlist(attrs)
        return obj

    def attrs_from_pairlist(self, pl):
        if not isinstance(pl, RObject) or pl.kind != "pairlist":
            return {}
        return dict(pl.value)

    def altrep(self, cls, state):
        if cls == "compact_intseq":
            n, start, step = state.value
            vals = start + step * np.arange(int(n), dtype=np.int64)
            return RObject("integer", vals.astype(np.int64))
        if cls == "compact_realseq":
            n, start, step = state.value
            return RObject("double", start + step * np.arange(int(n), dtype=np.float64))
        if cls in ("wrap_integer", "wrap_logical", "wrap_real", "wrap_string", "wrap_list"):
            return state.items[0][1] if state.kind == "pairlist" else state.value[0]
        if cls == "deferred_string":
            src = state.value[0] if isinstance(state, RObject) and state.kind == "pairlist" else state
            if isinstance(state, RObject) and state.kind == "pairlist":
                src = state.items[0][1]
            vals = src.value
            return RObject("character", [str(int(v)) if float(v).is_integer() else repr(float(v)) for v in vals])
        raise ValueError(f"unsupported ALTREP class {cls}")


def read_rds(path):
    with open(path, "rb") as f:
        raw = f.read()
    if raw[:2] == b"\x1f\x8b":
        raw = gzip.decompress(raw)
    elif raw[:6] == b"\xfd7zXZ\x00":
        raw = lzma.decompress(raw)
    r = _Reader(raw)
    r.header()
    return r.item()
