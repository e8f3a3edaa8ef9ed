"""TF-Lattice speech MOS mapping, restated in numpy (test infrastructure).

An independent restatement of the reference's mapper (src/lattice.zig:14-71)
and of the TFLite op semantics it relies on (src/tflite.zig:464-800): a
flatbuffer reader, numpy broadcasting for element-wise ops, f32 dot products
accumulated one fused multiply-add at a time from zero. Used by the tests as
the checker of the library's C++ interpreter; never by the product.
"""

from __future__ import annotations

import struct
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
DEFAULT_MODEL = (HERE.parent / "akvisqol_b200" / "model" /
                 "lattice_tcditugenmeetpackhref_ls2_nl60_lr12_bs2048_learn.005_ep2400_train1_7_raw.tflite")

F32, I32, BOOL = 0, 2, 6
FEATURES = ("fvnsim", "fvnsim10_", "fstdnsim", "fvdegenergy")


class _T:
    """A flatbuffer table at byte offset pos."""

    def __init__(self, buf: bytes, pos: int):
        self.buf, self.pos = buf, pos

    def _field(self, i: int):
        vt = self.pos - struct.unpack_from("<i", self.buf, self.pos)[0]
        size = struct.unpack_from("<H", self.buf, vt)[0]
        slot = 4 + 2 * i
        if slot + 2 > size:
            return None
        off = struct.unpack_from("<H", self.buf, vt + slot)[0]
        return self.pos + off if off else None

    def scalar(self, i: int, fmt: str, default=0):
        p = self._field(i)
        return default if p is None else struct.unpack_from("<" + fmt, self.buf, p)[0]

    def table(self, i: int):
        p = self._field(i)
        return None if p is None else _T(self.buf, p + struct.unpack_from("<I", self.buf, p)[0])

    def vector(self, i: int):
        p = self._field(i)
        if p is None:
            return None
        v = p + struct.unpack_from("<I", self.buf, p)[0]
        return v + 4, struct.unpack_from("<I", self.buf, v)[0]

    def tables(self, i: int):
        v = self.vector(i)
        if v is None:
            return []
        start, n = v
        return [_T(self.buf, start + 4 * k + struct.unpack_from("<I", self.buf, start + 4 * k)[0]) for k in range(n)]

    def ints(self, i: int, fmt: str = "i"):
        v = self.vector(i)
        if v is None:
            return None
        start, n = v
        return list(struct.unpack_from("<%d%s" % (n, fmt), self.buf, start))

    def string(self, i: int):
        v = self.vector(i)
        return None if v is None else self.buf[v[0]:v[0] + v[1]].decode()


def _fma32(p: float, q: float, c: float) -> np.float32:
    """fmaf(p, q, c) exactly, for f32 values given as floats: p*q is exact in
    f64; the f64 sum s = p*q + c and its error e (TwoSum, exact) give the
    exact result s + e. Rounding s to f32 equals rounding s + e unless s sits
    exactly on a midpoint between two f32 values and e != 0; then the
    neighbour on e's side is the correctly rounded result."""
    prod = p * q
    s = prod + c
    bb = s - prod
    e = (prod - (s - bb)) + (c - bb)
    r = np.float32(s)
    fr = float(r)
    if e != 0.0 and fr != s:
        other = np.nextafter(r, np.float32(np.inf) if s > fr else np.float32(-np.inf))
        if float(other) - s == s - fr:  # s is the midpoint of r and other
            up = e > 0.0
            r = max(r, other) if up else min(r, other)
    return np.float32(r)


def _fma_dot(x: np.ndarray, w: np.ndarray) -> np.float32:
    """Sequential f32 FMA from zero, each step rounded once to f32."""
    acc = 0.0
    for p, q in zip(x.astype(np.float64).tolist(), w.astype(np.float64).tolist()):
        acc = float(_fma32(p, q, acc))
    return np.float32(acc)


class Lattice:
    """The mapper: load once, then predict(fvnsim, fvnsim10, fstdnsim, fvdegenergy)."""

    def __init__(self, path: Path = DEFAULT_MODEL, nb: int = 21):
        buf = Path(path).read_bytes()
        root = _T(buf, struct.unpack_from("<I", buf, 0)[0])
        codes = [max(c.scalar(0, "b"), c.scalar(3, "i")) for c in root.tables(1)]
        g = root.tables(2)[0]
        buffers = root.tables(4)
        self.tensors = g.tables(0)
        self.types = [t.scalar(1, "b") for t in self.tensors]
        self.consts = {}
        for k, t in enumerate(self.tensors):
            bi = t.scalar(2, "I")
            if bi == 0 or bi >= len(buffers):
                continue
            data = buffers[bi].vector(0)
            if not data or data[1] == 0:
                continue
            shape = tuple(t.ints(0) or [])
            raw = buf[data[0]:data[0] + data[1]]
            dt = {F32: np.float32, I32: np.int32, BOOL: np.bool_}[self.types[k]]
            self.consts[k] = np.frombuffer(raw, dtype=dt).reshape(shape).copy()
        self.ops = []
        for op in g.tables(3):
            kind = codes[op.scalar(0, "I")]
            opt = op.table(4)
            self.ops.append((kind, op.ints(1) or [], op.ints(2) or [], opt))
        sig = next(s for s in root.tables(7) if s.string(2) == "predict" or len(root.tables(7)) == 1)
        self.inputs = {m.string(0): m.scalar(1, "I") for m in sig.tables(0)}
        self.outputs = {m.string(0): m.scalar(1, "I") for m in sig.tables(1)}
        self.nb = nb

    @staticmethod
    def _act(x, code):
        if code == 1:
            return np.maximum(x, np.float32(0))
        if code == 2:
            return np.clip(x, np.float32(-1), np.float32(1))
        if code == 3:
            return np.clip(x, np.float32(0), np.float32(6))
        return x

    def run(self, feeds: dict) -> dict:
        v = dict(self.consts)
        v.update(feeds)
        for kind, ins, outs, opt in self.ops:
            a = [v[i] if i >= 0 else None for i in ins]
            o = outs[0]
            act = opt.scalar(0, "b") if opt is not None and kind in (0, 18, 41, 9) else 0
            if kind == 0:
                v[o] = self._act(a[0] + a[1], act)
            elif kind == 41:
                v[o] = self._act(a[0] - a[1], act)
            elif kind == 18:
                v[o] = self._act(a[0] * a[1], act)
            elif kind == 57:
                v[o] = np.minimum(a[0], a[1])
            elif kind == 55:
                v[o] = np.maximum(a[0], a[1])
            elif kind == 71:
                v[o] = a[0] == a[1]
            elif kind == 19:
                v[o] = np.maximum(a[0], np.float32(0))
            elif kind == 21:
                v[o] = np.clip(a[0], np.float32(0), np.float32(6))
            elif kind == 101:
                v[o] = np.abs(a[0])
            elif kind == 53:
                to = self.types[o]
                x = a[0]
                if to == F32:
                    v[o] = x.astype(np.float32)
                elif to == I32:
                    v[o] = np.trunc(x).astype(np.int32) if x.dtype == np.float32 else x.astype(np.int32)
                else:
                    v[o] = x != 0
            elif kind == 2:
                axis = opt.scalar(0, "i") if opt is not None else 0
                cact = opt.scalar(1, "b") if opt is not None else 0
                v[o] = self._act(np.concatenate(a, axis=axis), cact)
            elif kind == 9:
                x, w = a[0], a[1]
                bias = a[2] if len(a) > 2 else None
                keep = bool(opt.scalar(2, "B")) if opt is not None else False
                n_out, n_in = w.shape
                rows = x.reshape(-1, n_in)
                y = np.empty((rows.shape[0], n_out), np.float32)
                for r in range(rows.shape[0]):
                    for j in range(n_out):
                        s = _fma_dot(rows[r], w[j])
                        if bias is not None:
                            s = np.float32(s + bias[j])
                        y[r, j] = s
                y = self._act(y, act)
                v[o] = y.reshape(x.shape[:-1] + (n_out,)) if keep else y
            elif kind == 126:
                x, y = a[0], a[1]
                adj_x = bool(opt.scalar(0, "B")) if opt is not None else False
                adj_y = bool(opt.scalar(1, "B")) if opt is not None else False
                xm = np.swapaxes(x, -1, -2) if adj_x else x
                ym = np.swapaxes(y, -1, -2) if adj_y else y
                bshape = np.broadcast_shapes(xm.shape[:-2], ym.shape[:-2])
                xb = np.broadcast_to(xm, bshape + xm.shape[-2:])
                yb = np.broadcast_to(ym, bshape + ym.shape[-2:])
                m, k, n = xm.shape[-2], xm.shape[-1], ym.shape[-1]
                if k == 1:
                    # one product per output: fma(p, q, 0) rounds p*q once
                    out = (xb.astype(np.float64) * yb.astype(np.float64)).astype(np.float32)
                else:
                    out = np.empty(bshape + (m, n), np.float32)
                    for idx in np.ndindex(*bshape):
                        for i in range(m):
                            for j in range(n):
                                out[idx + (i, j)] = _fma_dot(xb[idx + (i,)], yb[idx + (slice(None), j)])
                v[o] = out
            elif kind == 22:
                spec = a[1] if len(a) > 1 and a[1] is not None else np.array(opt.ints(0), np.int32)
                v[o] = a[0].reshape(tuple(int(d) for d in np.asarray(spec).reshape(-1)))
            elif kind == 70:
                v[o] = np.expand_dims(a[0], int(np.asarray(a[1]).reshape(-1)[0]))
            elif kind == 77:
                v[o] = np.array(a[0].shape, np.int32)
            elif kind == 94:
                v[o] = np.full(tuple(int(d) for d in a[0]), np.asarray(a[1]).reshape(-1)[0])
            elif kind == 49:
                parts = np.split(a[1], len(outs), axis=int(np.asarray(a[0]).reshape(-1)[0]))
                for t, p in zip(outs, parts):
                    v[t] = p
            else:
                raise ValueError(f"unsupported builtin {kind}")
        return v

    def predict(self, fvnsim, fvnsim10, fstdnsim, fvdegenergy) -> float:
        feeds = {}
        for name, vals in zip(FEATURES, (fvnsim, fvnsim10, fstdnsim, fvdegenergy)):
            for b in range(self.nb):
                feeds[self.inputs[f"{name}{b}"]] = np.array([vals[b]], np.float32)
        feeds[self.inputs["tau"]] = np.array([0.5], np.float32)
        out = self.run(feeds)[self.outputs["predictions"]]
        return float(np.asarray(out, np.float32).reshape(-1)[0])
