"""Encoded FastLanes columns: host encoding (C++ encoders of the library) and
device residency (torch tensors holding the packed words and metadata).

An encoded column is a contiguous array of 1024-value vectors, each with a
16-byte metadata entry {word offset, FOR base, scheme, bit width, aux}; the
uniform form (one scheme/bit width/base for all vectors, no metadata) is the
reference's layout (fastlanes/src/ssb/fls_q11.cu:202-223).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import (LAYOUT_NORMAL, LAYOUT_TRANSPOSED, SCHEME_DELTA, SCHEME_FOR, Column, check, lib)

META_DTYPE = np.dtype([("offset", "<u8"), ("base", "<i4"), ("scheme", "u1"), ("bw", "u1"), ("aux", "<u2")])
assert META_DTYPE.itemsize == 16


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def n_vectors(n_values: int) -> int:
    return (n_values + 1023) // 1024


@dataclass
class EncodedColumn:
    """A column encoded on the host."""
    words: np.ndarray            # uint32 payload words
    meta: np.ndarray | None      # META_DTYPE per vector, or None for a uniform column
    n_values: int
    layout: int
    scheme: int = SCHEME_FOR     # uniform columns
    bw: int = 0                  # uniform columns
    base: int = 0                # uniform columns
    max_vec_words: int = 0
    scheme_mask: int = 0
    payload_words: int = -1      # encoded words (words may carry padding past them)

    @property
    def n_vec(self) -> int:
        return n_vectors(self.n_values)

    @property
    def nbytes(self) -> int:
        """Encoded bytes a decode must read: payload plus per-vector metadata."""
        pw = int(self.words.size) if self.payload_words < 0 else self.payload_words
        return pw * 4 + (0 if self.meta is None else int(self.meta.size) * 16)

    # -- encoders -----------------------------------------------------------
    @classmethod
    def uniform(cls, values: np.ndarray, scheme: int = SCHEME_FOR, layout: int = LAYOUT_NORMAL,
                bw: int | None = None, base: int = 0) -> "EncodedColumn":
        """One scheme, bit width and FOR base for every vector (the reference's
        column format).  bw=None picks the smallest width that fits."""
        v = np.ascontiguousarray(values, dtype=np.int32)
        n = int(v.size)
        out = np.zeros(int(lib().fls_encode_bound_words(n)), dtype=np.uint32)
        n_words = ctypes.c_uint64()
        out_bw = ctypes.c_uint8()
        check(lib().fls_encode_uniform(_ptr(v), n, scheme, layout, 0xFF if bw is None else bw, base, _ptr(out),
                                       ctypes.addressof(n_words), ctypes.addressof(out_bw)), "fls_encode_uniform")
        words = out[:max(n_words.value, 4)].copy()
        return cls(words=words, meta=None, n_values=n, layout=layout, scheme=scheme, bw=out_bw.value, base=base,
                   max_vec_words=0, scheme_mask=1 << scheme, payload_words=int(n_words.value))

    @classmethod
    def encode(cls, values: np.ndarray, schemes: np.ndarray | int = SCHEME_FOR,
               layout: int = LAYOUT_TRANSPOSED, round4: bool = False) -> "EncodedColumn":
        """Per-vector encoding: `schemes` is one scheme for all vectors or an
        array with one scheme per vector (e.g. from the selector)."""
        v = np.ascontiguousarray(values, dtype=np.int32)
        n = int(v.size)
        nv = n_vectors(n)
        out = np.zeros(int(lib().fls_encode_bound_words(n)), dtype=np.uint32)
        meta = np.zeros(nv, dtype=META_DTYPE)
        n_words, mvw, mask = ctypes.c_uint64(), ctypes.c_uint32(), ctypes.c_uint32()
        if isinstance(schemes, (int, np.integer)):
            sp, s0 = None, int(schemes)
        else:
            sch = np.ascontiguousarray(schemes, dtype=np.uint8)
            assert sch.size == nv
            sp, s0 = _ptr(sch), 0
        check(lib().fls_encode_column(_ptr(v), n, sp, s0, layout, int(round4), _ptr(out), ctypes.addressof(n_words),
                                      _ptr(meta), ctypes.addressof(mvw), ctypes.addressof(mask)),
              "fls_encode_column")
        words = out[:max(n_words.value, 4)].copy()
        return cls(words=words, meta=meta, n_values=n, layout=layout, max_vec_words=mvw.value,
                   scheme_mask=mask.value, payload_words=int(n_words.value))

    def to_device(self, device=None) -> "DeviceColumn":
        return DeviceColumn(self, device)

    # -- container (fls_column_write_container / fls_column_open_container) --
    def to_bytes(self) -> bytes:
        """The column as an encoded-column container (payload, metadata and a
        checksummed footer)."""
        words = np.ascontiguousarray(self.words, dtype=np.uint32)
        meta = None if self.meta is None else np.ascontiguousarray(self.meta)
        d = Column(data=words.ctypes.data, meta=0 if meta is None else meta.ctypes.data, n_values=self.n_values,
                   n_words=int(words.size), layout=self.layout, scheme=self.scheme, bw=self.bw, base=self.base,
                   max_vec_words=self.max_vec_words, scheme_mask=self.scheme_mask)
        n = int(lib().fls_column_container_bytes(ctypes.byref(d)))
        out = _aligned16(n)
        check(lib().fls_column_write_container(ctypes.byref(d), out.ctypes.data, n, None), "fls_column_write_container")
        return out.tobytes()

    @classmethod
    def from_bytes(cls, b) -> "EncodedColumn":
        """A column from an encoded-column container; damaged or foreign bytes
        raise FlsError (checked by the library before anything is read)."""
        buf = _aligned16(len(b))
        buf[:] = np.frombuffer(b, dtype=np.uint8)
        d = Column()
        check(lib().fls_column_open_container(buf.ctypes.data, buf.size, ctypes.byref(d)), "fls_column_open_container")
        words = buf[: 4 * d.n_words].view(np.uint32).copy()
        meta = None
        if d.meta:
            off = int(d.meta) - buf.ctypes.data
            meta = buf[off: off + 16 * n_vectors(d.n_values)].view(META_DTYPE).copy()
        return cls(words=words, meta=meta, n_values=int(d.n_values), layout=int(d.layout), scheme=int(d.scheme),
                   bw=int(d.bw), base=int(d.base), max_vec_words=int(d.max_vec_words), scheme_mask=int(d.scheme_mask))

    def save(self, path: str) -> None:
        with open(path, "wb") as f:
            f.write(self.to_bytes())

    @classmethod
    def load(cls, path: str) -> "EncodedColumn":
        with open(path, "rb") as f:
            return cls.from_bytes(f.read())


class DeviceColumn:
    """An EncodedColumn resident in device memory, with its C descriptor."""

    def __init__(self, col: EncodedColumn, device=None):
        import torch
        dev = torch.device("cuda") if device is None else torch.device(device)
        self.host = col
        self.data = torch.from_numpy(col.words.view(np.int32)).to(dev)
        self.meta = None if col.meta is None else torch.from_numpy(col.meta.view(np.int32).reshape(-1)).to(dev)
        self.desc = Column(data=self.data.data_ptr(), meta=0 if self.meta is None else self.meta.data_ptr(),
                           n_values=col.n_values, n_words=int(col.words.size), layout=col.layout,
                           scheme=col.scheme, bw=col.bw, base=col.base, max_vec_words=col.max_vec_words,
                           scheme_mask=col.scheme_mask)

    @property
    def n_values(self) -> int:
        return self.host.n_values

    @property
    def n_vec(self) -> int:
        return self.host.n_vec

    @property
    def nbytes(self) -> int:
        return self.host.nbytes


class DeviceUniformColumn:
    """A uniform column (one scheme, bit width and FOR base, the reference's
    column format) whose packed words are already in device memory (int32
    tensor, 16-byte aligned): vector v at word 32*bw*v (FOR) or (32+32*bw)*v
    (DELTA, transposed).  Same interface as DeviceColumn."""

    def __init__(self, data, n_values: int, bw: int, base: int = 0, scheme: int = SCHEME_FOR,
                 layout: int = LAYOUT_NORMAL):
        self.host = None
        self.data, self.meta = data, None
        self._n_values, self.bw = n_values, bw
        per = 32 * bw if scheme == SCHEME_FOR else 32 + 32 * bw
        self.payload_words = n_vectors(n_values) * per
        if int(data.numel()) < self.payload_words:
            raise ValueError("device words smaller than the column")
        self.desc = Column(data=data.data_ptr(), meta=0, n_values=n_values, n_words=int(data.numel()), layout=layout,
                           scheme=scheme, bw=bw, base=base, max_vec_words=0, scheme_mask=1 << scheme)

    @property
    def n_values(self) -> int:
        return self._n_values

    @property
    def n_vec(self) -> int:
        return n_vectors(self._n_values)

    @property
    def nbytes(self) -> int:
        return self.payload_words * 4


class DeviceEncodedColumn:
    """A per-vector encoded column produced on the GPU (fls_encode_column_gpu):
    the device words and metadata with their C descriptor; same interface as
    DeviceColumn."""

    def __init__(self, data, meta, n_values: int, layout: int, payload_words: int, max_vec_words: int,
                 scheme_mask: int):
        self.host = None
        self.data, self.meta = data, meta
        self._n_values, self.layout, self.payload_words = n_values, layout, payload_words
        self.desc = Column(data=data.data_ptr(), meta=meta.data_ptr(), n_values=n_values, n_words=int(data.numel()),
                           layout=layout, scheme=0, bw=0, base=0, max_vec_words=max_vec_words,
                           scheme_mask=scheme_mask)

    @property
    def n_values(self) -> int:
        return self._n_values

    @property
    def n_vec(self) -> int:
        return n_vectors(self._n_values)

    @property
    def nbytes(self) -> int:
        return self.payload_words * 4 + self.n_vec * 16

    def to_host(self) -> EncodedColumn:
        """The same column as a host EncodedColumn (words and metadata copied back)."""
        words = self.data.cpu().numpy().view(np.uint32).copy()
        meta = self.meta.cpu().numpy().view(META_DTYPE).copy()
        return EncodedColumn(words=words, meta=meta, n_values=self._n_values, layout=self.layout,
                             max_vec_words=self.desc.max_vec_words, scheme_mask=self.desc.scheme_mask,
                             payload_words=self.payload_words)


def encode_column_gpu(values, schemes=0, layout: int = LAYOUT_TRANSPOSED, round4: bool = False,
                      compact: bool = True) -> DeviceEncodedColumn:
    """Encodes a device int32 column on the GPU: `schemes` is one scheme for
    every vector or a device uint8 tensor with one per vector (for example the
    learned selector's picks).  compact=True trims the output to the payload."""
    import torch
    n = int(values.numel())
    nv = n_vectors(n)
    dev = values.device
    bound = int(lib().fls_encode_bound_words(n))
    out = torch.empty(bound + 4, dtype=torch.int32, device=dev)
    meta = torch.empty(nv * 4, dtype=torch.int32, device=dev)
    info = torch.zeros(3, dtype=torch.int64, device=dev)
    ws_bytes = int(lib().fls_encode_gpu_workspace_bytes(n))
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    per_vec = not isinstance(schemes, (int, np.integer))
    if per_vec:
        assert schemes.dtype == torch.uint8 and schemes.numel() == nv and schemes.device == dev
    check(lib().fls_encode_column_gpu(values.data_ptr(), n, schemes.data_ptr() if per_vec else None,
                                      0 if per_vec else int(schemes), layout, int(round4), out.data_ptr(), bound + 4,
                                      meta.data_ptr(), info.data_ptr(), ws.data_ptr(), ws_bytes,
                                      torch.cuda.current_stream().cuda_stream), "fls_encode_column_gpu")
    total, mx, mask = (int(x) for x in info.cpu())
    if compact:
        out = out[:max(total, 4)].clone()
    return DeviceEncodedColumn(out, meta, n, layout, total, mx, mask)


class PendingEncode:
    """A GPU encode enqueued without reading its results back: finish() reads
    the encoder's info words (one device-to-host copy) and returns what
    encode_column_learned_gpu returns.  Deferring the read lets many columns
    be encoded back to back with no host round trip in between."""

    def __init__(self, out, meta, info, schemes, n, layout, compact):
        self.out, self.meta, self.info, self.schemes = out, meta, info, schemes
        self.n, self.layout, self.compact = n, layout, compact

    def finish(self):
        total, mx, mask, n_fb = (int(x) for x in self.info.cpu())
        out = self.out[:max(total, 4)].clone() if self.compact else self.out
        return DeviceEncodedColumn(out, self.meta, self.n, self.layout, total, mx, mask), self.schemes, n_fb


def encode_column_learned_gpu(values, params, threshold: float = 0.9, kappa: float = 0.0,
                              layout: int = LAYOUT_TRANSPOSED, compact: bool = True, defer: bool = False):
    """The learned encoder in one device call (fls_encode_learned_gpu): the MLP
    with `params` (device float32, FLS_MLP_N_PARAMS) picks each vector's scheme,
    the exhaustive choice replaces picks whose confidence is below
    `threshold`, and the column is encoded on the GPU.  Returns
    (DeviceEncodedColumn, per-vector schemes, number of fallback vectors), or
    with defer=True a PendingEncode whose finish() returns them."""
    import torch
    n = int(values.numel())
    nv = n_vectors(n)
    dev = values.device
    bound = int(lib().fls_encode_bound_words(n))
    out = torch.empty(bound + 4, dtype=torch.int32, device=dev)
    meta = torch.empty(nv * 4, dtype=torch.int32, device=dev)
    info = torch.empty(4, dtype=torch.int64, device=dev)  # the call sets all four words
    schemes = torch.empty(nv, dtype=torch.uint8, device=dev)
    ws_bytes = int(lib().fls_encode_learned_workspace_bytes(n))
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    check(lib().fls_encode_learned_gpu(values.data_ptr(), n, params.data_ptr(), threshold, kappa, layout,
                                       out.data_ptr(), bound + 4, meta.data_ptr(), info.data_ptr(), schemes.data_ptr(),
                                       ws.data_ptr(), ws_bytes, torch.cuda.current_stream().cuda_stream),
          "fls_encode_learned_gpu")
    pending = PendingEncode(out, meta, info, schemes, n, layout, compact)
    return pending if defer else pending.finish()


@dataclass
class RforColumn:
    """A column in the reference's tile-based run-length format (RFOR,
    tile_based/src/rlebinpack.cpp): per 512-value tile the runs' values and
    lengths, each FOR bit-packed in its own stream, with per-tile word
    offsets into both streams."""
    values: np.ndarray       # uint32 value stream
    run_lengths: np.ndarray  # uint32 run-length stream
    val_offsets: np.ndarray  # uint32, tiles + 1
    rl_offsets: np.ndarray   # uint32, tiles + 1
    n_values: int

    @property
    def n_tiles(self) -> int:
        return (self.n_values + _lib.RFOR_TILE - 1) // _lib.RFOR_TILE

    @property
    def nbytes(self) -> int:
        """Encoded bytes a decode reads: both streams and both offset arrays."""
        return 4 * (self.values.size + self.run_lengths.size + self.val_offsets.size + self.rl_offsets.size)

    @classmethod
    def encode(cls, values: np.ndarray) -> "RforColumn":
        v = np.ascontiguousarray(values).view(np.uint32)
        n = int(v.size)
        bound = int(lib().fls_rfor_bound_words(n))
        tiles = (n + _lib.RFOR_TILE - 1) // _lib.RFOR_TILE
        vs, rs = np.zeros(bound, np.uint32), np.zeros(bound, np.uint32)
        vo, ro = np.zeros(tiles + 1, np.uint32), np.zeros(tiles + 1, np.uint32)
        nv, nr = ctypes.c_uint64(), ctypes.c_uint64()
        check(lib().fls_rfor_encode(_ptr(v), n, _ptr(vs), _ptr(rs), _ptr(vo), _ptr(ro), ctypes.addressof(nv),
                                    ctypes.addressof(nr)), "fls_rfor_encode")
        return cls(vs[:nv.value].copy(), rs[:nr.value].copy(), vo, ro, n)

    def to_device(self, device=None) -> "DeviceRforColumn":
        return DeviceRforColumn(self, device)


class DeviceRforColumn:
    """An RforColumn in device memory, with its C descriptor."""

    def __init__(self, col: RforColumn, device=None):
        import torch
        dev = torch.device("cuda") if device is None else torch.device(device)
        self.host = col
        t = lambda a: torch.from_numpy(a.view(np.int32)).to(dev)  # noqa: E731
        self.values, self.run_lengths = t(col.values), t(col.run_lengths)
        self.val_offsets, self.rl_offsets = t(col.val_offsets), t(col.rl_offsets)
        self.desc = _lib.RforColumnDesc(values=self.values.data_ptr(), run_lengths=self.run_lengths.data_ptr(),
                                        val_offsets=self.val_offsets.data_ptr(), rl_offsets=self.rl_offsets.data_ptr(),
                                        n_values=col.n_values, n_val_words=int(col.values.size),
                                        n_rl_words=int(col.run_lengths.size))

    @property
    def n_values(self) -> int:
        return self.host.n_values

    @property
    def nbytes(self) -> int:
        return self.host.nbytes


def _aligned16(n: int) -> np.ndarray:
    """A uint8 array of n bytes starting on a 16-byte boundary."""
    raw = np.zeros(n + 16, dtype=np.uint8)
    off = (-raw.ctypes.data) % 16
    return raw[off: off + n]


def columns_array(cols) -> ctypes.Array:
    arr = (Column * len(cols))()
    for i, c in enumerate(cols):
        arr[i] = c.desc
    return arr


__all__ = ["EncodedColumn", "DeviceColumn", "DeviceUniformColumn", "DeviceEncodedColumn", "RforColumn",
           "DeviceRforColumn", "encode_column_gpu", "encode_column_learned_gpu",
           "META_DTYPE", "columns_array",
           "n_vectors", "_lib",
           "SCHEME_DELTA", "LAYOUT_TRANSPOSED"]
