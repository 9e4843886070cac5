"""The encoded-column container (fls_column_write_container /
fls_column_open_container) on the host: round trips of uniform and
per-vector columns of every scheme, and refusal of damaged, truncated,
foreign or inconsistent bytes -- including metadata that points outside the
payload under valid checksums, and every single-bit change of the footer."""
import struct

import numpy as np
import pytest

from fastlanesgpu_b200 import EncodedColumn, FlsError, datagen
from fastlanesgpu_b200._lib import (LAYOUT_NORMAL, LAYOUT_TRANSPOSED, SCHEME_CONST, SCHEME_DELTA, SCHEME_DICT,
                                    SCHEME_FOR, SCHEME_RLE)

FOOTER = 96
CRC_FOOTER = 68  # footer offset of the footer's own checksum


def _crc32c(data: bytes) -> int:
    poly, c = 0x82F63B78, 0xFFFFFFFF
    table = []
    for i in range(256):
        x = i
        for _ in range(8):
            x = (x >> 1) ^ poly if x & 1 else x >> 1
        table.append(x)
    for byte in data:
        c = table[(c ^ byte) & 0xFF] ^ (c >> 8)
    return c ^ 0xFFFFFFFF


def _reseal(d: bytearray):
    """Recomputes the footer checksum after a deliberate change of a footer
    field, so the open reaches the checks behind it."""
    foot = len(d) - FOOTER
    struct.pack_into("<I", d, foot + CRC_FOOTER, 0)
    struct.pack_into("<I", d, foot + CRC_FOOTER, _crc32c(bytes(d[foot:])))


def _same(a: EncodedColumn, b: EncodedColumn):
    assert np.array_equal(a.words, b.words)
    assert (a.meta is None) == (b.meta is None)
    if a.meta is not None:
        assert a.meta.tobytes() == b.meta.tobytes()
    for f in ("n_values", "layout", "scheme", "bw", "base", "max_vec_words", "scheme_mask"):
        assert getattr(a, f) == getattr(b, f), f


def _columns():
    vals = datagen.for_bitpack_mixed(10 * 1024 + 333, seed=2)
    yield EncodedColumn.uniform(vals)
    yield EncodedColumn.uniform(datagen.sorted_geometric(5000, seed=1), SCHEME_DELTA, layout=LAYOUT_TRANSPOSED)
    yield EncodedColumn.encode(vals, SCHEME_FOR)
    yield EncodedColumn.encode(datagen.sorted_geometric(7 * 1024 + 5, seed=4), SCHEME_DELTA, layout=LAYOUT_TRANSPOSED)
    yield EncodedColumn.encode(datagen.geometric_runs(9000, seed=5), SCHEME_RLE, layout=LAYOUT_TRANSPOSED)
    yield EncodedColumn.encode(np.full(3000, 77, np.int32), SCHEME_CONST)
    yield EncodedColumn.encode(np.random.default_rng(3).integers(0, 300, 4100).astype(np.int32), SCHEME_DICT,
                               layout=LAYOUT_TRANSPOSED)
    from fastlanesgpu_b200.selector import training_corpus
    from fastlanesgpu_b200 import ops
    corpus = training_corpus(200, seed=8)
    _, best = ops.encode_exhaustive(corpus)
    yield EncodedColumn.encode(corpus, best, layout=LAYOUT_TRANSPOSED)


@pytest.mark.parametrize("i", range(8))
def test_round_trip(i, tmp_path):
    col = list(_columns())[i]
    b = col.to_bytes()
    assert len(b) % 16 == 0 and b[-8:] == b"FLSCOLv1"
    _same(col, EncodedColumn.from_bytes(b))
    p = tmp_path / "c.flsc"
    col.save(str(p))
    _same(col, EncodedColumn.load(str(p)))


def _per_vector():
    return EncodedColumn.encode(datagen.geometric_runs(6 * 1024, seed=9), SCHEME_RLE, layout=LAYOUT_TRANSPOSED)


def _refused(b, status=1, text=""):
    with pytest.raises(FlsError) as e:
        EncodedColumn.from_bytes(bytes(b))
    assert e.value.status == status and text in str(e.value)


def test_damaged_bytes_are_refused():
    b = bytearray(_per_vector().to_bytes())
    for pos, text in ((5, "payload checksum"), (len(b) - FOOTER - 3, "metadata checksum")):
        d = bytearray(b)
        d[pos] ^= 0x40
        _refused(d, 1, text)
    _refused(b[:-1], 1)                       # truncated: footer no longer at the end
    _refused(b[:50], 1)
    _refused(b"x" * 10, 1)
    d = bytearray(b)
    d[-8:] = b"NOTACOL!"
    _refused(d, 1, "magic")
    d = bytearray(b)
    d[-12:-8] = struct.pack("<I", 1)          # version field of the footer (1: no footer checksum)
    _refused(d, 7, "version")


def test_metadata_outside_payload_is_refused_despite_checksums():
    col = _per_vector()
    b = bytearray(col.to_bytes())
    n_vec = col.n_vec
    foot = len(b) - FOOTER
    n_words, _, meta_off = struct.unpack_from("<QQQ", b, foot + 8)
    for field, value in (("offset", n_words + 4), ("offset", 2), ("scheme", 9), ("bw", 40), ("aux", 0)):
        d = bytearray(b)
        rec = meta_off + 16 * (n_vec - 1)
        if field == "offset":
            struct.pack_into("<Q", d, rec, value)
        elif field == "scheme":
            d[rec + 12] = value
        elif field == "bw":
            d[rec + 13] = value
        else:
            struct.pack_into("<H", d, rec + 14, value)
        struct.pack_into("<I", d, foot + 64, _crc32c(bytes(d[meta_off: meta_off + 16 * n_vec])))
        _reseal(d)
        _refused(d, 1, "vector")


def test_inconsistent_description_is_refused():
    col = EncodedColumn.uniform(datagen.uniform_bits(4096, 12, seed=1), bw=12)
    b = bytearray(col.to_bytes())
    foot = len(b) - FOOTER
    d = bytearray(b)
    struct.pack_into("<I", d, foot + 40, 30)           # bit width larger than the payload holds
    _reseal(d)
    _refused(d, 1, "uniform")
    d = bytearray(b)
    struct.pack_into("<Q", d, foot + 0, 10 ** 7)       # rows the payload does not hold
    _reseal(d)
    _refused(d, 1)
    d = bytearray(b)
    struct.pack_into("<I", d, foot + 32, 5)            # layout
    _reseal(d)
    _refused(d, 1)
    d = bytearray(b)
    struct.pack_into("<I", d, foot + 72, 1)            # reserved word
    _reseal(d)
    _refused(d, 1, "inconsistent")


def test_row_count_that_would_wrap_is_refused():
    """A resealed footer whose row count makes (vector count x words per
    vector) wrap modulo 2^64 -- a uniform 32-bit DELTA column of about 1.8e19
    rows -- is refused (the library caps columns at FLS_MAX_VALUES = 2^40
    rows and compares sizes by division), as is a row count at the cap that
    the payload does not hold."""
    col = EncodedColumn.uniform(datagen.sorted_geometric(4096, seed=1), SCHEME_DELTA, layout=LAYOUT_TRANSPOSED)
    assert col.bw <= 32
    b = bytearray(col.to_bytes())
    foot = len(b) - FOOTER
    struct.pack_into("<I", b, foot + 40, 32)              # bit width 32: 1056 words per vector
    n_vec = (1 << 64) // 1056 + 1                          # n_vec * 1056 wraps to a few words
    assert (n_vec * 1056) % (1 << 64) < 4096 and n_vec * 1024 < (1 << 64)
    for n_values, vec in ((n_vec * 1024, n_vec), (1 << 40, 1 << 30), ((1 << 40) + 1, (1 << 30) + 1)):
        d = bytearray(b)
        struct.pack_into("<Q", d, foot + 0, n_values)
        struct.pack_into("<Q", d, foot + 16, vec)
        _reseal(d)
        _refused(d, 1)


def test_writer_refuses_what_the_reader_refuses():
    """The writer checks the same column description as the reader before
    writing any byte: a uniform DELTA column in the normal layout, a bit
    width above 32 and a payload too small for the rows are refused at write
    time."""
    for field, value in (("layout", LAYOUT_NORMAL), ("bw", 33), ("n_values", 10 ** 6)):
        col = EncodedColumn.uniform(datagen.sorted_geometric(4096, seed=1), SCHEME_DELTA, layout=LAYOUT_TRANSPOSED)
        setattr(col, field, value)
        with pytest.raises(FlsError) as e:
            col.to_bytes()
        assert e.value.status == 1 and "container" in str(e.value)


@pytest.mark.parametrize("uniform", [True, False])
def test_every_footer_bit_flip_is_refused(uniform):
    """A damaged descriptor would decode to other values without any fault
    (a FOR base, the layout, the row count), so the footer carries its own
    checksum: each of its 768 single-bit changes is refused."""
    col = EncodedColumn.uniform(datagen.uniform_bits(3000, 9, seed=3), bw=9) if uniform else _per_vector()
    b = col.to_bytes()
    foot = len(b) - FOOTER
    for bit in range(8 * FOOTER):
        d = bytearray(b)
        d[foot + bit // 8] ^= 1 << (bit % 8)
        with pytest.raises(FlsError):
            EncodedColumn.from_bytes(bytes(d))
    d = bytearray(b)
    struct.pack_into("<i", d, foot + 44, col.base + 1)  # the FOR base alone
    _refused(d, 1, "footer checksum")


def test_random_bit_flips_are_refused_or_harmless():
    """Seeded single-bit changes anywhere in a per-vector container: refused,
    or (in the zero padding between payload and metadata, which nothing
    reads) the same column."""
    col = _per_vector()
    b = col.to_bytes()
    g = np.random.default_rng(11)
    for pos in g.integers(0, len(b), 400):
        d = bytearray(b)
        d[int(pos)] ^= 1 << int(g.integers(0, 8))
        try:
            got = EncodedColumn.from_bytes(bytes(d))
        except FlsError:
            continue
        _same(col, got)
