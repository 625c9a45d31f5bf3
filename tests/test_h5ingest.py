"""CPU tests of the HDF5 filterbank ingest (the data path of test/heavytests.jl:11-14):
the library's host LZ4 block codec against hand-worked blocks, the oracle's restatement and
the system LZ4 library when present; the bitshuffle transpose against hand-worked vectors;
and the HDF5 structure reader on files the writer produces (no kernels launched)."""
import ctypes as C
import ctypes.util
import os

import numpy as np
import pytest


def _lz4_dec(lib, blob, cap):
    src = np.frombuffer(bytes(blob), dtype=np.uint8) if len(blob) else np.zeros(1, np.uint8)
    out = np.empty(max(1, cap), np.uint8)
    n = C.c_int64()
    st = lib.fdr_lz4_decompress(src.ctypes.data, len(blob), out.ctypes.data, cap, C.byref(n))
    return st, out[:n.value].tobytes()


def _lz4_enc(lib, data):
    src = np.frombuffer(bytes(data), dtype=np.uint8) if len(data) else np.zeros(1, np.uint8)
    cap = len(data) + len(data) // 255 + 16
    out = np.empty(cap, np.uint8)
    n = C.c_int64()
    assert lib.fdr_lz4_compress(src.ctypes.data, len(data), out.ctypes.data, cap, C.byref(n)) == 0
    return out[:n.value].tobytes()


# LZ4 blocks worked by hand from the block format: token = (literals << 4) | (match - 4),
# 15 in a nibble continues in following bytes, then the literals, a 2-byte little-endian
# offset and (last sequence) no match.
HAND_LZ4 = [
    (bytes([0x50]) + b"hello", b"hello"),                        # literals only
    (bytes([0x14]) + b"a" + bytes([1, 0]), b"a" * 9),           # match of 8 at offset 1
    (bytes([0x20]) + b"ab", b"ab"),
    (bytes([0x2F]) + b"ab" + bytes([2, 0, 3]) + bytes([0x10]) + b"z", b"ab" * 12 + b"z"),  # 4+15+3 = 22
    (bytes([0xF0, 1]) + b"0123456789abcdef", b"0123456789abcdef"),  # 15 + 1 literals
]


def test_lz4_hand_blocks(fdr, oracle):
    lib = fdr._lib.lib()
    for blob, want in HAND_LZ4:
        st, got = _lz4_dec(lib, blob, len(want))
        assert st == 0 and got == want
        assert oracle.lz4_block_decode(blob) == want


def test_lz4_malformed_blocks_are_rejected(fdr):
    lib = fdr._lib.lib()
    for blob, cap in [(bytes([0x14]) + b"a" + bytes([0, 0]), 16),   # offset 0
                      (bytes([0x14]) + b"a" + bytes([2, 0]), 16),   # offset before the start
                      (bytes([0x50]) + b"hel", 16),                  # truncated literals
                      (bytes([0x14]) + b"a" + bytes([1]), 16),       # truncated offset
                      (bytes([0x14]) + b"a" + bytes([1, 0]), 5)]:    # output beyond capacity
        st, _ = _lz4_dec(lib, blob, cap)
        assert st == fdr._lib.FDR_ERR_INVALID_ARGUMENT


def _samples():
    rng = np.random.default_rng(7)
    x = rng.exponential(1.0, 50000).astype(np.float32).tobytes()
    return [b"", b"a", b"abcd" * 3, bytes(1000), x, bytes(rng.integers(0, 4, 70000, dtype=np.uint8)),
            b"the quick brown fox jumps over the lazy dog " * 300]


def test_lz4_round_trip_and_oracle(fdr, oracle):
    lib = fdr._lib.lib()
    for data in _samples():
        blob = _lz4_enc(lib, data)
        st, got = _lz4_dec(lib, blob, len(data))
        assert st == 0 and got == data
        if data:
            assert oracle.lz4_block_decode(blob) == data


def test_lz4_against_the_system_library(fdr):
    name = ctypes.util.find_library("lz4") or "liblz4.so.1"
    try:
        sys_lz4 = C.CDLL(name)
    except OSError:
        pytest.skip("no system LZ4 library")
    sys_lz4.LZ4_compress_default.restype = C.c_int
    sys_lz4.LZ4_decompress_safe.restype = C.c_int
    lib = fdr._lib.lib()
    for data in _samples()[1:]:
        src = np.frombuffer(data, np.uint8)
        cap = len(data) + len(data) // 255 + 16
        buf = np.empty(cap, np.uint8)
        n = sys_lz4.LZ4_compress_default(C.c_void_p(src.ctypes.data), C.c_void_p(buf.ctypes.data),
                                         len(data), cap)
        assert n > 0
        st, got = _lz4_dec(lib, buf[:n].tobytes(), len(data))   # theirs -> ours
        assert st == 0 and got == data
        ours = np.frombuffer(_lz4_enc(lib, data), np.uint8)        # ours -> theirs
        back = np.empty(len(data), np.uint8)
        m = sys_lz4.LZ4_decompress_safe(C.c_void_p(ours.ctypes.data), C.c_void_p(back.ctypes.data),
                                        len(ours), len(data))
        assert m == len(data) and back.tobytes() == data


def test_bitshuffle_hand_vectors(oracle, fdr):
    # 8 one-byte elements: bit-row k holds bit k of every element, element e at bit e
    assert oracle.bitshuffle_block(bytes([1, 0, 0, 0, 0, 0, 0, 0]), 1) == bytes([1, 0, 0, 0, 0, 0, 0, 0])
    assert oracle.bitshuffle_block(bytes([0xFF, 0, 0, 0, 0, 0, 0, 0]), 1) == bytes([1] * 8)
    assert oracle.bitshuffle_block(bytes([0, 0x80, 0, 0, 0, 0, 0, 0]), 1) == bytes([0] * 7 + [2])
    # float32 1.0 = 0x3F800000 in every element: byte 2 bit 7 and byte 3 bits 0..5 set
    one = np.ones(8, np.float32).tobytes()
    rows = oracle.bitshuffle_block(one, 4)
    want = bytearray(32)
    want[8 * 2 + 7] = 0xFF
    for k in range(6):
        want[8 * 3 + k] = 0xFF
    assert rows == bytes(want)
    x = np.random.default_rng(2).standard_normal(4096).astype(np.float32).tobytes()
    assert oracle.bitunshuffle_block(oracle.bitshuffle_block(x, 4), 4) == x
    # the writer's forward transform equals the oracle's, block by block and with a raw tail
    from importlib import import_module
    h5 = import_module(fdr.__name__ + ".h5")
    y = np.random.default_rng(3).standard_normal(1000 + 5).astype(np.float32).tobytes()
    sh = h5._bitshuffle_host(y, 4, 256)
    exp = b"".join(oracle.bitshuffle_block(y[e * 4:min(1000, e + 256) * 4], 4) for e in range(0, 1000, 256))
    assert sh == exp + y[4000:]


@pytest.mark.parametrize("shape,chunk", [((16, 1, 70000), (16, 1, 1 << 14)), ((7, 2, 3001), (3, 1, 1000)),
                                         ((16, 1, 1 << 17), None)])
def test_fbh5_structure_and_chunks(fdr, oracle, tmp_path, shape, chunk):
    rng = np.random.default_rng(sum(shape))
    data = rng.exponential(1.0, shape).astype(np.float32)
    hdr = {"fch1": 8400.0, "foff": -2.7939677238464355e-06, "tsamp": 18.253611008, "nbits": 32,
           "nchans": shape[2], "source_name": "VOYAGER-1"}
    path = str(tmp_path / "t.h5")
    fdr.write_fbh5(path, hdr, data, chunk=chunk)
    f = fdr.H5File(path)
    assert f.root["attributes"] == {"CLASS": "FILTERBANK", "VERSION": "1.0"}
    ds = f.dataset("data")
    assert list(ds.shape) == list(shape) and ds.dtype == np.dtype("<f4")
    assert ds.maxshape[0] == 2 ** 64 - 1  # unlimited time axis
    assert ds.attrs == hdr
    assert ds.filters == [{"id": 32008, "flags": 1, "cd": [0, 3, 4, 0, 2]}]
    lib = fdr._lib.lib()
    ch = ds.chunk
    n = int(np.prod(ch))
    got = np.zeros([-(-s // c) * c for s, c in zip(shape, ch)], np.float32)
    for offs, (addr, size, mask) in ds.chunks().items():
        raw = np.frombuffer(f.buf, dtype=np.uint8, count=size, offset=addr)
        ref = oracle.bitshuffle_lz4_decode_chunk(raw.tobytes(), 4)  # the oracle decodes
        out = np.empty(n * 4, np.uint8)
        nb, bel = C.c_int64(), C.c_int64()
        assert lib.fdr_bitshuffle_lz4_decode(raw.ctypes.data, size, 4, out.ctypes.data, n * 4,
                                             C.byref(nb), C.byref(bel)) == 0
        assert nb.value == n * 4 and bel.value == 2048
        whole = n - n % 8  # the library's output is still bit-transposed per block
        unsh = b"".join(oracle.bitunshuffle_block(out[e * 4:min(whole, e + 2048) * 4].tobytes(), 4)
                        for e in range(0, whole, 2048)) + out[whole * 4:].tobytes()
        assert unsh == ref
        got[tuple(slice(o, o + c) for o, c in zip(offs, ch))] = np.frombuffer(ref, np.float32).reshape(ch)
    assert np.array_equal(got[:shape[0], :shape[1], :shape[2]], data)
    f.close()


def test_fbh5_rejects_other_formats(fdr, tmp_path):
    p = tmp_path / "x.h5"
    p.write_bytes(b"\x89HDF\r\n\x1a\n" + bytes([2]) + bytes(100))
    with pytest.raises(fdr.H5FormatError):
        fdr.H5File(str(p))
    p.write_bytes(b"not hdf5" * 100)
    with pytest.raises(fdr.H5FormatError):
        fdr.H5File(str(p))
