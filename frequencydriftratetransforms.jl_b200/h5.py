"""HDF5 filterbank products (rawspec's "FBH5" files), read and written without libhdf5.

test/heavytests.jl:11-14 of FrequencyDriftRateTransforms.jl reads a rawspec product with
HDF5.jl and H5Zbitshuffle.jl: ``h5["data"][freq_range, 1, :]``, i.e. channels of IF 1 at all
time steps of the float32 dataset "data", stored in C order as (time, IF, channel) and
chunked with the bitshuffle filter (HDF5 filter 32008) using LZ4.  libhdf5 and the filter
plugin are not installed here, so this module reads the file structure itself, for the
layout rawspec writes with libhdf5's default (earliest) file format:

* superblock version 0 or 1 (root group symbol-table entry),
* version-1 object headers, with continuation blocks,
* groups as symbol tables (version-1 B-tree of group nodes, symbol-table nodes, local heap),
* dataspace, datatype (IEEE float, fixed-point, fixed-length string), data layout version 3
  (contiguous or chunked with a version-1 B-tree chunk index), filter pipeline versions 1
  and 2, attributes versions 1 and 2.

Chunks filtered by bitshuffle+LZ4 are decompressed on the host by the library
(fdr_bitshuffle_lz4_decode) and bit-transposed back to float32 on the device
(fdr_bitunshuffle); a chunk whose filter mask skips the filter is copied as stored.
``write_fbh5`` writes the same layout (used by the tests and by callers who convert
filterbank files).
"""
from __future__ import annotations

import ctypes as C
import mmap
import struct

import numpy as np
import torch

from . import _lib

UNDEF = 0xFFFFFFFFFFFFFFFF
SIGNATURE = b"\x89HDF\r\n\x1a\n"
BITSHUFFLE_FILTER = 32008
BITSHUFFLE_LZ4 = 2

# object header message types
_MSG_NIL, _MSG_DATASPACE, _MSG_DATATYPE, _MSG_FILL_OLD, _MSG_FILL = 0x0, 0x1, 0x3, 0x4, 0x5
_MSG_LAYOUT, _MSG_FILTERS, _MSG_ATTRIBUTE, _MSG_CONT, _MSG_SYMTAB = 0x8, 0xB, 0xC, 0x10, 0x11


class H5FormatError(ValueError):
    """The file uses an HDF5 feature outside the layout this reader supports."""


def _u(buf, off, n):
    return int.from_bytes(buf[off:off + n], "little")


def _pad8(n):
    return (n + 7) & ~7


def _parse_dataspace(d):
    ver = d[0]
    rank = d[1]
    flags = d[2]
    off = 8 if ver == 1 else 4
    dims = [_u(d, off + 8 * i, 8) for i in range(rank)]
    off += 8 * rank
    maxdims = None
    if flags & 1:
        maxdims = [_u(d, off + 8 * i, 8) for i in range(rank)]
    return dims, maxdims


def _parse_datatype(d):
    """numpy dtype (or ("S", n) for fixed-length strings) of a datatype message."""
    cls = d[0] & 0x0F
    bits0 = d[1]
    size = _u(d, 4, 4)
    if cls == 1:  # IEEE floating point
        if size not in (4, 8):
            raise H5FormatError(f"float of {size} bytes")
        return np.dtype((">" if bits0 & 1 else "<") + f"f{size}")
    if cls == 0:  # fixed-point
        signed = bool(bits0 & 0x08)
        return np.dtype((">" if bits0 & 1 else "<") + ("i" if signed else "u") + str(size))
    if cls == 3:  # fixed-length string
        return ("S", size)
    raise H5FormatError(f"datatype class {cls}")


def _datatype_len(d):
    """Encoded length of a datatype message (for attribute v2 payload offsets)."""
    cls = d[0] & 0x0F
    return 8 + {1: 12, 0: 4, 3: 0}.get(cls, 0)


def _parse_layout(d):
    ver = d[0]
    if ver != 3:
        raise H5FormatError(f"data layout message version {ver}")
    cls = d[1]
    if cls == 1:
        return {"class": "contiguous", "address": _u(d, 2, 8), "size": _u(d, 10, 8)}
    if cls == 2:
        nd = d[2]
        addr = _u(d, 3, 8)
        dims = [_u(d, 11 + 4 * i, 4) for i in range(nd)]
        return {"class": "chunked", "btree": addr, "chunk": dims[:-1], "elem": dims[-1]}
    if cls == 0:
        size = _u(d, 2, 2)
        return {"class": "compact", "data": bytes(d[4:4 + size])}
    raise H5FormatError(f"layout class {cls}")


def _parse_filters(d):
    ver, n = d[0], d[1]
    off = 8 if ver == 1 else 2
    out = []
    for _ in range(n):
        fid = _u(d, off, 2)
        off += 2
        nlen = 0
        if ver == 1 or fid >= 256:
            nlen = _u(d, off, 2)
            off += 2
        flags = _u(d, off, 2)
        ncd = _u(d, off + 2, 2)
        off += 4
        if nlen:
            off += _pad8(nlen) if ver == 1 else nlen
        cd = [_u(d, off + 4 * i, 4) for i in range(ncd)]
        off += 4 * ncd
        if ver == 1 and ncd % 2:
            off += 4
        out.append({"id": fid, "flags": flags, "cd": cd})
    return out


def _parse_attribute(d):
    ver = d[0]
    nsz, tsz, ssz = _u(d, 2, 2), _u(d, 4, 2), _u(d, 6, 2)
    off = 8 if ver in (1, 2) else 9
    pad = _pad8 if ver == 1 else (lambda x: x)
    name = bytes(d[off:off + nsz]).split(b"\0")[0].decode()
    off += pad(nsz)
    dt = d[off:off + tsz]
    off += pad(tsz)
    sp = d[off:off + ssz]
    off += pad(ssz)
    try:
        dtype = _parse_datatype(dt)
        dims, _ = _parse_dataspace(sp)
    except H5FormatError:
        return name, None  # variable-length strings and other types: not decoded
    count = int(np.prod(dims)) if dims else 1
    if isinstance(dtype, tuple):
        n = dtype[1]
        vals = [bytes(d[off + i * n:off + (i + 1) * n]).split(b"\0")[0].decode(errors="replace")
                for i in range(count)]
    else:
        vals = np.frombuffer(bytes(d[off:off + count * dtype.itemsize]), dtype=dtype).tolist()
    return name, (vals[0] if not dims else vals)


class H5File:
    """The structure of an HDF5 file (memory-mapped): ``root`` (attributes and members of
    the root group) and ``dataset(name)``."""

    def __init__(self, path):
        self.path = path
        with open(path, "rb") as fh:
            self.buf = mmap.mmap(fh.fileno(), 0, access=mmap.ACCESS_READ)
        b = self.buf
        base = None
        for off in [0] + [512 << i for i in range(20)]:  # the superblock may follow a user block
            if off + 8 <= len(b) and b[off:off + 8] == SIGNATURE:
                base = off
                break
        if base is None:
            raise H5FormatError(f"{path}: no HDF5 superblock")
        ver = b[base + 8]
        if ver not in (0, 1):
            raise H5FormatError(f"superblock version {ver} (files written with libver 'latest')")
        if b[base + 13] != 8 or b[base + 14] != 8:
            raise H5FormatError("offsets and lengths other than 8 bytes")
        p = base + 24 + (4 if ver == 1 else 0)
        self.base = _u(b, p, 8)  # base address of the file's addresses
        entry = p + 32            # root group symbol-table entry
        self.root_header = self.base + _u(b, entry + 8, 8)

    def close(self):
        try:
            self.buf.close()
        except BufferError:  # views of the mapping are still alive; it closes with them
            pass

    def _a(self, addr):
        return self.base + addr

    # -- object headers --------------------------------------------------------------
    def messages(self, addr):
        """(type, data) of every message of the version-1 object header at file offset addr,
        following continuation blocks."""
        b = self.buf
        if b[addr] != 1:
            raise H5FormatError(f"object header version {b[addr]} at {addr}")
        nmsg = _u(b, addr + 2, 2)
        blocks = [(addr + 16, _u(b, addr + 8, 4))]
        out = []
        while blocks and len(out) < nmsg:
            start, size = blocks.pop(0)
            p = start
            while p + 8 <= start + size and len(out) < nmsg:
                mtype, msize = _u(b, p, 2), _u(b, p + 2, 2)
                data = memoryview(b)[p + 8:p + 8 + msize]
                if mtype == _MSG_CONT:
                    blocks.append((self._a(_u(data, 0, 8)), _u(data, 8, 8)))
                out.append((mtype, data))
                p += 8 + msize
        return out

    def attributes(self, addr):
        return dict(_parse_attribute(d) for t, d in self.messages(addr) if t == _MSG_ATTRIBUTE)

    # -- groups ------------------------------------------------------------------------
    def members(self, addr):
        """name -> object header offset of a symbol-table group."""
        st = [d for t, d in self.messages(addr) if t == _MSG_SYMTAB]
        if not st:
            raise H5FormatError("group without a symbol table (compact or dense link storage)")
        btree, heap = self._a(_u(st[0], 0, 8)), self._a(_u(st[0], 8, 8))
        b = self.buf
        if b[heap:heap + 4] != b"HEAP":
            raise H5FormatError("bad local heap")
        heap_data = self._a(_u(b, heap + 24, 8))
        out = {}

        def name_at(off):
            end = b.find(b"\0", heap_data + off)
            return b[heap_data + off:end].decode()

        def walk(node):
            if b[node:node + 4] != b"TREE" or b[node + 4] != 0:
                raise H5FormatError("bad group B-tree node")
            level, n = b[node + 5], _u(b, node + 6, 2)
            for i in range(n):
                child = self._a(_u(b, node + 24 + 8 + 16 * i, 8))
                if level > 0:
                    walk(child)
                    continue
                if b[child:child + 4] != b"SNOD":
                    raise H5FormatError("bad symbol-table node")
                for k in range(_u(b, child + 6, 2)):
                    e = child + 8 + 40 * k
                    out[name_at(_u(b, e, 8))] = self._a(_u(b, e + 8, 8))

        walk(btree)
        return out

    @property
    def root(self):
        return {"attributes": self.attributes(self.root_header),
                "members": self.members(self.root_header)}

    def dataset(self, name):
        return H5Dataset(self, self.members(self.root_header)[name])


class H5Dataset:
    """A dataset: ``shape``, ``dtype``, ``attrs``, ``chunk`` and the chunk index."""

    def __init__(self, f, addr):
        self.f = f
        msgs = f.messages(addr)
        kinds = {t for t, _ in msgs}
        if _MSG_DATASPACE not in kinds or _MSG_DATATYPE not in kinds or _MSG_LAYOUT not in kinds:
            raise H5FormatError("not a dataset")
        for t, d in msgs:
            if t == _MSG_DATASPACE:
                self.shape, self.maxshape = _parse_dataspace(d)
            elif t == _MSG_DATATYPE:
                self.dtype = _parse_datatype(d)
            elif t == _MSG_LAYOUT:
                self.layout = _parse_layout(d)
        self.filters = next((_parse_filters(d) for t, d in msgs if t == _MSG_FILTERS), [])
        self.attrs = dict(_parse_attribute(d) for t, d in msgs if t == _MSG_ATTRIBUTE)
        self.chunk = self.layout.get("chunk")
        self._chunks = None

    def chunks(self):
        """{chunk offset tuple: (file offset, stored size, filter mask)} from the B-tree."""
        if self._chunks is not None:
            return self._chunks
        if self.layout["class"] != "chunked":
            raise H5FormatError("not chunked")
        b, f = self.f.buf, self.f
        rank = len(self.shape)
        ksz = 8 + 8 * (rank + 1)
        out = {}

        def walk(node):
            if b[node:node + 4] != b"TREE" or b[node + 4] != 1:
                raise H5FormatError("bad chunk B-tree node")
            level, n = b[node + 5], _u(b, node + 6, 2)
            p = node + 24
            for _ in range(n):
                size, mask = _u(b, p, 4), _u(b, p + 4, 4)
                offs = tuple(_u(b, p + 8 + 8 * i, 8) for i in range(rank))
                child = f._a(_u(b, p + ksz, 8))
                if level > 0:
                    walk(child)
                else:
                    out[offs] = (child, size, mask)
                p += ksz + 8

        walk(f._a(self.layout["btree"]))
        self._chunks = out
        return out

    def _bitshuffle(self):
        for i, flt in enumerate(self.filters):
            if flt["id"] == BITSHUFFLE_FILTER:
                return i, flt
        return None, None

    def read_chunk_device(self, offs, stage=None):
        """The chunk at offset tuple offs as a device tensor of self.chunk elements."""
        addr, size, mask = self.chunks()[offs]
        es = self.dtype.itemsize
        n = int(np.prod(self.chunk))
        raw = np.frombuffer(self.f.buf, dtype=np.uint8, count=size, offset=addr)
        fi, flt = self._bitshuffle()
        others = [x for x in self.filters if x["id"] != BITSHUFFLE_FILTER]
        if any(not (mask >> i) & 1 for i, x in enumerate(self.filters) if x["id"] != BITSHUFFLE_FILTER):
            raise H5FormatError(f"unsupported filters {[x['id'] for x in others]}")
        out = torch.empty(n * es, dtype=torch.uint8, device="cuda")
        if flt is None or (mask >> fi) & 1:
            out.copy_(torch.from_numpy(raw[:n * es].copy()))
            return out.view(_torch_dtype(self.dtype))
        host = torch.empty(n * es, dtype=torch.uint8).pin_memory() if stage is None else stage
        nbytes, bel = C.c_int64(), C.c_int64()
        comp = flt["cd"][4] if len(flt["cd"]) > 4 else BITSHUFFLE_LZ4
        if comp == BITSHUFFLE_LZ4:
            _lib.check(_lib.lib().fdr_bitshuffle_lz4_decode(
                raw.ctypes.data, size, es, host.data_ptr(), n * es, C.byref(nbytes), C.byref(bel)))
            if nbytes.value != n * es:
                raise H5FormatError(f"chunk decoded to {nbytes.value} bytes, expected {n * es}")
        elif comp == 0:  # bitshuffle alone: the default block of 8 KB (at least 128 elements)
            host[:n * es].copy_(torch.from_numpy(raw[:n * es].copy()))
            bs = flt["cd"][3] if len(flt["cd"]) > 3 and flt["cd"][3] else max(128, (8192 // es) // 8 * 8)
            bel.value = bs
        else:
            raise H5FormatError(f"bitshuffle compression {comp}")
        dev_in = host[:n * es].to("cuda", non_blocking=True)
        _lib.check(_lib.lib().fdr_bitunshuffle(dev_in.data_ptr(), n, es, bel.value, out.data_ptr(),
                                               C.c_void_p(torch.cuda.current_stream().cuda_stream)))
        return out.view(_torch_dtype(self.dtype))

    def read_device(self, sel):
        """dataset[sel] (a tuple of slices, C order) as a device tensor, decoding only the
        chunks that overlap the selection."""
        rank = len(self.shape)
        sl = [s.indices(self.shape[i]) for i, s in enumerate(sel)]
        if any(st != 1 for _, _, st in sl):
            raise ValueError("unit-step slices only")
        lo = [a for a, _, _ in sl]
        hi = [b for _, b, _ in sl]
        out = torch.empty([b - a for a, b in zip(lo, hi)], dtype=_torch_dtype(self.dtype), device="cuda")
        if self.layout["class"] == "contiguous":
            es = self.dtype.itemsize
            full = np.frombuffer(self.f.buf, dtype=self.dtype, count=int(np.prod(self.shape)),
                                 offset=self.f._a(self.layout["address"])).reshape(self.shape)
            out.copy_(torch.from_numpy(np.ascontiguousarray(full[tuple(slice(a, b) for a, b in zip(lo, hi))])))
            return out
        ch = self.chunk
        first = [a // c for a, c in zip(lo, ch)]
        last = [(b - 1) // c for b, c in zip(hi, ch)]
        stage = torch.empty(int(np.prod(ch)) * self.dtype.itemsize, dtype=torch.uint8).pin_memory()
        idx = [range(f0, l0 + 1) for f0, l0 in zip(first, last)]
        for cidx in np.ndindex(*[len(r) for r in idx]):
            offs = tuple((idx[i][cidx[i]]) * ch[i] for i in range(rank))
            if offs not in self.chunks():
                continue  # never written: the fill value (zero)
            blk = self.read_chunk_device(offs, stage).view(ch)
            torch.cuda.current_stream().synchronize()  # the staging buffer is reused
            src, dst = [], []
            for i in range(rank):
                a = max(lo[i], offs[i])
                b = min(hi[i], offs[i] + ch[i])
                src.append(slice(a - offs[i], b - offs[i]))
                dst.append(slice(a - lo[i], b - lo[i]))
            out[tuple(dst)] = blk[tuple(src)]
        return out


def _torch_dtype(dt):
    dt = np.dtype(dt)
    table = {np.dtype("<f4"): torch.float32, np.dtype("<f8"): torch.float64,
             np.dtype("u1"): torch.uint8}
    if dt not in table:
        raise H5FormatError(f"dataset element type {dt}")
    return table[dt]


class H5Filterbank:
    """A rawspec HDF5 filterbank product: ``header`` (the "data" dataset's attributes),
    ``nsamples``, ``nifs``, ``nchans`` and ``spectrogram`` (decoded on the device)."""

    decodes_on_device = True  # SearchPipeline reads its coarse channels with spectrogram()

    def __init__(self, path, dataset="data"):
        self.f = H5File(path)
        self.path = path
        self.ds = self.f.dataset(dataset)
        if len(self.ds.shape) != 3:
            raise H5FormatError(f"dataset shape {self.ds.shape}, expected (time, IF, channel)")
        self.nsamples, self.nifs, nch = self.ds.shape
        self.header = dict(self.ds.attrs)
        self.header.setdefault("nchans", nch)

    @property
    def nchans(self):
        return self.ds.shape[2]

    def spectrogram(self, lo, hi, ifno=0, t0=0, nt=None, out=None):
        """Channels [lo, hi) of IF ``ifno`` at steps [t0, t0+nt) as an (hi-lo, nt) float32
        CUDA tensor in Julia's column-major layout (frequency fastest), as heavytests.jl:14
        slices ``h5["data"][freq_range, 1, :]``.  ``out``, if given, is a device tensor of
        (hi-lo)*nt float32 that receives it."""
        nt = self.nsamples - t0 if nt is None else nt
        blk = self.ds.read_device((slice(t0, t0 + nt), slice(ifno, ifno + 1), slice(lo, hi)))
        blk = blk.reshape(nt, hi - lo).to(torch.float32)
        if out is None:
            out = torch.empty((nt, hi - lo), dtype=torch.float32, device="cuda")
        out = out.view(nt, hi - lo)
        out.copy_(blk)
        return out.t()

    def close(self):
        self.f.close()


# ----------------------------------------------------------------------------------------
# Writer: superblock 0, version-1 object headers, a symbol-table root group holding the
# chunked, bitshuffle+LZ4 filtered float32 dataset "data" (time, IF, channel) with the
# header fields as attributes -- the layout rawspec produces.
# ----------------------------------------------------------------------------------------

def _p8(b):
    return b + b"\0" * (_pad8(len(b)) - len(b))


def _msg(mtype, data, flags=0):
    data = _p8(data)
    return struct.pack("<HHB3x", mtype, len(data), flags) + data


def _object_header(msgs):
    body = b"".join(msgs)
    return struct.pack("<BBHII4x", 1, 0, len(msgs), 1, len(body)) + body


def _dt_f32():
    return bytes([0x11, 0x20, 0x1F, 0x00]) + struct.pack("<IHHBBBBI", 4, 0, 32, 23, 8, 0, 23, 127)


def _dt_f64():
    return bytes([0x11, 0x20, 0x3F, 0x00]) + struct.pack("<IHHBBBBI", 8, 0, 64, 52, 11, 0, 52, 1023)


def _dt_i32():
    return bytes([0x10, 0x08, 0x00, 0x00]) + struct.pack("<IHH", 4, 0, 32)


def _dt_str(n):
    return bytes([0x13, 0x00, 0x00, 0x00]) + struct.pack("<I", n)


_SCALAR = bytes([1, 0, 0, 0, 0, 0, 0, 0])


def _attribute(name, value):
    nm = name.encode() + b"\0"
    if isinstance(value, str):
        v = value.encode() + b"\0"
        dt, data = _dt_str(len(v)), v
    elif isinstance(value, (int, np.integer)) and not isinstance(value, bool):
        dt, data = _dt_i32(), struct.pack("<i", int(value))
    else:
        dt, data = _dt_f64(), struct.pack("<d", float(value))
    body = struct.pack("<BBHHH", 1, 0, len(nm), len(dt), len(_SCALAR)) + _p8(nm) + _p8(dt) + _p8(_SCALAR) + data
    return _msg(_MSG_ATTRIBUTE, body)


def _bitshuffle_host(raw, es, block_elems):
    """Bit transpose of each block (block_elems elements; the last holds the remaining whole
    groups of 8; the final elements mod 8 stay raw), the bitshuffle filter's forward step."""
    a = np.frombuffer(raw, dtype=np.uint8).reshape(-1, es)
    n = a.shape[0]
    whole = n - n % 8
    out = bytearray()
    for e0 in range(0, whole, block_elems):
        blk = a[e0:min(whole, e0 + block_elems)]
        planes = np.unpackbits(blk, axis=1, bitorder="little").reshape(len(blk), es * 8).T
        out += np.packbits(planes, axis=1, bitorder="little").tobytes()
    out += a[whole:].tobytes()
    return bytes(out)


def write_fbh5(path, header, data, chunk=None, block_elems=2048):
    """Write ``data`` (nsamples x nifs x nchans float32) as a rawspec-style HDF5 filterbank
    product: dataset "data" chunked as ``chunk`` (default: all steps, one IF, up to 2^16
    channels), each chunk bitshuffled in blocks of ``block_elems`` elements and LZ4
    compressed (filter 32008 with client data (0, 3, 4, 0, 2)); ``header`` fields (numbers
    and strings) become attributes of "data", CLASS and VERSION attributes of the root."""
    data = np.ascontiguousarray(np.asarray(data, dtype=np.float32))
    if data.ndim == 2:
        data = data[:, None, :]
    shape = data.shape
    chunk = tuple(chunk) if chunk else (shape[0], 1, min(shape[2], 1 << 16))
    es = 4
    # chunks, compressed
    grid = [-(-s // c) for s, c in zip(shape, chunk)]
    stored = []
    for idx in np.ndindex(*grid):
        offs = tuple(i * c for i, c in zip(idx, chunk))
        blk = np.zeros(chunk, dtype=np.float32)
        src = data[tuple(slice(o, min(o + c, s)) for o, c, s in zip(offs, chunk, shape))]
        blk[tuple(slice(0, n) for n in src.shape)] = src
        raw = blk.tobytes()
        sh = _bitshuffle_host(raw, es, block_elems)
        cap = 12 + (len(raw) // (block_elems * es) + 1) * (4 + block_elems * es + block_elems * es // 255 + 16) + 64
        buf = np.empty(cap, dtype=np.uint8)
        osz = C.c_int64()
        _lib.check(_lib.lib().fdr_bitshuffle_lz4_encode(sh, len(sh), es, block_elems, buf.ctypes.data,
                                                        cap, C.byref(osz)))
        stored.append((offs, buf[:osz.value].tobytes()))
    # addresses
    sb_size = 96
    root_msgs_wo = [_msg(_MSG_SYMTAB, bytes(16)), _attribute("CLASS", "FILTERBANK"),
                    _attribute("VERSION", "1.0")]
    root_addr = sb_size
    root_size = len(_object_header(root_msgs_wo))
    heap_addr = root_addr + root_size
    heap_data = b"\0" * 8 + _p8(b"data\0")
    gtree_addr = heap_addr + 32 + len(heap_data)
    gtree_size = 24 + 33 * 8 + 32 * 8
    snod_addr = gtree_addr + gtree_size
    snod_size = 8 + 8 * 40
    ds_addr = snod_addr + snod_size
    rank = 3
    dspace = struct.pack("<BBBB4x", 1, rank, 1, 0) + struct.pack("<3Q", *shape) + \
        struct.pack("<3Q", UNDEF, *shape[1:])
    fname = b"bitshuffle; see https://github.com/kiyo-masui/bitshuffle\0"
    cd = (0, 3, es, 0, BITSHUFFLE_LZ4)
    filt = struct.pack("<BB6x", 1, 1) + struct.pack("<HHHH", BITSHUFFLE_FILTER, len(fname), 1, len(cd)) + \
        _p8(fname) + struct.pack(f"<{len(cd)}I", *cd) + (b"\0" * 4 if len(cd) % 2 else b"")

    def ds_msgs(btree):
        layout = struct.pack("<BBB", 3, 2, rank + 1) + struct.pack("<Q", btree) + \
            struct.pack(f"<{rank + 1}I", *chunk, es)
        m = [_msg(_MSG_DATASPACE, dspace), _msg(_MSG_DATATYPE, _dt_f32(), 1),
             _msg(_MSG_FILL, bytes([2, 2, 2, 0])), _msg(_MSG_LAYOUT, layout),
             _msg(_MSG_FILTERS, filt)]
        for k, v in header.items():
            m.append(_attribute(k, v))
        return m

    ds_size = len(_object_header(ds_msgs(0)))
    ctree_addr = ds_addr + ds_size
    ksz = 8 + 8 * (rank + 1)
    node_size = 24 + 65 * ksz + 64 * 8
    nleaf = -(-len(stored) // 64)
    ntree = nleaf + (1 if nleaf > 1 else 0)
    data_addr = ctree_addr + ntree * node_size
    addrs = []
    a = data_addr
    for _, blob in stored:
        addrs.append(a)
        a += len(blob)
    eof = a

    def key(size, offs):
        return struct.pack("<II", size, 0) + struct.pack(f"<{rank + 1}Q", *offs, 0)

    def node(level, entries, upper):
        b = b"TREE" + struct.pack("<BBHQQ", 1, level, len(entries), UNDEF, UNDEF)
        for size, offs, child in entries:
            b += key(size, offs) + struct.pack("<Q", child)
        b += key(0, upper)
        return b + b"\0" * (node_size - len(b))

    leaves = []
    for i in range(nleaf):
        part = [(len(blob), offs, addrs[j]) for j, (offs, blob) in enumerate(stored)][64 * i:64 * (i + 1)]
        leaves.append(node(0, part, tuple(shape)))
    if nleaf > 1:
        if nleaf > 64:
            raise ValueError("more than 4096 chunks")
        leaf0 = ctree_addr + node_size
        root = node(1, [(0, stored[64 * i][0], leaf0 + i * node_size) for i in range(nleaf)], tuple(shape))
        trees = root + b"".join(leaves)
    else:
        trees = leaves[0]
    root_msgs = [_msg(_MSG_SYMTAB, struct.pack("<QQ", gtree_addr, heap_addr))] + root_msgs_wo[1:]
    out = bytearray()
    out += SIGNATURE + bytes([0, 0, 0, 0, 0, 8, 8, 0]) + struct.pack("<HHI", 4, 16, 0)
    out += struct.pack("<QQQQ", 0, UNDEF, eof, UNDEF)
    out += struct.pack("<QQII", 0, root_addr, 1, 0) + struct.pack("<QQ", gtree_addr, heap_addr)
    assert len(out) == sb_size
    out += _object_header(root_msgs)
    out += b"HEAP" + struct.pack("<B3xQQQ", 0, len(heap_data), UNDEF, heap_addr + 32) + heap_data
    gt = b"TREE" + struct.pack("<BBHQQ", 0, 0, 1, UNDEF, UNDEF) + struct.pack("<QQQ", 0, snod_addr, 8)
    out += gt + b"\0" * (gtree_size - len(gt))
    sn = b"SNOD" + struct.pack("<BBH", 1, 0, 1) + struct.pack("<QQII", 8, ds_addr, 0, 0) + bytes(16)
    out += sn + b"\0" * (snod_size - len(sn))
    out += _object_header(ds_msgs(ctree_addr))
    assert len(out) == ctree_addr
    out += trees
    assert len(out) == data_addr
    for _, blob in stored:
        out += blob
    with open(path, "wb") as fh:
        fh.write(out)
