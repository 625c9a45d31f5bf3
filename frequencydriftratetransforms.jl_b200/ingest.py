"""Spectrogram ingest and a multi-coarse-channel drift search.

The reference's own data path reads a rawspec product with HDF5 (test/heavytests.jl:11-14:
``h5["data"][freq_range, 1, :]``, a (channel, IF, time) view of a (time, IF, channel)
dataset) and leaves the search pipeline to DopplerDriftSearchPipeline.jl (the reference's README.md:68-71).
HDF5 with the bitshuffle filter needs libhdf5 and its plugin, which this environment does
not have; rawspec writes the same spectra as SIGPROC filterbank files, which are read here:
a keyword header (HEADER_START ... HEADER_END) followed by time-major samples, each
``nifs * nchans`` values of ``nbits`` bits.

``SearchPipeline`` runs zdtfdr! + findprotohits + proto-hit clustering over the coarse
channels of a file: each coarse channel's spectrogram (Nf fine channels x Nt steps, Julia
column-major layout, which is exactly the time-major file layout of that channel range) is
gathered by a pool of host threads into one of two pinned host buffers, copied to the
device on a copy stream, and searched on the compute stream while the next channel is
gathered.
"""
from __future__ import annotations

import os
import struct
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import torch

from . import _lib
from .arrays import fortran_empty
from .fdrutils import cluster_protohits
from .zdt import ZDTWorkspace, zdtfdr_protohits_

# SIGPROC header keywords and their value types
_INT = {"telescope_id", "machine_id", "data_type", "barycentric", "pulsarcentric", "nbits",
        "nsamples", "nchans", "nifs", "nbeams", "ibeam"}
_DOUBLE = {"az_start", "za_start", "src_raj", "src_dej", "tstart", "tsamp", "fch1", "foff",
           "refdm", "period"}
_STRING = {"rawdatafile", "source_name"}


def _put_str(fh, s):
    b = s.encode()
    fh.write(struct.pack("<i", len(b)))
    fh.write(b)


def _get_str(fh):
    (n,) = struct.unpack("<i", fh.read(4))
    if not 0 < n < 256:
        raise ValueError("not a SIGPROC filterbank header")
    return fh.read(n).decode()


def write_filterbank(path, header, data):
    """Write ``data`` (nsamples x nifs x nchans, float32 / uint8 / uint16 per header nbits)
    with ``header`` (dict of SIGPROC keywords; nbits, nchans, nifs are set from data)."""
    data = np.asarray(data)
    if data.ndim == 2:
        data = data[:, None, :]
    dt = {32: np.float32, 16: np.uint16, 8: np.uint8}
    hdr = dict(header)
    hdr["nchans"], hdr["nifs"] = int(data.shape[2]), int(data.shape[1])
    hdr.setdefault("nbits", 32)
    data = data.astype(dt[hdr["nbits"]], copy=False)
    with open(path, "wb") as fh:
        _put_str(fh, "HEADER_START")
        for k, v in hdr.items():
            _put_str(fh, k)
            if k in _INT:
                fh.write(struct.pack("<i", int(v)))
            elif k in _DOUBLE:
                fh.write(struct.pack("<d", float(v)))
            elif k in _STRING:
                _put_str(fh, str(v))
            else:
                raise ValueError(f"unknown SIGPROC keyword {k!r}")
        _put_str(fh, "HEADER_END")
        fh.write(np.ascontiguousarray(data).tobytes())


class Filterbank:
    """A SIGPROC filterbank file: ``header`` (dict) and ``data``, a read-only memory map of
    shape (nsamples, nifs, nchans)."""

    def __init__(self, path):
        with open(path, "rb") as fh:
            if _get_str(fh) != "HEADER_START":
                raise ValueError(f"{path}: not a SIGPROC filterbank file")
            hdr = {}
            while True:
                k = _get_str(fh)
                if k == "HEADER_END":
                    break
                if k in _INT:
                    hdr[k] = struct.unpack("<i", fh.read(4))[0]
                elif k in _DOUBLE:
                    hdr[k] = struct.unpack("<d", fh.read(8))[0]
                elif k in _STRING:
                    hdr[k] = _get_str(fh)
                else:
                    raise ValueError(f"{path}: unknown SIGPROC keyword {k!r}")
            off = fh.tell()
        self.path, self.header = path, hdr
        nbits, nchans, nifs = hdr.get("nbits", 32), hdr["nchans"], hdr.get("nifs", 1)
        dt = {32: np.float32, 16: np.uint16, 8: np.uint8}[nbits]
        nbytes = os.path.getsize(path) - off
        per = nchans * nifs * np.dtype(dt).itemsize
        self.nsamples = nbytes // per
        self.data = np.memmap(path, dtype=dt, mode="r", offset=off,
                              shape=(self.nsamples, nifs, nchans))

    @property
    def nchans(self):
        return self.header["nchans"]

    def spectrogram(self, lo, hi, ifno=0, t0=0, nt=None, out=None):
        """Channels [lo, hi) of IF ``ifno``, steps [t0, t0+nt): an (hi-lo, nt) float32 array
        in Julia's column-major layout (frequency fastest), as heavytests.jl:14 slices."""
        nt = self.nsamples - t0 if nt is None else nt
        src = self.data[t0:t0 + nt, ifno, lo:hi]
        if out is None:
            out = np.empty((nt, hi - lo), dtype=np.float32)
        else:
            out = out.reshape(nt, hi - lo)
        out[...] = src
        return out.T  # (Nf, Nt) view with column-major strides


class SearchPipeline:
    """Doppler drift search over coarse channels: for each coarse channel (``nfpc`` fine
    channels of a Filterbank), zdtfdr! over the rates r0 + j*dr (j < Nr), findprotohits at
    ``snr`` and proto-hit clustering (di, dj); host->device copies double-buffered against
    the device work."""

    def __init__(self, nfpc, nt, r0, dr, Nr, snr=10.0, di=1, dj=1):
        self.nfpc, self.nt, self.snr, self.di, self.dj = nfpc, nt, snr, di, dj
        self.ws = ZDTWorkspace(None, r0, dr, Nr, shape=(nfpc, nt))
        self.dest = fortran_empty(nfpc, Nr)
        self.pinned = [torch.empty(nfpc * nt, dtype=torch.float32).pin_memory() for _ in range(2)]
        self.dev = [torch.empty(nfpc * nt, dtype=torch.float32, device="cuda") for _ in range(2)]
        self.copy_stream = torch.cuda.Stream()
        self.ready = [torch.cuda.Event(), torch.cuda.Event()]
        self.nthreads = max(1, min(8, os.cpu_count() or 1))
        self.pool = ThreadPoolExecutor(max_workers=self.nthreads)
        self.r0, self.dr, self.Nr = r0, dr, Nr

    def _spec_view(self, k):
        return self.dev[k].view(self.nt, self.nfpc).t()  # (Nf, Nt), column-major

    def search_channel(self, spec):
        """Proto-hits and clusters of one device spectrogram."""
        hits = zdtfdr_protohits_(self.dest, self.ws, spec, threshold=self.snr, snr=True)
        labels, clusters = cluster_protohits(hits, self.nfpc, self.Nr, self.di, self.dj, fdr=self.dest)
        return hits, labels, clusters

    def _gather(self, fb, c, k, ifno, t0):
        """Copy coarse channel c into pinned buffer k, the time steps split over the pool."""
        out = self.pinned[k].numpy().reshape(self.nt, self.nfpc)
        lo, hi = c * self.nfpc, (c + 1) * self.nfpc
        step = max(1, self.nt // self.nthreads)

        def rows(a, b):
            out[a:b] = fb.data[t0 + a:t0 + b, ifno, lo:hi]

        return [self.pool.submit(rows, a, min(self.nt, a + step)) for a in range(0, self.nt, step)]

    def _copy(self, k, futures):
        for f in futures:
            f.result()
        with torch.cuda.stream(self.copy_stream):
            self.dev[k].copy_(self.pinned[k], non_blocking=True)
            self.ready[k].record(self.copy_stream)

    def run(self, fb, channels=None, ifno=0, t0=0):
        """Search the coarse channels ``channels`` (default: all) of Filterbank ``fb``;
        returns a list of (channel, hits, labels, clusters).  While channel i is searched,
        host threads gather channel i+1 into the other pinned buffer; its copy to the
        device is issued as soon as the gather is done."""
        nco = fb.nchans // self.nfpc
        channels = list(range(nco)) if channels is None else list(channels)
        if fb.nsamples - t0 < self.nt:
            raise ValueError("the file holds fewer time steps than the pipeline's Nt")
        results = []
        if getattr(fb, "decodes_on_device", False):  # HDF5 products: chunks decoded on the device
            for c in channels:
                spec = fb.spectrogram(c * self.nfpc, (c + 1) * self.nfpc, ifno, t0, self.nt,
                                      out=self.dev[0])
                results.append((c,) + self.search_channel(spec))
            return results
        cur = torch.cuda.current_stream()
        if channels:
            self._copy(0, self._gather(fb, channels[0], 0, ifno, t0))
        for i, c in enumerate(channels):
            k = i % 2
            nxt = None
            if i + 1 < len(channels):
                # buffer 1-k was last used by channel i-1, whose search has returned (it
                # synchronises), so both its pinned and its device copy are free
                nxt = self._gather(fb, channels[i + 1], 1 - k, ifno, t0)
            cur.wait_event(self.ready[k])
            hits, labels, clusters = self.search_channel(self._spec_view(k))
            results.append((c, hits, labels, clusters))
            if nxt is not None:
                self._copy(1 - k, nxt)
        return results

    def hit_table(self, fb, results):
        """Clusters as physical quantities: coarse channel, peak fine channel, frequency of the
        peak (fch1 + foff * channel, header units), drift rate (Hz/s from foff in MHz and tsamp
        in s), peak FDR value and proto-hit count."""
        foff, fch1, tsamp = fb.header.get("foff", 1.0), fb.header.get("fch1", 0.0), fb.header.get("tsamp", 1.0)
        rows = []
        for c, _, _, cl in results:
            for k in cl:
                ch = c * self.nfpc + int(k["peak_i"])
                rate = self.r0 + int(k["peak_j"]) * self.dr
                rows.append({"coarse": c, "channel": ch, "freq": fch1 + foff * ch,
                             "rate_ch_per_step": rate, "drift_hz_per_s": rate * foff * 1e6 / tsamp,
                             "peak": float(k["peak_value"]), "count": int(k["count"])})
        return rows
