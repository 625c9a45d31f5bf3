"""FDR utilities (src/fdrutils.jl) over the C ABI."""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .arrays import as_device_f32, fortran_empty, host_hit_buffer, ptr, stream_handle


def _mats(fdr):
    if isinstance(fdr, torch.Tensor):
        return [fdr], True
    return list(fdr), False


def _ptr_array(mats):
    return (C.c_void_p * len(mats))(*[m.data_ptr() for m in mats])


def create_fdr(spectrogram, Nr_or_rates):
    """create_fdr (fdrutils.jl:11-26): uninitialised (Nf, Nr) float32 device matrix."""
    Nr = Nr_or_rates if isinstance(Nr_or_rates, int) else len(Nr_or_rates)
    return fortran_empty(spectrogram.shape[0], Nr)


def fdrstats(fdr, stream=None):
    """fdrstats (fdrutils.jl:39-50) -> (m, s) as float32 values, computed on the device in
    Float32 in the order of the reference's pairwise sums (fdr_stats)."""
    mats, _ = _mats(fdr)
    Nf, Nrb = mats[0].shape
    m, s = C.c_double(), C.c_double()
    _lib.check(_lib.lib().fdr_stats(_ptr_array(mats), len(mats), Nf, Nrb, C.byref(m),
                                    C.byref(s), stream_handle(stream)))
    return np.float32(m.value), np.float32(s.value)


def fdrnormalize(x, m, s):
    """fdrnormalize(scalar, m, s) (fdrutils.jl:65-68)."""
    return (x - m) / s


def fdrnormalize_(fdr, m=None, s=None, stream=None):
    """fdrnormalize! (fdrutils.jl:70-90), in place on one matrix or a list of them."""
    mats, single = _mats(fdr)
    if m is None or s is None:
        m, s = fdrstats(fdr, stream)
    Nf, Nrb = mats[0].shape
    _lib.check(_lib.lib().fdr_normalize(_ptr_array(mats), len(mats), Nf, Nrb,
                                        float(np.float32(m)), float(np.float32(s)),
                                        stream_handle(stream)))
    return fdr


def fdrdenormalize(snr, m_or_fdr, s=None, stream=None):
    """fdrdenormalize (fdrutils.jl:104-119): snr*s + m in Julia's promoted type -- Float32
    for an integer or numpy float32 snr with Float32 m and s (each operation rounded),
    Float64 for a Python float snr."""
    if s is None:
        m, s = fdrstats(m_or_fdr, stream)
    else:
        m = m_or_fdr
    if (isinstance(snr, (bool, int, np.integer, np.float32)) and isinstance(m, np.float32)
            and isinstance(s, np.float32)):
        return np.float32(np.float32(np.float32(snr) * s) + m)
    return float(snr) * float(s) + float(m)


def fdrsynchronize(_type=None):
    """fdrsynchronize (fdrutils.jl:129-130; CuArray method ext:26-28)."""
    _lib.check(_lib.lib().fdr_synchronize(C.c_void_p(None)))


def findprotohits(fdr, threshold, snr=False, capacity=None, stream=None, return_threshold=False):
    """findprotohits (fdrutils.jl:148-169) -> int64 numpy array (nhits, 2) of ZERO-based
    (i, j) in column-major order (j offset by b*Nrb for the b-th matrix of a list).  With
    ``snr`` the threshold is fdrdenormalize(threshold, fdr) in the type Julia promotes
    ``threshold`` to: an int (or numpy float32) threshold gives Float32 arithmetic and
    comparison, a float gives Float64."""
    mats, _ = _mats(fdr)
    Nf, Nrb = mats[0].shape
    for mm in mats:
        if tuple(mm.shape) != (Nf, Nrb):
            raise _lib.FDRError(_lib.FDR_ERR_INVALID_ARGUMENT, "matrices differ in size")
    if capacity is None:
        capacity = 1 << 20
    while True:
        hits = host_hit_buffer(capacity)
        count = C.c_int64()
        thr = C.c_double()
        st = _lib.lib().fdr_findprotohits(_ptr_array(mats), len(mats), Nf, Nrb,
                                          float(threshold), _lib.snr_mode(threshold, snr), ptr(hits),
                                          capacity, C.byref(count), C.byref(thr),
                                          stream_handle(stream))
        if st == _lib.FDR_ERR_CAPACITY:
            capacity = int(count.value)
            continue
        _lib.check(st)
        break
    out = hits[: count.value].numpy().copy()
    return (out, thr.value) if return_threshold else out


CLUSTER_DTYPE = np.dtype([("peak_i", "<i8"), ("peak_j", "<i8"), ("peak_value", "<f4"),
                          ("reserved", "<i4"), ("count", "<i8"), ("i_min", "<i8"), ("i_max", "<i8"),
                          ("j_min", "<i8"), ("j_max", "<i8"), ("first", "<i8")])


def cluster_protohits(hits, Nf, Nj, di=1, dj=1, fdr=None, capacity=None, stream=None):
    """Clusters of proto-hits (fdr_cluster_protohits): the connected components of ``hits``
    (zero-based (i, j) pairs in the column-major order findprotohits returns, numpy or a
    CUDA int64 tensor) where proto-hits within di channels and dj drift-rate columns touch.
    ``fdr`` (one matrix or a list of rate batches covering the Nj columns) supplies the peak
    values.  Returns (labels, clusters): per-hit cluster numbers (numpy int64) and a numpy
    structured array with peak_i, peak_j, peak_value, count, i_min, i_max, j_min, j_max,
    first, ordered by each cluster's first proto-hit."""
    if isinstance(hits, torch.Tensor):
        h = hits.to(device="cuda", dtype=torch.int64).reshape(-1, 2).contiguous()
    else:
        h = torch.from_numpy(np.ascontiguousarray(np.asarray(hits, dtype=np.int64).reshape(-1, 2))).cuda()
    n = h.shape[0]
    if n == 0:
        return np.zeros(0, np.int64), np.zeros(0, CLUSTER_DTYPE)
    if fdr is not None:
        mats, _ = _mats(fdr)
        arr, nb, Nrb = _ptr_array(mats), len(mats), mats[0].shape[1]
    else:
        arr, nb, Nrb = None, 0, 0
    labels = torch.empty(n, dtype=torch.int64, device="cuda")
    cap = n if capacity is None else int(capacity)
    out = torch.empty((max(1, cap), CLUSTER_DTYPE.itemsize), dtype=torch.uint8, device="cuda")
    count = C.c_int64()
    _lib.check(_lib.lib().fdr_cluster_protohits(ptr(h), n, int(Nf), int(Nj), int(di), int(dj), arr,
                                                nb, Nrb, ptr(labels), ptr(out), cap, C.byref(count),
                                                stream_handle(stream)))
    clusters = np.frombuffer(out[: count.value].cpu().numpy().tobytes(), dtype=CLUSTER_DTYPE)
    return labels.cpu().numpy(), clusters
