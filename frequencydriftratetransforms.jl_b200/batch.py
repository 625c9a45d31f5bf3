"""Batches of coarse channels in one CUDA-graph launch (fdr_batch_* in the C ABI).

The reference computes one zdtfdr! per spectrogram and leaves the loop over coarse channels
to the pipeline (the reference's README.md:57-71).  ZDTBatch plans that loop once: channels of any shapes
(Nf, Nt, rate set) share fused plans by shape, run over several streams, are tuned by the
library's autotuner and replay as a single CUDA graph.
"""
from __future__ import annotations

import ctypes as C
from fractions import Fraction

import numpy as np
import torch

from . import _lib
from .arrays import as_device_f32, fortran_empty, stream_handle


class ZDTBatch:
    """``channels``: sequence of (spectrogram, r0, dr, Nr).  ``outputs[i]`` is channel i's
    (Nf, Nr) FDR, rewritten by every :meth:`launch`."""

    def __init__(self, channels, slots=4, stream=None):
        self.spectrograms, self.outputs = [], []
        arr = (_lib.fdr_batch_channel * len(channels))()
        for i, (spec, r0, dr, Nr) in enumerate(channels):
            x = as_device_f32(spec)
            out = fortran_empty(x.shape[0], int(Nr))
            self.spectrograms.append(x)
            self.outputs.append(out)
            arr[i] = _lib.fdr_batch_channel(x.shape[0], x.shape[1], int(Nr),
                                            float(np.float32(float(Fraction(r0)))),
                                            float(np.float32(float(Fraction(dr)))),
                                            x.data_ptr(), out.data_ptr())
        h = C.c_void_p()
        _lib.check(_lib.lib().fdr_batch_create(C.byref(h), arr, len(channels), int(slots),
                                               stream_handle(stream)))
        self._h = h

    def autotune(self, stream=None):
        _lib.check(_lib.lib().fdr_batch_autotune(self._h, stream_handle(stream)))
        return self.tuning()

    def capture(self, stream=None):
        s = stream if stream is not None else torch.cuda.current_stream()
        if s.cuda_stream == 0:
            raise _lib.FDRError(_lib.FDR_ERR_INVALID_ARGUMENT,
                                "capture needs a non-default stream (use torch.cuda.Stream())")
        _lib.check(_lib.lib().fdr_batch_capture(self._h, C.c_void_p(s.cuda_stream)))

    def launch(self, stream=None):
        _lib.check(_lib.lib().fdr_batch_launch(self._h, stream_handle(stream)))
        return self.outputs

    def tuning(self):
        g = (C.c_int * 64)()
        n, k = C.c_int(), C.c_int()
        _lib.check(_lib.lib().fdr_batch_get_tuning(self._h, g, 64, C.byref(n), C.byref(k)))
        return {"groups_per_shape": [g[i] for i in range(min(64, n.value))],
                "active_slots": k.value}

    def info(self):
        n, f, b = C.c_int64(), C.c_int64(), C.c_int64()
        c = C.c_int()
        _lib.check(_lib.lib().fdr_batch_info(self._h, C.byref(n), C.byref(f), C.byref(b), C.byref(c)))
        return {"channels": n.value, "fused": f.value, "bytes": b.value, "captured": bool(c.value)}

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.lib().fdr_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
