"""Pointer alignment at the C ABI: the fused ZDT kernels read the spectrogram and write the
FDR in 8-byte pairs of floats, so a device pointer that is only 4-byte aligned (a float*
one element past an allocation's start) is rejected with FDR_ERR_INVALID_ARGUMENT before any
kernel is launched, and the workspace stays usable.  Every call below stops at the host
check; none reaches a kernel with the misaligned pointer."""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _misaligned(t):
    return C.c_void_p(t.data_ptr() + 4)


def test_fused_path_rejects_misaligned_pointers(fdr, oracle):
    L = fdr._lib
    lib = L.lib()
    Nf, Nt, Nr = 1 << 12, 16, 17
    spec, _ = oracle.synth_spectrogram(Nf, Nt, 2, 20.0, 20.0, 2.0, seed=5)
    d = fdr.as_device_f32(spec)
    ws = fdr.ZDTWorkspace(d, -1.0, 0.25, Nr)
    assert ws.fused
    big = torch.zeros(Nf * Nt + 8, dtype=torch.float32, device="cuda")  # room past the offset
    dst = torch.zeros(Nf * Nr + 8, dtype=torch.float32, device="cuda")
    s = fdr.arrays.stream_handle()
    torch.cuda.synchronize()

    def rejected(st):
        assert st == L.FDR_ERR_INVALID_ARGUMENT, st
        assert "8-byte aligned" in lib.fdr_last_error_string().decode()

    rejected(lib.fdr_zdt_input(ws._h, _misaligned(big), s))
    dests = (C.c_void_p * 1)(_misaligned(dst).value)
    rejected(lib.fdr_zdt_execute(ws._h, None, None, 1, dests, L.FDR_WINDOW_RECT, None, s))
    dests_ok = (C.c_void_p * 1)(dst.data_ptr())
    rejected(lib.fdr_zdt_execute(ws._h, _misaligned(big), None, 1, dests_ok, L.FDR_WINDOW_RECT,
                                 None, s))
    blocks = (C.c_int32 * 1)(0)
    rejected(lib.fdr_zdt_execute_blocks(ws._h, None, blocks, 1, _misaligned(dst),
                                        L.FDR_WINDOW_RECT, None, s))
    ch = (L.fdr_batch_channel * 1)()
    ch[0] = L.fdr_batch_channel(Nf, Nt, Nr, -1.0, 0.25, d.data_ptr(), _misaligned(dst).value)
    h = C.c_void_p()
    rejected(lib.fdr_batch_create(C.byref(h), ch, 1, 1, s))
    assert not h.value
    torch.cuda.synchronize()
    # the workspace still runs, and matches a fresh one
    a = fdr.zdtfdr(ws).cpu().numpy()
    b = fdr.zdtfdr(fdr.ZDTWorkspace(d, -1.0, 0.25, Nr)).cpu().numpy()
    fdr.fdrsynchronize()
    assert np.array_equal(a, b)
