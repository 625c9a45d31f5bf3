"""B200-native frequency-drift-rate (FDR) transforms.

Host-side mirror of FrequencyDriftRateTransforms.jl's API (src/FrequencyDriftRateTransforms.jl
exports, :3-24) over the C ABI of libfdrb200.so (include/fdr_b200.h).  Every transform runs
in the library's hand-written sm_100a CUDA kernels; torch supplies device memory and
streams.  Julia's mutating names end in "_" instead of "!".

Matrices use the reference's column-major layout: a logical (Nf, Nt) matrix is a torch
tensor of shape (Nf, Nt) with strides (1, Nf).  Returned indices are zero-based.
"""
from . import _lib
from ._lib import FDRError, CapacityError
from .arrays import fortran_empty, fortran_zeros, as_device_f32
from .zdtutils import calcNl, growNr, estimate_memory, driftrates
from .batchrates import batchrates, RateRange
from .zdt import (ZDTWorkspace, input_, preprocess_, convolve_, postprocess_, output_,
                  zdtfdr_, zdtfdr_nodest_, zdtfdr, zdtfdr_protohits_, zdtfdr_blocks_,
                  zdtfdr_blocks_protohits_, fused_split)
from .batch import ZDTBatch
from . import proposal
from . import ingest
from .ingest import Filterbank, SearchPipeline, write_filterbank
from .h5 import H5File, H5Filterbank, H5FormatError, write_fbh5
from .intfdr import intshift, intshift_, intfdr, intfdr_, taylor_shifts, taylorfdr, taylorfdr_
from .fftfdr import (FFTFDRWorkspace, fftfdr_workspace, fftfdr_workspace_, fdshiftsum,
                     fdshiftsum_, fdshift, fdshift_, fftfdr, fftfdr_)
from .fdrutils import (create_fdr, fdrstats, fdrnormalize, fdrnormalize_, fdrdenormalize,
                       fdrsynchronize, findprotohits, cluster_protohits)

_lib.load()  # fail loudly at import when the CUDA library is missing

__all__ = [
    "FDRError", "ingest", "Filterbank", "H5File", "H5Filterbank", "H5FormatError", "write_fbh5", "SearchPipeline", "write_filterbank", "taylor_shifts", "taylorfdr", "taylorfdr_", "CapacityError", "fortran_empty", "fortran_zeros", "as_device_f32",
    "calcNl", "growNr", "estimate_memory", "driftrates", "batchrates", "RateRange",
    "ZDTWorkspace", "input_", "preprocess_", "convolve_", "postprocess_", "output_",
    "zdtfdr_", "zdtfdr_nodest_", "zdtfdr", "zdtfdr_protohits_", "zdtfdr_blocks_",
    "zdtfdr_blocks_protohits_", "fused_split", "ZDTBatch", "proposal",
    "intshift", "intshift_", "intfdr", "intfdr_",
    "FFTFDRWorkspace", "fftfdr_workspace", "fftfdr_workspace_", "fdshiftsum", "fdshiftsum_",
    "fdshift", "fdshift_", "fftfdr", "fftfdr_",
    "create_fdr", "fdrstats", "fdrnormalize", "fdrnormalize_", "fdrdenormalize",
    "fdrsynchronize", "findprotohits", "cluster_protohits",
]
