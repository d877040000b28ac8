"""huntian_b200: B200-native (sm_100a) halo-finding hot path of Huntian.jl.

Peak finding on the filtered density field and the radial-shell ellipsoidal collapse,
computed by libhuntian_b200.so (C ABI, include/huntian_b200.h).  This package is the
host-side mirror of the reference's GPU entry points; see host.py.
"""
from ._lib import (HT_CONV_CPU, HT_CONV_GPU, HT_MODE_BATCHED, HT_MODE_PLAIN, HTError,
                   LIB_PATH, RESULT_NAMES, RESULT_WIDTH, SYMBOLS)
from .host import (HaloFinder, PeakCandidate, ShellTables, analyse_peaks_gpu_cuda_multirf,
                   build_shell_tables, ir2min_of, nhunt_of, peak_find_tile_gpu)
from .tables import log_filterbank, read_filterbank, read_homeltab, write_homeltab
from . import bracket, catalog, collapse, dist

__all__ = ["HaloFinder", "PeakCandidate", "ShellTables", "build_shell_tables",
           "peak_find_tile_gpu",
           "analyse_peaks_gpu_cuda_multirf", "ir2min_of",
           "nhunt_of", "read_homeltab", "write_homeltab", "read_filterbank",
           "log_filterbank", "HTError", "LIB_PATH", "SYMBOLS", "RESULT_NAMES",
           "RESULT_WIDTH", "HT_CONV_GPU", "HT_CONV_CPU", "HT_MODE_PLAIN", "HT_MODE_BATCHED"]
