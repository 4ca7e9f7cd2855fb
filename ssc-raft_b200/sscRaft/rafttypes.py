"""ctypes layer of the B200 sscRaft drop-in (mirrors sscRaft/rafttypes.py of
cnpem/ssc-raft: library loading, prototypes, CNICE, FilterNumber, logger).

Only the parallel-beam hot path is bound.  The shared library is
``sscRaft/lib/libraft.so`` (built by ``make -C ssc-raft_b200/csrc``); there is
no CPU fallback -- importing this module fails loudly if the library is
missing.  Unlike the reference module, no heavy optional packages (h5py,
skimage, matplotlib, SharedArray) are imported.
"""
import ctypes
import logging
import os
import sys

import numpy

logger = logging.getLogger("sscRaft")
if not logger.handlers:
    _h = logging.StreamHandler(sys.stdout)
    _h.setFormatter(logging.Formatter('%(asctime)s - %(name)s - %(levelname)s - %(message)s'))
    logger.addHandler(_h)
logger.setLevel(logging.WARNING)

_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libraft.so")


def load_library(path=_LIB_PATH):
    if not os.path.exists(path):
        raise OSError(f"sscRaft: CUDA library not built: {path} (run `make -C ssc-raft_b200/csrc`)")
    return ctypes.CDLL(path)


libraft = load_library()

_P = ctypes.c_void_p
_I = ctypes.c_int
_F = ctypes.c_float

# Reference prototypes (rafttypes.py:126-198,311-323 of cnpem/ssc-raft)
libraft.getFBPMultiGPU.argtypes = [_P, _I, _P, _P, _P, _P, _P]
libraft.getFBPMultiGPU.restype = None
libraft.getFilterLowPassMultiGPU.argtypes = [_P, _I, _P, _P, _P]
libraft.getFilterLowPassMultiGPU.restype = None
libraft.getRadonRTMultiGPU.argtypes = [_P, _I, _P, _P, _P, _I, _I, _I, _I, _I, _F, _F]
libraft.getRadonRTMultiGPU.restype = None
libraft.get_tEM_RT_MultiGPU.argtypes = [_P, _I, _P, _P, _P, _P, _P, _P]
libraft.get_tEM_RT_MultiGPU.restype = None
libraft.get_eEM_RT_MultiGPU.argtypes = [_P, _I, _P, _P, _P, _P, _P]
libraft.get_eEM_RT_MultiGPU.restype = None
libraft.getBSTMultiGPU.argtypes = [_P, _I, _P, _P, _P, _P, _P, _I]
libraft.getBSTMultiGPU.restype = None
libraft.get_tEM_FQ_MultiGPU.argtypes = [_P, _I, _P, _P, _P, _P, _P, _P]
libraft.get_tEM_FQ_MultiGPU.restype = None
libraft.getBackgroundCorrectionMultiGPU.argtypes = [_P, _I, _P, _P, _P, _I, _I, _I, _I, _I, _I]
libraft.getBackgroundCorrectionMultiGPU.restype = None
# Extensions
libraft.raft_last_error.argtypes = [ctypes.c_char_p, _I]
libraft.raft_last_error.restype = _I
libraft.raft_clear_error.argtypes = []
libraft.raft_clear_error.restype = None
libraft.raft_inject_alloc_failures.argtypes = [_I]
libraft.raft_inject_alloc_failures.restype = None
libraft.raft_selftest_bounded_wait.argtypes = [_I, _I, ctypes.c_uint]
libraft.raft_selftest_bounded_wait.restype = _I
libraft.raft_abi_version.argtypes = []
libraft.raft_abi_version.restype = _I
libraft.raft_fbp_ext.argtypes = [_P, _I, _P, _P, _P, _P, _P, _I, _I]
libraft.raft_fbp_ext.restype = _I
libraft.raft_fbp_device.argtypes = [_I, _P, _P, _P, _P, _P, _I, _I, _P]
libraft.raft_fbp_device.restype = _I
libraft.raft_fbp_device_noalloc.argtypes = [_I, _P, _P, _P, _P, _P, _I, _I, _P]
libraft.raft_fbp_device_noalloc.restype = _I
libraft.raft_em_ext.argtypes = [_I, _I, _P, _P, _P, _P, _I, _I, _I, _I, _P, _I]
libraft.raft_em_ext.restype = _I
libraft.raft_em_device.argtypes = [_I, _I, _P, _P, _P, _P, _I, _I, _I, _I, _P, _I, _P]
libraft.raft_radon_device.argtypes = [_I, _P, _P, _P, _I, _I, _I, _I, _I, _F, _F, _P]
libraft.raft_radon_device.restype = _I
libraft.raft_background_device.argtypes = [_I, _P, _P, _P, _I, _I, _I, _I, _I, _P]
libraft.raft_bst_device.argtypes = [_I, _P, _P, _P, _P, _P]
libraft.raft_bst_device.restype = _I
libraft.raft_temfq_device.argtypes = [_I, _P, _P, _P, _P, _P, _P, _P]
libraft.raft_temfq_device.restype = _I
libraft.raft_background_device.restype = _I
libraft.raft_em_device.restype = _I

libraft.raft_launch_count.argtypes = []
libraft.raft_launch_count.restype = ctypes.c_longlong
libraft.raft_autotune_table.argtypes = [ctypes.c_char_p, _I]
libraft.raft_autotune_table.restype = _I
libraft.raft_profile_enable.argtypes = [_I]
libraft.raft_profile_enable.restype = None
libraft.raft_profile_read.argtypes = [_P, _P, _I]
libraft.raft_profile_read.restype = _I
libraft.raft_filter_set_fixed.argtypes = [_I]
libraft.raft_filter_set_fixed.restype = _I

libraft.raft_slab_partition.argtypes = [_I, _I, _P, _P]
libraft.raft_slab_partition.restype = _I
libraft.raft_plan_window.argtypes = [_P, _P, _I, _I, _P]
libraft.raft_plan_window.restype = _I
libraft.raft_fast_sincos.argtypes = [_I, _P, _I, _I, _P, _P]
libraft.raft_fast_sincos.restype = _I

GEOMETRY = {"nearest": 0, "linear": 1}


def autotune_table():
    """Backprojector launch shapes chosen by the autotuner in this process."""
    import json
    buf = ctypes.create_string_buffer(1 << 16)
    libraft.raft_autotune_table(buf, 1 << 16)
    return json.loads(buf.value.decode() or "[]")


def fast_sincos(angles, kind=0, gpu=0):
    """(cos, sin) of angles with the GPU fast intrinsics (kind 0: __sinf/__cosf,
    1: __sincosf) -- the values the reference's index rules use."""
    a = numpy.ascontiguousarray(angles, dtype=numpy.float32)
    c = numpy.zeros_like(a)
    s = numpy.zeros_like(a)
    libraft.raft_fast_sincos(gpu, _ptr(a), a.size, kind, _ptr(c), _ptr(s))
    check_error("fast_sincos")
    return c, s
STORE = {"float32": 1, "bfloat16": 2}


def check_error(what=""):
    """Raise RuntimeError if the last library call on this thread failed."""
    buf = ctypes.create_string_buffer(1024)
    if libraft.raft_last_error(buf, 1024):
        msg = buf.value.decode(errors="replace")
        logger.error(f"{what}: {msg}")
        raise RuntimeError(f"sscRaft {what}: {msg}")


def CNICE(darray, dtype=numpy.float32):
    """Contiguous copy in dtype only when needed (rafttypes.py:485-491)."""
    if darray.dtype != dtype:
        return numpy.ascontiguousarray(darray.astype(dtype))
    elif darray.flags['C_CONTIGUOUS'] is False:
        return numpy.ascontiguousarray(darray)
    else:
        return darray


def FilterNumber(mfilter):
    """Filter name -> id (rafttypes.py:501-519); unknown names map to hamming
    as in the reference.  'shepp-logan' (9) is new."""
    table = {'none': 0, 'gaussian': 1, 'lorentz': 2, 'cosine': 3, 'rectangle': 4,
             'hann': 5, 'hamming': 6, 'ramp': 7, 'shepp-logan': 9, 'shepp_logan': 9}
    return table.get(str(mfilter).lower(), 6)


def setInterpolation(name):
    if name.lower() == 'nearest':
        return 0
    elif name.lower() == 'bilinear':
        return 1
    logger.warning("Interpolation invalid. Using default 'nearest' interpolation.")
    return 0


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _gpus(gpus):
    g = numpy.ascontiguousarray(numpy.array(gpus).astype(numpy.intc))
    return g, len(g)
