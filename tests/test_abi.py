"""CPU tests of the C ABI boundary: the library loads, exports every symbol
include/raft_b200.h declares, and fails without a GPU by raising (never by
exiting the process).  No compute call is made."""
import ctypes
import os
import re
import subprocess
import sys

import numpy as np
import pytest

from conftest import REPO

LIB = os.path.join(REPO, "ssc-raft_b200", "sscRaft", "lib", "libraft.so")
HDR = os.path.join(REPO, "include", "raft_b200.h")


def declared():
    src = open(HDR).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(?:void|int|long long)\s+\*?\s*([A-Za-z_]\w*)\s*\(", src)))


def test_header_declares_reference_entry_points():
    names = declared()
    for ref in ("getFBPMultiGPU", "getFilterLowPassMultiGPU", "getRadonRTMultiGPU",
                "get_tEM_RT_MultiGPU", "get_eEM_RT_MultiGPU", "raft_last_error"):
        assert ref in names


def test_library_exports_every_declared_symbol():
    out = subprocess.check_output(["nm", "-D", "--defined-only", LIB], text=True)
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [n for n in declared() if n not in exported]
    assert not missing, missing
    lib = ctypes.CDLL(LIB)
    for n in declared():
        assert hasattr(lib, n)


def test_library_is_sm100a_build():
    out = subprocess.check_output(["cuobjdump", "--list-elf", LIB], text=True)
    assert "sm_100a" in out


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="checks the no-GPU error path")
def test_no_gpu_raises_instead_of_exiting():
    code = (
        "import sys, numpy as np; sys.path.insert(0, %r)\n"
        "import sscRaft\n"
        "try:\n"
        "    sscRaft.fbp(np.zeros((1, 8, 16), np.float32), dic={'gpu': [0], 'angles[rad]': np.zeros(8)})\n"
        "except RuntimeError as e:\n"
        "    print('RAISED', e)\n"
        "print('ALIVE')\n" % os.path.join(REPO, "ssc-raft_b200"))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert "RAISED" in r.stdout and "ALIVE" in r.stdout, r.stdout + r.stderr


def test_invalid_parameters_are_reported():
    import sscRaft
    from sscRaft.rafttypes import libraft, _ptr
    buf = ctypes.create_string_buffer(256)
    pi = np.array([1, 10, 1, 1, 2, 0, 0, 7, 0, 0], np.int32)      # nrays < 2
    pf = np.array([0, 0, 1, 0, 1, 1, 0], np.float32)
    out = np.zeros(4, np.int32)
    assert libraft.raft_plan_window(_ptr(pf), _ptr(pi), 0, 0, _ptr(out)) == 1
    assert libraft.raft_last_error(buf, 256) == 1 and b"invalid sizes" in buf.value
    pi[0] = 64
    pi[7] = 12                                                     # unknown filter id
    assert libraft.raft_plan_window(_ptr(pf), _ptr(pi), 0, 0, _ptr(out)) == 1
    pi[7] = 7
    pf[4] = 0.0                                                    # pixel size 0
    assert libraft.raft_plan_window(_ptr(pf), _ptr(pi), 0, 0, _ptr(out)) == 1
    pf[4] = 1.0
    assert libraft.raft_plan_window(_ptr(pf), _ptr(pi), 0, 0, _ptr(out)) == 0
    assert libraft.raft_last_error(buf, 256) == 0


def test_device_entries_validate_arguments_before_any_gpu_call():
    """The device-pointer entry points refuse a bad operator/storage pair, a
    bad EM kind and null data pointers (when there are slices) with an error
    status and message -- checked before any device is touched, so this runs
    without a GPU.  An empty batch may pass null pointers."""
    import sscRaft  # noqa: F401  (binds the argtypes)
    from sscRaft.processing.alignments import rotationaxis  # noqa: F401
    from sscRaft.rafttypes import libraft, _ptr
    buf = ctypes.create_string_buffer(512)

    def err(rc):
        assert rc == 1
        assert libraft.raft_last_error(buf, 512) == 1
        return buf.value.decode()

    N, A, n = 64, 30, 2
    ang = np.linspace(0, np.pi, A, endpoint=False).astype(np.float32)
    pf = np.array([0, 0, 1, 0, 1, 1, 0], np.float32)
    pi = np.array([N, A, n, N, 2, 0, 0, 7, 0, 0], np.int32)
    fake = ctypes.c_void_p(16)          # never dereferenced: the calls stop before any device work
    for g, s in ((0, 1), (1, 0), (2, 0), (1, 3)):
        assert "geometry/store" in err(libraft.raft_fbp_device(0, fake, fake, _ptr(ang), _ptr(pf), _ptr(pi),
                                                               g, s, None))
    assert "null data pointer" in err(libraft.raft_fbp_device(0, None, fake, _ptr(ang), _ptr(pf), _ptr(pi),
                                                              0, 0, None))
    assert "kind" in err(libraft.raft_em_device(2, 0, fake, fake, fake, _ptr(ang), N, A, n, 1, None, 1, None))
    assert "null data pointer" in err(libraft.raft_em_device(0, 0, fake, fake, None, _ptr(ang), N, A, n, 1,
                                                             None, 1, None))
    assert "null data pointer" in err(libraft.raft_radon_device(0, fake, None, _ptr(ang), N, N, N, A, n, 1.0, 1.0,
                                                                None))
    assert "null data pointer" in err(libraft.raft_background_device(0, fake, None, fake, N, A, n, 1, 1, None))
    pb = np.array([N, A, n, N, 2, 0, 0, 7, 0, 0], np.int32)
    assert "null data pointer" in err(libraft.raft_bst_device(0, None, fake, _ptr(pf), _ptr(pb), None))
    pq = np.array([N, A, n, N, 1, 0, 0, 1, 2, 0, 0], np.int32)
    pqf = np.array([0.0, 0.0, 0.0], np.float32)
    assert "null data pointer" in err(libraft.raft_temfq_device(0, fake, fake, None, _ptr(ang), _ptr(pqf), _ptr(pq),
                                                                None))
    res = ctypes.c_double(0)
    assert "null data pointer" in err(libraft.raft_centersino_device(0, None, fake, fake, fake, 64, 64, 0,
                                                                     ctypes.byref(res), None))
    # an empty batch with null pointers passes the argument checks (it then
    # needs a device: without one the call reports that instead)
    pi[2] = 0
    if libraft.raft_fbp_device(0, None, None, _ptr(ang), _ptr(pf), _ptr(pi), 0, 0, None):
        libraft.raft_last_error(buf, 512)
        assert "null data pointer" not in buf.value.decode()
