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
