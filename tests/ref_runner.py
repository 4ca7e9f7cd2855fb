"""Run one call of the REFERENCE library (oracle/_ref/libraft_ref.so, built
from the reference's own CUDA sources) in a process of its own, so that its
exports never meet this repository's libraft.so in one address space.

    python tests/ref_runner.py fbp|bst|eem IN.npz OUT.npz

IN.npz holds the arguments with the reference's packing (`sino`, `angles`,
`paramf`, `parami`); OUT.npz receives `out`.  Test infrastructure only."""
import ctypes
import os
import sys

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(REPO, "oracle", "_ref", "libraft_ref.so")


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def run_fbp(d):
    """getFBPMultiGPU (fbp.cu:238-302) on GPU 0 with host buffers."""
    lib = ctypes.CDLL(REF_LIB)
    P, I = ctypes.c_void_p, ctypes.c_int
    lib.getFBPMultiGPU.argtypes = [P, I, P, P, P, P, P]
    sino = np.ascontiguousarray(d["sino"], np.float32)
    ang = np.ascontiguousarray(d["angles"], np.float32)
    pf = np.ascontiguousarray(d["paramf"], np.float32)
    pi = np.ascontiguousarray(d["parami"], np.int32)
    No = int(pi[3])
    obj = np.zeros((sino.shape[0], No, No), np.float32)
    g = np.array([0], np.intc)
    lib.getFBPMultiGPU(_p(g), 1, _p(obj), _p(sino), _p(ang), _p(pf), _p(pi))
    return obj


def run_bst(d):
    """getBSTMultiGPU (bst.cu:674-734) on GPU 0 with host buffers."""
    lib = ctypes.CDLL(REF_LIB)
    P, I = ctypes.c_void_p, ctypes.c_int
    lib.getBSTMultiGPU.argtypes = [P, I, P, P, P, P, P, I]
    sino = np.ascontiguousarray(d["sino"], np.float32)
    ang = np.ascontiguousarray(d["angles"], np.float32)
    pf = np.ascontiguousarray(d["paramf"], np.float32)
    pi = np.ascontiguousarray(d["parami"], np.int32)
    obj = np.zeros((sino.shape[0], int(pi[3]), int(pi[3])), np.float32)
    g = np.array([0], np.intc)
    lib.getBSTMultiGPU(_p(g), 1, _p(obj), _p(sino), _p(ang), _p(pf), _p(pi), 0)
    return obj


def run_eem(d):
    """get_eEM_RT_MultiGPU (em_rt.cu:201-262) on GPU 0 from the uniform start."""
    lib = ctypes.CDLL(REF_LIB)
    P, I = ctypes.c_void_p, ctypes.c_int
    lib.get_eEM_RT_MultiGPU.argtypes = [P, I, P, P, P, P, P]
    tomo = np.ascontiguousarray(d["tomo"], np.float32)
    ang = np.ascontiguousarray(d["angles"], np.float32)
    B, A, N = tomo.shape
    pi = np.array([N, A, B, N, 0, 0, 0, 1, int(d["iterations"]), 0], np.int32)
    pf = np.zeros(1, np.float32)
    obj = np.ones((B, N, N), np.float32)
    g = np.array([0], np.intc)
    lib.get_eEM_RT_MultiGPU(_p(g), 1, _p(obj), _p(tomo), _p(ang), _p(pf), _p(pi))
    return obj


def main():
    kind, src, dst = sys.argv[1:4]
    d = np.load(src)
    out = {"fbp": run_fbp, "bst": run_bst, "eem": run_eem}[kind](d)
    np.savez(dst, out=out)


if __name__ == "__main__":
    main()
