"""Ragged batches: many reconstruction requests of different sizes and angle
counts (FBP and emission EM) run together on one GPU (no reference
counterpart; the reference reconstructs one size per call).

Inputs and outputs are device arrays exposing ``data_ptr()`` (e.g. torch CUDA
tensors); angles are host arrays."""
import ctypes

import numpy

from ...rafttypes import GEOMETRY, STORE, FilterNumber, _ptr, check_error, libraft


class RaftRequest(ctypes.Structure):
    """Mirror of ``raft_request`` (include/raft_b200.h)."""
    _fields_ = [("kind", ctypes.c_int), ("nrays", ctypes.c_int), ("nangles", ctypes.c_int),
                ("pad", ctypes.c_int), ("filter", ctypes.c_int), ("niter", ctypes.c_int),
                ("pixel", ctypes.c_float), ("offset", ctypes.c_float),
                ("angles", ctypes.c_void_p), ("d_data", ctypes.c_void_p), ("d_out", ctypes.c_void_p)]


libraft.raft_ragged_device.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
libraft.raft_ragged_device.restype = ctypes.c_int


def reconstruct_ragged(requests, gpu=0, operator="nearest", precision="float32", stream=None):
    """Run a ragged batch.

    requests: list of dicts with keys
      kind ('fbp' | 'eem'), data (device [nangles, nrays]), out (device [nrays, nrays];
      eEM: initial guess in, result out), angles (host, radians),
      FBP: filter (name, default 'ramp'), padding (2), pixel (1.0), offset (0.0);
      eEM: iterations (equal for all eEM requests).
    Returns (latency_ms per request, total_ms), measured on the device from the batch start.
    """
    n = len(requests)
    arr = (RaftRequest * n)()
    keep = []
    for i, r in enumerate(requests):
        data, out = r["data"], r["out"]
        ang = numpy.ascontiguousarray(r["angles"], dtype=numpy.float32)
        keep.append(ang)
        A, N = int(data.shape[-2]), int(data.shape[-1])
        arr[i].kind = 0 if r["kind"] == "fbp" else 1
        arr[i].nrays, arr[i].nangles = N, A
        arr[i].pad = int(r.get("padding", 2))
        arr[i].filter = FilterNumber(r.get("filter", "ramp"))
        arr[i].niter = int(r.get("iterations", 0))
        arr[i].pixel = float(r.get("pixel", 1.0))
        arr[i].offset = float(r.get("offset", 0.0))
        arr[i].angles = ang.ctypes.data
        arr[i].d_data = data.data_ptr()
        arr[i].d_out = out.data_ptr()
    lat = numpy.zeros(n, numpy.float64)
    tot = numpy.zeros(1, numpy.float64)
    g = GEOMETRY[operator]
    st = 0 if g == 0 else STORE[precision]
    rc = libraft.raft_ragged_device(gpu, ctypes.cast(arr, ctypes.c_void_p), n, g, st, _ptr(lat), _ptr(tot),
                                    stream)
    if rc:
        check_error("reconstruct_ragged")
    return lat, float(tot[0])
