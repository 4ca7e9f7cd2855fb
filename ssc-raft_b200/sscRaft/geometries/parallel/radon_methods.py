"""Radon transform wrapper (sscRaft/geometries/parallel/radon_methods.py:3-61 of cnpem/ssc-raft)."""
from ...rafttypes import CNICE, _gpus, _ptr, check_error, libraft
import numpy


def radon_RT(phantom, angles, gpus, pixel=1.0):
    """Ray-tracing Radon transform of a 3-D phantom [slices, y, x] ->
    [slices, angles, x], scaled by nrays*pixel/2 as the reference does."""
    a = 1.0
    gpus_arr, ngpus = _gpus(gpus)
    nslices = 1 if len(phantom.shape) == 2 else phantom.shape[0]
    nrays = phantom.shape[2]
    _, img_sizey, img_sizex = phantom.shape
    phantom = CNICE(phantom)
    angles = CNICE(numpy.array(angles))
    nangles = angles.shape[0]
    tomogram = -numpy.ones((nslices, nangles, nrays), dtype=numpy.float32)
    libraft.getRadonRTMultiGPU(_ptr(gpus_arr), ngpus, _ptr(tomogram), _ptr(phantom), _ptr(angles),
                               img_sizex, img_sizey, nrays, nangles, nslices, a, a)
    check_error("radon_RT")
    return tomogram * nrays * pixel / 2
