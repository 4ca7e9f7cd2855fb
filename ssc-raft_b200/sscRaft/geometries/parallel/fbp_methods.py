"""FBP wrappers (sscRaft/geometries/parallel/fbp_methods.py:4-205 of cnpem/ssc-raft)."""
from ...rafttypes import (CNICE, FilterNumber, GEOMETRY, STORE, _gpus, _ptr, check_error, libraft, logger)
import numpy


def _fbp_params(tomogram, dic):
    nrays = tomogram.shape[-1]
    nangles = tomogram.shape[-2]
    nslices = 1 if len(tomogram.shape) == 2 else tomogram.shape[0]
    filter_type = FilterNumber(dic['filter'])
    beta_delta = dic['beta/delta']
    regularization = dic['regularization']
    offset = dic['rotation axis offset']
    blocksize = dic['blocksize']
    energy = dic['energy[eV]']
    z2 = dic['z2[m]']
    pixelx, pixely = dic['detectorPixel[m]'], dic['detectorPixel[m]']
    if beta_delta != 0.0:                       # fbp_methods.py:57-62
        beta_delta = 1.0 / beta_delta
    else:
        beta_delta, z2, energy = 0.0, 0.0, 1.0
    padx, pady, padz = dic['padding'], 0, 0
    objsize = nrays
    param_int = CNICE(numpy.array([nrays, nangles, nslices, objsize, padx, pady, padz,
                                   filter_type, 0, blocksize]), numpy.int32)
    param_float = CNICE(numpy.array([beta_delta, regularization, energy, z2, pixelx, pixely,
                                     offset]), numpy.float32)
    return nrays, nangles, nslices, objsize, param_int, param_float


def fbpGPU(tomogram, angles, gpus, dic, obj=None):
    """Filtered backprojection of a parallel-beam tomogram [slices, angles, rays]
    (or [angles, rays]) -> object [z, y, x] (fbp_methods.py:4-103).

    Dictionary keys as the reference ('filter', 'detectorPixel[m]', 'beta/delta',
    'z2[m]', 'energy[eV]', 'regularization', 'padding', 'blocksize',
    'rotation axis offset'), plus the optional extensions
    'operator' ('nearest' = the reference's truncating backprojector [default],
    'linear' = linear interpolation with true ramp-family filters) and
    'precision' ('float32' [default] or 'bfloat16' filtered-sinogram storage,
    'linear' operator only; accumulation is always float32).
    """
    gpus_arr, ngpus = _gpus(gpus)
    nrays, nangles, nslices, objsize, param_int, param_float = _fbp_params(tomogram, dic)
    tomogram = CNICE(tomogram)
    if obj is None:
        obj = numpy.zeros([nslices, objsize, objsize], dtype=numpy.float32)
    obj = CNICE(obj)
    angles = CNICE(numpy.array(angles))
    operator = dic.get('operator', 'nearest')
    precision = dic.get('precision', 'float32')
    if operator not in GEOMETRY:
        raise ValueError(f"operator must be one of {list(GEOMETRY)}")
    geometry = GEOMETRY[operator]
    if geometry == 0:
        if precision != 'float32':
            raise ValueError("precision 'bfloat16' needs operator 'linear'")
        libraft.getFBPMultiGPU(_ptr(gpus_arr), ngpus, _ptr(obj), _ptr(tomogram), _ptr(angles),
                               _ptr(param_float), _ptr(param_int))
    else:
        if precision not in STORE:
            raise ValueError(f"precision must be one of {list(STORE)}")
        libraft.raft_fbp_ext(_ptr(gpus_arr), ngpus, _ptr(obj), _ptr(tomogram), _ptr(angles),
                             _ptr(param_float), _ptr(param_int), geometry, STORE[precision])
    check_error("fbpGPU")
    return obj


def bstGPU(tomogram, angles, gpus, dic, obj=None, nstreams=0):
    """FBP by the Backprojection Slice Theorem (fbp_methods.py:105-205 of the
    reference): same dictionary as fbpGPU; the rotation axis offset is
    truncated to an integer and the angles must be uniform over [0, pi)
    (fbp() passes linspace(0, pi, A, endpoint=False)).  The padded length
    N*(1+padding) must fit the shared-memory transforms: at most 14528 when its
    prime factors are 2, 3, 5, 7, about 7000 otherwise (Bluestein's algorithm).
    Returns obj [slices, N, N] (written in place when given)."""
    gpus_arr, ngpus = _gpus(gpus)
    nrays = tomogram.shape[-1]
    nangles = tomogram.shape[-2]
    nslices = 1 if len(tomogram.shape) == 2 else tomogram.shape[0]
    filter_type = FilterNumber(dic['filter'])
    beta_delta = dic['beta/delta']
    regularization = dic['regularization']
    offset = int(dic['rotation axis offset'])
    blocksize = dic['blocksize']
    energy = dic['energy[eV]']
    z2 = dic['z2[m]']
    pixelx, pixely = dic['detectorPixel[m]'], dic['detectorPixel[m]']
    if beta_delta != 0.0:
        beta_delta = 1.0 / beta_delta
    else:
        beta_delta, z2, energy = 0.0, 0.0, 1.0
    padx, pady, padz = dic['padding'], 0, 0
    objsize = nrays
    tomogram = CNICE(tomogram)
    if obj is None:
        obj = numpy.zeros([nslices, objsize, objsize], dtype=numpy.float32)
    obj = CNICE(obj)
    angles = CNICE(numpy.array(angles))
    param_int = CNICE(numpy.array([nrays, nangles, nslices, objsize, padx, pady, padz, filter_type, 0,
                                   blocksize]), numpy.int32)
    param_float = CNICE(numpy.array([beta_delta, regularization, energy, z2, pixelx, pixely, offset]),
                        numpy.float32)
    libraft.getBSTMultiGPU(_ptr(gpus_arr), ngpus, _ptr(obj), _ptr(tomogram), _ptr(angles), _ptr(param_float),
                           _ptr(param_int), int(nstreams))
    check_error("bstGPU")
    return obj
