"""EM wrappers (sscRaft/geometries/parallel/em_methods.py:3-151 of cnpem/ssc-raft)."""
from ...rafttypes import CNICE, _gpus, _ptr, check_error, libraft
import numpy


def _em_params(nrays, nangles, nslices, objsize, nflats, iterations, blocksize):
    param_int = CNICE(numpy.array([nrays, nangles, nslices, objsize, 0, 0, 0, nflats,
                                   iterations, blocksize]), numpy.int32)
    param_float = CNICE(numpy.array([0]), numpy.float32)
    return param_int, param_float


def eEMRT_GPU_(tomo, angles, iterations, gpus, blocksize, obj=None):
    """Emission EM with ray-tracing operators; obj is the initial guess
    (default ones) and is updated in place when it is a contiguous float32
    array (em_methods.py:3-70)."""
    nslices = 1 if len(tomo.shape) == 2 else tomo.shape[0]
    nangles, nrays = tomo.shape[-2], tomo.shape[-1]
    objsize = nrays
    gpus_arr, ngpus = _gpus(gpus)
    obj = CNICE(obj) if obj is not None else numpy.ones([nslices, objsize, objsize], dtype=numpy.float32)
    tomo = CNICE(tomo)
    angles = CNICE(numpy.array(angles))
    param_int, param_float = _em_params(nrays, nangles, nslices, objsize, 1, iterations, blocksize)
    libraft.get_eEM_RT_MultiGPU(_ptr(gpus_arr), ngpus, _ptr(obj), _ptr(tomo), _ptr(angles),
                                _ptr(param_float), _ptr(param_int))
    check_error("eEMRT_GPU_")
    return obj


def tEMRT_GPU_(counts, flat, angles, iterations, gpus, blocksize, obj=None):
    """Transmission EM with ray-tracing operators (em_methods.py:72-151).

    As in the reference, ``counts`` (-log transmission) is overwritten in
    place by exp(-counts) when it is a float array."""
    nslices = 1 if len(counts.shape) == 2 else counts.shape[0]
    nflats = 1 if len(counts.shape) == 2 else flat.shape[0]
    nangles, nrays = counts.shape[-2], counts.shape[-1]
    objsize = nrays
    counts = numpy.exp(-counts, counts)
    gpus_arr, ngpus = _gpus(gpus)
    obj = CNICE(obj) if obj is not None else numpy.ones([nslices, objsize, objsize], dtype=numpy.float32)
    counts = CNICE(counts)
    flat = CNICE(flat)
    angles = CNICE(numpy.array(angles))
    param_int, param_float = _em_params(nrays, nangles, nslices, objsize, nflats, iterations, blocksize)
    libraft.get_tEM_RT_MultiGPU(_ptr(gpus_arr), ngpus, _ptr(obj), _ptr(counts), _ptr(flat),
                                _ptr(angles), _ptr(param_float), _ptr(param_int))
    check_error("tEMRT_GPU_")
    return obj


def em_with_metrics(kind, data, angles, iterations, gpu=0, flat=None, obj=None, use_graph=True):
    """Single-GPU EM that also returns per-iteration FP64 metrics
    [iterations, slices, 3] = (sum (model-data)^2, sum data^2, NLL) of the
    iterate entering each iteration.  kind 'tEM' takes data already mapped
    through exp(-x); 'eEM' takes the emission tomogram.  New (the reference
    computes no residual)."""
    data = CNICE(data if data.ndim == 3 else data[None])
    nslices, nangles, nrays = data.shape
    obj = CNICE(obj) if obj is not None else numpy.ones([nslices, nrays, nrays], dtype=numpy.float32)
    k = {'tEM': 0, 'eEM': 1}[kind]
    if k == 0:
        flat = CNICE(numpy.ones((nslices, nrays)) if flat is None else flat)
    angles = CNICE(numpy.array(angles))
    metrics = numpy.zeros((iterations, nslices, 3), dtype=numpy.float64)
    libraft.raft_em_ext(k, gpu, _ptr(obj), _ptr(data), _ptr(flat) if flat is not None else None,
                        _ptr(angles), nrays, nangles, nslices, iterations, _ptr(metrics),
                        1 if use_graph else 0)
    check_error("em_with_metrics")
    return obj, metrics


def tEMFQ_GPU_(count, flat, angles, pad, interpolation, det_pixel, tv_reg, iterations, gpus, blocksize,
               obj=None):
    """Transmission EM with the Fourier-slice projector and the BST
    back-projector (em_methods.py:153-237 of the reference).  count: photon
    counts [slices, angles, rays] (not -log); flat [slices, rays]; angles
    uniform over [0, pi); pad = (padx, 0, 0): the Fourier-slice zero padding;
    interpolation 0 nearest / 1 bilinear; det_pixel = (x, y), the projection
    scale is det_pixel x / (rays (1 + padx)) (1 / that length when <= 0);
    tv_reg unused (as in the reference).  obj: initial guess [slices, N, N] (default ones),
    updated in place when float32 C-contiguous; returned."""
    nslices = 1 if len(count.shape) == 2 else count.shape[0]
    nflats = 1 if len(flat.shape) == 2 else flat.shape[0]
    nangles, nrays = count.shape[-2], count.shape[-1]
    objsize = nrays
    # the library reads one flat row per slice; a single row serves every slice
    flat = numpy.asarray(flat)
    if flat.size == nrays and nslices > 1:
        flat = numpy.broadcast_to(flat.reshape(1, nrays), (nslices, nrays))
    elif flat.size != nslices * nrays:
        raise ValueError(f'flat must hold one row of {nrays} rays per slice (or one row for all), '
                         f'got shape {flat.shape}')
    gpus_arr, ngpus = _gpus(gpus)
    if obj is not None:
        obj = CNICE(obj)
    else:
        obj = CNICE(numpy.ones([nslices, objsize, objsize], dtype=numpy.float32))
    count = CNICE(count)
    flat = CNICE(flat)
    angles = CNICE(numpy.array(angles))
    padx, pady, padz = pad
    det_pixelx, det_pixely = det_pixel
    param_int = CNICE(numpy.array([nrays, nangles, nslices, objsize, padx, pady, padz, nflats, iterations,
                                   interpolation, blocksize]), numpy.int32)
    param_float = CNICE(numpy.array([det_pixelx, det_pixely, tv_reg]), numpy.float32)
    libraft.get_tEM_FQ_MultiGPU(_ptr(gpus_arr), ngpus, _ptr(count), _ptr(obj), _ptr(angles), _ptr(flat),
                                _ptr(param_float), _ptr(param_int))
    check_error("tEMFQ_GPU_")
    return obj
