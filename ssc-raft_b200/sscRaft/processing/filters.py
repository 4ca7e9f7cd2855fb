"""lowpass() (sscRaft/processing/filters.py:5-89 of cnpem/ssc-raft)."""
from ..rafttypes import CNICE, FilterNumber, _gpus, _ptr, check_error, libraft
from ..io import SetDictionary
from ..geometries.methods import em  # noqa: F401  (the reference exposes em here too)
import numpy


def lowpass(tomogram, dic=None, **kwargs):
    """FBP row filter only (edge padding, axis offset 0), applied in place to
    a contiguous float32 tomogram [slices, angles, rays] and returned."""
    required = ('gpu',)
    optional = ('filter', 'padding', 'regularization', 'beta/delta', 'blocksize', 'energy[eV]', 'z2[m]',
                'detectorPixel[m]')
    default = ('ramp', 2, 0.0, 0.0, 0, 1.0, 1.0, 1.0)
    dic = SetDictionary(dic, required, optional, default)
    gpus_arr, ngpus = _gpus(dic['gpu'])
    nrays, nangles = tomogram.shape[-1], tomogram.shape[-2]
    nslices = 1 if len(tomogram.shape) == 2 else tomogram.shape[0]
    filter_type = FilterNumber(dic['filter'])
    beta_delta = dic['beta/delta']
    regularization = dic['regularization']
    energy, z2 = dic['energy[eV]'], dic['z2[m]']
    pixelx, pixely = dic['detectorPixel[m]'], dic['detectorPixel[m]']
    if beta_delta != 0.0:
        beta_delta = 1.0 / beta_delta
    else:
        beta_delta, z2, energy = 0.0, 0.0, 1.0
    padx = dic['padding']
    tomogram = CNICE(tomogram)
    param_int = CNICE(numpy.array([nrays, nangles, nslices, nrays, padx, 0, 0, filter_type, 0,
                                   dic['blocksize']]), numpy.int32)
    param_float = CNICE(numpy.array([beta_delta, regularization, energy, z2, pixelx, pixely, 0.0]),
                        numpy.float32)
    libraft.getFilterLowPassMultiGPU(_ptr(gpus_arr), ngpus, _ptr(tomogram), _ptr(param_float),
                                     _ptr(param_int))
    check_error("lowpass")
    return tomogram
