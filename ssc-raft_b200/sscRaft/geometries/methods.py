"""Public fbp() / em() (sscRaft/geometries/methods.py:7-186 of cnpem/ssc-raft)."""
from ..rafttypes import logger
from ..io import SetDictionary
from .parallel.fbp_methods import fbpGPU, bstGPU
from .parallel.em_methods import eEMRT_GPU_, tEMRT_GPU_, tEMFQ_GPU_
import numpy


def fbp(tomogram, angles=None, obj=None, dic=None, nstreams=0, **kwargs):
    """Filtered backprojection of a parallel-beam tomogram [slices, angles, rays].
    Same dictionary and defaults as the reference (methods.py:54-56); methods
    'RT' (ray-traced backprojection) and 'BST' (backprojection slice theorem,
    uniform angles over [0, pi) assumed)."""
    required = ('gpu',)
    optional = ('filter', 'rotation axis offset', 'padding', 'regularization', 'beta/delta',
                'blocksize', 'energy[eV]', 'z2[m]', 'method', 'detectorPixel[m]')
    default = ('ramp', 0.0, 2, 0.0, 0.0, 0, 1.0, 1.0, 'RT', 1.0)
    dic = SetDictionary(dic, required, optional, default)
    method = dic['method']
    gpus = dic['gpu']
    if method == 'RT':
        try:
            angles = dic['angles[rad]']
        except KeyError:
            if angles is None:
                logger.error('Missing angles list!! Finishing run...')
                raise ValueError('Missing angles list!!')
        return fbpGPU(tomogram, angles, gpus, dic, obj=obj)
    if method == 'BST':
        angles = numpy.linspace(0.0, numpy.pi, tomogram.shape[-2], endpoint=False)
        return bstGPU(tomogram, angles, gpus, dic, obj=obj, nstreams=nstreams)
    raise ValueError(f'Invalid FBP method: {method}')


def em(data, flat=None, angles=None, obj=None, dic=None, **kwargs):
    """Expectation maximisation, methods 'eEMRT', 'tEMRT' and 'tEMFQ' (methods.py:83-186)."""
    required = ('gpu',)
    optional = ('iterations', 'detectorPixel[m]', 'padding', 'beamgeometry', 'interpolation', 'blocksize')
    default = (10, 0.0, 2, 'parallel', 'bilinear', 0)
    dic = SetDictionary(dic, required, optional, default)
    blocksize = dic['blocksize']
    gpus = dic['gpu']
    method = dic['method']
    iterations = dic['iterations']
    if angles is None:
        try:
            angles = dic['angles[rad]']
        except KeyError:
            logger.error('Missing angles list!! Finishing run...')
            raise ValueError('Missing angles list!!')
    if method != 'eEMRT':
        if flat is None:
            try:
                flat = dic['flat']
            except KeyError:
                logger.warning('No flat provided.')
                flat = numpy.ones((data.shape[0], data.shape[-1]))
    if method == 'eEMRT':
        return eEMRT_GPU_(data, angles, iterations, gpus, blocksize, obj=obj)
    elif method == 'tEMRT':
        return tEMRT_GPU_(data, flat, angles, iterations, gpus, blocksize, obj=obj)
    elif method == 'tEMFQ':
        # methods.py:140-181: padding and detector pixel from the dictionary,
        # total variation off, the interpolation name mapped to 0/1
        from ..rafttypes import setInterpolation
        det_pixel = (dic['detectorPixel[m]'], dic['detectorPixel[m]'])
        pad = (dic['padding'], 0, 0)
        return tEMFQ_GPU_(data, flat, angles, pad, setInterpolation(dic['interpolation']), det_pixel, 0.0,
                          iterations, gpus, blocksize, obj=obj)
    logger.error(f'Invalid EM method:{method}')
    raise ValueError(f'Invalid EM method:{method}')
