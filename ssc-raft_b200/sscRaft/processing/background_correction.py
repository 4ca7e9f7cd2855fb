"""Flat/dark correction of projections (sscRaft/processing/background_correction.py
of cnpem/ssc-raft): correct_projections, correct_background and the GPU driver
_background_correctionGPU, with the same argument meaning, shape checks and
in-place behaviour.  The work runs in libraft.so (getBackgroundCorrectionMultiGPU,
kernel in csrc/background.cu)."""
import numpy

from ..io import SetDictionary
from ..rafttypes import CNICE, _gpus, _ptr, check_error, libraft, logger


def _background_correctionGPU(frames, flat, dark, gpus=[0], is_log=False, blocksize=0):
    """T = -log((D - D_d) / (D_f - D_d)) (is_log) or T = (D - D_d) / (D_f - D_d),
    each difference clamped below at 0.5.

    frames [slices, angles, rays] (or [angles, rays]), flat [slices, flats, rays]
    (or [slices, rays]), dark [slices, rays] (or [slices, 1, rays]).  With two or
    more flats the first two are interpolated linearly over the angles.  The
    result is written into the float32 C-contiguous frames array when it is one
    (else into a converted copy) and returned."""
    gpus_arr, ngpus = _gpus(gpus)
    nrays = frames.shape[-1]
    nangles = frames.shape[-2]
    if len(frames.shape) == 2:
        nslices = 1
    elif len(frames.shape) == 3:
        nslices = frames.shape[0]
    else:
        message = f'Incorrect data dimension: {frames.shape}! It accepts only 2- or 3-dimension array.'
        logger.error(message)
        raise ValueError(message)
    if len(flat.shape) == 2:
        nflats = 1
    elif len(flat.shape) == 3:
        nflats = flat.shape[-2]
    else:
        message = f'Incorrect flat dimension: {flat.shape}! It accepts only 2- or 3-dimension array.'
        logger.error(message)
        raise ValueError(message)
    if len(dark.shape) == 3:
        dark = dark[:, 0, :]
    elif len(dark.shape) != 2:
        message = f'Incorrect dark dimension: {dark.shape}! It accepts only 2- or 3-dimension array.'
        logger.error(message)
        raise ValueError(message)
    if flat.shape[-1] != nrays or flat.shape[0] != nslices:
        message = (f'Flat dimension ({flat.shape[0]},{flat.shape[-1]}) does not match data dimension '
                   f'({nslices},{nrays}).')
        logger.error(message)
        raise ValueError(message)
    if dark.shape[-1] != nrays or dark.shape[0] != nslices:
        message = (f'Dark dimension ({dark.shape[0]},{dark.shape[-1]}) does not match data dimension '
                   f'({nslices},{nrays}).')
        logger.error(message)
        raise ValueError(message)
    flat = CNICE(flat)
    dark = CNICE(dark)
    frames = CNICE(frames)
    libraft.getBackgroundCorrectionMultiGPU(_ptr(gpus_arr), ngpus, _ptr(frames), _ptr(flat), _ptr(dark),
                                            nrays, nangles, nslices, nflats, 1 if is_log else 0, int(blocksize))
    check_error("background correction")
    return frames


def correct_projections(frames, flat, dark, dic, **kwargs):
    """Flat/dark correction of projections laid out [angles, slices, rays]
    as acquired (flat [flats, slices, rays], dark [darks, slices, rays]: every
    array has its first two axes swapped, as the reference does, so the dark
    must be three-dimensional; the first dark is used); returns the corrected
    data as [slices, angles, rays].

    dic: 'gpu' (list, required), 'uselog' (default False), 'blocksize' (0 = automatic)."""
    dic = SetDictionary(dic, ('gpu',), ('uselog', 'blocksize'), (False, 0))
    frames = numpy.swapaxes(frames, 0, 1)
    flat = numpy.swapaxes(flat, 0, 1)
    dark = numpy.swapaxes(dark, 0, 1)
    return _background_correctionGPU(frames, flat, dark, dic['gpu'], dic['uselog'], dic['blocksize'])


def correct_background(frames, flat, dark, gpus=[0], is_log=False, blocksize=0):
    """Flat/dark correction of frames [slices, angles, rays]; see _background_correctionGPU."""
    return _background_correctionGPU(frames, flat, dark, gpus, is_log, blocksize)
