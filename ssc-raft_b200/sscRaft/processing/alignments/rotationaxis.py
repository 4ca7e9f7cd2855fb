"""Rotation-axis estimation and correction (sscRaft/processing/alignments/rotationaxis.py
of cnpem/ssc-raft): the GPU finders Centersino / Centersino_subpixel
(findcentersino*, csrc/rotation.cu), the GPU sub-pixel correction
correct_rotation_axis (getRotAxisCorrectionMultiGPU) and the host-side helpers,
with the reference's argument meaning and return values."""
import ctypes

import numpy

from ...rafttypes import CNICE, _gpus, _ptr, check_error, libraft, logger

libraft.findcentersino.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_int, ctypes.c_int]
libraft.findcentersino.restype = ctypes.c_int
libraft.findcentersino_subpixel.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_int, ctypes.c_int]
libraft.findcentersino_subpixel.restype = ctypes.c_float
libraft.findcentersino16.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_int, ctypes.c_int]
libraft.findcentersino16.restype = ctypes.c_int
libraft.correctRotationAxis.argtypes = [ctypes.c_void_p, ctypes.c_void_p] + [ctypes.c_int] * 4
libraft.correctRotationAxis.restype = None
libraft.getRotAxisCorrectionMultiGPU.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_float,
                                                 ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
libraft.getRotAxisCorrectionMultiGPU.restype = None
libraft.raft_centersino_device.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 4 + [ctypes.c_int] * 3 + \
    [ctypes.c_void_p, ctypes.c_void_p]
libraft.raft_centersino_device.restype = ctypes.c_int


def _frames(frame0, frame1, flat, dark, dtype=numpy.float32):
    arrs = [CNICE(a, dtype) for a in (frame0, frame1, dark, flat)]
    return arrs, frame0.shape[-1], frame0.shape[-2]


def Centersino(frame0, frame1, flat, dark):
    """Integer rotation-axis offset of a 180-degree scan from its first and
    last frames [slices, rays] by phase correlation of -log((I - dark) / (flat - dark))
    (flat and dark applied inside)."""
    (f0, f1, dk, ft), nrays, nslices = _frames(frame0, frame1, flat, dark)
    offset = libraft.findcentersino(_ptr(f0), _ptr(f1), _ptr(dk), _ptr(ft), nrays, nslices)
    check_error("Centersino")
    return offset


def Centersino16(frame0, frame1, flat, dark):
    """Centersino for uint16 frames (findcentersino16)."""
    (f0, f1, dk, ft), nrays, nslices = _frames(frame0, frame1, flat, dark, numpy.uint16)
    offset = libraft.findcentersino16(_ptr(f0), _ptr(f1), _ptr(dk), _ptr(ft), nrays, nslices)
    check_error("Centersino16")
    return offset


def Centersino_subpixel(frame0, frame1, flat, dark):
    """Sub-pixel variant of Centersino (the reference's search grid, x = i * 0.01)."""
    (f0, f1, dk, ft), nrays, nslices = _frames(frame0, frame1, flat, dark)
    offset = libraft.findcentersino_subpixel(_ptr(f0), _ptr(f1), _ptr(dk), _ptr(ft), nrays, nslices)
    check_error("Centersino_subpixel")
    return offset


def find_rotation_axis_360(tomo, nx_search=500, nx_window=500, nsinos=None):
    """CPU search of the rotation axis of a 360-degree scan tomo [angles, slices, rays]:
    the deviation (from rays//2) minimising the mismatch between the first half
    of the sinogram and the mirrored second half, summed over nsinos sinograms
    from the middle slice (default slices//20, or all when that is 0)."""
    ntheta, nz, nx = tomo.shape
    score = numpy.ones(2 * nx_search)
    if nsinos is None:
        nsinos = nz // 20
    if nsinos == 0:
        nsinos = nz
    last = ntheta if ntheta % 2 == 0 else ntheta - 1
    for k in range(nsinos):
        z = k + nz // 2
        for i in range(2 * nx_search):
            c = nx // 2 - nx_search + i
            left = tomo[:ntheta // 2, z, c - nx_window:c]
            right = numpy.flip(tomo[ntheta // 2:last, z, c:c + nx_window], axis=1)
            half_norm = numpy.linalg.norm(left + right) / 2
            score[i] += numpy.linalg.norm(left - right) / half_norm
    deviation = numpy.argmin(score) - nx_search
    logger.info(f'Automatic rotation axis correction deviation: {deviation}')
    return deviation


def correct_rotation_axis360(data, dic):
    """Pad a 360-degree tomogram [slices, angles, rays] by 2|shift| rays so the
    axis sits in the middle; dic['shift'] = (automatic, value),
    dic['findRotationAxis'] = (nx_search, nx_window, nsinos).  Returns (proj, shift)."""
    auto, shift = dic['shift'][0], dic['shift'][1]
    if auto:
        nx_search, nx_window, nsinos = dic['findRotationAxis']
        shift = find_rotation_axis_360(numpy.swapaxes(data, 0, 1), nx_search=nx_search, nx_window=nx_window,
                                       nsinos=nsinos)
        dic.update({'shift': [auto, shift]})
    a = numpy.abs(shift)
    proj = numpy.zeros((data.shape[0], data.shape[1], data.shape[2] + 2 * a))
    if shift < 0:
        proj[:, :, 2 * a:data.shape[2] + 2 * a] = data
    else:
        proj[:, :, 0:data.shape[2]] = data
    return proj, shift


def c_correct_rotation_axis(data, deviation, out=None):
    """Integer shift of every row by `deviation` rays (right if positive), zero
    fill, on the host (correctRotationAxis)."""
    data = CNICE(data)
    if out is None:
        out = numpy.empty_like(data)
    elif not out.flags.c_contiguous:
        raise ValueError('Output array must be contiguous')
    out = CNICE(out)
    sizez, sizey, sizex = data.shape if data.ndim == 3 else (1,) + data.shape
    libraft.correctRotationAxis(_ptr(data), _ptr(out), sizex, sizey, sizez, int(deviation))
    check_error("correctRotationAxis")
    return out


def correct_rotation_axis_int(data, deviation):
    """Widen [slices, angles, rays] by 2|deviation| rays placing the data so the
    axis Centersino reported is centred (deviation in Centersino's sign)."""
    d = -deviation
    a = numpy.abs(d)
    proj = numpy.zeros((data.shape[0], data.shape[1], data.shape[2] + 2 * a))
    if d < 0:
        proj[:, :, 2 * a:data.shape[2] + 2 * a] = data
    else:
        proj[:, :, 0:data.shape[2]] = data
    return proj


def correct_rotation_axis_cropped(data, deviation):
    """Shift rays by `deviation` in place, keeping the shape (zero fill)."""
    proj = numpy.zeros_like(data)
    if deviation < 0:
        proj[..., :deviation] = data[..., -deviation:]
    elif deviation > 0:
        proj[..., deviation:] = data[..., :-deviation]
    data[...] = proj
    return data


def correct_rotation_axis(data, axis_offset, gpus=[0], blocksize=0):
    """Sub-pixel axis correction on the GPU: every row shifted by axis_offset
    rays (Fourier phase ramp on 3x edge-padded rows); in place on the float32
    C-contiguous data [slices, angles, rays] (or a converted copy), returned."""
    gpus_arr, ngpus = _gpus(gpus)
    nrays, nangles = data.shape[-1], data.shape[-2]
    nslices = data.shape[0] if data.ndim == 3 else 1
    data = CNICE(data)
    libraft.getRotAxisCorrectionMultiGPU(_ptr(gpus_arr), ngpus, _ptr(data), float(axis_offset), nrays, nangles,
                                         nslices, int(blocksize))
    check_error("correct_rotation_axis")
    return data


def _blocks(n, block_size):
    return [(s, min(n, s + block_size)) for s in range(0, n, block_size)]


def Centersino_block(frame0, frame1, flat, dark, block_size):
    """Centersino per block of block_size slices; the list of offsets."""
    return [Centersino(frame0[a:b], frame1[a:b], flat[a:b], dark[a:b]) for a, b in _blocks(frame0.shape[0], block_size)]


def correct_rotation_axis_block(data, rotation_axis_list, block_size):
    """correct_rotation_axis per block of slices with the block's offset."""
    for k, (a, b) in enumerate(_blocks(data.shape[0], block_size)):
        data[a:b] = correct_rotation_axis(data[a:b], rotation_axis_list[k], [0], 0)
    return data
