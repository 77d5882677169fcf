"""ctypes binding of oracle/_ref/libref.so: the reference's own OpenCL kernels compiled for the CPU.
TEST INFRASTRUCTURE ONLY (pins the oracle). available() is False where the reference tree was not
present when the library was built."""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libref.so")
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(LIB_PATH)
        for name in ("ref_atom_sort_d", "ref_band_limit_d", "ref_band_pass_d", "ref_bilinear_translate_d",
                     "ref_complex_multiply_d",
                     "ref_complex_to_real_d", "ref_fft_shift_d", "ref_init_plane_wave_d", "ref_init_probe_wave_d",
                     "ref_ctem_image_d", "ref_propagator_d", "ref_sqabs_d", "ref_sum_reduction_d",
                     "ref_transmission_projected_d", "ref_transmission_full3d_d"):
            getattr(_lib, name).restype = None
        _lib.ref_atom_sort_d.argtypes = [_dp, _dp, _dp, C.c_int] + [C.c_double] * 6 + [C.c_int, C.c_int, _ip, _ip,
                                                                                        C.c_double, C.c_int]
        _lib.ref_band_limit_d.argtypes = [_dp, C.c_uint, C.c_uint, C.c_double, C.c_double, _dp, _dp]
        _lib.ref_band_pass_d.argtypes = [_dp, _dp, C.c_uint, C.c_uint] + [C.c_double] * 4
        _lib.ref_bilinear_translate_d.argtypes = [_dp, _dp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_uint, C.c_uint]
        _lib.ref_fft_shift_d.argtypes = [_dp, _dp, C.c_uint, C.c_uint]
        _lib.ref_complex_to_real_d.argtypes = [_dp, _dp, C.c_int, C.c_uint, C.c_uint]
        _lib.ref_sum_reduction_d.argtypes = [_dp, _dp, C.c_uint]
        _lib.ref_propagator_d.argtypes = [_dp, _dp, _dp, C.c_uint, C.c_uint] + [C.c_double] * 6
        _lib.ref_init_probe_wave_d.argtypes = [_dp, C.c_uint, C.c_uint, _dp, _dp] + [C.c_double] * 6 + [_dp, C.c_double,
                                                                                                     C.c_double]
        _lib.ref_ctem_image_d.argtypes = [_dp, _dp, C.c_uint, C.c_uint, _dp, _dp] + [C.c_double] * 4 + [_dp] + [C.c_double] * 4
        _lib.ref_sqabs_d.argtypes = [_dp, _dp, C.c_uint, C.c_uint]
        _lib.ref_transmission_projected_d.argtypes = [_dp, _dp, _dp, _dp, _ip, _dp, _ip, _dp, _ip]
        _lib.ref_transmission_full3d_d.argtypes = [_dp, _dp, _dp, _dp, _ip, _dp, _ip, _dp, _ip]
    return _lib


def d(a):
    return a.ctypes.data_as(_dp)


def i(a):
    return a.ctypes.data_as(_ip)


def inter(a):
    out = np.empty(a.size * 2)
    out[0::2] = a.real.ravel()
    out[1::2] = a.imag.ravel()
    return out


def cplx(flat, shape):
    return (flat[0::2] + 1j * flat[1::2]).reshape(shape)


def aberr_array(cfg):
    """(re, im) of C12, C21, C23, C32, C34, C41, C43, C45, C52, C54, C56 (ComplexAberration::getComplex)."""
    out = []
    for nm in ("C12", "C21", "C23", "C32", "C34", "C41", "C43", "C45", "C52", "C54", "C56"):
        a = getattr(cfg, nm)
        out += [a.mag * np.cos(a.ang), a.mag * np.sin(a.ang)]   # std::polar(mag, ang)
    return np.asarray(out)
