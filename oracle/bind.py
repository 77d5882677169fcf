"""ctypes binding of the CPU oracle (oracle/_build/liborc.so). TEST INFRASTRUCTURE ONLY.

Imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm, as the checker
and the timed CPU baseline. The engine (cltem_b200) never imports this module.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from cltem_b200 import abi  # noqa: E402

LIB_PATH = os.path.join(HERE, "_build", "liborc.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def build(quiet=True):
    r = subprocess.run(["make", "-C", HERE], capture_output=quiet, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + (r.stdout or "") + (r.stderr or ""))


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.orc_last_error.restype = C.c_char_p
        L.orc_potential_value.restype = C.c_double
        L.orc_potential_value.argtypes = [C.c_int, C.c_int, _dp, C.c_int, C.c_int, C.c_double]
        L.orc_bessk0.restype = C.c_double
        L.orc_bessk0.argtypes = [C.c_double]
        L.orc_bessk1.restype = C.c_double
        L.orc_bessk1.argtypes = [C.c_double]
        L.orc_sim_create.argtypes = [C.POINTER(abi.Config), C.c_int, C.c_int, _dp, C.c_size_t, C.c_int, C.POINTER(C.c_void_p)]
        L.orc_sim_destroy.argtypes = [C.c_void_p]
        L.orc_set_atoms.argtypes = [C.c_void_p, C.c_size_t, _ip, _dp, _dp, _dp]
        L.orc_get_sorted_atoms.argtypes = [C.c_void_p, _ip, _dp, _dp, _dp, C.c_size_t, _ip, C.c_size_t, _ip, _ip,
                                           C.POINTER(C.c_size_t)]
        L.orc_build_transmission.argtypes = [C.c_void_p]
        L.orc_get_transmission.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp]
        L.orc_get_propagator.argtypes = [C.c_void_p, _dp]
        L.orc_get_probe.argtypes = [C.c_void_p, C.c_double, C.c_double, _dp]
        L.orc_stem_run.argtypes = [C.c_void_p, _ip, C.c_size_t, _dp]
        L.orc_cbed_run.argtypes = [C.c_void_p, _dp]
        L.orc_ctem_run.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.orc_fft2.argtypes = [C.c_int, C.c_int, _dp, _dp]
        L.orc_geometry.argtypes = [C.POINTER(abi.Config), C.POINTER(abi.Geometry), _dp, _dp]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_k_stem_pixel.restype = C.c_double
        L.orc_k_stem_pixel.argtypes = [_dp, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double]
        L.orc_k_ctem_image.argtypes = [C.POINTER(abi.Config), _dp, _dp, _dp, _dp]
        L.orc_run_staged.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_size_t), _ip, _dp, _dp, _dp, _dp]
        L.orc_draws.argtypes = [C.POINTER(abi.Config), C.c_int, _ip, C.c_size_t, _dp, _ip, C.c_int, C.c_int, _dp]
        L.orc_set_ccd.argtypes = [C.c_void_p, _dp, _dp, C.c_size_t, C.c_int, C.c_double]
        L.orc_poisson.argtypes = [C.c_uint64, C.c_int, _dp, C.c_size_t, _dp]
        L.orc_k_bilinear_translate.argtypes = [_dp, _dp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int]
        L.orc_plasmon_depths.argtypes = [C.POINTER(abi.Config), C.c_ulonglong, C.c_double, _dp, C.c_size_t,
                                         C.POINTER(C.c_size_t)]
        _lib = L
    return _lib


def _chk(rc):
    if rc != 0:
        raise RuntimeError("oracle: " + lib().orc_last_error().decode())


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def cplx(flat):
    return flat[0::2] + 1j * flat[1::2]


def geometry(cfg):
    g = abi.Geometry()
    kx = np.zeros(cfg.resolution)
    ky = np.zeros(cfg.resolution)
    _chk(lib().orc_geometry(C.byref(cfg), C.byref(g), _d(kx), _d(ky)))
    return g, kx, ky


def fft2(a, inverse=False):
    n = a.shape[0]
    flat = np.empty(2 * n * n)
    flat[0::2] = a.real.ravel()
    flat[1::2] = a.imag.ravel()
    out = np.empty_like(flat)
    _chk(lib().orc_fft2(n, int(inverse), _d(flat), _d(out)))
    return cplx(out).reshape(n, n)


def stem_pixel(recip, angle_scale, inner, outer, xc=0.0, yc=0.0):
    n = recip.shape[0]
    flat = np.empty(2 * n * n)
    flat[0::2] = recip.real.ravel()
    flat[1::2] = recip.imag.ravel()
    return lib().orc_k_stem_pixel(_d(flat), n, angle_scale, inner, outer, xc, yc)


def ctem_image(cfg, recip):
    g, kx, ky = geometry(cfg)
    n = recip.shape[0]
    flat = np.empty(2 * n * n)
    flat[0::2] = recip.real.ravel()
    flat[1::2] = recip.imag.ravel()
    out = np.empty_like(flat)
    _chk(lib().orc_k_ctem_image(C.byref(cfg), _d(kx), _d(ky), _d(flat), _d(out)))
    return cplx(out).reshape(n, n)


def draws(cfg, pass_, pixels, n_slices, n_builds):
    """(defocus changes per pixel, sets [pixel, slice], frame shifts [build, 2]) of one incoherent pass."""
    pixels = np.ascontiguousarray(pixels, dtype=np.int32)
    df = np.zeros(len(pixels))
    sets = np.zeros((len(pixels), n_slices), np.int32)
    shift = np.zeros((n_builds, 2))
    _chk(lib().orc_draws(C.byref(cfg), pass_, _i(pixels), len(pixels), _d(df), _i(sets), n_slices, n_builds, _d(shift)))
    return df, sets, shift


def poisson(seed, pass_, lam):
    """The oracle's seeded Poisson deviates of means `lam` (pixel i of dose pass `pass_`)."""
    lam = np.ascontiguousarray(lam, dtype=np.float64)
    out = np.zeros_like(lam)
    _chk(lib().orc_poisson(int(seed), int(pass_), _d(lam), lam.size, _d(out)))
    return out


def bilinear_translate(img, ix, iy, sx, sy):
    """bilinear_translate_d restated (FP64) on a real image [h, w]."""
    a = np.ascontiguousarray(img, dtype=np.float64)
    out = np.empty_like(a)
    _chk(lib().orc_k_bilinear_translate(_d(a), _d(out), int(ix), int(iy), float(sx), float(sy), a.shape[1], a.shape[0]))
    return out


def plasmon_depths(cfg, job, thickness, cap=4096):
    out = np.zeros(cap)
    n = C.c_size_t()
    _chk(lib().orc_plasmon_depths(C.byref(cfg), int(job), float(thickness), _d(out), cap, C.byref(n)))
    return out[: n.value]


def set_threads(n):
    lib().orc_set_threads(int(n))


def num_threads():
    return lib().orc_num_threads()


class OracleSim:
    """One simulation (one atom configuration at a time), FP64 (`_d`) unless double_precision=False."""

    def __init__(self, cfg, params, double_precision=True):
        self.cfg = cfg
        self.res = cfg.resolution
        self.N = self.res * self.res
        vals = np.ascontiguousarray(params.values, dtype=np.float64)
        h = C.c_void_p()
        _chk(lib().orc_sim_create(C.byref(cfg), params.form, params.i_per_atom, _d(vals), vals.size,
                                  int(double_precision), C.byref(h)))
        self.h = h
        self.geo = geometry(cfg)[0]

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_sim_destroy(self.h)
            self.h = None

    def set_atoms(self, st):
        Z = np.ascontiguousarray(st.Z, dtype=np.int32)
        x, y, z = (np.ascontiguousarray(v, dtype=np.float64) for v in (st.x, st.y, st.z))
        _chk(lib().orc_set_atoms(self.h, len(Z), _i(Z), _d(x), _d(y), _d(z)))

    def sorted_atoms(self, cap):
        g = self.geo
        nbs = g.n_slices * g.blocks_x * g.blocks_y + 1
        Z = np.zeros(cap, np.int32)
        x, y, z = np.zeros(cap), np.zeros(cap), np.zeros(cap)
        bs = np.zeros(nbs, np.int32)
        bid = np.zeros(cap, np.int32)
        zid = np.zeros(cap, np.int32)
        n = C.c_size_t()
        _chk(lib().orc_get_sorted_atoms(self.h, _i(Z), _d(x), _d(y), _d(z), cap, _i(bs), nbs, _i(bid), _i(zid), C.byref(n)))
        n = n.value
        return dict(Z=Z[:n], x=x[:n], y=y[:n], z=z[:n], block_start=bs, block_ids=bid[:n], z_ids=zid[:n])

    def build_transmission(self):
        _chk(lib().orc_build_transmission(self.h))

    def transmission(self, s, band_limited=True):
        out = np.empty(2 * self.N)
        _chk(lib().orc_get_transmission(self.h, s, int(band_limited), _d(out)))
        return cplx(out).reshape(self.res, self.res)

    def propagator(self):
        out = np.empty(2 * self.N)
        _chk(lib().orc_get_propagator(self.h, _d(out)))
        return cplx(out).reshape(self.res, self.res)

    def probe(self, x, y):
        out = np.empty(2 * self.N)
        _chk(lib().orc_get_probe(self.h, x, y, _d(out)))
        return cplx(out).reshape(self.res, self.res)

    def stem(self, pixels):
        pixels = np.ascontiguousarray(pixels, dtype=np.int32)
        g = self.geo
        out = np.zeros(g.n_outputs * self.cfg.n_detectors * len(pixels))
        _chk(lib().orc_stem_run(self.h, _i(pixels), len(pixels), _d(out)))
        return out.reshape(g.n_outputs, self.cfg.n_detectors, len(pixels))

    def set_ccd(self, ccd, binning=1, dose=10000.0):
        dqe = np.ascontiguousarray(ccd.dqe, dtype=np.float64)
        ntf = np.ascontiguousarray(ccd.ntf, dtype=np.float64)
        _chk(lib().orc_set_ccd(self.h, _d(dqe), _d(ntf), dqe.size, int(binning), float(dose)))

    def run_staged(self, configs):
        """Average over the passes of a staged run (STEM [o, d, pixel] or CBED [o, ky, kx]) with the config's
        incoherence options: mixed static sets, chromatic defocus, source-size shifts, moving frame."""
        from cltem_b200.structure import concat_configs
        cnt, Z, x, y, z = concat_configs(configs)
        cnt = np.ascontiguousarray(cnt, dtype=np.uint64)
        g = self.geo
        if self.cfg.mode == abi.MODE_STEM:
            npx = self.cfg.stem_pixels_x * self.cfg.stem_pixels_y
            shape = (g.n_outputs, self.cfg.n_detectors, npx)
        else:
            shape = (g.n_outputs, self.res, self.res)
        out = np.zeros(int(np.prod(shape)))
        _chk(lib().orc_run_staged(self.h, len(configs), cnt.ctypes.data_as(C.POINTER(C.c_size_t)), _i(Z), _d(x), _d(y),
                                  _d(z), _d(out)))
        return out.reshape(shape)

    def cbed(self):
        out = np.zeros(self.geo.n_outputs * self.N)
        _chk(lib().orc_cbed_run(self.h, _d(out)))
        return out.reshape(self.geo.n_outputs, self.res, self.res)

    def ctem(self):
        no = self.geo.n_outputs
        ew = np.zeros(no * 2 * self.N)
        diff = np.zeros(no * self.N)
        img = np.zeros(no * self.N)
        _chk(lib().orc_ctem_run(self.h, _d(ew), _d(diff), _d(img)))
        return (cplx(ew).reshape(no, self.res, self.res), diff.reshape(no, self.res, self.res),
                img.reshape(no, self.res, self.res))
