"""Python host binding of libmslice.so (include/mslice.h) through ctypes.

The classes mirror the reference's job interface for the multislice path: a Context per device (the
reference's clContext + one worker thread per device, src/simulation/threading/threadpool.cpp:9-19),
a Simulation holding one SimulationManager-like configuration (src/simulation/simulationmanager.h)
whose mode drivers correspond to SimulationStem/Cbed/Ctem::simulate, and simulate(), the
SimulationRunner-level entry that runs every frozen-phonon configuration and averages the images
(src/simulation/threading/simulationrunner.cpp:16-134, SimulationManager::updateImages :274-350).

There is no CPU fallback: every compute call runs CUDA kernels, and importing this module fails with
RuntimeError if the compiled library is missing.
"""
import ctypes as C
import os

import numpy as np

from . import abi
from .params import Parameterisation

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmslice.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_szp = C.POINTER(C.c_size_t)

_lib = None


class MsliceError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"mslice error {code}: {msg}")
        self.code = code


def load_library(path=None):
    """Load libmslice.so (built by `make -C cltem_b200/csrc`). Raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise RuntimeError(f"libmslice.so not found at {path}: build it with `make -C cltem_b200/csrc` "
                           "(or __graft_entry__.build()); there is no CPU fallback")
    L = C.CDLL(path)
    L.mslice_version.restype = C.c_char_p
    L.mslice_last_error.restype = C.c_char_p
    sig = {
        "mslice_ctx_create": [C.c_int, C.POINTER(C.c_void_p)],
        "mslice_ctx_destroy": [C.c_void_p],
        "mslice_ctx_set_memory_limit": [C.c_void_p, C.c_size_t],
        "mslice_params_load": [C.c_void_p, C.c_int, C.c_int, _dp, C.c_size_t],
        "mslice_geometry_compute": [C.POINTER(abi.Config), C.POINTER(abi.Geometry)],
        "mslice_sim_create": [C.c_void_p, C.POINTER(abi.Config), C.POINTER(C.c_void_p)],
        "mslice_sim_destroy": [C.c_void_p],
        "mslice_sim_geometry": [C.c_void_p, C.POINTER(abi.Geometry)],
        "mslice_set_progress": [C.c_void_p, C.c_void_p, C.c_void_p],
        "mslice_cancel": [C.c_void_p],
        "mslice_set_atoms": [C.c_void_p, _ip, _dp, _dp, _dp, C.c_size_t],
        "mslice_get_sorted_atoms": [C.c_void_p, _ip, _dp, _dp, _dp, C.c_size_t, _ip, C.c_size_t, _ip, _ip, _szp],
        "mslice_build_transmission": [C.c_void_p],
        "mslice_get_transmission": [C.c_void_p, C.c_int, C.c_int, _dp],
        "mslice_get_propagator": [C.c_void_p, _dp],
        "mslice_get_probe": [C.c_void_p, C.c_double, C.c_double, _dp],
        "mslice_stem_run": [C.c_void_p, _ip, C.c_size_t, _dp],
        "mslice_cbed_run": [C.c_void_p, _dp],
        "mslice_ctem_run": [C.c_void_p, _dp, _dp, _dp],
        "mslice_stage_configs": [C.c_void_p, C.c_int, _szp, _ip, _dp, _dp, _dp],
        "mslice_stem_run_staged": [C.c_void_p],
        "mslice_stem_run_staged_async": [C.c_void_p],
        "mslice_sim_wait": [C.c_void_p],
        "mslice_cbed_run_staged": [C.c_void_p],
        "mslice_staged_result": [C.c_void_p, _dp, C.c_size_t],
        "mslice_stem_simulate": [C.c_void_p, C.c_int, _szp, _ip, _dp, _dp, _dp, _dp, C.c_size_t],
        "mslice_stem_run_plain": [C.c_void_p, _ip, C.c_size_t, _dp],
        "mslice_fft2": [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, _dp, _dp],
        "mslice_ctx_stream": [C.c_void_p, C.POINTER(C.c_void_p)],
        "mslice_ctx_launch_count": [C.c_void_p, C.POINTER(C.c_ulonglong)],
        "mslice_last_timing": [C.c_void_p, _dp],
        "mslice_profile_enable": [C.c_void_p, C.c_int],
        "mslice_ctem_loss_grad": [C.c_void_p, _dp, _dp, _dp, _dp, _dp, C.c_int],
        "mslice_ctem_loss": [C.c_void_p, _dp, _dp],
        "mslice_ctem_loss_forward": [C.c_void_p, _dp, _dp, C.c_int, C.POINTER(C.c_ulonglong)],
        "mslice_ctem_loss_backward": [C.c_void_p, C.c_ulonglong, _dp, _dp, _dp],
        "mslice_profile_read": [C.c_void_p, C.c_int, _dp, C.POINTER(C.c_ulonglong), _dp, C.c_int],
        "mslice_incoherence_draws": [C.POINTER(abi.Config), C.c_int, _ip, C.c_size_t, _dp, _ip, C.c_int, C.c_int, _dp],
        "mslice_plasmon_draws": [C.POINTER(abi.Config), C.c_ulonglong, C.c_double, _dp, C.c_size_t, _szp, C.c_int, _dp],
        "mslice_tune_batch": [C.c_void_p, _ip, C.c_int, C.c_int, _ip, _dp],
        "mslice_set_step_variant": [C.c_void_p, C.c_int, C.c_int],
        "mslice_step_variant_name": [C.c_void_p, C.c_int, C.c_int, C.c_char_p, C.c_size_t],
        "mslice_get_tuning": [C.c_void_p, _ip, _ip, _ip, _ip, _ip],
        "mslice_set_ccd": [C.c_void_p, _dp, _dp, C.c_size_t, C.c_int, C.c_double],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = C.c_int
    _lib = L
    return L


def _check(rc):
    if rc != abi.OK:
        raise MsliceError(rc, _lib.mslice_last_error().decode())


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def _cplx(flat):
    return flat[0::2] + 1j * flat[1::2]


def _interleave(a):
    a = np.asarray(a, dtype=np.complex128)
    out = np.empty(a.size * 2)
    out[0::2] = a.real.ravel()
    out[1::2] = a.imag.ravel()
    return out


PROGRESS_CB = C.CFUNCTYPE(None, C.c_double, C.c_void_p)


def geometry(cfg: abi.Config) -> abi.Geometry:
    L = load_library()
    g = abi.Geometry()
    _check(L.mslice_geometry_compute(C.byref(cfg), C.byref(g)))
    return g


def incoherence_draws(cfg: abi.Config, pass_: int, pixels, n_slices: int, n_builds: int):
    """The random draws of one pass (host only): defocus change per pixel (Å), transmission set per pixel and
    slice, and the source-size frame shift (Å) of each transmission build."""
    L = load_library()
    pixels = np.ascontiguousarray(pixels, dtype=np.int32)
    df = np.zeros(len(pixels))
    sets = np.zeros((len(pixels), n_slices), np.int32)
    shift = np.zeros((n_builds, 2))
    _check(L.mslice_incoherence_draws(C.byref(cfg), int(pass_), _i(pixels), len(pixels), _d(df), _i(sets), int(n_slices),
                                      int(n_builds), _d(shift)))
    return df, sets, shift


def plasmon_draws(cfg: abi.Config, job: int, thickness: float, n_events: int = 0, cap: int = 4096):
    """The seeded plasmon draws of one job (host only): scattering depths (Å, the last +inf) and the
    (polar mrad, azimuth rad) of its first n_events events."""
    L = load_library()
    d = np.zeros(cap)
    n = C.c_size_t()
    ang = np.zeros(2 * max(n_events, 1))
    _check(L.mslice_plasmon_draws(C.byref(cfg), int(job), float(thickness), _d(d), cap, C.byref(n), int(n_events), _d(ang)))
    return d[: n.value], ang[: 2 * n_events].reshape(n_events, 2)


class Context:
    """A device context (one CUDA device, one stream)."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        import weakref
        h = C.c_void_p()
        _check(self.lib.mslice_ctx_create(device, C.byref(h)))
        self.h = h
        self.device = device
        self.params = None
        self._sims = weakref.WeakSet()

    def close(self):
        """Destroy the context; simulations still open on it are destroyed with it."""
        if getattr(self, "h", None):
            for sim in list(getattr(self, "_sims", ())):
                sim.h = None   # the library frees them with the context
            self.lib.mslice_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def load_params(self, p: Parameterisation):
        vals = np.ascontiguousarray(p.values, dtype=np.float64)
        _check(self.lib.mslice_params_load(self.h, p.form, p.i_per_atom, _d(vals), vals.size))
        self.params = p

    def set_memory_limit(self, nbytes: int):
        _check(self.lib.mslice_ctx_set_memory_limit(self.h, int(nbytes)))

    def stream(self) -> int:
        s = C.c_void_p()
        _check(self.lib.mslice_ctx_stream(self.h, C.byref(s)))
        return s.value or 0

    def launch_count(self) -> int:
        n = C.c_ulonglong()
        _check(self.lib.mslice_ctx_launch_count(self.h, C.byref(n)))
        return n.value

    def fft2(self, a, inverse=False, double_precision=True):
        """Unitary 2-D DFT of a (batch, n, n) or (n, n) complex array with the engine's FFT kernels."""
        a = np.asarray(a)
        single = a.ndim == 2
        if single:
            a = a[None]
        b, n, _ = a.shape
        flat = _interleave(a)
        out = np.empty_like(flat)
        _check(self.lib.mslice_fft2(self.h, n, int(inverse), int(double_precision), b, _d(flat), _d(out)))
        r = _cplx(out).reshape(b, n, n)
        return r[0] if single else r


class Simulation:
    """One simulation configuration on a context (SimulationWorker state for one manager)."""

    def __init__(self, ctx: Context, cfg: abi.Config):
        self.ctx = ctx
        self.lib = ctx.lib
        self.cfg = cfg
        h = C.c_void_p()
        _check(self.lib.mslice_sim_create(ctx.h, C.byref(cfg), C.byref(h)))
        self.h = h
        ctx._sims.add(self)
        g = abi.Geometry()
        _check(self.lib.mslice_sim_geometry(self.h, C.byref(g)))
        self.geo = g
        self.res = cfg.resolution
        self.N = self.res * self.res
        self._cb = None

    def close(self):
        if getattr(self, "h", None):
            if getattr(self.ctx, "h", None):   # a closed context has already freed its simulations
                self.lib.mslice_sim_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def set_progress(self, fn):
        self._cb = PROGRESS_CB(lambda f, u: fn(f)) if fn else None
        _check(self.lib.mslice_set_progress(self.h, C.cast(self._cb, C.c_void_p) if fn else None, None))

    def cancel(self):
        self.lib.mslice_cancel(self.h)

    @property
    def n_outputs(self):
        return self.geo.n_outputs

    def set_atoms(self, st):
        Z = np.ascontiguousarray(st.Z, dtype=np.int32)
        x, y, z = (np.ascontiguousarray(v, dtype=np.float64) for v in (st.x, st.y, st.z))
        _check(self.lib.mslice_set_atoms(self.h, _i(Z), _d(x), _d(y), _d(z), len(Z)))

    def sorted_atoms(self, cap):
        g = self.geo
        nbs = g.n_slices * g.blocks_x * g.blocks_y + 1
        Z = np.zeros(max(cap, 1), np.int32)
        x, y, z = np.zeros(max(cap, 1)), np.zeros(max(cap, 1)), np.zeros(max(cap, 1))
        bs = np.zeros(nbs, np.int32)
        bid = np.zeros(max(cap, 1), np.int32)
        zid = np.zeros(max(cap, 1), np.int32)
        n = C.c_size_t()
        _check(self.lib.mslice_get_sorted_atoms(self.h, _i(Z), _d(x), _d(y), _d(z), cap, _i(bs), nbs, _i(bid), _i(zid),
                                                C.byref(n)))
        n = n.value
        return dict(Z=Z[:n], x=x[:n], y=y[:n], z=z[:n], block_start=bs, block_ids=bid[:n], z_ids=zid[:n])

    def build_transmission(self):
        _check(self.lib.mslice_build_transmission(self.h))

    def transmission(self, s, band_limited=True):
        out = np.empty(2 * self.N)
        _check(self.lib.mslice_get_transmission(self.h, s, int(band_limited), _d(out)))
        return _cplx(out).reshape(self.res, self.res)

    def propagator(self):
        out = np.empty(2 * self.N)
        _check(self.lib.mslice_get_propagator(self.h, _d(out)))
        return _cplx(out).reshape(self.res, self.res)

    def probe(self, x, y):
        out = np.empty(2 * self.N)
        _check(self.lib.mslice_get_probe(self.h, float(x), float(y), _d(out)))
        return _cplx(out).reshape(self.res, self.res)

    def stem(self, pixels):
        pixels = np.ascontiguousarray(pixels, dtype=np.int32)
        out = np.zeros(max(1, self.n_outputs * self.cfg.n_detectors * len(pixels)))
        _check(self.lib.mslice_stem_run(self.h, _i(pixels), len(pixels), _d(out)))
        return out[: self.n_outputs * self.cfg.n_detectors * len(pixels)].reshape(
            self.n_outputs, self.cfg.n_detectors, len(pixels))

    def stem_plain(self, pixels):
        pixels = np.ascontiguousarray(pixels, dtype=np.int32)
        out = np.zeros(max(1, self.n_outputs * self.cfg.n_detectors * len(pixels)))
        _check(self.lib.mslice_stem_run_plain(self.h, _i(pixels), len(pixels), _d(out)))
        return out[: self.n_outputs * self.cfg.n_detectors * len(pixels)].reshape(
            self.n_outputs, self.cfg.n_detectors, len(pixels))

    def cbed(self):
        out = np.zeros(self.n_outputs * self.N)
        _check(self.lib.mslice_cbed_run(self.h, _d(out)))
        return out.reshape(self.n_outputs, self.res, self.res)

    def ctem(self):
        no = self.n_outputs
        ew = np.zeros(no * 2 * self.N)
        diff = np.zeros(no * self.N)
        img = np.zeros(no * self.N)
        _check(self.lib.mslice_ctem_run(self.h, _d(ew), _d(diff), _d(img)))
        return (_cplx(ew).reshape(no, self.res, self.res), diff.reshape(no, self.res, self.res),
                img.reshape(no, self.res, self.res))

    # ---- differentiable CTEM ----------------------------------------------------------------------
    def ctem_loss(self, target):
        """L = sum (I - target)^2 of the CTEM image of the current atoms (forward only)."""
        t = np.ascontiguousarray(target, dtype=np.float64).reshape(-1)
        L = C.c_double()
        _check(self.lib.mslice_ctem_loss(self.h, _d(t), C.byref(L)))
        return L.value

    def ctem_loss_grad(self, target, n_atoms, checkpoint_every=0):
        """(L, dL/dxyz [n_atoms, 3] in the order given to set_atoms, dL/dC10, dL/dC30) by the adjoint."""
        t = np.ascontiguousarray(target, dtype=np.float64).reshape(-1)
        L, g10, g30 = C.c_double(), C.c_double(), C.c_double()
        gx = np.zeros(3 * max(n_atoms, 1))
        _check(self.lib.mslice_ctem_loss_grad(self.h, _d(t), C.byref(L), _d(gx), C.byref(g10), C.byref(g30),
                                              int(checkpoint_every)))
        return L.value, gx[: 3 * n_atoms].reshape(n_atoms, 3), g10.value, g30.value

    def ctem_loss_forward(self, target, checkpoint_every=0):
        """The loss, keeping the adjoint's state: (L, token) for ctem_loss_backward."""
        t = np.ascontiguousarray(target, dtype=np.float64).reshape(-1)
        L, tok = C.c_double(), C.c_ulonglong()
        _check(self.lib.mslice_ctem_loss_forward(self.h, _d(t), C.byref(L), int(checkpoint_every), C.byref(tok)))
        return L.value, tok.value

    def ctem_loss_backward(self, token, n_atoms):
        """(dL/dxyz [n_atoms, 3], dL/dC10, dL/dC30) from the state of forward `token`."""
        g10, g30 = C.c_double(), C.c_double()
        gx = np.zeros(3 * max(n_atoms, 1))
        _check(self.lib.mslice_ctem_loss_backward(self.h, int(token), _d(gx), C.byref(g10), C.byref(g30)))
        return gx[: 3 * n_atoms].reshape(n_atoms, 3), g10.value, g30.value

    # ---- frozen-phonon runs ---------------------------------------------------------------------
    def stage(self, configs):
        from .structure import concat_configs
        counts, Z, x, y, z = concat_configs(configs)
        self._staged = (counts, Z, x, y, z)
        _check(self.lib.mslice_stage_configs(self.h, len(configs), counts.ctypes.data_as(_szp), _i(Z), _d(x), _d(y), _d(z)))

    def run_staged(self):
        if self.cfg.mode == abi.MODE_STEM:
            _check(self.lib.mslice_stem_run_staged(self.h))
        else:
            _check(self.lib.mslice_cbed_run_staged(self.h))

    def run_staged_async(self):
        """Queue a staged STEM run and return (mslice_stem_run_staged_async); wait() or staged_result() waits."""
        _check(self.lib.mslice_stem_run_staged_async(self.h))

    def wait(self):
        _check(self.lib.mslice_sim_wait(self.h))

    def result_size(self):
        if self.cfg.mode == abi.MODE_STEM:
            return self.n_outputs * self.cfg.n_detectors * self.cfg.stem_pixels_x * self.cfg.stem_pixels_y
        return self.n_outputs * self.N

    def staged_result(self, out=None):
        n = self.result_size()
        if out is None:
            out = np.zeros(n)
        _check(self.lib.mslice_staged_result(self.h, _d(out), n))
        return self._shape(out)

    def _shape(self, flat):
        if self.cfg.mode == abi.MODE_STEM:
            return flat.reshape(self.n_outputs, self.cfg.n_detectors, self.cfg.stem_pixels_y, self.cfg.stem_pixels_x)
        return flat.reshape(self.n_outputs, self.res, self.res)

    def stem_simulate(self, configs, out=None):
        """One end-to-end call: host atom arrays in, averaged detector images out."""
        from .structure import concat_configs
        counts, Z, x, y, z = concat_configs(configs)
        n = self.result_size()
        if out is None:
            out = np.zeros(n)
        _check(self.lib.mslice_stem_simulate(self.h, len(configs), counts.ctypes.data_as(_szp), _i(Z), _d(x), _d(y),
                                             _d(z), _d(out), n))
        return self._shape(out)

    def set_ccd(self, ccd=None, binning=1, dose=10000.0):
        """CTEM dose simulation with a CCD (cltem_b200.params.CCD: 725-value DQE and NTF tables), `binning` and
        `dose` electrons per Å^2 (SimulationManager defaults: binning 1, dose 10000); None restores the perfect
        image."""
        if ccd is None:
            _check(self.lib.mslice_set_ccd(self.h, None, None, 0, 1, 1.0))
            return
        dqe = np.ascontiguousarray(ccd.dqe, dtype=np.float64)
        ntf = np.ascontiguousarray(ccd.ntf, dtype=np.float64)
        if dqe.size != ntf.size:
            raise ValueError("DQE and NTF tables differ in length")
        _check(self.lib.mslice_set_ccd(self.h, _d(dqe), _d(ntf), dqe.size, int(binning), float(dose)))

    def tune_batch(self, candidates=None, reps=3):
        """Autotune the probe batch (mslice_tune_batch); returns (batch, waves per second)."""
        best = C.c_int()
        rate = C.c_double()
        if candidates is None:
            _check(self.lib.mslice_tune_batch(self.h, None, 0, int(reps), C.byref(best), C.byref(rate)))
        else:
            c = np.ascontiguousarray(candidates, dtype=np.int32)
            _check(self.lib.mslice_tune_batch(self.h, _i(c), len(c), int(reps), C.byref(best), C.byref(rate)))
        return best.value, rate.value

    def set_step_variant(self, col_variant, row_variant=None):
        """Kernels of the batched STEM step (mslice_set_step_variant): column 0 one block per tile, then the
        size's other column kernels (step_variant_name(0, v)); row 0 plain, 1 / 2 with an L2 prefetch one / two
        grid residencies ahead, 3 in wave-fastest order, and where the size's default row plan is a wide one,
        4-7 the same four with the plain Stockham plan. The row variant is kept when not given."""
        if row_variant is None:
            row_variant = self.tuning()["row_variant"]
        _check(self.lib.mslice_set_step_variant(self.h, int(col_variant), int(row_variant)))

    def step_variant_name(self, which, index):
        """A description of column (which = 0) or row (1) step variant `index` (mslice_step_variant_name)."""
        buf = C.create_string_buffer(256)
        _check(self.lib.mslice_step_variant_name(self.h, int(which), int(index), buf, 256))
        return buf.value.decode()

    def tuning(self):
        """{"batch", "col_variant", "col_variants", "row_variant", "row_variants"} the next STEM run uses
        (mslice_get_tuning)."""
        b, v, n, rv, rn = C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_int()
        _check(self.lib.mslice_get_tuning(self.h, C.byref(b), C.byref(v), C.byref(n), C.byref(rv), C.byref(rn)))
        return {"batch": b.value, "col_variant": v.value, "col_variants": n.value, "row_variant": rv.value,
                "row_variants": rn.value}

    KERNELS = ("row_step", "col_step", "potential", "bandlimit", "probe")

    def profile(self, on=True):
        _check(self.lib.mslice_profile_enable(self.h, int(on)))

    def profile_read(self, reset=False):
        """{kernel: (total device ms, launches, algorithmic bytes)} accumulated while profiling was on."""
        out = {}
        for k, name in enumerate(self.KERNELS):
            ms, n, by = C.c_double(), C.c_ulonglong(), C.c_double()
            _check(self.lib.mslice_profile_read(self.h, k, C.byref(ms), C.byref(n), C.byref(by), 0))
            out[name] = (ms.value, n.value, by.value)
        if reset:
            ms, n, by = C.c_double(), C.c_ulonglong(), C.c_double()
            _check(self.lib.mslice_profile_read(self.h, 0, C.byref(ms), C.byref(n), C.byref(by), 1))
        return out

    def last_timing(self):
        t = np.zeros(3)
        _check(self.lib.mslice_last_timing(self.h, _d(t)))
        return {"build_ms": t[0], "propagate_ms": t[1], "total_ms": t[2]}


def simulate(settings, structure, params: Parameterisation, n_configs: int = 1, u_rms: float = 0.0, seed: int = 0,
             device: int = 0):
    """Run a whole simulation (every frozen-phonon configuration) and return the averaged images:
    STEM -> {detector name: array[n_out, py, px]}, CBED -> {"Diff": array[n_out, res, res]},
    CTEM -> {"EW": complex array, "Diff": ..., "Image": ...} averaged over configurations."""
    from .structure import phonon_configs
    ctx = Context(device)
    ctx.load_params(params)
    sim = Simulation(ctx, settings.cfg)
    configs = phonon_configs(structure, n_configs, u_rms, seed) if (n_configs > 1 or u_rms > 0) else [structure]
    mode = settings.cfg.mode
    if mode == abi.MODE_STEM:
        r = sim.stem_simulate(configs)
        return {settings.detectors[d][0]: r[:, d] for d in range(settings.cfg.n_detectors)}
    if mode == abi.MODE_CBED:
        sim.stage(configs)
        sim.run_staged()
        return {"Diff": sim.staged_result()}
    ew = diff = img = None
    for c in configs:
        sim.set_atoms(c)
        e, d, i = sim.ctem()
        ew = e if ew is None else ew + e
        diff = d if diff is None else diff + d
        img = i if img is None else img + i
    n = len(configs)
    out = {"EW": ew / n, "Diff": diff / n}
    if settings.cfg.ctem_image:
        out["Image"] = img / n
    return out
