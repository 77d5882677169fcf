"""Simulation configuration: clTEM's JSON config <-> the engine's POD config.

read_config mirrors JSONUtils::JsonToManager (src/simulation/utilities/jsonutils.cpp:15-366): the same
keys, the same unit conversions (C10/C12/C21/C23 nm -> Å x10, C30..C56 um -> Å x1e4, delta nm -> Å,
angles deg -> rad, beam-tilt azimuth deg -> rad), the same defaults for keys that are absent
(SimulationManager defaults, src/simulation/simulationmanager.cpp:8-50) and the same truncation of
detector radii/centres to unsigned int (jsonutils.cpp:234-237).

attach_structure mirrors SimulationManager::setStructure (simulationmanager.cpp:133-152): unless
"maintain areas" is set, the CTEM/STEM areas take the structure's x/y limits and the CBED position its
centre.
"""
import json
from dataclasses import dataclass
import math

from . import abi


def _get(j, *keys):
    for k in keys:
        if not isinstance(j, dict) or k not in j:
            raise KeyError(k)
        j = j[k]
    return j


def _try(j, setter, *keys, conv=lambda v: v):
    try:
        setter(conv(_get(j, *keys)))
        return True
    except (KeyError, TypeError, ValueError):
        return False


@dataclass
class PlasmonSettings:
    """PlasmonScattering's settings (src/simulation/incoherence/inelastic/plasmon.h, read by
    jsonutils.cpp:331-360; mean free path converted from nm to Å).

    With plasmons on, clTEM_cmd draws a table of scattering depths per job before the run
    (src/console/main.cpp:710-727: initDepthVectors, generateScatteringDepths over the crystal's
    thickness), and each job's slice loop tilts its beam at every depth it reaches
    (simulationstem.cpp:191-232, simulationcbed.cpp:145-187, simulationctem.cpp:316-357). apply() copies
    these settings into the engine's config, where the same events are made from seeded draws. Enabling
    them also sets the incoherence iterations count (IncoherentEffects::enabled) and turns mixed static
    potentials off (precalculateTransmission is false, so parallelPotentialsCount is 1)."""
    enabled: bool = False
    kind: str = "full"             # "full" or "individual"
    individual: int = 1
    mean_free_path: float = 100.0  # Å (10 nm)
    characteristic_angle: float = 1.0   # mrad
    critical_angle: float = 0.1         # mrad


def apply_plasmon(cfg, p: "PlasmonSettings"):
    """The plasmon fields of the engine's config (include/mslice.h) from the settings: "individual" n is
    passed as n, "full" as 0."""
    cfg.plasmon = int(bool(p.enabled))
    cfg.plasmon_individual = max(1, int(p.individual)) if p.kind == "individual" else 0
    cfg.plasmon_mfp = float(p.mean_free_path)
    cfg.plasmon_char_angle = float(p.characteristic_angle)
    cfg.plasmon_crit_angle = float(p.critical_angle)


def _read_plasmon(j):
    p = PlasmonSettings()
    pl = ("incoherence", "inelastic scattering", "plasmon")
    _try(j, lambda v: setattr(p, "enabled", v), *pl, "enabled", conv=bool)
    _try(j, lambda v: setattr(p, "kind", v if v in ("full", "individual") else p.kind), *pl, "type", conv=str)
    _try(j, lambda v: setattr(p, "individual", v), *pl, "individual", conv=int)
    _try(j, lambda v: setattr(p, "mean_free_path", v * 10.0), *pl, "mean free path", "value", conv=float)
    _try(j, lambda v: setattr(p, "characteristic_angle", v), *pl, "characteristic angle", "value", conv=float)
    _try(j, lambda v: setattr(p, "critical_angle", v), *pl, "critical angle", "value", conv=float)
    return p


def _read_vibrations(j, default):
    """JsonToThermalVibrations (src/simulation/utilities/jsonutils.cpp:368-418): flags default to false;
    per-element values that are not numbers (the "units" entry) are skipped."""
    from .structure import Vibrations, symbol_to_z
    v = Vibrations(default=float(default))
    ph = ("incoherence", "inelastic scattering", "phonon")
    _try(j, lambda b: setattr(v, "force_default", b), *ph, "force default", conv=bool)
    _try(j, lambda b: setattr(v, "force_xyz", b), *ph, "force xyz displacements", conv=bool)
    _try(j, lambda b: setattr(v, "force_defined", b), *ph, "override file", conv=bool)
    try:
        table = _get(j, *ph, "values")
        for name, val in (table.items() if isinstance(table, dict) else []):
            if isinstance(val, (int, float)) and not isinstance(val, bool):
                try:
                    v.values[symbol_to_z(name)] = float(val)
                except RuntimeError:
                    pass
    except (KeyError, TypeError):
        pass
    return v


class SimulationSettings:
    """Host-side view of a clTEM simulation (the subset of SimulationManager the path reads)."""

    def __init__(self):
        self.cfg = abi.config_defaults()
        self.maintain_area = False
        self.potentials = "kirkland"
        self.iterations = 1
        self.phonon_enabled = False
        self.phonon_default_u2 = 0.0
        self.vibrations = None       # structure.Vibrations, set by read_config
        self.parallel_pixels = 1
        self.ccd_name = ""          # "ctem/ccd/name" ("" or "Perfect": no dose simulation)
        self.ccd_dose = 10000.0     # e- per Å^2 (SimulationManager default)
        self.ccd_binning = 1
        self.mixed_static_count = 1
        self.mixed_static_enabled = False
        self.precalculate_transmission = True   # "precalculate transmission" (SimulationManager default)
        self.plasmon = PlasmonSettings()
        self.detectors = []

    def effective_iterations(self) -> int:
        """IncoherentEffects::iterations (src/simulation/incoherence/incoherenteffects.h:40-54): the stored
        count when any effect of the mode is on (phonons or plasmons; chromatic or source size outside
        CTEM), else 1."""
        c = self.cfg
        on = self.phonon_enabled or self.plasmon.enabled or (c.mode != abi.MODE_CTEM and (c.chromatic or c.source_size))
        return max(1, int(self.iterations)) if on else 1

    def mixed_static_sets(self) -> int:
        """SimulationManager::useParallelPotentials / parallelPotentialsCount (simulationmanager.h:185-232):
        mixed static potentials need frozen phonons and precalculated transmissions (which plasmons turn
        off); STEM uses them only with the static frame, the other modes only when there are fewer sets
        than iterations. Returns the set count, or 0 when the reference would not use them."""
        c = self.cfg
        precalc = self.precalculate_transmission and not self.plasmon.enabled
        do_parallel = self.phonon_enabled and precalc and self.mixed_static_enabled
        n = int(self.mixed_static_count)
        if c.mode == abi.MODE_STEM:
            count = n if (do_parallel and not c.stem_moving_frame) else 1
        else:
            count = n if (do_parallel and n < self.effective_iterations()) else 1
        return count if (self.mixed_static_enabled and count > 1) else 0

    # -- detectors -------------------------------------------------------------------------------
    def set_detectors(self, dets):
        """dets: list of (name, inner, outer, xc, yc) in mrad."""
        if len(dets) > abi.MAX_DETECTORS:
            raise ValueError("too many detectors")
        self.detectors = list(dets)
        self.cfg.n_detectors = len(dets)
        for i, (n, a, b, xc, yc) in enumerate(dets):
            d = self.cfg.detectors[i]
            d.name = n.encode()[:47]
            d.inner, d.outer, d.xcentre, d.ycentre = float(a), float(b), float(xc), float(yc)

    def attach_structure(self, structure):
        lim = structure.limits()
        self.cfg.struct_limits[:] = lim
        if not self.maintain_area:
            self.cfg.ctem_area[:] = [lim[0], lim[1], lim[2], lim[3]]
            self.cfg.stem_area[:] = [lim[0], lim[1], lim[2], lim[3]]
            self.cfg.cbed_x = (lim[0] + lim[1]) / 2
            self.cfg.cbed_y = (lim[2] + lim[3]) / 2


def read_config(path_or_dict) -> SimulationSettings:
    if isinstance(path_or_dict, dict):
        j = path_or_dict
    else:
        with open(path_or_dict) as f:
            j = json.load(f)
    s = SimulationSettings()
    c = s.cfg

    def setc(name):
        return lambda v: setattr(c, name, v)

    _try(j, setc("double_precision"), "double precision", conv=lambda v: int(bool(v)))
    if _try(j, setc("mode"), "mode", "id", conv=int) and c.mode == 0:
        c.mode = abi.MODE_CTEM
    _try(j, setc("resolution"), "resolution", conv=int)
    _try(j, setc("slice_thickness"), "slice thickness", "val", conv=float)
    _try(j, setc("slice_offset"), "slice offset", "val", conv=float)
    interval = [0, False]
    _try(j, lambda v: interval.__setitem__(0, v), "intermediate output", "slice interval", conv=int)
    _try(j, lambda v: interval.__setitem__(1, v), "intermediate output", "enabled", conv=bool)
    c.intermediate_slices = interval[0] if interval[1] else 0
    _try(j, setc("full3d"), "full 3d", "state", conv=lambda v: int(bool(v)))
    _try(j, setc("full3d_integrals"), "full 3d", "integrals", conv=int)
    _try(j, lambda v: setattr(s, "maintain_area", v), "maintain areas", conv=bool)
    _try(j, lambda v: setattr(s, "potentials", v), "potentials", conv=str)
    _try(j, setc("padding_xy"), "default padding", "xy", "val", conv=float)
    _try(j, setc("padding_z"), "default padding", "z", "val", conv=float)

    mic = ("microscope",)
    _try(j, setc("voltage"), *mic, "voltage", "val", conv=float)
    _try(j, setc("cond_ap"), *mic, "condenser aperture", "semi-angle", conv=float)
    _try(j, setc("cond_ap_smooth"), *mic, "condenser aperture", "smoothing", conv=float)
    _try(j, setc("obj_ap"), *mic, "objective aperture", "semi-angle", conv=float)
    _try(j, setc("obj_ap_smooth"), *mic, "objective aperture", "smoothing", conv=float)
    _try(j, setc("beam_tilt"), *mic, "beam tilt", "inclination", "val", conv=float)
    _try(j, setc("beam_azimuth"), *mic, "beam tilt", "azimuth", "val", conv=lambda v: (math.pi / 180) * float(v))
    _try(j, setc("alpha"), *mic, "alpha", "val", conv=float)
    _try(j, setc("delta"), *mic, "delta", "val", conv=lambda v: 10 * float(v))
    ab = mic + ("aberrations",)
    _try(j, setc("C10"), *ab, "C10", "val", conv=lambda v: 10 * float(v))
    _try(j, setc("C30"), *ab, "C30", "val", conv=lambda v: 10000 * float(v))
    _try(j, setc("C50"), *ab, "C50", "val", conv=lambda v: 10000 * float(v))
    for name, scale in (("C12", 10), ("C21", 10), ("C23", 10), ("C32", 1e4), ("C34", 1e4), ("C41", 1e4),
                        ("C43", 1e4), ("C45", 1e4), ("C52", 1e4), ("C54", 1e4), ("C56", 1e4)):
        try:
            mag = scale * float(_get(j, *ab, name, "mag"))
            ang = (math.pi / 180) * float(_get(j, *ab, name, "ang"))
            getattr(c, name).mag = mag
            getattr(c, name).ang = ang
        except (KeyError, TypeError, ValueError):
            pass

    _try(j, setc("ctem_image"), "ctem", "simulate image", conv=lambda v: int(bool(v)))
    try:
        c.ctem_area[:] = [float(_get(j, "ctem", "area", "x", "start")), float(_get(j, "ctem", "area", "x", "finish")),
                          float(_get(j, "ctem", "area", "y", "start")), float(_get(j, "ctem", "area", "y", "finish"))]
    except (KeyError, TypeError, ValueError):
        pass
    try:
        xs, xf = float(_get(j, "stem", "area", "x", "start")), float(_get(j, "stem", "area", "x", "finish"))
        xp = int(_get(j, "stem", "scan", "x", "pixels"))
        ys, yf = float(_get(j, "stem", "area", "y", "start")), float(_get(j, "stem", "area", "y", "finish"))
        yp = int(_get(j, "stem", "scan", "y", "pixels"))
        pad = float(_get(j, "stem", "area", "padding", "val"))
        c.stem_area[:] = [xs, xf, ys, yf]
        c.stem_pixels_x, c.stem_pixels_y, c.stem_padding = xp, yp, pad
    except (KeyError, TypeError, ValueError):
        pass
    _try(j, lambda v: setattr(s, "parallel_pixels", v), "stem", "static area", "concurrent pixels", conv=int)
    c.stem_job_pixels = max(1, int(s.parallel_pixels))
    # "static area" off: every job simulates its own window (SimulationManager::currentAreaBase)
    _try(j, lambda v: setattr(c, "stem_moving_frame", 0 if v else 1), "stem", "static area", "enabled", conv=bool)
    dets = []
    try:
        for name, d in _get(j, "stem", "detectors").items():
            try:
                # readJsonEntry<unsigned int>: fractional mrad are truncated
                dets.append((name, int(_get(d, "radius", "inner")), int(_get(d, "radius", "outer")),
                             int(_get(d, "centre", "x")), int(_get(d, "centre", "y"))))
            except (KeyError, TypeError, ValueError):
                pass
    except (KeyError, TypeError):
        pass
    s.set_detectors(dets)
    try:
        c.cbed_x = float(_get(j, "cbed", "position", "x"))
        c.cbed_y = float(_get(j, "cbed", "position", "y"))
        c.cbed_padding = float(_get(j, "cbed", "position", "padding"))
    except (KeyError, TypeError, ValueError):
        pass
    _try(j, lambda v: setattr(s, "iterations", v), "incoherence", "iterations", conv=int)
    ph = ("incoherence", "inelastic scattering", "phonon")
    _try(j, lambda v: setattr(s, "phonon_enabled", v), *ph, "enabled", conv=bool)
    _try(j, lambda v: setattr(s, "phonon_default_u2", v), *ph, "default", "value", conv=float)
    s.vibrations = _read_vibrations(j, s.phonon_default_u2)
    # mixed static potentials (jsonutils.cpp:319-326; SimulationManager::useParallelPotentials)
    _try(j, lambda v: setattr(s, "mixed_static_count", v), *ph, "mixed static potentials", "count", conv=int)
    _try(j, lambda v: setattr(s, "mixed_static_enabled", v), *ph, "mixed static potentials", "enabled", conv=bool)
    _try(j, lambda v: setattr(s, "precalculate_transmission", v), "precalculate transmission", conv=bool)
    s.plasmon = _read_plasmon(j)
    apply_plasmon(c, s.plasmon)
    # probe incoherence (jsonutils.cpp:276-308)
    pr = ("incoherence", "probe")
    _try(j, lambda v: setattr(c, "chromatic", int(v)), *pr, "chromatic", "enabled", conv=bool)
    _try(j, lambda v: setattr(c, "chromatic_cc", v), *pr, "chromatic", "Cc", "val", conv=float)
    _try(j, lambda v: setattr(c, "chromatic_hwhm_pos", v), *pr, "chromatic", "dE", "HWHM +", conv=float)
    _try(j, lambda v: setattr(c, "chromatic_hwhm_neg", v), *pr, "chromatic", "dE", "HWHM -", conv=float)
    _try(j, lambda v: setattr(c, "source_size", int(v)), *pr, "source size", "enabled", conv=bool)
    _try(j, lambda v: setattr(c, "source_fwhm", v), *pr, "source size", "FWHM", "val", conv=float)
    if c.mode != abi.MODE_STEM:
        c.stem_moving_frame = 0   # the static-area switch is read only by STEM
    c.mixed_static = s.mixed_static_sets()
    # CTEM CCD (jsonutils.cpp:176-184)
    _try(j, lambda v: setattr(s, "ccd_name", v), "ctem", "ccd", "name", conv=str)
    _try(j, lambda v: setattr(s, "ccd_dose", v), "ctem", "ccd", "dose", "val", conv=float)
    _try(j, lambda v: setattr(s, "ccd_binning", v), "ctem", "ccd", "binning", conv=int)
    return s


# ---------------------------------------------------------------------------------------------------
# The named workloads (synthetic, seeded)
# ---------------------------------------------------------------------------------------------------
def perovskite_ctem(n=(5, 5, 10), resolution=256, double_precision=True):
    """CTEM plane-wave exit wave of a cubic perovskite (a = 3.905 Å, Sr/Ti/O) supercell over the
    periodic field [0, n_x a], 200 kV, projected Kirkland potential, 1.9525 Å slices."""
    from .structure import perovskite
    st = perovskite(*n)
    s = SimulationSettings()
    c = s.cfg
    c.mode = abi.MODE_CTEM
    c.double_precision = int(double_precision)
    c.resolution = resolution
    c.padding_xy = 0.0
    c.padding_z = 0.0
    c.slice_thickness = 1.9525
    c.slice_offset = 0.97625
    c.voltage = 200.0
    s.maintain_area = True
    L = n[0] * 3.905
    c.ctem_area[:] = [0.0, L, 0.0, L]
    c.ctem_image = 1
    c.C10 = 0.0
    c.C30 = 0.0
    c.obj_ap = 25.0
    c.alpha = 0.0
    c.delta = 0.0
    s.attach_structure(st)
    return s, st


def perovskite_stem(n=(10, 10, 20), resolution=512, scan=64, double_precision=False, area=(13.125, 25.925)):
    """Batched STEM ADF over a perovskite supercell: 300 kV, 24 mrad probe, Cs = 1 um, C1 = 0,
    scan x scan probes on a 0.2 Å raster (12.8 Å at 64), ADF 70-200 mrad, 8 Å xy padding."""
    from .structure import perovskite
    st = perovskite(*n)
    s = SimulationSettings()
    c = s.cfg
    c.mode = abi.MODE_STEM
    c.double_precision = int(double_precision)
    c.resolution = resolution
    c.padding_xy = 8.0
    c.padding_z = 0.0
    c.slice_thickness = 1.9525
    c.slice_offset = 0.97625
    c.voltage = 300.0
    c.cond_ap = 24.0
    c.C10 = 0.0
    c.C30 = 1.0e4
    s.maintain_area = True
    lo, hi = area
    if scan != 64:
        hi = lo + 0.2 * scan
    c.stem_area[:] = [lo, hi, lo, hi]
    c.stem_pixels_x = scan
    c.stem_pixels_y = scan
    c.stem_padding = 0.0
    s.set_detectors([("ADF", 70.0, 200.0, 0.0, 0.0)])
    s.attach_structure(st)
    return s, st


def fcc_cbed(n=(20, 20, 60), resolution=1024, double_precision=False, integrals=4):
    """CBED with the full-3D Lobato potential through an FCC Au-like crystal (a = 4.08 Å), 200 kV,
    10 mrad probe at the field centre, 2.04 Å slices, cbed padding 65.6 Å."""
    from .structure import fcc
    st = fcc(*n)
    s = SimulationSettings()
    c = s.cfg
    c.mode = abi.MODE_CBED
    c.double_precision = int(double_precision)
    c.resolution = resolution
    c.padding_xy = 8.0
    c.padding_z = 0.0
    c.slice_thickness = 2.04
    c.slice_offset = 1.02
    c.voltage = 200.0
    c.cond_ap = 10.0
    c.C10 = 0.0
    c.C30 = 0.0
    c.full3d = 1
    c.full3d_integrals = integrals
    s.potentials = "lobato"
    s.maintain_area = False
    c.cbed_padding = 65.6
    s.attach_structure(st)
    return s, st


def perovskite_dctem(n=(8, 8, 16), resolution=512, double_precision=False):
    """Differentiable CTEM: perovskite 8x8x16 cells (5,120 atoms) over the periodic 31.24 Å field, 300 kV,
    32 slices of 1.9525 Å, C1 = -10 nm, Cs = -15 um, objective aperture 25 mrad, no partial coherence."""
    from .structure import perovskite
    st = perovskite(*n)
    s = SimulationSettings()
    c = s.cfg
    c.mode = abi.MODE_CTEM
    c.double_precision = int(double_precision)
    c.resolution = resolution
    c.padding_xy = 0.0
    c.padding_z = 0.0
    c.slice_thickness = 1.9525
    c.slice_offset = 0.97625
    c.voltage = 300.0
    s.maintain_area = True
    L = n[0] * 3.905
    c.ctem_area[:] = [0.0, L, 0.0, L]
    c.ctem_image = 1
    c.C10 = -100.0
    c.C30 = -1.5e5
    c.obj_ap = 25.0
    c.alpha = 0.0
    c.delta = 0.0
    s.attach_structure(st)
    return s, st


def uneven_stem_cell(rng):
    """One cell of the uneven batched STEM workload, drawn from `rng` (numpy Generator): a perovskite or FCC
    supercell 4-16 cells wide and 10-80 slices thick (two slices per cell), a grid from {256, 384, 512, 768,
    1024}, 80-300 kV, a 16-32 mrad probe (Cs = 1 um), a 16x16 raster over the whole cell, an ADF detector at
    2-5 times the convergence angle and 8 Å xy padding."""
    from .structure import fcc, perovskite
    kind = rng.choice(["perovskite", "fcc"])
    lat = int(rng.integers(4, 17))
    slices = int(rng.integers(10, 81))
    grid = int(rng.choice([256, 384, 512, 768, 1024]))
    kv = float(rng.uniform(80.0, 300.0))
    mrad = float(rng.uniform(16.0, 32.0))
    nz = max(5, (slices + 1) // 2)
    if kind == "perovskite":
        a = 3.905
        st = perovskite(lat, lat, nz)
    else:
        a = 4.08
        st = fcc(lat, lat, nz)
    s = SimulationSettings()
    c = s.cfg
    c.mode = abi.MODE_STEM
    c.double_precision = 0
    c.resolution = grid
    c.allow_any_resolution = 1
    c.padding_xy = 8.0
    c.padding_z = 0.0
    c.slice_thickness = a / 2
    c.slice_offset = a / 4
    c.voltage = kv
    c.cond_ap = mrad
    c.C10 = 0.0
    c.C30 = 1.0e4
    s.maintain_area = True
    c.stem_area[:] = [0.0, lat * a, 0.0, lat * a]
    c.stem_pixels_x = c.stem_pixels_y = 16
    c.stem_padding = 0.0
    s.set_detectors([("ADF", 2.0 * mrad, 5.0 * mrad, 0.0, 0.0)])
    s.attach_structure(st)
    return s, st
