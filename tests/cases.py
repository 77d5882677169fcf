"""Small seeded workloads shared by the parity tests (sizes the CPU oracle finishes in seconds)."""
from cltem_b200 import abi, config
from cltem_b200.structure import fcc, perovskite, phonon_configs


def small_stem(double_precision=True, res=256, n=(4, 4, 4), scan=4, interval=0, detectors=None):
    """STEM through a small perovskite block: 300 kV, 24 mrad, Cs = 1 um, 8 Å padding."""
    s, st = config.perovskite_stem(n=n, resolution=res, scan=scan, double_precision=double_precision,
                                   area=(3.905, 3.905 + 0.2 * scan))
    c = s.cfg
    c.stem_area[:] = [3.905, 3.905 + 0.2 * scan, 3.905, 3.905 + 0.2 * scan]
    s.set_detectors(detectors or [("ADF", 40.0, 100.0, 0.0, 0.0), ("BF", 0.0, 20.0, 0.0, 0.0)])
    c.intermediate_slices = interval
    s.attach_structure(st)
    return s, st


def small_ctem(double_precision=True, res=256, n=(5, 5, 4)):
    s, st = config.perovskite_ctem(n=n, resolution=res, double_precision=double_precision)
    c = s.cfg
    c.C10 = -100.0      # Å
    c.C30 = -1.5e5      # Å
    c.obj_ap = 25.0
    c.alpha = 0.3
    c.delta = 30.0
    c.C12.mag, c.C12.ang = 20.0, 0.3
    c.C23.mag, c.C23.ang = 50.0, 1.1
    s.attach_structure(st)
    return s, st


def small_cbed(double_precision=True, res=256, n=(4, 4, 3), full3d=True, integrals=2, form="lobato"):
    s, st = config.fcc_cbed(n=n, resolution=res, double_precision=double_precision, integrals=integrals)
    c = s.cfg
    c.full3d = int(full3d)
    c.cbed_padding = 4.0
    s.potentials = form
    s.attach_structure(st)
    return s, st


def phonons(st, n=2, u=0.08, seed=7):
    return phonon_configs(st, n, u, seed)
