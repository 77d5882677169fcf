"""CLI front end and file formats (no GPU): TIFF layout, .xyz reading, JSON config reading."""
import json
import os

import numpy as np
import pytest

from cltem_b200 import abi
from cltem_b200.cli import main as cli_main
from cltem_b200.config import read_config
from cltem_b200.structure import perovskite, read_xyz, write_xyz
from cltem_b200.tiff import read_tiff, write_tiff


def test_tiff_roundtrip_and_tags(tmp_path):
    a = np.arange(12, dtype=np.float64).reshape(3, 4) * 0.5
    p = tmp_path / "x.tif"
    write_tiff(str(p), a)
    b, tags = read_tiff(str(p))
    assert np.array_equal(b, a.astype(np.float32))
    assert tags[256] == 4 and tags[257] == 3 and tags[258] == 32 and tags[339] == 3   # float32 samples
    assert tags[274] == 4 and tags[259] == 1 and tags[278] == 3                        # BOTLEFT, raw, one strip


def test_xyz_roundtrip_single_precision(tmp_path):
    st = perovskite(2, 2, 1)
    p = tmp_path / "s.xyz"
    write_xyz(st, str(p))
    r = read_xyz(str(p))
    assert np.array_equal(r.Z, st.Z)
    assert np.allclose(r.x, st.x, atol=1e-5)
    assert all(v == float(np.float32(v)) for v in r.x)   # std::stof semantics


def test_xyz_header_variants(tmp_path):
    p = tmp_path / "h.xyz"
    p.write_text("2\nx y z A occ nm\n0.1 0.2 0.3 Sr 1\n0.4 0.5 0.6 O 1\n")
    r = read_xyz(str(p))
    assert list(r.Z) == [38, 8]
    assert abs(r.x[0] - 1.0) < 1e-6   # nm -> Å
    p.write_text("3\nwrong count\nSr 0 0 0\n")
    with pytest.raises(RuntimeError):
        read_xyz(str(p))


def _cfg_json():
    return {
        "mode": {"id": 2, "name": "STEM"}, "resolution": 256, "double precision": False,
        "slice thickness": {"units": "Å", "val": 1.9525}, "slice offset": {"units": "Å", "val": 0.97625},
        "potentials": "kirkland", "maintain areas": True,
        "default padding": {"xy": {"units": "Å", "val": 8.0}, "z": {"units": "Å", "val": 0.0}},
        "full 3d": {"integrals": 4, "state": False},
        "intermediate output": {"enabled": True, "slice interval": 2},
        "microscope": {"voltage": {"units": "kV", "val": 300.0},
                       "condenser aperture": {"semi-angle": 24.0, "smoothing": 0.0, "units": "mrad"},
                       "aberrations": {"C10": {"units": "nm", "val": 1.5}, "C30": {"units": "μm", "val": 1.0},
                                       "C12": {"mag": 2.0, "ang": 30.0, "units": "nm, °"}},
                       "delta": {"units": "nm", "val": 3.0}, "alpha": {"units": "mrad", "val": 0.3},
                       "beam tilt": {"azimuth": {"units": "°", "val": 90.0}, "inclination": {"units": "mrad", "val": 0.0}}},
        "stem": {"area": {"padding": {"units": "Å", "val": 0.0}, "x": {"start": 3.905, "finish": 4.705, "units": "Å"},
                          "y": {"start": 3.905, "finish": 4.705, "units": "Å"}},
                 "scan": {"x": {"pixels": 2}, "y": {"pixels": 2}},
                 "detectors": {"ADF": {"radius": {"inner": 40.7, "outer": 100.0}, "centre": {"x": 0.0, "y": 0.0}}}},
        "incoherence": {"iterations": 2, "inelastic scattering": {"phonon": {"enabled": True, "force default": True,
                                                                                 "default": {"value": 0.0064}}}},
    }


def test_json_config_units_and_defaults():
    s = read_config(_cfg_json())
    c = s.cfg
    assert c.mode == abi.MODE_STEM and c.resolution == 256 and c.double_precision == 0
    assert c.C10 == 15.0 and c.C30 == 1.0e4                      # nm -> Å, um -> Å
    assert abs(c.C12.mag - 20.0) < 1e-12 and abs(c.C12.ang - np.pi / 6) < 1e-12
    assert c.delta == 30.0 and abs(c.beam_azimuth - np.pi / 2) < 1e-12
    assert c.intermediate_slices == 2 and c.stem_pixels_x == 2
    assert s.detectors[0][1] == 40                               # detector radii truncated to unsigned int
    assert c.obj_ap == 100.0 and c.cond_ap == 24.0               # objective aperture keeps its default
    assert s.phonon_enabled and s.iterations == 2


def test_cli_rejects_cif_and_missing_args(tmp_path, capsys):
    assert cli_main([]) == 1
    p = tmp_path / "c.json"
    p.write_text(json.dumps(_cfg_json()))
    assert cli_main([str(tmp_path / "s.cif"), "-c", str(p), "-o", str(tmp_path / "o")]) == 1
    assert cli_main(["-v"]) == 0


def test_xyz_site_occupancy(tmp_path):
    # consecutive atoms at one position form a site; one draw keeps the atom whose cumulative occupancy
    # interval holds it, or none (CrystalStructure::processOccupancyList)
    lines = []
    for k in range(400):
        lines.append(f"Sr {k}.0 0.0 0.0 0.5")
        lines.append(f"Ti {k}.0 0.0 0.0 0.25")   # same site: Sr 1/2, Ti 1/4, vacancy 1/4
        lines.append(f"O {k}.5 0.0 0.0 1.0")      # a full site of its own
    p = tmp_path / "occ.xyz"
    p.write_text(f"{len(lines)}\nA x y z occ\n" + "\n".join(lines) + "\n")
    s = read_xyz(str(p), seed=3, occupancy_draw="uniform")
    z = np.asarray(s.Z)
    assert (z == 8).sum() == 400
    n_sr, n_ti = (z == 38).sum(), (z == 22).sum()
    assert abs(n_sr - 200) < 45 and abs(n_ti - 100) < 35 and n_sr + n_ti < 400
    # the reference's draw is a standard normal: Sr kept with P(0 <= r < 1/2) = 0.191, Ti with 0.082
    s = read_xyz(str(p), seed=3)
    z = np.asarray(s.Z)
    n_sr, n_ti = (z == 38).sum(), (z == 22).sum()
    assert abs(n_sr - 76.6) < 28 and abs(n_ti - 32.8) < 19 and (z == 8).sum() == 400
    # one atom per site at most, and the draw is repeatable
    xs = np.asarray(s.x)[z != 8]
    assert len(np.unique(xs)) == len(xs)
    s2 = read_xyz(str(p), seed=3)
    assert np.array_equal(np.asarray(s2.Z), z)
    p.write_text("2\nA x y z occ\nSr 0 0 0 0.7\nTi 0 0 0 0.6\n")
    with pytest.raises(RuntimeError):
        read_xyz(str(p))
