"""The CLI front end end to end on the GPU: outputs named and laid out as clTEM_cmd writes them."""
import json
import os

import numpy as np
import pytest

from cltem_b200.cli import main as cli_main
from cltem_b200.config import read_config
from cltem_b200.engine import Context, Simulation
from cltem_b200.params import load_default
from cltem_b200.structure import perovskite, phonon_configs, read_xyz, write_xyz
from cltem_b200.tiff import read_tiff
from tests.test_cpu_cli import _cfg_json

pytestmark = pytest.mark.gpu


def test_cli_stem_stack_matches_engine(tmp_path):
    st = perovskite(3, 3, 2)
    xyz = tmp_path / "s.xyz"
    write_xyz(st, str(xyz))
    cfg = _cfg_json()
    cj = tmp_path / "c.json"
    cj.write_text(json.dumps(cfg))
    out = tmp_path / "out"
    assert cli_main([str(xyz), "-c", str(cj), "-o", str(out), "--seed", "5"]) == 0
    files = sorted(os.listdir(out))
    s = read_config(cfg)
    s2 = read_xyz(str(xyz))
    s.attach_structure(s2)
    ctx = Context(0)
    ctx.load_params(load_default("kirkland"))
    sim = Simulation(ctx, s.cfg)
    n_sl = sim.geo.n_slices
    width = len(str(n_sl - 1))
    expect = [f"ADF_{min((i + 1) * 2 - 1, n_sl - 1):0{width}d}.tif" for i in range(sim.n_outputs)]
    assert "ADF.json" in files and all(e in files for e in expect), files
    confs = phonon_configs(s2, 2, np.sqrt(0.0064), seed=5)
    ref = sim.stem_simulate(confs)   # [n_out, n_det, py, px]
    for i, e in enumerate(expect):
        img, tags = read_tiff(str(out / e))
        assert tags[274] == 4
        assert np.allclose(img, ref[i, 0].astype(np.float32), rtol=1e-6)
    sim.close()
    ctx.close()


def test_cli_ctem_outputs(tmp_path):
    st = perovskite(3, 3, 2)
    xyz = tmp_path / "s.xyz"
    write_xyz(st, str(xyz))
    cfg = _cfg_json()
    cfg["mode"] = {"id": 1, "name": "CTEM"}
    cfg["maintain areas"] = False
    cfg["ctem"] = {"simulate image": True}
    cfg["intermediate output"] = {"enabled": False, "slice interval": 0}
    cfg["incoherence"]["inelastic scattering"]["phonon"]["enabled"] = False
    cj = tmp_path / "c.json"
    cj.write_text(json.dumps(cfg))
    out = tmp_path / "out"
    assert cli_main([str(xyz), "-c", str(cj), "-o", str(out)]) == 0
    files = set(os.listdir(out))
    for nm in ("EW_amplitude", "EW_phase", "Diff", "Image"):
        assert nm + ".tif" in files and nm + ".json" in files
    amp, _ = read_tiff(str(out / "EW_amplitude.tif"))
    assert amp.shape == (256, 256) and np.all(np.isfinite(amp))


def test_cli_cif_supercell_ctem_matches_engine(tmp_path):
    from cltem_b200.cif import SuperCellInfo, read_cif_structure
    from tests.test_cpu_cif import PEROVSKITE
    cif = tmp_path / "sto.cif"
    cif.write_text(PEROVSKITE)
    cfg = _cfg_json()
    cfg["mode"] = {"id": 1, "name": "CTEM"}
    cfg["maintain areas"] = False
    cfg["ctem"] = {"simulate image": False}
    cfg["intermediate output"] = {"enabled": False, "slice interval": 0}
    cfg["incoherence"]["inelastic scattering"]["phonon"]["enabled"] = False
    cj = tmp_path / "c.json"
    cj.write_text(json.dumps(cfg))
    out = tmp_path / "out"
    args = [str(cif), "-c", str(cj), "-o", str(out), "-s", "15.5,15.5,8", "-z", "0,0,1", "-n", "1,0,0"]
    assert cli_main(args) == 0
    amp, _ = read_tiff(str(out / "EW_amplitude.tif"))
    st = read_cif_structure(str(cif), SuperCellInfo(uvw=(0, 0, 1), abc=(1, 0, 0), widths=(15.5, 15.5, 8)))
    # Sr on 4 x 4 x 3 lattice points (z = 8 is inside [0, 8] by rounding), Ti 4 x 4 x 2, O 48 + 32 + 32
    assert [(st.Z == z).sum() for z in (38, 22, 8)] == [48, 32, 112]
    s = read_config(cfg)
    s.attach_structure(st)
    ctx = Context(0)
    ctx.load_params(load_default("kirkland"))
    sim = Simulation(ctx, s.cfg)
    sim.set_atoms(st)
    ew, _, _ = sim.ctem()
    assert np.allclose(amp, np.abs(ew[-1]).astype(np.float32), rtol=1e-6, atol=1e-6)
    sim.close()
    ctx.close()
