"""Incoherence effects on the CPU: the engine's random draws (host code, no device) equal the oracle's
restatement draw for draw, have the reference's distributions, and the oracle's moving-frame geometry and
staged driver reduce to the plain paths when every option is off."""
import numpy as np
import pytest

from cltem_b200 import abi
from cltem_b200.engine import geometry, incoherence_draws
from tests.cases import phonons, small_stem


def _cfg(**kw):
    s, st = small_stem(double_precision=True, scan=4)
    for k, v in kw.items():
        setattr(s.cfg, k, v)
    return s, st


@pytest.mark.parametrize("opts", [dict(chromatic=1, chromatic_cc=1.4, chromatic_hwhm_neg=0.3, chromatic_hwhm_pos=0.6),
                                  dict(mixed_static=5), dict(source_size=1, source_fwhm=0.7),
                                  dict(chromatic=1, chromatic_cc=2.0, chromatic_hwhm_neg=0.0, chromatic_hwhm_pos=0.5,
                                       mixed_static=3, source_size=1, source_fwhm=1.0)])
def test_engine_draws_equal_oracle(oracle, opts):
    s, _ = _cfg(seed=1234, **opts)
    pix = np.arange(37, dtype=np.int32) * 3
    for p in (0, 1, 7):
        e = incoherence_draws(s.cfg, p, pix, 11, 9)
        o = oracle.draws(s.cfg, p, pix, 11, 9)
        for a, b in zip(e, o):
            assert np.array_equal(a, b)


def test_draws_off_are_zero():
    s, _ = _cfg(seed=5)
    df, sets, shift = incoherence_draws(s.cfg, 3, np.arange(10), 4, 3)
    assert not df.any() and not sets.any() and not shift.any()


def test_draw_distributions():
    # defocus: ChromaticAberration::generateDist, a half-normal of sigma_pos with weight 1/(1+r) and of
    # sigma_neg with weight r/(1+r), r = sigma_neg/sigma_pos; focus change = 1e4 Cc dE / kV
    s, _ = _cfg(seed=99, chromatic=1, chromatic_cc=1.0, chromatic_hwhm_neg=0.5, chromatic_hwhm_pos=1.0,
                mixed_static=4, source_size=1, source_fwhm=2.0)
    pix = np.arange(40000, dtype=np.int32)
    df, sets, shift = incoherence_draws(s.cfg, 0, pix, 3, 40000)
    k = 2.0 * np.sqrt(2.0 * np.log(2.0))
    sp, sn = 2.0 * 1.0 / k, 2.0 * 0.5 / k
    scale = 1e4 * 1.0 / s.cfg.voltage
    pos = df[df > 0] / scale
    neg = -df[df < 0] / scale
    r = sn / sp
    assert abs(len(neg) / len(df) - r / (1 + r)) < 0.01
    assert abs(np.sqrt(np.mean(pos ** 2)) - sp) < 0.02 * sp
    assert abs(np.sqrt(np.mean(neg ** 2)) - sn) < 0.03 * sn
    counts = np.bincount(sets.ravel(), minlength=4)
    assert counts.min() > 0.23 * sets.size and counts.max() < 0.27 * sets.size
    sd = 2.0 / k
    assert abs(shift.std() - sd) < 0.02 * sd and abs(shift.mean()) < 0.02 * sd
    # the pass number changes every draw
    df1, sets1, _ = incoherence_draws(s.cfg, 1, pix[:100], 3, 0)
    assert not np.array_equal(df1, df[:100]) and not np.array_equal(sets1, sets[:100])


def test_moving_frame_geometry(oracle):
    s, _ = _cfg(stem_moving_frame=1, stem_padding=6.0)
    g = geometry(s.cfg)
    og = oracle.geometry(s.cfg)[0]
    for f in ("sim_x", "sim_y", "full_x", "full_y", "real_scale", "k_max"):
        assert np.allclose(getattr(g, f)[:] if hasattr(getattr(g, f), "__len__") else getattr(g, f),
                           getattr(og, f)[:] if hasattr(getattr(og, f), "__len__") else getattr(og, f), rtol=0, atol=0), f
    # the window is stem_padding wide plus the cell padding on both sides, at the scan origin
    assert abs((g.sim_x[1] - g.sim_x[0]) - (6.0 + 2 * s.cfg.padding_xy)) < 1e-12
    assert abs((g.sim_x[0] + g.sim_x[1]) / 2 - s.cfg.stem_area[0]) < 1e-12
    # the binning range stays the full padded scan area
    s2, _ = _cfg(stem_padding=6.0)
    g2 = geometry(s2.cfg)
    assert list(g.full_x) == list(g2.full_x) and g.blocks_x == g2.blocks_x


def test_moving_frame_rejections():
    from cltem_b200.engine import MsliceError
    s, _ = _cfg(stem_moving_frame=1, mixed_static=2)
    with pytest.raises(MsliceError):
        geometry(s.cfg)


def test_oracle_staged_reduces_to_plain_average(oracle, kirkland):
    s, st = _cfg()
    s.cfg.resolution = 64
    s.cfg.allow_any_resolution = 1
    confs = phonons(st, 2)
    o = oracle.OracleSim(s.cfg, kirkland)
    got = o.run_staged(confs)
    pix = np.arange(16, dtype=np.int32)
    ref = 0
    for c in confs:
        o.set_atoms(c)
        o.build_transmission()
        ref = ref + o.stem(pix)
    assert np.allclose(got, ref / 2, rtol=1e-14, atol=0)


def test_json_incoherence_keys():
    from cltem_b200.config import read_config
    j = {"mode": {"id": 2}, "resolution": 256,
         "stem": {"static area": {"enabled": False, "concurrent pixels": 5}},
         "incoherence": {"iterations": 7,
                         "probe": {"chromatic": {"enabled": True, "Cc": {"val": 1.3}, "dE": {"HWHM +": 0.9, "HWHM -": 0.4}},
                                   "source size": {"enabled": True, "FWHM": {"val": 0.8}}},
                         "inelastic scattering": {"phonon": {"enabled": True,
                                                             "mixed static potentials": {"enabled": True, "count": 4}}}}}
    s = read_config(j)
    c = s.cfg
    # STEM uses mixed static potentials only with the static frame (parallelPotentialsCount)
    assert (c.stem_moving_frame, c.stem_job_pixels, c.mixed_static) == (1, 5, 0)
    assert (c.chromatic, c.chromatic_cc, c.chromatic_hwhm_pos, c.chromatic_hwhm_neg) == (1, 1.3, 0.9, 0.4)
    assert (c.source_size, c.source_fwhm) == (1, 0.8)
    assert s.effective_iterations() == 7
    j["stem"]["static area"]["enabled"] = True
    assert read_config(j).cfg.mixed_static == 4
    # they need count > 1, frozen phonons and precalculated transmissions, which plasmons turn off
    ph = j["incoherence"]["inelastic scattering"]
    ph["phonon"]["mixed static potentials"]["count"] = 1
    assert read_config(j).cfg.mixed_static == 0
    ph["phonon"]["mixed static potentials"]["count"] = 4
    ph["plasmon"] = {"enabled": True, "mean free path": {"value": 12.0}, "type": "individual", "individual": 2}
    s = read_config(j)
    assert s.cfg.mixed_static == 0 and s.plasmon.enabled and s.plasmon.mean_free_path == 120.0
    assert s.plasmon.kind == "individual" and s.plasmon.individual == 2
    ph["plasmon"]["enabled"] = False
    j["precalculate transmission"] = False
    assert read_config(j).cfg.mixed_static == 0
    j["precalculate transmission"] = True
    ph["phonon"]["enabled"] = False
    assert read_config(j).cfg.mixed_static == 0
    ph["phonon"]["enabled"] = True
    # CBED: only with fewer sets than iterations
    j["mode"]["id"] = 3
    assert read_config(j).cfg.mixed_static == 4
    j["incoherence"]["iterations"] = 4
    assert read_config(j).cfg.mixed_static == 0
    j["incoherence"]["iterations"] = 7
    j["mode"]["id"] = 2
    j["stem"]["static area"]["enabled"] = False
    # plasmons alone switch the incoherence iterations on
    ph["phonon"]["enabled"] = False
    j["incoherence"]["probe"]["chromatic"]["enabled"] = False
    j["incoherence"]["probe"]["source size"]["enabled"] = False
    assert read_config(j).effective_iterations() == 1
    ph["plasmon"]["enabled"] = True
    assert read_config(j).effective_iterations() == 7
    ph["plasmon"]["enabled"] = False
    ph["phonon"]["enabled"] = True
    j["incoherence"]["probe"]["chromatic"]["enabled"] = True
    j["incoherence"]["probe"]["source size"]["enabled"] = True
    # CTEM: chromatic / source size do not count as incoherence (IncoherentEffects::enabled), the moving
    # frame is a STEM switch
    j["mode"]["id"] = 0
    j["incoherence"]["inelastic scattering"]["phonon"]["enabled"] = False
    s = read_config(j)
    assert s.effective_iterations() == 1 and s.cfg.stem_moving_frame == 0


def test_ccd_tables_and_json_keys():
    from cltem_b200.config import read_config
    from cltem_b200.params import CCD_TABLE_SIZE, load_ccds
    ccds = load_ccds()
    assert set(ccds) == {"k2", "orius"}
    for c in ccds.values():
        assert c.dqe.shape == (CCD_TABLE_SIZE,) and c.ntf.shape == (CCD_TABLE_SIZE,)
        assert np.all(c.dqe >= 0) and np.all(c.ntf >= 0)
    s = read_config({"mode": {"id": 0}, "ctem": {"ccd": {"name": "K2", "dose": {"val": 50.0}, "binning": 2}}})
    assert (s.ccd_name, s.ccd_dose, s.ccd_binning) == ("K2", 50.0, 2)
    assert read_config({}).ccd_name == ""


def test_ccd_reader_stream_semantics(tmp_path):
    # the reference reads each table line with `stringstream >> double`, which splits runs like "0.70.6"
    from cltem_b200.params import read_ccd
    vals = " ".join(["0.5"] * 723) + " 0.70.6"
    p = tmp_path / "cam.dat"
    p.write_text("Cam\n\nDQE\n" + vals + "\nNTF\n" + vals + "\n")
    c = read_ccd(str(p))
    assert c.name == "Cam" and c.dqe.size == 725 and c.dqe[-2] == 0.7 and c.dqe[-1] == 0.6
    p.write_text("Cam\nDQE\n0.1 0.2\nNTF\n" + vals + "\n")
    with pytest.raises(RuntimeError):
        read_ccd(str(p))


@pytest.mark.parametrize("lam", [0.0, 0.3, 4.0, 9.9, 10.0, 55.0, 3000.0])
def test_oracle_poisson_moments(oracle, lam):
    x = oracle.poisson(7, 0, np.full(40000, lam))
    assert np.all(x == np.floor(x)) and np.all(x >= 0)
    if lam == 0:
        assert not x.any()
        return
    se = np.sqrt(lam / x.size)
    assert abs(x.mean() - lam) < 5 * se
    assert abs(x.var() / lam - 1) < 0.05
