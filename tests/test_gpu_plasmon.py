"""Plasmon scattering on the GPU against the oracle (FP64 <= 1e-12, FP32 <= 1e-5 relative L2).

Each job's beam is turned at the scattering depths of its seeded table (simulationstem.cpp:190-232,
simulationcbed.cpp:145-187, simulationctem.cpp:316-357): the propagator is rebuilt for the new wavevector, the
full 3-D transmissions that follow get the new sub-slice shifts (both taken from kx, as modifyBeamTilt writes
them), and diffraction outputs and STEM detectors read the pattern translated by the tilt
(translateDiffImage / bilinear_translate_d). With the projected potential the reference's modifyBeamTilt
fails at the first event, and so do the engine and the oracle.
"""
import numpy as np
import pytest

from cltem_b200 import abi
from cltem_b200.engine import MsliceError, Simulation, plasmon_draws
from tests.cases import small_cbed, small_ctem, small_stem
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL = {True: 1e-12, False: 1e-5}


def _plasmon(c, mfp=4.0, char=6.0, crit=60.0, kind=0, seed=5):
    c.plasmon = 1
    c.plasmon_individual = kind
    c.plasmon_mfp = mfp
    c.plasmon_char_angle = char
    c.plasmon_crit_angle = crit
    c.seed = seed


def _events(c, job):
    d, _ = plasmon_draws(c, job, c.struct_limits[5] - c.struct_limits[4])
    return len(d) - 1


def _cbed_case(dp):
    s, st = small_cbed(double_precision=dp, res=128, n=(3, 3, 3), integrals=2)
    s.cfg.allow_any_resolution = 1
    s.cfg.intermediate_slices = 2
    _plasmon(s.cfg)
    return s, st


@pytest.mark.parametrize("dp", [True, False])
def test_cbed_plasmon_parity(gpu_ctx, oracle, lobato, dp):
    s, st = _cbed_case(dp)
    assert _events(s.cfg, 0) >= 2
    gpu_ctx.load_params(lobato)
    sim = Simulation(gpu_ctx, s.cfg)
    sim.set_atoms(st)
    got = sim.cbed()
    o = oracle.OracleSim(s.cfg, lobato, double_precision=True)
    o.set_atoms(st)
    o.build_transmission()
    ref = o.cbed()
    assert rel_l2(got, ref) < TOL[dp]
    # the events change the pattern, and a second run (the beam restored in between) repeats it
    assert np.array_equal(sim.cbed(), got)
    s.cfg.plasmon = 0
    plain = Simulation(gpu_ctx, s.cfg)
    plain.set_atoms(st)
    assert rel_l2(plain.cbed()[-1], got[-1]) > 1e-3
    sim.close()
    plain.close()


def test_cbed_plasmon_staged_passes(gpu_ctx, oracle, lobato):
    """Staged CBED: each pass is its own job with its own depth table (job = pass)."""
    s, st = _cbed_case(True)
    s.cfg.iterations = 3
    gpu_ctx.load_params(lobato)
    sim = Simulation(gpu_ctx, s.cfg)
    sim.stage([st])
    sim.run_staged()
    got = sim.staged_result()
    o = oracle.OracleSim(s.cfg, lobato, double_precision=True)
    ref = o.run_staged([st])
    assert rel_l2(got, ref) < 1e-12
    sim.close()


@pytest.mark.parametrize("dp", [True, False])
def test_ctem_plasmon_parity(gpu_ctx, oracle, lobato, dp):
    s, st = small_ctem(double_precision=dp, res=128, n=(3, 3, 3))
    s.cfg.allow_any_resolution = 1
    s.cfg.full3d = 1
    s.cfg.full3d_integrals = 2
    s.cfg.intermediate_slices = 2
    _plasmon(s.cfg, mfp=3.0)
    assert _events(s.cfg, 0) >= 2
    gpu_ctx.load_params(lobato)
    sim = Simulation(gpu_ctx, s.cfg)
    sim.set_atoms(st)
    ew, diff, img = sim.ctem()
    o = oracle.OracleSim(s.cfg, lobato, double_precision=True)
    o.set_atoms(st)
    o.build_transmission()
    oew, odiff, oimg = o.ctem()
    assert rel_l2(ew, oew) < TOL[dp]
    assert rel_l2(diff, odiff) < TOL[dp]
    assert rel_l2(img, oimg) < TOL[dp]
    sim.close()


@pytest.mark.parametrize("dp", [True, False])
def test_stem_plasmon_parity(gpu_ctx, oracle, lobato, dp):
    """STEM jobs of 2 consecutive pixels, each with its own tilt history; detectors on the translated pattern."""
    s, st = small_stem(double_precision=dp, res=128, n=(3, 3, 3), scan=2, interval=2)
    s.cfg.allow_any_resolution = 1
    s.cfg.full3d = 1
    s.cfg.full3d_integrals = 2
    s.cfg.stem_job_pixels = 2
    _plasmon(s.cfg, mfp=3.0)
    assert _events(s.cfg, 0) >= 1 and _events(s.cfg, 1) >= 1
    gpu_ctx.load_params(lobato)
    sim = Simulation(gpu_ctx, s.cfg)
    sim.set_atoms(st)
    pix = np.arange(4, dtype=np.int32)
    got = sim.stem(pix)
    o = oracle.OracleSim(s.cfg, lobato, double_precision=True)
    o.set_atoms(st)
    o.build_transmission()
    ref = o.stem(pix)
    for d in range(s.cfg.n_detectors):
        assert rel_l2(got[:, d], ref[:, d]) < TOL[dp], (d, got[:, d], ref[:, d])
    sim.close()


def test_stem_plasmon_staged(gpu_ctx, oracle, lobato):
    s, st = small_stem(double_precision=True, res=128, n=(3, 3, 3), scan=2)
    s.cfg.allow_any_resolution = 1
    s.cfg.full3d = 1
    s.cfg.full3d_integrals = 2
    s.cfg.stem_job_pixels = 3
    s.cfg.iterations = 2
    _plasmon(s.cfg, mfp=3.0)
    gpu_ctx.load_params(lobato)
    sim = Simulation(gpu_ctx, s.cfg)
    sim.stage([st])
    sim.run_staged()
    got = sim.staged_result().reshape(sim.n_outputs, s.cfg.n_detectors, -1)
    o = oracle.OracleSim(s.cfg, lobato, double_precision=True)
    ref = o.run_staged([st])
    assert rel_l2(got, ref) < 1e-12
    sim.close()


def test_projected_plasmon_event_fails_like_the_reference(gpu_ctx, oracle, kirkland):
    """Projected potential: the first event stops the run (the reference's modifyBeamTilt sets an argument the
    projected kernel does not have); a table with no event runs normally."""
    s, st = small_cbed(double_precision=True, res=128, n=(3, 3, 3), full3d=False)
    s.cfg.allow_any_resolution = 1
    s.potentials = "kirkland"
    _plasmon(s.cfg, mfp=3.0)
    gpu_ctx.load_params(kirkland)
    sim = Simulation(gpu_ctx, s.cfg)
    sim.set_atoms(st)
    with pytest.raises(MsliceError) as e:
        sim.cbed()
    assert e.value.code == abi.ERR_UNSUPPORTED
    o = oracle.OracleSim(s.cfg, kirkland, double_precision=True)
    o.set_atoms(st)
    o.build_transmission()
    with pytest.raises(RuntimeError):
        o.cbed()
    # "individual" 1 means a table of +inf alone: no event, the plain result
    s.cfg.plasmon_individual = 1
    sim1 = Simulation(gpu_ctx, s.cfg)
    sim1.set_atoms(st)
    s.cfg.plasmon = 0
    sim0 = Simulation(gpu_ctx, s.cfg)
    sim0.set_atoms(st)
    assert np.array_equal(sim1.cbed(), sim0.cbed())
    sim.close()
    sim1.close()
    sim0.close()
