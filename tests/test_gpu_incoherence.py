"""Incoherence effects on the GPU against the oracle's staged driver (same seeded draws): mixed static
potentials, chromatic defocus spread, source-size frame shifts, the moving STEM frame and iterations that
cycle through the staged configurations. FP64 engine <= 1e-12, FP32 engine <= 1e-5 relative L2 against
the FP64 oracle."""
import numpy as np
import pytest

from cltem_b200.engine import MsliceError, Simulation
from tests.cases import phonons, small_cbed, small_stem
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL = {True: 1e-12, False: 1e-5}


def _staged(gpu_ctx, oracle, params, s, confs):
    gpu_ctx.load_params(params)
    sim = Simulation(gpu_ctx, s.cfg)
    sim.stage(confs)
    sim.run_staged()
    got = sim.staged_result()
    ref = oracle.OracleSim(s.cfg, params).run_staged(confs)
    return got.reshape(ref.shape), ref


@pytest.mark.parametrize("dp", [True, False])
def test_mixed_static_stem(gpu_ctx, oracle, kirkland, dp):
    s, st = small_stem(double_precision=dp, scan=3, interval=3)
    s.cfg.mixed_static, s.cfg.iterations, s.cfg.seed = 3, 2, 11
    got, ref = _staged(gpu_ctx, oracle, kirkland, s, phonons(st, 3, seed=21))
    assert rel_l2(got, ref) < TOL[dp]
    # the mixture differs from any single set
    s1, _ = small_stem(double_precision=dp, scan=3, interval=3)
    one, _ = _staged(gpu_ctx, oracle, kirkland, s1, phonons(st, 1, seed=21))
    assert rel_l2(got, one) > 10 * TOL[dp]


@pytest.mark.parametrize("dp", [True, False])
def test_chromatic_and_source_size_stem(gpu_ctx, oracle, kirkland, dp):
    s, st = small_stem(double_precision=dp, scan=3)
    c = s.cfg
    c.chromatic, c.chromatic_cc, c.chromatic_hwhm_neg, c.chromatic_hwhm_pos = 1, 1.5, 0.4, 0.8
    c.source_size, c.source_fwhm, c.seed = 1, 0.6, 5
    got, ref = _staged(gpu_ctx, oracle, kirkland, s, phonons(st, 2, seed=3))
    assert rel_l2(got, ref) < TOL[dp]


@pytest.mark.parametrize("dp,job_pixels,source", [(True, 1, False), (True, 4, True), (False, 3, True)])
def test_moving_frame_stem(gpu_ctx, oracle, kirkland, dp, job_pixels, source):
    s, st = small_stem(double_precision=dp, scan=3)
    c = s.cfg
    c.stem_moving_frame, c.stem_job_pixels, c.stem_padding = 1, job_pixels, 6.0
    c.source_size, c.source_fwhm, c.seed = int(source), 0.4, 8
    got, ref = _staged(gpu_ctx, oracle, kirkland, s, phonons(st, 2, seed=4))
    assert rel_l2(got, ref) < TOL[dp]


def test_moving_frame_single_run_is_pass_zero(gpu_ctx, oracle, kirkland):
    s, st = small_stem(double_precision=True, scan=3)
    s.cfg.stem_moving_frame, s.cfg.stem_job_pixels, s.cfg.stem_padding = 1, 2, 6.0
    gpu_ctx.load_params(kirkland)
    conf = phonons(st, 1, seed=2)
    sim = Simulation(gpu_ctx, s.cfg)
    sim.set_atoms(conf[0])
    got = sim.stem(np.arange(9, dtype=np.int32))
    ref = oracle.OracleSim(s.cfg, kirkland).run_staged(conf)
    assert rel_l2(got, ref) < 1e-12


def test_iterations_cycle_configurations(gpu_ctx, oracle, kirkland):
    s, st = small_stem(double_precision=True, scan=2)
    s.cfg.iterations, s.cfg.chromatic, s.cfg.chromatic_cc = 3, 1, 1.0
    s.cfg.chromatic_hwhm_neg = s.cfg.chromatic_hwhm_pos = 0.5
    got, ref = _staged(gpu_ctx, oracle, kirkland, s, phonons(st, 2, seed=6))
    assert rel_l2(got, ref) < 1e-12


@pytest.mark.parametrize("dp", [True, False])
def test_cbed_incoherent(gpu_ctx, oracle, lobato, dp):
    s, st = small_cbed(double_precision=dp, full3d=False)
    c = s.cfg
    c.mixed_static, c.iterations, c.seed = 2, 3, 17
    c.chromatic, c.chromatic_cc, c.chromatic_hwhm_neg, c.chromatic_hwhm_pos = 1, 1.2, 0.6, 0.6
    c.source_size, c.source_fwhm = 1, 0.5
    got, ref = _staged(gpu_ctx, oracle, lobato, s, phonons(st, 2, seed=12))
    assert rel_l2(got, ref) < TOL[dp]


def test_mixed_static_needs_staging(gpu_ctx, kirkland):
    s, st = small_stem(double_precision=True, scan=2)
    s.cfg.mixed_static = 2
    gpu_ctx.load_params(kirkland)
    sim = Simulation(gpu_ctx, s.cfg)
    sim.set_atoms(st)
    with pytest.raises(MsliceError):
        sim.stem(np.arange(4, dtype=np.int32))
    sim.stage(phonons(st, 1))
    with pytest.raises(MsliceError):   # fewer configurations than sets
        sim.run_staged()
