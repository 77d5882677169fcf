"""CTEM dose simulation (DQE filter, seeded Poisson counts, NTF filter) on the GPU against the oracle with the
same seed: the FP64 engine reproduces the oracle's counts, each dosed image draws a new pass, and clearing the
CCD gives the perfect image back."""
import numpy as np
import pytest

from cltem_b200.engine import MsliceError, Simulation
from cltem_b200.params import load_ccds
from tests.cases import small_ctem
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ccd,binning,dose", [("k2", 1, 50.0), ("orius", 2, 1.0e5)])
def test_dosed_image_matches_oracle(gpu_ctx, oracle, kirkland, ccd, binning, dose):
    s, st = small_ctem(double_precision=True)
    s.cfg.seed = 31
    cam = load_ccds()[ccd]
    gpu_ctx.load_params(kirkland)
    sim = Simulation(gpu_ctx, s.cfg)
    sim.set_atoms(st)
    _, _, perfect = sim.ctem()
    sim.set_ccd(cam, binning, dose)
    img0 = sim.ctem()[2]
    img1 = sim.ctem()[2]
    o = oracle.OracleSim(s.cfg, kirkland)
    o.set_atoms(st)
    o.build_transmission()
    o.set_ccd(cam, binning, dose)
    ref0 = o.ctem()[2]
    ref1 = o.ctem()[2]
    assert rel_l2(img0, ref0) < 1e-12 and rel_l2(img1, ref1) < 1e-12
    assert rel_l2(img0, img1) > 1e-3                    # a new noise pass per image
    # the counts are unbiased: the dosed image has the perfect image's mean scaled by the dose per pixel,
    # times the DQE/NTF gain at k = 0
    npix = dose * sim.geo.real_scale ** 2 * binning ** 2
    gain = np.sqrt(cam.dqe[0]) * cam.ntf[0]
    assert abs(img0.mean() / (npix * perfect.mean() * gain) - 1) < 0.05
    sim.set_ccd(None)
    assert np.array_equal(sim.ctem()[2], perfect)


def test_dosed_fp32_close_to_fp64(gpu_ctx, kirkland):
    cam = load_ccds()["k2"]
    imgs = []
    for dp in (True, False):
        s, st = small_ctem(double_precision=dp)
        s.cfg.seed = 5
        gpu_ctx.load_params(kirkland)
        sim = Simulation(gpu_ctx, s.cfg)
        sim.set_atoms(st)
        sim.set_ccd(cam, 1, 1.0e5)
        imgs.append(sim.ctem()[2])
    # the FP32 means differ from FP64 by ~1e-6, which moves a few Poisson counts by one
    assert rel_l2(imgs[1], imgs[0]) < 1e-3


def test_ccd_argument_checks(gpu_ctx, kirkland):
    s, st = small_ctem(double_precision=True)
    gpu_ctx.load_params(kirkland)
    sim = Simulation(gpu_ctx, s.cfg)
    cam = load_ccds()["k2"]
    with pytest.raises(MsliceError):
        sim.set_ccd(cam, 0, 10.0)
    with pytest.raises(MsliceError):
        sim.set_ccd(cam, 1, -1.0)
