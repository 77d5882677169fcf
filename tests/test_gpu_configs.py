"""Parity of the engine with the CPU oracle at the sizes of the five benchmark workloads.

The smaller parity tests (test_gpu_parity.py) cover every kernel and plan; these run the workloads
themselves, at the size and through the path the benchmark times:
- batched STEM ADF: perovskite 10x10x20 cells, 512^2, 64x64 probes, 40 slices, ADF 70-200 mrad, the
  autotuned probe batch with CUDA-graph replays, staged configuration (seeded u_rms 0.08 Å), compared with
  the FP64 oracle on 8 seeded scan pixels;
- plane-wave CTEM: perovskite 5x5x10 cells, 256^2, 200 kV, 20 slices, exit wave, diffraction and image;
- differentiable CTEM: perovskite 8x8x16 cells, 512^2, 32 slices, C1 = -10 nm, Cs = -15 um, 25 mrad, the
  adjoint gradient against FP64 central differences (h = 1e-4 Å) and the FP32 adjoint against the FP64 one;
- full-3D CBED: FCC Au 20x20x6 cells (the workload's lateral size and grid at a tenth of its thickness),
  1024^2, Lobato, 4 sub-slices, diffraction pattern;
- uneven batched STEM: the first cell of each grid (256^2 to 1024^2) of the seeded 48-cell workload, 4 scan
  pixels against the oracle.

Tolerances: FP64 engine vs FP64 oracle <= 1e-12 relative L2, FP32 engine vs FP64 oracle <= 1e-5.
"""
import numpy as np
import pytest

from cltem_b200 import config
from cltem_b200.engine import Simulation
from cltem_b200.structure import Structure, phonon_configs
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL = {True: 1e-12, False: 1e-5}


def _oracle_stem(oracle, params, cfg, conf, pix):
    o = oracle.OracleSim(cfg, params, double_precision=True)
    o.set_atoms(conf)
    o.build_transmission()
    return o.stem(pix)


def test_stem_headline_workload(gpu_ctx, oracle, kirkland):
    """The benchmark's STEM workload as benchmarked: the autotuned batch, two staged runs (the second replays
    the CUDA graphs of both batch shapes), FP32 against the FP64 oracle, then the FP64 engine."""
    gpu_ctx.load_params(kirkland)
    s, st = config.perovskite_stem(n=(10, 10, 20), resolution=512, scan=64, double_precision=False)
    conf = phonon_configs(st, 1, 0.08, seed=2718)[0]
    pix = np.sort(np.random.default_rng(31).choice(64 * 64, 8, replace=False)).astype(np.int32)
    ref = _oracle_stem(oracle, kirkland, s.cfg, conf, pix)          # [1 output, 1 detector, 8]

    sim = Simulation(gpu_ctx, s.cfg)
    batch, _ = sim.tune_batch()
    assert batch >= 256
    assert sim.geo.n_slices == 40
    sim.stage([conf])
    sim.run_staged()
    first = sim.staged_result().reshape(-1)
    sim.run_staged()                                                 # graph replays
    img = sim.staged_result().reshape(-1)
    assert np.array_equal(first, img)
    err32 = rel_l2(img[pix], ref[0, 0])
    assert err32 < TOL[False], err32
    sim.close()

    s64, _ = config.perovskite_stem(n=(10, 10, 20), resolution=512, scan=64, double_precision=True)
    sim = Simulation(gpu_ctx, s64.cfg)
    sim.set_atoms(conf)
    got = sim.stem(pix)
    assert rel_l2(got[0, 0], ref[0, 0]) < TOL[True]
    sim.close()


@pytest.mark.parametrize("dp", [True, False])
def test_ctem_plane_wave_workload(gpu_ctx, oracle, kirkland, dp):
    """Plane-wave CTEM at full size: perovskite 5x5x10 cells (1,250 atoms), 256^2 over the periodic 19.525 Å
    field, 200 kV, 20 slices; exit wave, diffraction pattern and objective-lens image."""
    gpu_ctx.load_params(kirkland)
    s, st = config.perovskite_ctem(n=(5, 5, 10), resolution=256, double_precision=dp)
    assert len(st) == 1250
    sim = Simulation(gpu_ctx, s.cfg)
    assert sim.geo.n_slices == 20
    o = oracle.OracleSim(s.cfg, kirkland, double_precision=True)
    sim.set_atoms(st)
    o.set_atoms(st)
    o.build_transmission()
    ew, diff, img = sim.ctem()
    oew, odiff, oimg = o.ctem()
    assert rel_l2(ew, oew) < TOL[dp]
    assert rel_l2(diff, odiff) < TOL[dp]
    assert rel_l2(img, oimg) < TOL[dp]
    sim.close()


def _dctem_target(ctx):
    ts, st = config.perovskite_dctem(double_precision=True)
    ts.cfg.C10 += 30.0
    tsim = Simulation(ctx, ts.cfg)
    tsim.set_atoms(phonon_configs(st, 1, 0.05, seed=77)[0])
    target = tsim.ctem()[2][0]
    tsim.close()
    return target


def test_differentiable_ctem_workload(gpu_ctx, kirkland):
    """Gradients at the differentiable-CTEM workload's size (5,120 atoms, 512^2, 32 slices, checkpoints every
    6 slices): FP64 adjoint against FP64 central differences for 4 interior atoms (x and y), C10 and C30; the
    FP32 adjoint against the FP64 adjoint."""
    from copy import deepcopy
    gpu_ctx.load_params(kirkland)
    target = _dctem_target(gpu_ctx)
    s64, st = config.perovskite_dctem(double_precision=True)
    sim = Simulation(gpu_ctx, s64.cfg)
    assert sim.geo.n_slices == 32
    sim.set_atoms(st)
    L, g, g10, g30 = sim.ctem_loss_grad(target, len(st))
    assert abs(L - sim.ctem_loss(target)) <= 1e-9 * L

    def loss(cfg, x, y):
        sm = Simulation(gpu_ctx, cfg)
        sm.set_atoms(Structure(st.Z, x, y, st.z))
        v = sm.ctem_loss(target)
        sm.close()
        return v

    h = 1e-4
    Lf = s64.cfg.ctem_area[1]
    inner = np.where((st.x > 1.0) & (st.y > 1.0) & (st.x < Lf - 1.0) & (st.y < Lf - 1.0))[0]
    for i in np.random.default_rng(5).choice(inner, 4, replace=False):
        for axis in (0, 1):
            xp, yp, xm, ym = st.x.copy(), st.y.copy(), st.x.copy(), st.y.copy()
            (xp if axis == 0 else yp)[i] += h
            (xm if axis == 0 else ym)[i] -= h
            fd = (loss(s64.cfg, xp, yp) - loss(s64.cfg, xm, ym)) / (2 * h)
            assert abs(g[i, axis] - fd) <= 2e-5 * max(abs(fd), 1e-3 * np.abs(g).max()), (i, axis, g[i, axis], fd)
    for name, d, ref in (("C10", 1e-2, g10), ("C30", 10.0, g30)):
        cp, cm = deepcopy(s64.cfg), deepcopy(s64.cfg)
        setattr(cp, name, getattr(cp, name) + d)
        setattr(cm, name, getattr(cm, name) - d)
        fd = (loss(cp, st.x, st.y) - loss(cm, st.x, st.y)) / (2 * d)
        assert abs(ref - fd) <= 1e-5 * max(abs(fd), 1e-12), (name, ref, fd)
    sim.close()

    s32, _ = config.perovskite_dctem(double_precision=False)
    sim = Simulation(gpu_ctx, s32.cfg)
    sim.set_atoms(st)
    L32, g32, g10_32, g30_32 = sim.ctem_loss_grad(target, len(st))
    # the FP32 tolerances of the small-case adjoint test
    assert abs(L32 - L) <= 1e-4 * L
    assert np.linalg.norm(g32 - g) <= 1e-3 * np.linalg.norm(g)
    assert abs(g10_32 - g10) <= 1e-3 * abs(g10) and abs(g30_32 - g30) <= 1e-3 * abs(g30)
    sim.close()


@pytest.fixture(scope="module")
def cbed3d_reference(oracle, lobato):
    """The oracle's diffraction pattern of the reduced full-3D CBED workload (one build serves both
    precisions: about a minute of host time)."""
    s, st = config.fcc_cbed(n=(20, 20, 6), resolution=1024, double_precision=True, integrals=4)
    o = oracle.OracleSim(s.cfg, lobato, double_precision=True)
    o.set_atoms(st)
    o.build_transmission()
    return o.cbed()


@pytest.mark.parametrize("dp", [False, True])
def test_cbed_full3d_workload_reduced_thickness(gpu_ctx, cbed3d_reference, lobato, kirkland, dp):
    """Full-3D CBED at the workload's lateral size and grid (FCC Au 20x20 cells, 1024^2, Lobato, 4 sub-slices,
    cbed padding 65.6 Å) over 6 cells (12 slices) of its 60: the diffraction pattern of one probe."""
    gpu_ctx.load_params(lobato)
    s, st = config.fcc_cbed(n=(20, 20, 6), resolution=1024, double_precision=dp, integrals=4)
    sim = Simulation(gpu_ctx, s.cfg)
    assert sim.geo.n_slices == 12
    sim.set_atoms(st)
    got = sim.cbed()
    sim.close()
    gpu_ctx.load_params(kirkland)
    assert rel_l2(got, cbed3d_reference) < TOL[dp]


def _uneven_first_cells():
    rng = np.random.default_rng(2024)   # the uneven workload's seed
    cells = {}
    for i in range(48):
        s, st = config.uneven_stem_cell(rng)
        cells.setdefault(s.cfg.resolution, (i, s, st))
    return cells


@pytest.mark.parametrize("grid", [256, 384, 512, 768, 1024])
def test_uneven_workload_cells(gpu_ctx, oracle, kirkland, grid):
    """The first cell of each grid in the seeded uneven-batch workload, FP32 with the autotuned batch over its
    whole 16x16 raster (staged, one phonon configuration), 4 seeded pixels against the oracle."""
    gpu_ctx.load_params(kirkland)
    i, s, st = _uneven_first_cells()[grid]
    conf = phonon_configs(st, 1, 0.08, seed=2024 + i)[0]
    sim = Simulation(gpu_ctx, s.cfg)
    sim.tune_batch()
    sim.stage([conf])
    sim.run_staged()
    img = sim.staged_result().reshape(-1)
    sim.close()
    pix = np.sort(np.random.default_rng(grid).choice(256, 4, replace=False)).astype(np.int32)
    ref = _oracle_stem(oracle, kirkland, s.cfg, conf, pix)
    assert rel_l2(img[pix], ref[0, 0]) < TOL[False], (grid, img[pix], ref[0, 0])
