"""Differentiable CTEM under the full 3-D potential: the gradient with respect to atom x, y and z (a true
derivative here, where the projected model's z only selects a slice) against FP64 central finite differences,
and the FP32 engine against the FP64 one.

The full 3-D trapezoid pairs each sub-slice sample with the previous passing sample of its bin row, also across
atoms, so the adjoint replays the forward loops per pixel (gather3d.cu). The finite differences see the same
pairing. Perovskite 4x4x2 cells, 256², Kirkland and Lobato parameterisations, 2 sub-slice integrals: the atoms
sit at multiples of a/2 = 1.9525 Å in z and the sub-slice samples every 0.976 Å, so no atom lies within
0.07 Å of the one-sided 3 Å z test's threshold (a step of 1e-5 Å never flips a test). The central difference's
truncation error falls as h^2 (relative 1e-4 at h = 1e-3 Å, 1e-6 at 1e-4 Å where the potential is curved most);
h = 1e-5 Å leaves it near 1e-8, below the 2e-5 tolerance by far, with FP64 rounding still well under it.

The loss itself jumps where an atom crosses a bin edge: the atom moves to another place in its bin row's sorted
order, and the trapezoid pairs other samples across atoms. The adjoint is the derivative within one binning, so
the finite differences take atoms at least 0.1 Å from every xy bin edge (a quarter of the perovskite's atoms sit
on the edge x = 7.81 Å of this 2 x 2 binning); z bin edges lie 0.976 Å from every atom.
"""
from copy import deepcopy

import numpy as np
import pytest

from cltem_b200.engine import Context, Simulation, geometry
from cltem_b200.structure import Structure, phonon_configs
from tests.cases import small_ctem

pytestmark = pytest.mark.gpu


def _cfg(dp, tilt=False, n=(4, 4, 2)):
    s, st = small_ctem(double_precision=dp, n=n)
    c = s.cfg
    c.C10, c.C30 = -100.0, -1.5e5
    if tilt:    # the 3-D kernel shifts every sub-slice sample by the tilt (shift_x, shift_y), cumulatively
        c.beam_tilt, c.beam_azimuth = 6.0, 0.7
    c.alpha, c.delta = 0.0, 0.0
    c.C12.mag = c.C23.mag = 0.0
    c.full3d, c.full3d_integrals = 1, 2
    return s, st


def _setup(dp, params, tilt=False):
    s, st = _cfg(dp, tilt)
    ctx = Context(0)
    ctx.load_params(params)
    ts, _ = _cfg(True, tilt)
    ts.cfg.C10 = -70.0
    tsim = Simulation(ctx, ts.cfg)
    tsim.set_atoms(phonon_configs(st, 1, 0.05, seed=4)[0])
    _, _, img = tsim.ctem()
    tsim.close()
    return ctx, s, st, img[0]


def _sim64(ctx, s, st, step=None, dc10=0.0):
    cfg = deepcopy(s.cfg)
    cfg.double_precision = 1
    cfg.C10 += dc10
    sim = Simulation(ctx, cfg)
    xyz = [st.x.copy(), st.y.copy(), st.z.copy()]
    if step is not None:
        i, axis, h = step
        xyz[axis][i] += h
    sim.set_atoms(Structure(st.Z, *xyz))
    return sim


@pytest.mark.parametrize("form,tilt", [("kirkland", False), ("lobato", False), ("kirkland", True)])
def test_full3d_adjoint_matches_finite_differences(form, tilt, kirkland, lobato):
    params = kirkland if form == "kirkland" else lobato
    ctx, s, st, target = _setup(True, params, tilt)
    sim = Simulation(ctx, s.cfg)
    sim.set_atoms(st)
    L, g, g10, g30 = sim.ctem_loss_grad(target, len(st))
    assert abs(L - sim.ctem_loss(target)) <= 1e-9 * L
    assert np.abs(g[:, 2]).max() > 0            # z is a real coordinate of the 3-D potential
    geo = geometry(s.cfg)
    ex = np.linspace(geo.full_x[0], geo.full_x[1], geo.blocks_x + 1)
    ey = np.linspace(geo.full_y[0], geo.full_y[1], geo.blocks_y + 1)
    off_edges = (np.abs(st.x[:, None] - ex).min(1) > 0.1) & (np.abs(st.y[:, None] - ey).min(1) > 0.1)
    inner = np.where(off_edges)[0]
    h = 1e-5
    for i in np.random.default_rng(7).choice(inner, 4, replace=False):
        for axis in (0, 1, 2):
            lp = _sim64(ctx, s, st, (i, axis, +h)).ctem_loss(target)
            lm = _sim64(ctx, s, st, (i, axis, -h)).ctem_loss(target)
            fd = (lp - lm) / (2 * h)
            assert abs(g[i, axis] - fd) <= 2e-5 * max(abs(fd), 1e-3 * np.abs(g).max()), (i, axis, g[i, axis], fd)
    fd10 = (_sim64(ctx, s, st, dc10=1e-2).ctem_loss(target) - _sim64(ctx, s, st, dc10=-1e-2).ctem_loss(target)) / 2e-2
    assert abs(g10 - fd10) <= 1e-5 * abs(fd10)


def test_full3d_adjoint_fp32_close_to_fp64_and_checkpoints(kirkland):
    ctx, s, st, target = _setup(False, kirkland)
    sim = Simulation(ctx, s.cfg)
    sim.set_atoms(st)
    L32, g32, c10_32, c30_32 = sim.ctem_loss_grad(target, len(st))
    s64 = _sim64(ctx, s, st)
    L64, g64, c10_64, c30_64 = s64.ctem_loss_grad(target, len(st))
    assert abs(L32 - L64) <= 1e-4 * L64
    assert np.linalg.norm(g32 - g64) <= 1e-3 * np.linalg.norm(g64)
    assert abs(c10_32 - c10_64) <= 1e-3 * abs(c10_64)
    # the gradient does not depend on how the slices are checkpointed (FP64 atomics: equal to rounding)
    L1, g1, _, _ = s64.ctem_loss_grad(target, len(st), checkpoint_every=1)
    assert abs(L1 - L64) <= 1e-12 * L64
    assert np.abs(g1 - g64).max() <= 1e-10 * np.abs(g64).max()
