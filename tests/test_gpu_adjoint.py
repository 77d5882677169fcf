"""Differentiable CTEM: the hand-written adjoint against FP64 central finite differences.

Loss L = sum (I - I_target)^2 of the CTEM image; the target comes from the same structure with seeded
Gaussian displacements (0.05 Å) and the defocus shifted by 30 Å (the differentiable-CTEM workload).
"""
import numpy as np
import pytest

from cltem_b200.engine import Context, Simulation
from cltem_b200.structure import Structure, phonon_configs
from tests.cases import small_ctem

pytestmark = pytest.mark.gpu


def _setup(dp, kirkland, n=(4, 4, 2)):
    s, st = small_ctem(double_precision=dp, n=n)
    s.cfg.C10, s.cfg.C30 = -100.0, -1.5e5
    s.cfg.alpha, s.cfg.delta = 0.0, 0.0
    s.cfg.C12.mag = s.cfg.C23.mag = 0.0
    ctx = Context(0)
    ctx.load_params(kirkland)
    # target: displaced structure, defocus + 30 Å
    tgt_s, _ = small_ctem(double_precision=True, n=n)
    tgt_s.cfg.C10, tgt_s.cfg.C30 = -70.0, -1.5e5
    tgt_s.cfg.alpha, tgt_s.cfg.delta = 0.0, 0.0
    tgt_s.cfg.C12.mag = tgt_s.cfg.C23.mag = 0.0
    tsim = Simulation(ctx, tgt_s.cfg)
    tsim.set_atoms(phonon_configs(st, 1, 0.05, seed=4)[0])
    _, _, img = tsim.ctem()
    tsim.close()
    return ctx, s, st, img[0]


def _loss64(ctx, s, st, dx=None, dc10=0.0, dc30=0.0):
    from copy import deepcopy
    cfg = deepcopy(s.cfg)
    cfg.double_precision = 1
    cfg.C10 += dc10
    cfg.C30 += dc30
    sim = Simulation(ctx, cfg)
    x, y = st.x.copy(), st.y.copy()
    if dx is not None:
        i, axis, h = dx
        (x if axis == 0 else y)[i] += h
    sim.set_atoms(Structure(st.Z, x, y, st.z))
    return sim


def test_loss_matches_ctem_image(kirkland):
    ctx, s, st, target = _setup(True, kirkland)
    sim = Simulation(ctx, s.cfg)
    sim.set_atoms(st)
    _, _, img = sim.ctem()
    L = sim.ctem_loss(target)
    assert abs(L - np.sum((img[0] - target) ** 2)) <= 1e-10 * L


@pytest.mark.parametrize("ck", [0, 1, 3])
def test_adjoint_fp64_matches_finite_differences(kirkland, ck):
    ctx, s, st, target = _setup(True, kirkland)
    sim = Simulation(ctx, s.cfg)
    sim.set_atoms(st)
    L, g, g10, g30 = sim.ctem_loss_grad(target, len(st), checkpoint_every=ck)
    assert abs(L - sim.ctem_loss(target)) <= 1e-9 * L
    # interior atoms: with zero padding the reference's strict range filter drops atoms on the field edge
    # (x or y = 0), so their gradient is zero while a finite step brings them into the model
    L_ = s.cfg.ctem_area[1]
    inner = np.where((st.x > 0.5) & (st.y > 0.5) & (st.x < L_ - 0.5) & (st.y < L_ - 0.5))[0]
    rng = np.random.default_rng(0)
    h = 1e-4
    for i in rng.choice(inner, 4, replace=False):
        for axis in (0, 1):
            lp = _loss64(ctx, s, st, (i, axis, +h)).ctem_loss(target)
            lm = _loss64(ctx, s, st, (i, axis, -h)).ctem_loss(target)
            fd = (lp - lm) / (2 * h)
            assert abs(g[i, axis] - fd) <= 2e-5 * max(abs(fd), 1e-3 * np.abs(g).max()), (i, axis, g[i, axis], fd)
    assert np.all(g[:, 2] == 0)
    for (dc, ref, name) in ((1e-2, g10, "C10"), (10.0, g30, "C30")):
        kw = {"dc10": dc} if name == "C10" else {"dc30": dc}
        kwm = {"dc10": -dc} if name == "C10" else {"dc30": -dc}
        fd = (_loss64(ctx, s, st, **kw).ctem_loss(target) - _loss64(ctx, s, st, **kwm).ctem_loss(target)) / (2 * dc)
        assert abs(ref - fd) <= 1e-5 * max(abs(fd), 1e-12), (name, ref, fd)


def test_adjoint_fp32_close_to_fp64(kirkland):
    ctx, s, st, target = _setup(False, kirkland)
    sim = Simulation(ctx, s.cfg)
    sim.set_atoms(st)
    L32, g32, c10_32, c30_32 = sim.ctem_loss_grad(target, len(st))
    s64 = _loss64(ctx, s, st)
    L64, g64, c10_64, c30_64 = s64.ctem_loss_grad(target, len(st))
    assert abs(L32 - L64) <= 1e-4 * L64
    assert np.linalg.norm(g32 - g64) <= 1e-3 * np.linalg.norm(g64)
    assert abs(c10_32 - c10_64) <= 1e-3 * abs(c10_64) and abs(c30_32 - c30_64) <= 1e-3 * abs(c30_64)


def test_torch_autograd_function(kirkland):
    import torch
    from cltem_b200.autograd import ctem_image_loss
    ctx, s, st, target = _setup(True, kirkland)
    sim = Simulation(ctx, s.cfg)
    xyz = torch.tensor(np.stack([st.x, st.y, st.z], 1), dtype=torch.float64, requires_grad=True)
    lens = torch.tensor([s.cfg.C10, s.cfg.C30], dtype=torch.float64, requires_grad=True)
    loss = ctem_image_loss(sim, torch.tensor(st.Z), xyz, lens, torch.tensor(target))
    loss.backward()
    sim2 = Simulation(ctx, s.cfg)
    sim2.set_atoms(st)
    L, g, g10, g30 = sim2.ctem_loss_grad(target, len(st))
    assert abs(loss.item() - L) <= 1e-12 * L
    assert np.allclose(xyz.grad.numpy(), g, rtol=0, atol=1e-12 * np.abs(g).max())
    assert np.allclose(lens.grad.numpy(), [g10, g30], rtol=1e-12)


@pytest.mark.parametrize("dp", [True, False])
def test_gradient_independent_of_checkpoint_segments(kirkland, dp):
    """The adjoint band-limits gT, forms gV and gathers the atom gradients once per checkpoint segment (up to
    32 slices a launch): thin slices (0.2 Å, ~40 slices, most of them empty) give the same loss and gradients
    for one slice a segment, 5 slices a segment and every slice in one segment (two atom launches)."""
    ctx, s, st, target = _setup(dp, kirkland)
    s.cfg.slice_thickness = 0.2
    s.cfg.slice_offset = 0.1
    sim = Simulation(ctx, s.cfg)
    sim.set_atoms(st)
    runs = [sim.ctem_loss_grad(target, len(st), checkpoint_every=ck) for ck in (1, 5, 10000)]
    L1, g1, c10, c30 = runs[0]
    assert np.abs(g1).max() > 0
    tol = 1e-12 if dp else 1e-6
    for L, g, d10, d30 in runs[1:]:
        assert abs(L - L1) <= tol * L1
        assert np.abs(g - g1).max() <= tol * np.abs(g1).max()
        assert abs(d10 - c10) <= tol * abs(c10) and abs(d30 - c30) <= tol * abs(c30)


def test_forward_backward_halves_equal_loss_grad(kirkland):
    """mslice_ctem_loss_forward + mslice_ctem_loss_backward give mslice_ctem_loss_grad's numbers; a run in
    between invalidates the forward state."""
    from cltem_b200 import abi
    from cltem_b200.engine import MsliceError
    ctx, s, st, target = _setup(True, kirkland)
    sim = Simulation(ctx, s.cfg)
    sim.set_atoms(st)
    L, g, g10, g30 = sim.ctem_loss_grad(target, len(st))
    L2, tok = sim.ctem_loss_forward(target)
    g2, h10, h30 = sim.ctem_loss_backward(tok, len(st))
    assert L2 == L and np.array_equal(g2, g) and h10 == g10 and h30 == g30
    L3, tok3 = sim.ctem_loss_forward(target)
    sim.ctem()                                          # another run: the forward state is gone
    with pytest.raises(MsliceError) as e:
        sim.ctem_loss_backward(tok3, len(st))
    assert e.value.code == abi.ERR_STATE
    _, tok4 = sim.ctem_loss_forward(target)
    with pytest.raises(MsliceError):
        sim.ctem_loss_backward(tok4 - 1, len(st))       # a stale token


@pytest.mark.parametrize("dp", [True, False])
def test_adjoint_with_beam_tilt_matches_finite_differences(kirkland, dp):
    """Beam tilt (6 mrad at azimuth 0.7 rad): the projected kernel's tilt-corrected radius in the atom gradient,
    the tilted propagator in the adjoint; FP64 against FP64 central differences, FP32 against FP64."""
    ctx, s, st, target = _setup(True, kirkland)
    s.cfg.beam_tilt, s.cfg.beam_azimuth = 6.0, 0.7
    sim = Simulation(ctx, s.cfg)
    sim.set_atoms(st)
    L, g, g10, g30 = sim.ctem_loss_grad(target, len(st))
    L_ = s.cfg.ctem_area[1]
    inner = np.where((st.x > 0.5) & (st.y > 0.5) & (st.x < L_ - 0.5) & (st.y < L_ - 0.5))[0]
    h = 1e-4
    if dp:
        for i in np.random.default_rng(3).choice(inner, 4, replace=False):
            for axis in (0, 1):
                lp = _loss64(ctx, s, st, (i, axis, +h)).ctem_loss(target)
                lm = _loss64(ctx, s, st, (i, axis, -h)).ctem_loss(target)
                fd = (lp - lm) / (2 * h)
                assert abs(g[i, axis] - fd) <= 2e-5 * max(abs(fd), 1e-3 * np.abs(g).max()), (i, axis, g[i, axis], fd)
        fd10 = (_loss64(ctx, s, st, dc10=1e-2).ctem_loss(target) - _loss64(ctx, s, st, dc10=-1e-2).ctem_loss(target)) / 2e-2
        assert abs(g10 - fd10) <= 1e-5 * abs(fd10)
    else:
        from copy import deepcopy
        c32 = deepcopy(s.cfg)
        c32.double_precision = 0
        s32 = Simulation(ctx, c32)
        s32.set_atoms(st)
        c64 = deepcopy(s.cfg)
        c64.double_precision = 1
        s64 = Simulation(ctx, c64)
        s64.set_atoms(st)
        L64, g64, c10_64, c30_64 = s64.ctem_loss_grad(target, len(st))
        L32, g32, c10_32, c30_32 = s32.ctem_loss_grad(target, len(st))
        assert abs(L32 - L64) <= 1e-4 * L64
        assert np.linalg.norm(g32 - g64) <= 1e-3 * np.linalg.norm(g64)
