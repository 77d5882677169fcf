"""Parity at the largest grids of clTEM's resolution list (3072², 4096², 8192²) against the CPU oracle.

At these sizes every plan changes shape: one row or one column a block at 1024 threads (8192²), the FP32
one-column tile at 8192², and at FP64 8192² the twiddle table read from global memory because the table
and one transform's data do not both fit in a block's shared memory. A few atoms at random positions in a
400 Å field keep the oracle's potential sums small (0.05-0.13 Å pixels), so the oracle's time goes to its
transforms; each oracle result is computed once and shared by the FP64 and FP32 cases.
"""
import functools

import numpy as np
import pytest

from cltem_b200.engine import Simulation
from cltem_b200.params import load_default
from cltem_b200.structure import Structure
from tests.cases import small_ctem, small_stem
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL = {True: 1e-12, False: 1e-5}
FIELD = 400.0   # Å
SIZES = [3072, 4096, 8192]


def _atoms(n=24, seed=11, lo=1.0, hi=FIELD - 1.0, z=(0.2, 3.6)):
    rng = np.random.default_rng(seed)
    return Structure(rng.choice([8, 22, 38], n).astype(np.int32), rng.uniform(lo, hi, n), rng.uniform(lo, hi, n),
                     rng.uniform(*z, n))


def _ctem_case(res, dp):
    s, _ = small_ctem(double_precision=dp, res=res, n=(3, 3, 2))
    st = _atoms()
    s.cfg.ctem_area[:] = [0.0, FIELD, 0.0, FIELD]
    s.attach_structure(st)
    return s, st


def _stem_case(res, dp):
    # one probe at the field centre; 192 Å of padding on each side makes the field ~400 Å
    s, _ = small_stem(double_precision=dp, res=res, scan=1)
    c = s.cfg
    c.stem_area[:] = [0.0, 0.2, 0.0, 0.2]
    c.padding_xy = 192.0
    # one slice (the oracle's STEM transforms dominate its time); six Sr atoms within 1.5 Å of the probe so
    # the ADF ring carries a signal well above FP32 rounding of the whole wave
    far = _atoms(lo=-40.0, hi=40.0, z=(0.2, 1.7))
    ang = np.arange(6) * (np.pi / 3)
    rad = np.linspace(0.3, 1.5, 6)
    st = Structure(np.concatenate([far.Z, np.full(6, 38, np.int32)]), np.concatenate([far.x, 0.1 + rad * np.cos(ang)]),
                   np.concatenate([far.y, 0.1 + rad * np.sin(ang)]), np.concatenate([far.z, np.full(6, 1.0)]))
    s.attach_structure(st)
    return s, st


@functools.lru_cache(maxsize=None)
def _oracle_ctem(res):
    from oracle import bind
    s, st = _ctem_case(res, True)
    o = bind.OracleSim(s.cfg, load_default("kirkland"), double_precision=True)
    o.set_atoms(st)
    o.build_transmission()
    return o.ctem()


@functools.lru_cache(maxsize=None)
def _oracle_stem(res):
    from oracle import bind
    s, st = _stem_case(res, True)
    o = bind.OracleSim(s.cfg, load_default("kirkland"), double_precision=True)
    o.set_atoms(st)
    o.build_transmission()
    return o.stem(np.zeros(1, np.int32))


@pytest.mark.parametrize("dp", [True, False])
@pytest.mark.parametrize("res", SIZES)
def test_ctem_parity_large(gpu_ctx, kirkland, dp, res):
    s, st = _ctem_case(res, dp)
    gpu_ctx.load_params(kirkland)
    sim = Simulation(gpu_ctx, s.cfg)
    sim.set_atoms(st)
    ew, diff, img = sim.ctem()
    sim.close()
    oew, odiff, oimg = _oracle_ctem(res)
    assert np.abs(oew - 1.0).max() > 1e-3   # the atoms scatter
    assert rel_l2(ew, oew) < TOL[dp], res
    assert rel_l2(diff, odiff) < TOL[dp], res
    assert rel_l2(img, oimg) < TOL[dp], res


@pytest.mark.parametrize("dp", [True, False])
def test_stem_parity_4096(gpu_ctx, kirkland, dp):
    s, st = _stem_case(4096, dp)
    gpu_ctx.load_params(kirkland)
    sim = Simulation(gpu_ctx, s.cfg)
    sim.set_atoms(st)
    got = sim.stem(np.zeros(1, np.int32))
    sim.close()
    ref = _oracle_stem(4096)
    assert ref[:, 0].max() > 1e-4 * ref[:, 1].max()   # ADF against BF
    for d in range(s.cfg.n_detectors):
        assert rel_l2(got[:, d], ref[:, d]) < TOL[dp], d


_PLAIN = {}


def _plain_stem_8192(gpu_ctx, kirkland):
    if "out" in _PLAIN:
        return _PLAIN["out"]
    s, st = _stem_case(8192, True)
    gpu_ctx.load_params(kirkland)
    sim = Simulation(gpu_ctx, s.cfg)
    sim.set_atoms(st)
    _PLAIN["out"] = sim.stem_plain(np.zeros(1, np.int32))
    sim.close()
    return _PLAIN["out"]


@pytest.mark.parametrize("dp", [True, False])
def test_stem_8192_matches_plain_path(gpu_ctx, kirkland, dp):
    """The oracle's STEM takes minutes at 8192², so the fused probe, row and detector kernels of that size are
    checked against the engine's plain FP64 path instead: cuFFT transforms and the reference's unfused
    kernel sequence, itself held to the fused FP64 path at 1e-12 at the other sizes."""
    s, st = _stem_case(8192, dp)
    gpu_ctx.load_params(kirkland)
    sim = Simulation(gpu_ctx, s.cfg)
    sim.set_atoms(st)
    got = sim.stem(np.zeros(1, np.int32))
    sim.close()
    ref = _plain_stem_8192(gpu_ctx, kirkland)
    assert ref[:, 0].max() > 1e-4 * ref[:, 1].max()   # ADF against BF
    for d in range(s.cfg.n_detectors):
        assert rel_l2(got[:, d], ref[:, d]) < TOL[dp], d
