"""mslice_bin_atoms_noalloc: atom binning for callers that cannot allocate device memory.

A host application that hands the library only buffers from its own device-memory pool (and forbids
side allocations), or a pipeline stage that cannot afford cudaMalloc's implicit device synchronisation,
needs binning that works entirely in memory it already owns plus the library's fixed scratch. This test
gives the entry point device buffers owned by the caller (here: torch tensors) and checks that two calls
in a row reproduce, bit for bit, what the allocating entry point (mslice_set_atoms) produces. It lives in
a file of its own that pytest collects last.
"""
import ctypes as C

import numpy as np
import pytest

from cltem_b200 import abi
from cltem_b200.engine import Context, Simulation, load_library
from tests.cases import phonons, small_stem

pytestmark = pytest.mark.gpu


def _bind():
    L = load_library()
    f = L.mslice_bin_atoms_noalloc
    f.argtypes = [C.POINTER(abi.Geometry)] + [C.c_void_p] * 4 + [C.c_size_t] + [C.c_void_p] * 6
    f.restype = C.c_int
    return f


def test_noalloc_binning_matches_set_atoms_on_two_calls(kirkland):
    import torch
    fn = _bind()
    ctx = Context(0)
    ctx.load_params(kirkland)
    s, st = small_stem(double_precision=True)
    sim = Simulation(ctx, s.cfg)
    g = sim.geo
    n_bins = g.n_slices * g.blocks_x * g.blocks_y
    dev = torch.device("cuda", 0)
    for call, conf in enumerate(phonons(st, 2, seed=123)):   # two calls in a row, different configurations
        sim.set_atoms(conf)
        ref = sim.sorted_atoms(len(conf))
        n = len(conf)
        dZ = torch.from_numpy(conf.Z.astype(np.int32)).to(dev)
        dx, dy, dz = (torch.from_numpy(np.ascontiguousarray(v)).to(dev) for v in (conf.x, conf.y, conf.z))
        bs = torch.full((n_bins + 1,), -7, dtype=torch.int32, device=dev)
        oZ = torch.zeros(n, dtype=torch.int32, device=dev)
        ox, oy, oz = (torch.zeros(n, dtype=torch.float64, device=dev) for _ in range(3))
        stream = torch.cuda.current_stream(dev).cuda_stream
        rc = fn(C.byref(g), dZ.data_ptr(), dx.data_ptr(), dy.data_ptr(), dz.data_ptr(), n, bs.data_ptr(), oZ.data_ptr(),
                ox.data_ptr(), oy.data_ptr(), oz.data_ptr(), stream)
        assert rc == abi.OK, load_library().mslice_last_error()
        torch.cuda.synchronize(dev)
        got_bs = bs.cpu().numpy()
        assert np.array_equal(got_bs, ref["block_start"]), f"call {call}"
        n_in = int(got_bs[-1])
        assert np.array_equal(oZ.cpu().numpy()[:n_in], ref["Z"][:n_in])
        for k, t in (("x", ox), ("y", oy), ("z", oz)):
            assert np.array_equal(t.cpu().numpy()[:n_in], ref[k][:n_in]), (call, k)
    sim.close()
    ctx.close()


def test_noalloc_binning_at_its_limit(kirkland):
    """131,072 atoms (the limit) over 62,500 bins (a 200 Å field, 100 slices): the tightest carve of the
    scratch, bit-exact against mslice_set_atoms."""
    import torch
    from cltem_b200.structure import Structure
    fn = _bind()
    ctx = Context(0)
    ctx.load_params(kirkland)
    rng = np.random.default_rng(99)
    n = 131072
    conf = Structure(rng.choice([8, 22, 38], n).astype(np.int32), rng.uniform(0, 184, n), rng.uniform(0, 184, n),
                     rng.uniform(0, 195, n))
    s, _ = small_stem(double_precision=False)
    s.maintain_area = True
    s.cfg.stem_area[:] = [0.0, 184.0, 0.0, 184.0]
    s.cfg.slice_thickness, s.cfg.slice_offset = 1.95, 0.0
    s.attach_structure(conf)
    sim = Simulation(ctx, s.cfg)
    g = sim.geo
    n_bins = g.n_slices * g.blocks_x * g.blocks_y
    assert 60000 <= n_bins <= 65535, n_bins
    sim.set_atoms(conf)
    ref = sim.sorted_atoms(n)
    dev = torch.device("cuda", 0)
    dZ = torch.from_numpy(conf.Z).to(dev)
    dx, dy, dz = (torch.from_numpy(np.ascontiguousarray(v)).to(dev) for v in (conf.x, conf.y, conf.z))
    bs = torch.full((n_bins + 1,), -7, dtype=torch.int32, device=dev)
    oZ = torch.zeros(n, dtype=torch.int32, device=dev)
    ox, oy, oz = (torch.zeros(n, dtype=torch.float64, device=dev) for _ in range(3))
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = fn(C.byref(g), dZ.data_ptr(), dx.data_ptr(), dy.data_ptr(), dz.data_ptr(), n, bs.data_ptr(), oZ.data_ptr(),
            ox.data_ptr(), oy.data_ptr(), oz.data_ptr(), stream)
    assert rc == abi.OK, load_library().mslice_last_error()
    torch.cuda.synchronize(dev)
    got_bs = bs.cpu().numpy()
    assert np.array_equal(got_bs, ref["block_start"])
    n_in = int(got_bs[-1])
    assert n_in > 0.9 * n
    assert np.array_equal(oZ.cpu().numpy()[:n_in], ref["Z"][:n_in])
    for k, t in (("x", ox), ("y", oy), ("z", oz)):
        assert np.array_equal(t.cpu().numpy()[:n_in], ref[k][:n_in]), k
    sim.close()
    ctx.close()


def test_noalloc_rejects_sizes_beyond_its_limit(kirkland):
    fn = _bind()
    s, _ = small_stem()
    from cltem_b200.engine import geometry
    g = geometry(s.cfg)
    rc = fn(C.byref(g), 1, 1, 1, 1, 131073, 1, 1, 1, 1, 1, None)   # rejected before any pointer is used
    assert rc == abi.ERR_ARG
    assert b"131072" in load_library().mslice_last_error()
    bad = geometry(s.cfg)
    bad.n_slices = 1                       # does not cover z_lims at thickness dz
    rc = fn(C.byref(bad), 1, 1, 1, 1, 4, 1, 1, 1, 1, 1, None)
    assert rc == abi.ERR_ARG
    assert b"n_slices" in load_library().mslice_last_error()
