"""Parity of the CUDA engine (through the C ABI) with the CPU oracle on seeded inputs.

Tolerances (stated by the task's north star): FP64 engine vs FP64 oracle <= 1e-12 relative L2,
FP32 engine vs FP64 oracle <= 1e-5 relative L2, atom binning bit-exact.
"""
import numpy as np
import pytest

from cltem_b200 import abi
from cltem_b200.engine import Simulation, MsliceError
from cltem_b200.structure import Structure, perovskite
from tests.cases import small_cbed, small_ctem, small_stem, phonons
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL = {True: 1e-12, False: 1e-5}


def _sim(gpu_ctx, params, settings):
    gpu_ctx.load_params(params)
    return Simulation(gpu_ctx, settings.cfg)


def _osim(oracle, params, settings):
    return oracle.OracleSim(settings.cfg, params, double_precision=True)


# ---------------------------------------------------------------------------------------------------
# FFT
# ---------------------------------------------------------------------------------------------------
@pytest.mark.parametrize("dp", [True, False])
@pytest.mark.parametrize("n", [64, 96, 256, 384, 512, 768, 1024])
def test_fft2_matches_oracle_and_numpy(gpu_ctx, oracle, dp, n):
    rng = np.random.default_rng(n)
    a = rng.standard_normal((2, n, n)) + 1j * rng.standard_normal((2, n, n))
    for inverse in (False, True):
        got = gpu_ctx.fft2(a, inverse=inverse, double_precision=dp)
        ref = np.stack([oracle.fft2(a[i], inverse=inverse) for i in range(2)])
        assert rel_l2(got, ref) < (1e-13 if dp else 2e-6)
        if (n & (n - 1)) == 0:
            npref = np.fft.ifft2(a, norm="ortho") if inverse else np.fft.fft2(a, norm="ortho")
            assert rel_l2(got, npref) < (1e-13 if dp else 2e-6)


def test_fft2_of_delta(gpu_ctx):
    n = 256
    a = np.zeros((n, n), complex)
    a[0, 0] = 1.0
    got = gpu_ctx.fft2(a, double_precision=True)
    assert np.allclose(got, np.full((n, n), 1.0 / n), atol=1e-15)


# ---------------------------------------------------------------------------------------------------
# Atom binning: bit-exact
# ---------------------------------------------------------------------------------------------------
def _compare_sorted(a, b):
    assert len(a["Z"]) == len(b["Z"])
    n_in = int(b["block_start"][-1])
    assert np.array_equal(a["block_start"], b["block_start"])
    for k in ("Z", "x", "y", "z"):
        assert np.array_equal(a[k][:n_in], b[k][:n_in]), k
    assert np.array_equal(a["block_ids"], b["block_ids"])
    assert np.array_equal(a["z_ids"], b["z_ids"])


@pytest.mark.parametrize("dp", [True, False])
def test_sort_atoms_bit_exact(gpu_ctx, oracle, kirkland, dp):
    s, st = small_stem(double_precision=dp)
    sim = _sim(gpu_ctx, kirkland, s)
    osim = _osim(oracle, kirkland, s)
    for conf in [st] + phonons(st, 2):
        sim.set_atoms(conf)
        osim.set_atoms(conf)
        _compare_sorted(sim.sorted_atoms(len(conf)), osim.sorted_atoms(len(conf)))


@pytest.mark.parametrize("dp", [True, False])
def test_sort_edge_cases(gpu_ctx, oracle, kirkland, dp):
    s, st = small_stem(double_precision=dp)
    g = oracle.geometry(s.cfg)[0]
    bx = (g.full_x[1] - g.full_x[0]) / g.blocks_x
    # atoms exactly on bin edges, on / just inside the padded limits, out of range, many in one bin row
    xs = [g.full_x[0], g.full_x[0] + bx, g.full_x[0] + 2 * bx, np.nextafter(g.full_x[1], 0), g.full_x[1],
          g.full_x[0] - 1.0, g.full_x[1] + 1.0]
    zs = [g.z_lims[0] + 1e-9, g.z_lims[1] - 1e-9, g.z_lims[0] + g.dz, g.z_lims[1] - g.dz, g.z_lims[1]]
    Z, X, Y, W = [], [], [], []
    for x in xs:
        for z in zs:
            Z.append(8); X.append(x); Y.append(g.full_y[0] + bx); W.append(z)
    rng = np.random.default_rng(3)
    for _ in range(700):   # > 256 atoms in one bin row of one slice
        Z.append(22); X.append(g.full_x[0] + 0.5 * bx + rng.uniform(0, bx)); Y.append(g.full_y[0] + 0.5 * bx)
        W.append(g.z_lims[1] - 0.5 * g.dz)
    st2 = Structure(np.array(Z, np.int32), np.array(X), np.array(Y), np.array(W))
    sim = _sim(gpu_ctx, kirkland, s)
    osim = _osim(oracle, kirkland, s)
    sim.set_atoms(st2)
    osim.set_atoms(st2)
    _compare_sorted(sim.sorted_atoms(len(st2)), osim.sorted_atoms(len(st2)))
    # the long bin row must reach the potential (no 256-atom cap): compare the slice potential
    sim.build_transmission()
    osim.build_transmission()
    assert rel_l2(sim.transmission(0, band_limited=False), osim.transmission(0, band_limited=False)) < TOL[dp]


def test_sort_empty(gpu_ctx, oracle, kirkland):
    s, st = small_stem(double_precision=True)
    empty = Structure(np.zeros(0, np.int32), np.zeros(0), np.zeros(0), np.zeros(0))
    sim = _sim(gpu_ctx, kirkland, s)
    sim.set_atoms(empty)
    r = sim.sorted_atoms(0)
    assert r["block_start"][-1] == 0 and len(r["Z"]) == 0
    sim.build_transmission()
    t = sim.transmission(0)
    assert np.allclose(t, 1.0, atol=1e-12)   # vacuum: T = exp(0)


# ---------------------------------------------------------------------------------------------------
# Transmission functions
# ---------------------------------------------------------------------------------------------------
@pytest.mark.parametrize("dp", [True, False])
@pytest.mark.parametrize("form", ["kirkland", "peng", "lobato"])
@pytest.mark.parametrize("tilt", [0.0, 12.0])
def test_transmission_projected(gpu_ctx, oracle, params_all, dp, form, tilt):
    # tilt (mrad): the tilt-corrected distance of projected_d.cl:283-296
    s, st = small_stem(double_precision=dp)
    s.cfg.beam_tilt, s.cfg.beam_azimuth = tilt, 0.7
    p = params_all[form]
    sim = _sim(gpu_ctx, p, s)
    osim = _osim(oracle, p, s)
    sim.set_atoms(st)
    osim.set_atoms(st)
    sim.build_transmission()
    osim.build_transmission()
    for sl in range(sim.geo.n_slices):
        assert rel_l2(sim.transmission(sl, False), osim.transmission(sl, False)) < TOL[dp]
        assert rel_l2(sim.transmission(sl, True), osim.transmission(sl, True)) < TOL[dp]


@pytest.mark.parametrize("dp", [True, False])
@pytest.mark.parametrize("form", ["lobato", "kirkland", "peng"])
@pytest.mark.parametrize("tilt", [0.0, 12.0])
def test_transmission_full3d(gpu_ctx, oracle, params_all, dp, form, tilt):
    # tilt (mrad): the per-sub-slice shift moves the xy offsets between samples (full_3d_d.cl:244-246)
    s, st = small_cbed(double_precision=dp, form=form)
    s.cfg.beam_tilt, s.cfg.beam_azimuth = tilt, 0.7
    p = params_all[form]
    sim = _sim(gpu_ctx, p, s)
    osim = _osim(oracle, p, s)
    sim.set_atoms(st)
    osim.set_atoms(st)
    sim.build_transmission()
    osim.build_transmission()
    for sl in range(sim.geo.n_slices):
        assert rel_l2(sim.transmission(sl, True), osim.transmission(sl, True)) < TOL[dp]


@pytest.mark.parametrize("dp", [True, False])
def test_transmission_full3d_many_rows(gpu_ctx, oracle, params_all, dp):
    # 0.25 Å slices: each slice reads ±12 z bins, so a tile's list of bin rows (up to 25 x 3) is staged in
    # more than one pass of 64 rows, with the trapezoid's row resets across the passes
    s, st = small_cbed(double_precision=dp, n=(2, 2, 2))
    s.cfg.slice_thickness, s.cfg.slice_offset = 0.25, 0.125
    p = params_all["lobato"]
    sim = _sim(gpu_ctx, p, s)
    osim = _osim(oracle, p, s)
    assert sim.geo.load_blocks_z == 12 and sim.geo.n_slices == 25
    sim.set_atoms(st)
    osim.set_atoms(st)
    sim.build_transmission()
    osim.build_transmission()
    for sl in range(sim.geo.n_slices):
        assert rel_l2(sim.transmission(sl, False), osim.transmission(sl, False)) < TOL[dp], sl


@pytest.mark.parametrize("dp", [True, False])
@pytest.mark.parametrize("form", ["kirkland", "peng", "lobato"])
@pytest.mark.parametrize("full3d", [False, True])
def test_transmission_one_term(gpu_ctx, oracle, params_all, dp, form, full3d):
    # a parameterisation that uses only the first term of each kind (i_per_atom = 1): the kernels index the
    # table with the full per-element stride and sum fewer terms
    from cltem_b200.params import Parameterisation
    full = params_all[form]
    p = Parameterisation(full.name + "_1", full.form, 1, full.values)
    s, st = small_cbed(double_precision=dp, form=form) if full3d else small_stem(double_precision=dp)
    sim = _sim(gpu_ctx, p, s)
    osim = _osim(oracle, p, s)
    sim.set_atoms(st)
    osim.set_atoms(st)
    sim.build_transmission()
    osim.build_transmission()
    for sl in range(sim.geo.n_slices):
        t = sim.transmission(sl, False)
        assert np.all(np.isfinite(t))
        assert rel_l2(t, osim.transmission(sl, False)) < TOL[dp]
    gpu_ctx.load_params(params_all["kirkland"])


# ---------------------------------------------------------------------------------------------------
# Propagator and probe
# ---------------------------------------------------------------------------------------------------
@pytest.mark.parametrize("dp", [True, False])
def test_propagator_and_probe(gpu_ctx, oracle, kirkland, dp):
    s, st = small_stem(double_precision=dp)
    s.cfg.C12.mag, s.cfg.C12.ang = 30.0, 0.4
    s.cfg.C23.mag, s.cfg.C23.ang = 200.0, -0.7
    s.cfg.C10 = 25.0
    sim = _sim(gpu_ctx, kirkland, s)
    osim = _osim(oracle, kirkland, s)
    assert rel_l2(sim.propagator(), osim.propagator()) < (1e-14 if dp else 1e-6)
    for (x, y) in [(4.0, 4.3), (5.1, 3.9)]:
        assert rel_l2(sim.probe(x, y), osim.probe(x, y)) < (1e-12 if dp else 1e-6)


# ---------------------------------------------------------------------------------------------------
# Mode drivers
# ---------------------------------------------------------------------------------------------------
@pytest.mark.parametrize("dp", [True, False])
@pytest.mark.parametrize("interval", [0, 3])
def test_stem_parity(gpu_ctx, oracle, kirkland, dp, interval):
    s, st = small_stem(double_precision=dp, interval=interval)
    sim = _sim(gpu_ctx, kirkland, s)
    osim = _osim(oracle, kirkland, s)
    conf = phonons(st, 1)[0]
    sim.set_atoms(conf)
    osim.set_atoms(conf)
    osim.build_transmission()
    pixels = np.arange(s.cfg.stem_pixels_x * s.cfg.stem_pixels_y, dtype=np.int32)[::-1].copy()
    got = sim.stem(pixels)
    ref = osim.stem(pixels)
    assert got.shape == ref.shape
    for d in range(s.cfg.n_detectors):
        assert rel_l2(got[:, d], ref[:, d]) < TOL[dp], (d, got[:, d], ref[:, d])


@pytest.mark.parametrize("dp", [True, False])
@pytest.mark.parametrize("res", [64, 96, 128, 384, 512, 768, 1024, 1536, 2048])
def test_stem_parity_sizes(gpu_ctx, oracle, kirkland, dp, res):
    # the fused step kernels at every plan the engine picks: radix-8 and 3 * 2^k columns, the two-column
    # FP32 step, the wide FP32 rows at 512 and 1024, the two-row FP32 step elsewhere (one row pair a block
    # from 1536), the FP64 steps with their register budgets
    s, st = small_stem(double_precision=dp, res=res, n=(2, 2, 2), scan=2)
    s.cfg.allow_any_resolution = 1   # 64, 96, 128 and 384 are not in the reference's resolution list
    sim = _sim(gpu_ctx, kirkland, s)
    osim = _osim(oracle, kirkland, s)
    sim.set_atoms(st)
    osim.set_atoms(st)
    osim.build_transmission()
    pixels = np.arange(s.cfg.stem_pixels_x * s.cfg.stem_pixels_y, dtype=np.int32)
    got = sim.stem(pixels)
    ref = osim.stem(pixels)
    for d in range(s.cfg.n_detectors):
        assert rel_l2(got[:, d], ref[:, d]) < TOL[dp], (res, d)


def test_stem_staged_phonon_average(gpu_ctx, oracle, kirkland):
    s, st = small_stem(double_precision=True)
    confs = phonons(st, 3)
    sim = _sim(gpu_ctx, kirkland, s)
    got = sim.stem_simulate(confs)
    osim = _osim(oracle, kirkland, s)
    pix = np.arange(s.cfg.stem_pixels_x * s.cfg.stem_pixels_y, dtype=np.int32)
    acc = 0
    for c in confs:
        osim.set_atoms(c)
        osim.build_transmission()
        acc = acc + osim.stem(pix)
    ref = (acc / len(confs)).reshape(got.shape)
    assert rel_l2(got, ref) < 1e-12


def test_stem_plain_path_matches(gpu_ctx, kirkland):
    s, st = small_stem(double_precision=True, interval=4)
    sim = _sim(gpu_ctx, kirkland, s)
    sim.set_atoms(st)
    pix = np.arange(6, dtype=np.int32)
    assert rel_l2(sim.stem_plain(pix), sim.stem(pix)) < 1e-12


@pytest.mark.parametrize("dp", [True, False])
def test_cbed_full3d_parity(gpu_ctx, oracle, lobato, dp):
    s, st = small_cbed(double_precision=dp)
    sim = _sim(gpu_ctx, lobato, s)
    osim = _osim(oracle, lobato, s)
    sim.set_atoms(st)
    osim.set_atoms(st)
    osim.build_transmission()
    assert rel_l2(sim.cbed(), osim.cbed()) < TOL[dp]


def test_cbed_staged_average(gpu_ctx, oracle, lobato):
    s, st = small_cbed(double_precision=True, full3d=False)
    confs = phonons(st, 2, u=0.09)
    sim = _sim(gpu_ctx, lobato, s)
    sim.stage(confs)
    sim.run_staged()
    got = sim.staged_result()
    osim = _osim(oracle, lobato, s)
    acc = 0
    for c in confs:
        osim.set_atoms(c)
        osim.build_transmission()
        acc = acc + osim.cbed()
    assert rel_l2(got, acc / len(confs)) < 1e-12


@pytest.mark.parametrize("dp", [True, False])
def test_ctem_parity(gpu_ctx, oracle, kirkland, dp):
    s, st = small_ctem(double_precision=dp)
    s.cfg.intermediate_slices = 3
    sim = _sim(gpu_ctx, kirkland, s)
    osim = _osim(oracle, kirkland, s)
    sim.set_atoms(st)
    osim.set_atoms(st)
    osim.build_transmission()
    ew, diff, img = sim.ctem()
    oew, odiff, oimg = osim.ctem()
    assert rel_l2(ew, oew) < TOL[dp]
    assert rel_l2(diff, odiff) < TOL[dp]
    assert rel_l2(img, oimg) < TOL[dp]


@pytest.mark.parametrize("dp", [True, False])
@pytest.mark.parametrize("res", [384, 768, 1024])
def test_ctem_parity_sizes(gpu_ctx, oracle, kirkland, dp, res):
    # one plane wave through the step kernels of each plan (single-wave launches)
    s, st = small_ctem(double_precision=dp, res=res, n=(3, 3, 2))
    s.cfg.allow_any_resolution = 1
    sim = _sim(gpu_ctx, kirkland, s)
    osim = _osim(oracle, kirkland, s)
    sim.set_atoms(st)
    osim.set_atoms(st)
    osim.build_transmission()
    ew, diff, img = sim.ctem()
    oew, odiff, oimg = osim.ctem()
    assert rel_l2(ew, oew) < TOL[dp] and rel_l2(diff, odiff) < TOL[dp] and rel_l2(img, oimg) < TOL[dp]


def test_ctem_vacuum_is_unchanged(gpu_ctx, kirkland):
    s, st = small_ctem(double_precision=True)
    sim = _sim(gpu_ctx, kirkland, s)
    sim.set_atoms(Structure(np.zeros(0, np.int32), np.zeros(0), np.zeros(0), np.zeros(0)))
    ew, diff, img = sim.ctem()
    assert np.allclose(ew, 1.0, atol=1e-12)


# ---------------------------------------------------------------------------------------------------
# Errors through the ABI
# ---------------------------------------------------------------------------------------------------
def test_errors(gpu_ctx, kirkland):
    s, st = small_stem(double_precision=False)
    sim = _sim(gpu_ctx, kirkland, s)
    with pytest.raises(MsliceError) as e:
        sim.build_transmission()
    assert e.value.code == abi.ERR_STATE
    bad = Structure(np.array([200], np.int32), np.array([5.0]), np.array([5.0]), np.array([1.0]))
    with pytest.raises(MsliceError) as e:
        sim.set_atoms(bad)
    assert e.value.code == abi.ERR_ARG
    s2, _ = small_stem()
    s2.cfg.resolution = 300
    with pytest.raises(MsliceError) as e:
        Simulation(gpu_ctx, s2.cfg)
    assert e.value.code == abi.ERR_ARG
    with pytest.raises(MsliceError) as e:
        sim.stem_plain(np.arange(2, dtype=np.int32))
    assert e.value.code == abi.ERR_STATE


def test_cancel_from_progress(gpu_ctx, kirkland):
    s, st = small_stem(double_precision=False, scan=8)
    s.cfg.probe_batch = 4
    sim = _sim(gpu_ctx, kirkland, s)
    sim.set_atoms(st)
    sim.set_progress(lambda f: sim.cancel())
    with pytest.raises(MsliceError) as e:
        sim.stem(np.arange(64, dtype=np.int32))
    assert e.value.code == abi.ERR_CANCELLED
    sim.set_progress(None)
    r = sim.stem(np.arange(4, dtype=np.int32))   # the object stays usable
    assert np.all(np.isfinite(r))


def test_memory_limit(kirkland):
    from cltem_b200.engine import Context
    ctx = Context(0)
    ctx.load_params(kirkland)
    ctx.set_memory_limit(1 << 20)
    s, st = small_stem(double_precision=True)
    with pytest.raises(MsliceError) as e:
        Simulation(ctx, s.cfg)
    assert e.value.code == abi.ERR_OOM
    ctx.close()


# ---------------------------------------------------------------------------------------------------
# Directly against outputs of the reference's own kernels (tests/golden/ref_kernels.npz)
# ---------------------------------------------------------------------------------------------------
@pytest.mark.parametrize("dp", [True, False])
def test_engine_matches_reference_kernel_outputs(gpu_ctx, params_all, dp):
    import os
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_kernels.npz"))
    sub = int(g["sub"])
    conf = Structure(g["stem_atoms_Z"].astype(np.int32), g["stem_atoms_x"], g["stem_atoms_y"], g["stem_atoms_z"])
    s, _ = small_stem(double_precision=dp)
    sim = _sim(gpu_ctx, params_all["kirkland"], s)
    sim.set_atoms(conf)
    assert np.array_equal(sim.sorted_atoms(len(conf))["block_start"], g["stem_block_start"])
    for k in (0, 3):
        assert rel_l2(sim.transmission(k, band_limited=False)[::sub, ::sub], g[f"stem_kirkland_T{k}"]) < TOL[dp]
    assert rel_l2(sim.probe(4.3, 4.1)[::sub, ::sub], g["stem_probe_4.3_4.1"]) < TOL[dp]
    assert rel_l2(sim.propagator()[::sub, ::sub], g["stem_propagator"]) < (1e-14 if dp else 1e-6)
    s3, st3 = small_cbed(double_precision=dp)
    sim3 = _sim(gpu_ctx, params_all["lobato"], s3)
    sim3.set_atoms(st3)
    assert rel_l2(sim3.transmission(1, band_limited=False)[::sub, ::sub], g["cbed_lobato3d_T1"]) < TOL[dp]
