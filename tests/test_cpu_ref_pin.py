"""Pin the oracle to the reference's own kernels.

oracle/_ref/libref.so holds clTEM's kernels/*_d.cl compiled for the CPU (oracle/build_ref.py). Where it
exists, every restated kernel of the oracle must give bit-identical results on the same inputs (both
sides are built with -ffp-contract=off against the same libm). Inputs stay within the reference's
__local limit of 256 atoms per bin row, beyond which its kernels index past their arrays.
"""
import numpy as np
import pytest

from oracle import ref_bind as rb
from tests.cases import small_cbed, small_ctem, small_stem, phonons

pytestmark = pytest.mark.skipif(not rb.available(), reason="reference kernels not built (oracle/build_ref.py)")


def _pot_args(g, cfg, form, icount, slice_k, full3d):
    ia = np.array([form, icount, cfg.resolution, cfg.resolution, slice_k, g.n_slices, g.blocks_x, g.blocks_y,
                   g.load_blocks_x, g.load_blocks_y, g.load_blocks_z, cfg.full3d_integrals], np.int32)
    if full3d:
        cz = g.z_lims[0] + (g.n_slices - slice_k) * g.dz
        sx = (g.wavevector[0] / g.wavevector[2]) * g.dz / cfg.full3d_integrals
        sy = (g.wavevector[1] / g.wavevector[2]) * g.dz / cfg.full3d_integrals
        tail = [cz, sx, sy]
    else:
        tail = [cfg.beam_tilt, cfg.beam_azimuth]
    da = np.array([g.dz, g.real_scale, g.full_x[1], g.full_x[0], g.full_y[1], g.full_y[0], g.sigma, g.sim_x[0],
                   g.sim_y[0]] + tail, np.float64)
    return ia, da


def test_atom_sort_ids_bit_exact(oracle, kirkland):
    s, st = small_stem()
    g = oracle.geometry(s.cfg)[0]
    for conf in phonons(st, 2):
        o = oracle.OracleSim(s.cfg, kirkland)
        o.set_atoms(conf)
        r = o.sorted_atoms(len(conf))
        keep = ((conf.x > g.full_x[0]) & (conf.x < g.full_x[1]) & (conf.y > g.full_y[0]) & (conf.y < g.full_y[1]) &
                (conf.z > g.z_lims[0]) & (conf.z < g.z_lims[1]))
        x, y, z = (np.ascontiguousarray(v[keep]) for v in (conf.x, conf.y, conf.z))
        n = len(x)
        bid = np.zeros(n, np.int32)
        zid = np.zeros(n, np.int32)
        rb.lib().ref_atom_sort_d(rb.d(x), rb.d(y), rb.d(z), n, g.full_x[0], g.full_x[1], g.full_y[0], g.full_y[1],
                                 g.z_lims[0], g.z_lims[1], g.blocks_x, g.blocks_y, rb.i(bid), rb.i(zid), g.dz, g.n_slices)
        assert np.array_equal(bid, r["block_ids"]) and np.array_equal(zid, r["z_ids"])


@pytest.mark.parametrize("form", ["kirkland", "peng", "lobato"])
def test_projected_potential_bit_exact(oracle, params_all, form):
    s, st = small_stem()
    p = params_all[form]
    o = oracle.OracleSim(s.cfg, p)
    o.set_atoms(phonons(st, 1)[0])
    o.build_transmission()
    g = o.geo
    a = o.sorted_atoms(len(st))
    for k in (0, g.n_slices // 2):
        ia, da = _pot_args(g, s.cfg, p.form, p.i_per_atom, k, False)
        out = np.zeros(2 * s.cfg.resolution ** 2)
        vals = np.ascontiguousarray(p.values)
        rb.lib().ref_transmission_projected_d(rb.d(out), rb.d(a["x"]), rb.d(a["y"]), rb.d(a["z"]), rb.i(a["Z"]),
                                              rb.d(vals), rb.i(ia), rb.d(da), rb.i(a["block_start"]))
        ref = rb.cplx(out, (s.cfg.resolution, s.cfg.resolution))
        assert np.array_equal(ref, o.transmission(k, band_limited=False))


@pytest.mark.parametrize("form", ["lobato", "kirkland"])
def test_full3d_potential_bit_exact(oracle, params_all, form):
    s, st = small_cbed(form=form)
    p = params_all[form]
    o = oracle.OracleSim(s.cfg, p)
    o.set_atoms(st)
    o.build_transmission()
    g = o.geo
    a = o.sorted_atoms(len(st))
    for k in (0, g.n_slices - 1):
        ia, da = _pot_args(g, s.cfg, p.form, p.i_per_atom, k, True)
        out = np.zeros(2 * s.cfg.resolution ** 2)
        vals = np.ascontiguousarray(p.values)
        rb.lib().ref_transmission_full3d_d(rb.d(out), rb.d(a["x"]), rb.d(a["y"]), rb.d(a["z"]), rb.i(a["Z"]),
                                           rb.d(vals), rb.i(ia), rb.d(da), rb.i(a["block_start"]))
        assert np.array_equal(rb.cplx(out, (s.cfg.resolution,) * 2), o.transmission(k, band_limited=False))


def test_band_limit_bit_exact(oracle, kirkland):
    s, st = small_stem()
    o = oracle.OracleSim(s.cfg, kirkland)
    o.set_atoms(st)
    o.build_transmission()
    g, kx, ky = oracle.geometry(s.cfg)
    n = s.cfg.resolution
    t = oracle.fft2(o.transmission(1, band_limited=False))
    flat = rb.inter(t)
    rb.lib().ref_band_limit_d(rb.d(flat), n, n, g.k_max, s.cfg.inverse_limit_factor, rb.d(kx), rb.d(ky))
    got = oracle.fft2(rb.cplx(flat, (n, n)), inverse=True)
    assert np.array_equal(got, o.transmission(1, band_limited=True))


def test_propagator_bit_exact(oracle, kirkland):
    s, _ = small_stem()
    s.cfg.beam_tilt, s.cfg.beam_azimuth = 2.0, 0.3
    o = oracle.OracleSim(s.cfg, kirkland)
    g, kx, ky = oracle.geometry(s.cfg)
    n = s.cfg.resolution
    out = np.zeros(2 * n * n)
    rb.lib().ref_propagator_d(rb.d(out), rb.d(kx), rb.d(ky), n, n, g.dz, g.wavenumber, g.wavevector[0], g.wavevector[1],
                              g.wavevector[2], g.k_max * s.cfg.inverse_limit_factor)
    assert np.array_equal(rb.cplx(out, (n, n)), o.propagator())


def test_probe_bit_exact(oracle, kirkland):
    s, _ = small_stem()
    c = s.cfg
    c.C10, c.C30, c.C50 = 31.0, 1.2e4, 3.0e6
    for nm, (m, a) in {"C12": (12.0, 0.3), "C21": (40.0, -1.0), "C23": (25.0, 2.0), "C32": (900.0, 0.1),
                       "C34": (700.0, 0.5), "C41": (2e4, 1.0), "C43": (1e4, -0.4), "C45": (3e4, 0.9),
                       "C52": (1e6, 0.2), "C54": (2e6, 1.3), "C56": (5e5, -2.0)}.items():
        getattr(c, nm).mag, getattr(c, nm).ang = m, a
    c.cond_ap_smooth = 0.5
    o = oracle.OracleSim(c, kirkland)
    g, kx, ky = oracle.geometry(c)
    n = c.resolution
    for (x, y) in [(4.1, 4.4), (4.7, 3.95)]:
        out = np.zeros(2 * n * n)
        ab = rb.aberr_array(c)
        rb.lib().ref_init_probe_wave_d(rb.d(out), n, n, rb.d(kx), rb.d(ky), x - g.sim_x[0], y - g.sim_y[0], g.wavelength,
                                       c.C10, c.C30, c.C50, rb.d(ab), c.cond_ap, c.cond_ap_smooth)
        assert np.array_equal(rb.cplx(out, (n, n)), o.probe(x, y))


def test_stem_detector_chain_bit_exact(oracle):
    """fft_shift -> complex_to_real(4) -> band_pass -> sum_reduction -> host sum (simulationstem.cpp:42-132)."""
    n = 256
    rng = np.random.default_rng(5)
    recip = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    scale = 0.6836066131937237
    for (inner, outer, xc, yc) in [(40.0, 100.0, 0.0, 0.0), (0.0, 20.0, 3.0, -2.0), (70.0, 200.0, 0.0, 0.0)]:
        sh = np.zeros(2 * n * n)
        r2 = np.zeros(n * n)
        bp = np.zeros(n * n)
        rb.lib().ref_fft_shift_d(rb.d(rb.inter(recip)), rb.d(sh), n, n)
        rb.lib().ref_complex_to_real_d(rb.d(sh), rb.d(r2), 4, n, n)
        rb.lib().ref_band_pass_d(rb.d(r2), rb.d(bp), n, n, inner / scale, outer / scale, xc / scale, yc / scale)
        sums = np.zeros(n * n // 256)
        rb.lib().ref_sum_reduction_d(rb.d(bp), rb.d(sums), n * n)
        total = 0.0
        for v in sums:   # host loop of doSumReduction (simulationstem.cpp:67-69)
            total += v
        assert total == oracle.stem_pixel(recip, scale, inner, outer, xc, yc)


def test_ctem_image_bit_exact(oracle, kirkland):
    s, _ = small_ctem()
    c = s.cfg
    c.obj_ap_smooth = 1.5
    g, kx, ky = oracle.geometry(c)
    n = c.resolution
    rng = np.random.default_rng(9)
    recip = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    out = np.zeros(2 * n * n)
    ab = rb.aberr_array(c)
    rb.lib().ref_ctem_image_d(rb.d(rb.inter(recip)), rb.d(out), n, n, rb.d(kx), rb.d(ky), g.wavelength, c.C10, c.C30,
                              c.C50, rb.d(ab), c.obj_ap, c.obj_ap_smooth, c.alpha, c.delta)
    assert np.array_equal(rb.cplx(out, (n, n)), oracle.ctem_image(c, recip))
