"""Make tests/golden/ref_kernels.npz: outputs of the reference's own double-precision kernels on small
seeded inputs, for parity checks where the reference tree is absent (the GPU box).

Needs oracle/_ref/libref.so, built from the reference's kernels/*_d.cl by oracle/build_ref.py:
    python oracle/build_ref.py [reference_root] && python tests/golden/make_ref_golden.py
Inputs come from the seeded workloads of tests/cases.py; the binned atoms the potential kernels read are
produced by the reference's atom_sort kernel plus the host binning (restated in the oracle, whose ids this
script checks against atom_sort first).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from cltem_b200.params import read_params_json, default_bundle_path  # noqa: E402
from oracle import bind as ob  # noqa: E402
from oracle import ref_bind as rb  # noqa: E402
from tests.cases import phonons, small_cbed, small_ctem, small_stem  # noqa: E402


SUB = 4


def pot_args(g, cfg, form, icount, k, full3d):
    ia = np.array([form, icount, cfg.resolution, cfg.resolution, k, g.n_slices, g.blocks_x, g.blocks_y,
                   g.load_blocks_x, g.load_blocks_y, g.load_blocks_z, cfg.full3d_integrals], np.int32)
    tail = ([g.z_lims[0] + (g.n_slices - k) * g.dz, (g.wavevector[0] / g.wavevector[2]) * g.dz / cfg.full3d_integrals,
             (g.wavevector[1] / g.wavevector[2]) * g.dz / cfg.full3d_integrals] if full3d
            else [cfg.beam_tilt, cfg.beam_azimuth])
    da = np.array([g.dz, g.real_scale, g.full_x[1], g.full_x[0], g.full_y[1], g.full_y[0], g.sigma, g.sim_x[0],
                   g.sim_y[0]] + tail, np.float64)
    return ia, da


def main():
    if not rb.available():
        raise SystemExit("build the reference kernels first: python oracle/build_ref.py [reference_root]")
    P = read_params_json(default_bundle_path())
    L = rb.lib()
    out = {}
    # projected potential (Kirkland) of two slices of a phonon-displaced perovskite, 256^2
    s, st = small_stem()
    conf = phonons(st, 1, seed=11)[0]
    o = ob.OracleSim(s.cfg, P["kirkland"])
    o.set_atoms(conf)
    a = o.sorted_atoms(len(conf))
    g = o.geo
    keep = ((conf.x > g.full_x[0]) & (conf.x < g.full_x[1]) & (conf.y > g.full_y[0]) & (conf.y < g.full_y[1]) &
            (conf.z > g.z_lims[0]) & (conf.z < g.z_lims[1]))
    fx, fy, fz = (np.ascontiguousarray(v[keep]) for v in (conf.x, conf.y, conf.z))
    bid = np.zeros(len(fx), np.int32)
    zid = np.zeros(len(fx), np.int32)
    L.ref_atom_sort_d(rb.d(fx), rb.d(fy), rb.d(fz), len(fx), g.full_x[0], g.full_x[1], g.full_y[0], g.full_y[1],
                      g.z_lims[0], g.z_lims[1], g.blocks_x, g.blocks_y, rb.i(bid), rb.i(zid), g.dz, g.n_slices)
    assert np.array_equal(bid, a["block_ids"]) and np.array_equal(zid, a["z_ids"]), "binning differs from atom_sort"
    for k in (0, 3):
        ia, da = pot_args(g, s.cfg, 0, 3, k, False)
        buf = np.zeros(2 * s.cfg.resolution ** 2)
        L.ref_transmission_projected_d(rb.d(buf), rb.d(a["x"]), rb.d(a["y"]), rb.d(a["z"]), rb.i(a["Z"]),
                                       rb.d(np.ascontiguousarray(P["kirkland"].values)), rb.i(ia), rb.d(da),
                                       rb.i(a["block_start"]))
        out[f"stem_kirkland_T{k}"] = rb.cplx(buf, (s.cfg.resolution,) * 2)
    out["stem_atoms_x"], out["stem_atoms_y"], out["stem_atoms_z"] = conf.x, conf.y, conf.z
    out["stem_atoms_Z"] = conf.Z
    out["stem_block_start"] = a["block_start"]
    # probe (all aberrations) and propagator
    c = s.cfg
    gg, kx, ky = ob.geometry(c)
    n = c.resolution
    pr = np.zeros(2 * n * n)
    L.ref_init_probe_wave_d(rb.d(pr), n, n, rb.d(kx), rb.d(ky), 4.3 - gg.sim_x[0], 4.1 - gg.sim_y[0], gg.wavelength,
                            c.C10, c.C30, c.C50, rb.d(rb.aberr_array(c)), c.cond_ap, c.cond_ap_smooth)
    out["stem_probe_4.3_4.1"] = rb.cplx(pr, (n, n))
    pp = np.zeros(2 * n * n)
    L.ref_propagator_d(rb.d(pp), rb.d(kx), rb.d(ky), n, n, gg.dz, gg.wavenumber, gg.wavevector[0], gg.wavevector[1],
                       gg.wavevector[2], gg.k_max * c.inverse_limit_factor)
    out["stem_propagator"] = rb.cplx(pp, (n, n))
    # full-3D Lobato potential of a small FCC block
    s3, st3 = small_cbed()
    o3 = ob.OracleSim(s3.cfg, P["lobato"])
    o3.set_atoms(st3)
    a3 = o3.sorted_atoms(len(st3))
    ia, da = pot_args(o3.geo, s3.cfg, 2, 5, 1, True)
    buf = np.zeros(2 * s3.cfg.resolution ** 2)
    L.ref_transmission_full3d_d(rb.d(buf), rb.d(a3["x"]), rb.d(a3["y"]), rb.d(a3["z"]), rb.i(a3["Z"]),
                                rb.d(np.ascontiguousarray(P["lobato"].values)), rb.i(ia), rb.d(da), rb.i(a3["block_start"]))
    out["cbed_lobato3d_T1"] = rb.cplx(buf, (s3.cfg.resolution,) * 2)
    # CTEM image transfer applied to a seeded reciprocal wave
    sc, _ = small_ctem()
    cc = sc.cfg
    gc, kxc, kyc = ob.geometry(cc)
    rng = np.random.default_rng(21)
    rw = rng.standard_normal((cc.resolution,) * 2) + 1j * rng.standard_normal((cc.resolution,) * 2)
    im = np.zeros(2 * cc.resolution ** 2)
    L.ref_ctem_image_d(rb.d(rb.inter(rw)), rb.d(im), cc.resolution, cc.resolution, rb.d(kxc), rb.d(kyc), gc.wavelength,
                       cc.C10, cc.C30, cc.C50, rb.d(rb.aberr_array(cc)), cc.obj_ap, cc.obj_ap_smooth, cc.alpha, cc.delta)
    out["ctem_image_out"] = rb.cplx(im, (cc.resolution,) * 2)
    # keep every SUB-th pixel of each image (the comparisons index the same pixels); atoms are kept whole.
    # The CTEM input is regenerated at test time from its seed (np.random.default_rng(21)).
    for k in list(out):
        if out[k].ndim == 2:
            out[k] = out[k][::SUB, ::SUB].copy()
    out["sub"] = np.array(SUB)
    np.savez_compressed(os.path.join(HERE, "ref_kernels.npz"), **out)
    print({k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
