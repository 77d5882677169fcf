"""CIF input and the zone-axis supercell (no GPU): parsing, symmetry images, tiling, rotations, occupancy,
thermal parameters, frozen-phonon axes and the reference's error behaviour.

Expected values are worked out from the reference's algorithm (src/simulation/cif/*.cpp,
src/simulation/structure/crystalstructure.cpp) for small hand-written files."""
import itertools
import json
import math

import numpy as np
import pytest

from cltem_b200.cif import (CIFReader, SuperCellInfo, axis_rotation, calculate_tiling, make_supercell,
                            normalised_rotation, read_cif_structure, strip_comments_whitespace, wrap_position)
from cltem_b200.cli import main as cli_main
from cltem_b200.config import read_config
from cltem_b200.structure import Vibrations, frozen_phonon_configs, process_occupancy


def _cubic_ops():
    """The 48 operations of m-3m as signed permutations of x, y, z."""
    out = []
    for perm in itertools.permutations("xyz"):
        for signs in itertools.product("+-", repeat=3):
            out.append(",".join(s + p for s, p in zip(signs, perm)))
    return out


def _cif(sym_rows, atom_header, atom_rows, cell=(4.0, 4.0, 4.0, 90.0, 90.0, 90.0), extra=""):
    a, b, c, al, be, ga = cell
    sym = ""
    if sym_rows is not None:
        sym = "loop_\n_symmetry_equiv_pos_as_xyz\n" + "\n".join(sym_rows) + "\n\n"
    return (f"data_test\n# a comment line\n_cell_length_a {a}\n_cell_length_b {b}\n_cell_length_c {c}\n"
            f"_cell_angle_alpha {al}\n_cell_angle_beta {be}\n_cell_angle_gamma {ga}\n\n" + sym +
            "loop_\n" + "\n".join(atom_header) + "\n" + "\n".join(atom_rows) + "\n" + extra)


PEROVSKITE = _cif([f"'{o}'" for o in _cubic_ops()],
                  ["_atom_site_label", "_atom_site_type_symbol", "_atom_site_occupancy", "_atom_site_fract_x",
                   "_atom_site_fract_y", "_atom_site_fract_z"],
                  [" Sr1 Sr2+ 1.0 0.0 0.0 0.0   # A site", " Ti1 Ti4+ 1.0 0.5 0.5 0.5", " O1 O2- 1.0 0.5 0.5 0.0"])


def test_strip_comments_keeps_trailing_whitespace():
    out = strip_comments_whitespace("  a b  \n\n   # only a comment\nx # c # d\n  q\n")
    # leading whitespace goes, the text is cut at the last '#', trailing whitespace stays
    assert out == "a b  \nx # c \nq\n"


def test_wrap_position_semantics():
    assert wrap_position(1.25) == 0.25 and wrap_position(-0.25) == 0.75
    assert wrap_position(-1.0) == 1.0      # 1 + modf(-1) = 1 + (-0)
    assert wrap_position(0.5) == 0.5


def test_symmetry_images_of_perovskite_sites():
    cif = CIFReader(text=PEROVSKITE)
    assert len(cif.symmetries) == 48
    assert [s.elements for s in cif.sites] == [["Sr"], ["Ti"], ["O"]]
    assert cif.sites[0].positions == [[0.0, 0.0, 0.0]]
    assert cif.sites[1].positions == [[0.5, 0.5, 0.5]]
    o = cif.sites[2].positions
    assert len(o) == 3 and sorted(map(tuple, o)) == [(0.0, 0.5, 0.5), (0.5, 0.0, 0.5), (0.5, 0.5, 0.0)]
    assert o[0] == [0.5, 0.5, 0.0]         # the file position comes first
    g = cif.cell
    assert g.avec == [4.0, 0.0, 0.0] and abs(g.bvec[1] - 4.0) < 1e-15 and abs(g.cvec[2] - 4.0) < 1e-15


def test_fractional_translations_and_quoting():
    rows = ["1 x,y,z", '2 "x+1/2,y+1/2,z"', "3 'x+1/2, y, z+1/2'", "4 x,-y+1/2,1/2+z"]
    text = _cif(None, ["_atom_site_label", "_atom_site_type_symbol", "_atom_site_fract_x", "_atom_site_fract_y",
                       "_atom_site_fract_z"], ["Au1 Au 0.0 0.0 0.0"])
    text = text.replace("loop_\n_atom_site_label",
                        "loop_\n_symmetry_equiv_pos_site_id\n_symmetry_equiv_pos_as_xyz\n" + "\n".join(rows)
                        + "\n\nloop_\n_atom_site_label")
    cif = CIFReader(text=text)
    assert len(cif.symmetries) == 4
    op = cif.symmetries[3].ops
    assert (op[1].yf, op[1].c, op[2].zf, op[2].c) == (-1.0, 0.5, 1.0, 0.5)
    assert cif.sites[0].positions == [[0.0, 0.0, 0.0], [0.5, 0.5, 0.0], [0.5, 0.0, 0.5], [0.0, 0.5, 0.5]]


def test_supercell_counts_and_order():
    cif = CIFReader(text=PEROVSKITE)
    sc = make_supercell(cif, SuperCellInfo(widths=(19.0, 19.0, 19.0)))
    # one tile holds 5 atoms; per axis the positions 0, 4, .., 16 (Sr) and 2, .., 18 (Ti, O) lie in [0, 19]
    sym = np.asarray(sc.symbols)
    assert (sym == "Sr").sum() == 125 and (sym == "Ti").sum() == 125 and (sym == "O").sum() == 375
    assert len(sym) == 625
    # order: site, symmetry image, then tiles with z outermost and x innermost
    assert list(sym[:125]) == ["Sr"] * 125
    assert np.allclose(sc.x[:6], [0, 4, 8, 12, 16, 0]) and np.allclose(sc.y[:6], [0, 0, 0, 0, 0, 4])
    assert np.all(sc.z[:25] == 0.0) and abs(sc.z[25] - 4.0) < 1e-15   # c_z = 4 sqrt(..) / sin(90°)
    assert np.all((sc.x >= 0) & (sc.x <= 19) & (sc.y >= 0) & (sc.y <= 19) & (sc.z >= 0) & (sc.z <= 19))
    assert np.all(sc.occ == 1.0) and not sc.defined_u.any()


def test_tiling_range_includes_minus_one():
    basis = [[4.0, 0.0, 0.0], [0.0, 4.0, 0.0], [0.0, 0.0, 4.0]]
    mins, maxs = calculate_tiling(basis, 19.0, 10.0, 3.0)
    assert mins == [-1, -1, -1] and maxs == [5, 3, 1]
    mins, maxs = calculate_tiling([[0.0, 4.0, 0.0], [-4.0, 0.0, 0.0], [0.0, 0.0, 4.0]], 100.0, 100.0, 100.0)
    assert mins == [-1, -25, -1] and maxs == [25, 0, 25]


def test_minus_one_wraps_into_tile_minus_one():
    hdr = ["_atom_site_label", "_atom_site_type_symbol", "_atom_site_fract_x", "_atom_site_fract_y",
           "_atom_site_fract_z"]
    a = make_supercell(CIFReader(text=_cif(["x,y,z"], hdr, ["C1 C -1.0 0.0 0.0"])), SuperCellInfo(widths=(19, 5, 5)))
    b = make_supercell(CIFReader(text=_cif(["x,y,z"], hdr, ["C1 C 0.0 0.0 0.0"])), SuperCellInfo(widths=(19, 5, 5)))
    # -1 wraps to 1 and its identity image wraps to 0: the reference keeps both as positions of the site,
    # so every lattice point holds the atom twice (x = 0 reached from tile -1 by the first)
    bs = sorted(zip(b.x, b.y, b.z))
    assert len(b.x) == 20 and sorted(zip(a.x, a.y, a.z)) == sorted(bs + bs)


def test_rotations():
    R = normalised_rotation([1.0, 1.0, 0.0], [0.0, 0.0, 1.0])
    v = np.asarray(R) @ np.array([1.0, 1.0, 0.0]) / math.sqrt(2)
    assert np.allclose(v, [0, 0, 1], atol=1e-15)
    assert np.allclose(np.asarray(R) @ np.asarray(R).T, np.eye(3), atol=1e-15)
    assert normalised_rotation([0, 0, 2.0], [0, 0, 1.0]) == [[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]]
    Rz = np.asarray(axis_rotation([0, 0, 1.0], math.pi / 2))
    assert np.allclose(Rz @ [1, 0, 0], [0, 1, 0], atol=1e-15)


def test_zone_axis_normal_and_tilt():
    cif = CIFReader(text=PEROVSKITE)
    sc = make_supercell(cif, SuperCellInfo(uvw=(1, 1, 0), widths=(12, 12, 12)))
    a, b, c = (np.asarray(v) for v in sc.basis)
    assert np.allclose(a + b, [0, 0, 4 * math.sqrt(2)], atol=1e-12)    # [110] along z
    assert np.allclose([np.linalg.norm(a), np.linalg.norm(b), np.linalg.norm(c)], 4.0)
    # the in-plane axis: the reference applies the rotation taking x onto the projected [010], which
    # turns the cell by +90 degrees (b ends up along -x)
    sc = make_supercell(cif, SuperCellInfo(abc=(0, 1, 0), widths=(12, 12, 12)))
    a, b, c = (np.asarray(v) for v in sc.basis)
    assert np.allclose(a, [0, 4, 0], atol=1e-12) and np.allclose(b, [-4, 0, 0], atol=1e-12)
    # [-100] is antiparallel to x: a half turn about z
    sc = make_supercell(cif, SuperCellInfo(abc=(-1, 0, 0), widths=(12, 12, 12)))
    assert np.allclose(sc.basis[0], [-4, 0, 0], atol=1e-12)
    sc = make_supercell(cif, SuperCellInfo(tilts=(0, 0, 90), widths=(12, 12, 12)))
    assert np.allclose(sc.basis[0], [0, 4, 0], atol=1e-12)
    sc = make_supercell(cif, SuperCellInfo(tilts=(1.0, 0.5, 0), widths=(12, 12, 12)))
    assert np.allclose(np.linalg.norm(np.asarray(sc.basis), axis=1), 4.0)
    assert len(sc.symbols) > 0


def test_rotation_errors():
    cif = CIFReader(text=PEROVSKITE)
    with pytest.raises(RuntimeError, match="Zone axis rotation matrix contains NaNs"):
        make_supercell(cif, SuperCellInfo(uvw=(0, 0, 0)))
    with pytest.raises(RuntimeError, match="Normal rotation matrix contains NaNs"):
        make_supercell(cif, SuperCellInfo(abc=(0, 0, 1)))


def test_shared_sites_occupancy_and_thermals():
    hdr = ["_atom_site_label", "_atom_site_type_symbol", "_atom_site_occupancy", "_atom_site_fract_x",
           "_atom_site_fract_y", "_atom_site_fract_z", "_atom_site_B_iso_or_equiv"]
    aniso = ("\nloop_\n_atom_site_aniso_label\n_atom_site_aniso_U_11\n_atom_site_aniso_U_22\n_atom_site_aniso_U_33\n"
             "La1 0.011(2) 0.012 0.013\n")
    text = _cif(["x,y,z"], hdr, ["Sr1 Sr 0.5 0.0 0.0 0.0 0.004", "La1 La 0.25(1) 0.0 0.0 0.0 .",
                                 "O1 O 1.0 0.5 0.5 0.5 0.007"], extra=aniso)
    cif = CIFReader(text=text)
    assert len(cif.sites) == 2 and cif.sites[0].elements == ["Sr", "La"]
    assert cif.sites[0].occupancies == [0.5, 0.25]
    assert cif.sites[0].thermal_u == [[0.004, 0.004, 0.004], [0.011, 0.012, 0.013]]
    assert cif.sites[1].thermal_u == [[0.007, 0.007, 0.007]] and cif.sites[0].thermal_defined
    sc = make_supercell(cif, SuperCellInfo(widths=(39, 39, 3)))
    sym = np.asarray(sc.symbols)
    assert list(sym[:4]) == ["Sr", "La", "Sr", "La"]          # elements of a site stay together
    assert sc.defined_u.all()
    s = read_cif_structure(None, SuperCellInfo(widths=(39, 39, 3)), text=text, seed=4, occupancy_draw="uniform")
    n_site = 10 * 10 * 1
    n_sr, n_la, n_o = ((s.Z == z).sum() for z in (38, 57, 8))
    assert n_o == 10 * 10 and abs(n_sr - n_site / 2) < 20 and abs(n_la - n_site / 4) < 16
    assert s.axes.shape == (3, 3) and np.allclose(s.axes, np.eye(3), atol=1e-15)
    assert s.defined_u.all() and s.u2.shape == (len(s), 3)


def test_occupancy_draw_is_the_reference_normal():
    # one site per position: Sr 1/2, Ti 1/4; the reference draws r from N(0, 1)
    n = 20000
    X = np.repeat(np.arange(n, dtype=np.float64), 2)
    Y = np.zeros(2 * n)
    Zc = np.zeros(2 * n)
    occ = np.tile([0.5, 0.25], n)
    keep = process_occupancy(X, Y, Zc, occ, np.random.default_rng(1), "normal")
    p_sr = (keep % 2 == 0).sum() / n
    p_ti = (keep % 2 == 1).sum() / n
    phi = lambda t: 0.5 * (1 + math.erf(t / math.sqrt(2)))   # noqa: E731
    assert abs(p_sr - (phi(0.5) - 0.5)) < 0.01 and abs(p_ti - (phi(0.75) - phi(0.5))) < 0.01
    keep = process_occupancy(X, Y, Zc, occ, np.random.default_rng(1), "uniform")
    assert abs((keep % 2 == 0).sum() / n - 0.5) < 0.015 and abs((keep % 2 == 1).sum() / n - 0.25) < 0.015


def test_fixes_and_errors():
    hdr = ["_atom_site_label", "_atom_site_fract_x", "_atom_site_fract_y", "_atom_site_fract_z"]
    text = _cif(None, hdr, ["Sr1 0 0 0", "ti1 0.5 0.5 0.5"])
    with pytest.raises(RuntimeError) as e:
        CIFReader(text=text)
    assert "Cannot find _symmetry_equiv_pos_ block" in str(e.value)
    assert "Could not find _atom_site_type_symbol" in str(e.value)
    cif = CIFReader(text=text, fix=True)      # P1, symbols from labels, case corrected
    assert [s.elements for s in cif.sites] == [["Sr"], ["Ti"]] and len(cif.symmetries) == 1
    hdr = ["_atom_site_label", "_atom_site_type_symbol", "_atom_site_fract_x", "_atom_site_fract_y",
           "_atom_site_fract_z"]
    with pytest.raises(RuntimeError, match="Could not detect valid atom"):
        CIFReader(text=_cif(["x,y,z"], hdr, ["X1 Qq 0 0 0"]))
    with pytest.raises(RuntimeError, match="not a number"):
        CIFReader(text=_cif(["x,y,z"], hdr, ["Sr1 Sr ? 0 0"]))
    assert CIFReader(text=_cif(["x,y,z"], hdr, ["Sr1 sr 0 0 0"]), fix=True).sites[0].elements == ["Sr"]
    with pytest.raises(RuntimeError, match="Did not find any atoms inside limits"):
        make_supercell(CIFReader(text=_cif(["x,y,z"], hdr, ["Sr1 Sr 0.5 0.5 0.5"])), SuperCellInfo(widths=(1, 1, 1)))


def test_frozen_phonon_axes_and_vibration_table():
    text = PEROVSKITE
    s = read_cif_structure(None, SuperCellInfo(abc=(0, 1, 0), widths=(12, 12, 12)), text=text)
    assert np.allclose(s.axes[0], [0, 1, 0], atol=1e-15) and np.allclose(s.axes[1], [-1, 0, 0], atol=1e-15)
    vib = Vibrations(default=0.01, values={38: 0.02})
    u2 = vib.mean_square(s)
    assert np.all(u2[s.Z == 38] == 0.02) and np.all(u2[s.Z == 8] == 0.01)   # no file values: element table
    (c,) = frozen_phonon_configs(s, 1, vib, seed=3)
    d = np.stack([c.x - s.x, c.y - s.y, c.z - s.z], axis=1)
    rng = np.random.Generator(np.random.PCG64([3, 0]))
    n = rng.standard_normal((len(s), 3)) * np.sqrt(u2)
    # deviate 1 along a' = +y, deviate 2 along b' = -x
    assert np.allclose(d[:, 1], n[:, 0], atol=1e-15) and np.allclose(d[:, 0], -n[:, 1], atol=1e-15)
    (c2,) = frozen_phonon_configs(s, 1, Vibrations(default=0.01, values={38: 0.02}, force_xyz=True), seed=3)
    assert np.allclose(c2.x - s.x, n[:, 0], atol=1e-15)
    assert np.all(Vibrations(default=0.03, force_default=True).mean_square(s) == 0.03)


def test_vibrations_from_json():
    j = {"incoherence": {"inelastic scattering": {"phonon": {
        "enabled": True, "default": {"value": 0.005}, "override file": True, "force xyz displacements": True,
        "values": {"H": 0.002, "Sr": 0.008, "units": "Å²"}}}}}
    v = read_config(j).vibrations
    assert v.default == 0.005 and v.values == {1: 0.002, 38: 0.008}
    assert v.force_defined and v.force_xyz and not v.force_default


def test_cli_cif_options(tmp_path):
    p = tmp_path / "c.json"
    p.write_text(json.dumps({"mode": {"id": 1}}))
    cif = tmp_path / "s.cif"
    cif.write_text(PEROVSKITE)
    out = str(tmp_path / "o")
    assert cli_main([str(cif), "-c", str(p), "-o", out]) == 1                      # -s, -z required
    assert cli_main([str(cif), "-c", str(p), "-o", out, "-s", "10,10", "-z", "0,0,1"]) == 1
    assert cli_main([str(tmp_path / "s.pdb"), "-c", str(p), "-o", out]) == 1
