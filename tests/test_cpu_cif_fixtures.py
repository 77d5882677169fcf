"""The CIF reader and zone-axis supercell against hand-made CIF files whose atom lists are derived step by step
(tests/golden/cif/derive_expected.py, each step citing the clTEM source it restates; clTEM's own CIF code
needs Eigen and cannot be built here). Checked: the symmetry images of every site, the tile range, and the
kept atoms in order, element and occupancy, positions within 1e-9 Å."""
import json
import os

import numpy as np
import pytest

from cltem_b200.cif import CIFReader, SuperCellInfo, calculate_tiling, make_supercell

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cif")
with open(os.path.join(HERE, "expected.json")) as _f:
    EXPECTED = json.load(_f)


@pytest.mark.parametrize("name", sorted(EXPECTED))
def test_cif_fixture(name):
    e = EXPECTED[name]
    cif = CIFReader(os.path.join(HERE, e["cif"]))
    # step 1: symmetry images, in the order the operations produce them
    assert [[list(map(float, p)) for p in site.positions] for site in cif.sites] == e["fractional_positions"]
    info = SuperCellInfo(uvw=tuple(e["uvw"]), abc=tuple(e["abc"]), widths=tuple(e["widths"]), tilts=tuple(e["tilts"]))
    sc = make_supercell(cif, info)
    # steps 2-3: the rotated basis
    assert np.allclose(np.asarray(sc.basis, dtype=np.float64), np.asarray(e["basis"]), rtol=0, atol=1e-12)
    # step 4: the tile range
    mins, maxs = calculate_tiling(sc.basis, *e["widths"])
    assert list(mins) == e["tile_min"] and list(maxs) == e["tile_max"]
    # step 5: the atoms, in order
    want = e["atoms"]
    assert len(sc.symbols) == len(want)
    assert list(sc.symbols) == [a[0] for a in want]
    got = np.stack([sc.x, sc.y, sc.z], axis=1)
    assert np.allclose(got, np.asarray([a[1:4] for a in want]), rtol=0, atol=1e-9)
    assert np.array_equal(sc.occ, np.asarray([a[4] for a in want]))
