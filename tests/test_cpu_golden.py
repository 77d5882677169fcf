"""The oracle against outputs of the reference's own kernels (tests/golden/ref_kernels.npz, made by
tests/golden/make_ref_golden.py). Runs everywhere: the fixtures travel, the reference tree does not."""
import os

import numpy as np
import pytest

from cltem_b200.structure import Structure
from tests.cases import small_cbed, small_ctem, small_stem

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_kernels.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def stem_conf(g):
    return Structure(g["stem_atoms_Z"].astype(np.int32), g["stem_atoms_x"], g["stem_atoms_y"], g["stem_atoms_z"])


def test_oracle_projected_potential_matches_reference_output(oracle, kirkland, gold):
    s, _ = small_stem()
    o = oracle.OracleSim(s.cfg, kirkland)
    o.set_atoms(stem_conf(gold))
    o.build_transmission()
    sub = int(gold["sub"])
    assert np.array_equal(o.sorted_atoms(len(gold["stem_atoms_Z"]))["block_start"], gold["stem_block_start"])
    for k in (0, 3):
        assert np.array_equal(o.transmission(k, False)[::sub, ::sub], gold[f"stem_kirkland_T{k}"])


def test_oracle_probe_and_propagator_match_reference_output(oracle, kirkland, gold):
    s, _ = small_stem()
    o = oracle.OracleSim(s.cfg, kirkland)
    sub = int(gold["sub"])
    assert np.array_equal(o.probe(4.3, 4.1)[::sub, ::sub], gold["stem_probe_4.3_4.1"])
    assert np.array_equal(o.propagator()[::sub, ::sub], gold["stem_propagator"])


def test_oracle_full3d_matches_reference_output(oracle, lobato, gold):
    s, st = small_cbed()
    o = oracle.OracleSim(s.cfg, lobato)
    o.set_atoms(st)
    o.build_transmission()
    sub = int(gold["sub"])
    assert np.array_equal(o.transmission(1, False)[::sub, ::sub], gold["cbed_lobato3d_T1"])


def test_oracle_ctem_image_matches_reference_output(oracle, gold):
    s, _ = small_ctem()
    n = s.cfg.resolution
    rng = np.random.default_rng(21)
    rw = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    sub = int(gold["sub"])
    assert np.array_equal(oracle.ctem_image(s.cfg, rw)[::sub, ::sub], gold["ctem_image_out"])
