"""Plasmon scattering on the host: the seeded draws (depth tables, angles), the reference's table rules, the
output translation kernel pinned to the reference's own bilinear_translate_d, and the JSON settings.

The reference (PlasmonScattering, src/simulation/incoherence/inelastic/plasmon.cpp) draws depths and angles
from one clock-seeded stream; here every draw is a function of (seed, job, index), shared by the engine and the
oracle, so the tables must agree exactly and follow the reference's distributions.
"""
import math

import numpy as np
import pytest

from cltem_b200 import abi, config
from cltem_b200.engine import plasmon_draws
from oracle import ref_bind as rb


def _cfg(kind=0, mfp=20.0, char=2.0, crit=30.0, seed=11):
    c = abi.config_defaults()
    c.plasmon = 1
    c.plasmon_individual = kind
    c.plasmon_mfp = mfp
    c.plasmon_char_angle = char
    c.plasmon_crit_angle = crit
    c.seed = seed
    return c


@pytest.mark.parametrize("kind", [0, 2, 3])
def test_depth_tables_engine_equals_oracle(oracle, kind):
    c = _cfg(kind=kind)
    for job in range(12):
        d_e, _ = plasmon_draws(c, job, 60.0)
        d_o = oracle.plasmon_depths(c, job, 60.0)
        assert np.array_equal(d_e, d_o)
        assert np.isinf(d_e[-1]) and np.all(np.isfinite(d_e[:-1]))
        assert np.all(np.diff(d_e[:-1]) > 0) and (len(d_e) == 1 or d_e[-2] <= 60.0)
        if kind:
            assert len(d_e) == kind   # "individual" n: n entries counting the closing +inf (n - 1 events)


def test_individual_one_means_no_event():
    """getDistancesForIndividual keeps a table whose size (with the closing +inf) equals `individual`: for 1
    that is a table of +inf alone, so no job scatters."""
    c = _cfg(kind=1, mfp=5.0)
    for job in range(5):
        d, _ = plasmon_draws(c, job, 50.0)
        assert len(d) == 1 and np.isinf(d[0])


def test_event_count_is_poisson_in_thickness():
    """Full tables: the number of depths <= t is Poisson with mean t / mfp (exponential distances)."""
    c = _cfg(kind=0, mfp=10.0)
    counts = np.array([len(plasmon_draws(c, j, 40.0)[0]) - 1 for j in range(4000)])
    assert abs(counts.mean() - 4.0) < 0.15
    assert abs(counts.var() - 4.0) < 0.4


def test_angle_distributions():
    """Polar angle: theta^2 = char^2 (((crit^2 + char^2) / char^2)^u - 1), so
    P(theta <= t) = ln(1 + t^2 / char^2) / ln((crit^2 + char^2) / char^2); azimuth uniform on [0, 2 pi)."""
    c = _cfg(char=2.0, crit=30.0)
    ang = np.concatenate([plasmon_draws(c, j, 1.0, n_events=8)[1] for j in range(500)])
    theta, phi = ang[:, 0], ang[:, 1]
    assert np.all(theta >= 0) and np.all(theta <= 30.0 + 1e-9)
    assert np.all(phi >= 0) and np.all(phi < 2 * math.pi)
    R = (30.0 ** 2 + 2.0 ** 2) / 2.0 ** 2
    for t in (1.0, 3.0, 10.0):
        expect = math.log(1 + t * t / 4.0) / math.log(R)
        assert abs(np.mean(theta <= t) - expect) < 0.03
    assert abs(np.mean(phi < math.pi) - 0.5) < 0.03


@pytest.mark.skipif(not rb.available(), reason="reference kernels not built (oracle/build_ref.py)")
@pytest.mark.parametrize("shift", [(0, 0, 0.0, 0.0), (3, -2, 0.25, 0.75), (-1, -1, 1.0 - 1e-12, 0.5), (7, 5, 0.0, 0.3),
                                   (-6, 4, 0.9, 0.1)])
def test_bilinear_translate_pinned_to_reference_kernel(oracle, shift):
    """The oracle's translation of a diffraction pattern (bilinear_translate_d) against the reference's own
    kernel compiled for the CPU: identical bits."""
    ix, iy, sx, sy = shift
    img = np.random.default_rng(7).random((24, 32))
    got = oracle.bilinear_translate(img, ix, iy, sx, sy)
    L = rb.lib()
    ref = np.empty_like(img)
    L.ref_bilinear_translate_d(rb.d(img), rb.d(ref), ix, iy, sx, sy, img.shape[1], img.shape[0])
    assert np.array_equal(got, ref)


def test_config_maps_plasmon_settings():
    j = {"mode": {"id": 1}, "incoherence": {"iterations": 3, "inelastic scattering": {"plasmon": {
        "enabled": True, "type": "individual", "individual": 4, "mean free path": {"value": 12.5},
        "characteristic angle": {"value": 0.8}, "critical angle": {"value": 7.0}}}}}
    s = config.read_config(j)
    c = s.cfg
    assert c.plasmon == 1 and c.plasmon_individual == 4
    assert c.plasmon_mfp == pytest.approx(125.0) and c.plasmon_char_angle == 0.8 and c.plasmon_crit_angle == 7.0
    assert s.effective_iterations() == 3
    j["incoherence"]["inelastic scattering"]["plasmon"]["type"] = "full"
    assert config.read_config(j).cfg.plasmon_individual == 0
