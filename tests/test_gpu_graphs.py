"""The STEM batch loop replays a captured CUDA graph after the first batch of a shape; the replays must give
the same numbers, the same launch count and the same per-kernel profile as eager launches."""
import numpy as np
import pytest

from cltem_b200.engine import Simulation
from tests.cases import phonons, small_stem

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dp", [True, False])
def test_graph_replays_equal_one_eager_batch(gpu_ctx, kirkland, dp):
    gpu_ctx.load_params(kirkland)
    s1, st = small_stem(double_precision=dp, scan=5, interval=2)     # 25 probes
    conf = phonons(st, 1)[0]
    pix = np.arange(25, dtype=np.int32)[::-1].copy()
    s1.cfg.probe_batch = 25                                            # one eager batch
    one = Simulation(gpu_ctx, s1.cfg)
    one.set_atoms(conf)
    ref = one.stem(pix)
    l0 = gpu_ctx.launch_count()
    assert np.array_equal(one.stem(pix), ref)
    per_batch = gpu_ctx.launch_count() - l0                           # transmission already built
    s4, _ = small_stem(double_precision=dp, scan=5, interval=2)
    s4.cfg.probe_batch = 4                                             # 6 x 4 + 1: eager, capture, replays, eager tail
    sim = Simulation(gpu_ctx, s4.cfg)
    sim.set_atoms(conf)
    assert np.array_equal(sim.stem(pix), ref)
    for rep in range(2):                                               # these runs start from replays
        l0 = gpu_ctx.launch_count()
        assert np.array_equal(sim.stem(pix), ref), rep
        assert gpu_ctx.launch_count() - l0 == 7 * per_batch


def test_graph_profile_counts_every_replay(gpu_ctx, kirkland):
    gpu_ctx.load_params(kirkland)
    s, st = small_stem(double_precision=False, scan=4)                 # 16 probes
    s.cfg.probe_batch = 4
    sim = Simulation(gpu_ctx, s.cfg)
    sim.set_atoms(st)
    pix = np.arange(16, dtype=np.int32)
    sim.stem(pix)
    sim.profile(True)
    sim.profile_read(reset=True)
    sim.stage(phonons(st, 2))
    sim.run_staged()
    prof = sim.profile_read()
    sim.profile(False)
    S = sim.geo.n_slices
    # 2 configurations x 4 batches x S slices, each a row and a column launch with a positive duration
    assert prof["row_step"][1] == 2 * 4 * S and prof["col_step"][1] == 2 * 4 * S
    assert prof["row_step"][0] > 0 and prof["col_step"][0] > 0
    s.cfg.probe_batch = 16                                             # one batch per configuration
    other = Simulation(gpu_ctx, s.cfg)
    other.stage(phonons(st, 2))
    other.run_staged()
    assert np.array_equal(sim.staged_result(), other.staged_result())


def _staged_case(kirkland, chromatic=False):
    from tests.cases import phonons, small_stem
    s, st = small_stem(double_precision=False, scan=8)
    s.cfg.probe_batch = 24   # several batches a pass, the last one short
    if chromatic:
        s.cfg.chromatic = 1
        s.cfg.chromatic_cc = 1.5
        s.cfg.chromatic_hwhm_neg = s.cfg.chromatic_hwhm_pos = 0.4
    return s, phonons(st, 3, seed=21)


@pytest.mark.parametrize("chromatic", [False, True])
def test_whole_staged_run_graph_matches_eager(gpu_ctx, kirkland, chromatic, monkeypatch):
    """A staged STEM run captured as one graph (every pass's binning, build and batches) gives the eager run's
    bits, on its first launch (captured) and on replays."""
    from cltem_b200.engine import Simulation
    gpu_ctx.load_params(kirkland)
    s, confs = _staged_case(kirkland, chromatic)
    monkeypatch.setenv("MSLICE_NO_GRAPHS", "1")
    eager = Simulation(gpu_ctx, s.cfg)
    monkeypatch.delenv("MSLICE_NO_GRAPHS")
    eager.stage(confs)
    eager.run_staged()
    ref = eager.staged_result()
    sim = Simulation(gpu_ctx, s.cfg)
    sim.stage(confs)
    for _ in range(3):
        sim.run_staged()
        assert np.array_equal(sim.staged_result(), ref)
    assert sim.last_timing()["total_ms"] > 0 and sim.last_timing()["build_ms"] == -1
    eager.close()
    sim.close()


def test_async_runs_on_two_contexts_overlap_and_match(kirkland):
    """Queued staged runs on two contexts (two streams): each result equals its synchronous run."""
    from cltem_b200.engine import Context, Simulation
    from tests.cases import phonons, small_stem
    ctxs = [Context(0), Context(0)]
    sims, refs = [], []
    for k, c in enumerate(ctxs):
        c.load_params(kirkland)
        s, st = small_stem(double_precision=False, scan=6, res=256 if k == 0 else 128)
        s.cfg.allow_any_resolution = 1
        confs = phonons(st, 2, seed=30 + k)
        sim = Simulation(c, s.cfg)
        sim.stage(confs)
        sim.run_staged()
        refs.append(sim.staged_result().copy())
        sims.append(sim)
    for sim in sims:
        sim.run_staged_async()
    for sim, ref in zip(sims, refs):
        sim.wait()
        assert np.array_equal(sim.staged_result(), ref)
    for sim in sims:
        sim.close()
    for c in ctxs:
        c.close()
