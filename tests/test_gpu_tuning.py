"""The autotuner: it picks one of the candidate batches and step kernels, later runs use them, and the results
do not depend on the batch."""
import numpy as np
import pytest

from cltem_b200.engine import MsliceError, Simulation
from tests.cases import phonons, small_stem

pytestmark = pytest.mark.gpu


def test_tune_batch_picks_a_candidate_and_keeps_results(gpu_ctx, kirkland):
    gpu_ctx.load_params(kirkland)
    s, st = small_stem(double_precision=False, scan=5)
    conf = phonons(st, 1)[0]
    pix = np.arange(25, dtype=np.int32)
    sim = Simulation(gpu_ctx, s.cfg)
    sim.set_atoms(conf)
    best, rate = sim.tune_batch([4, 8, 16], reps=2)
    assert best in (4, 8, 16) and rate > 0
    # the reference: the same step kernels (the tuner may pick another FFT plan for the row pass, which rounds
    # differently) at the engine's default batch
    t = sim.tuning()
    ref_sim = Simulation(gpu_ctx, s.cfg)
    ref_sim.set_atoms(conf)
    ref_sim.set_step_variant(t["col_variant"], t["row_variant"])
    ref = ref_sim.stem(pix)
    sim.build_transmission()
    l0 = gpu_ctx.launch_count()
    got = sim.stem(pix)
    nbatch = -(-25 // best)
    per_batch = 1 + 2 * sim.geo.n_slices + sim.geo.n_outputs
    assert gpu_ctx.launch_count() - l0 == nbatch * per_batch
    assert np.allclose(got, ref, rtol=1e-12, atol=0)   # per-probe arithmetic does not depend on the batch


def test_tune_batch_default_candidates_are_cached(gpu_ctx, kirkland):
    gpu_ctx.load_params(kirkland)
    s, st = small_stem(double_precision=False, scan=2)
    a = Simulation(gpu_ctx, s.cfg)
    b1, r1 = a.tune_batch(reps=1)
    b = Simulation(gpu_ctx, s.cfg)
    b2, r2 = b.tune_batch(reps=1)   # same device, grid and precision: the cached result
    assert (b1, r1) == (b2, r2) and b1 in (64, 128, 256, 512, 1024, 2048)
    with pytest.raises(MsliceError):
        a.tune_batch([0, 4])


@pytest.mark.parametrize("res", [256, 512, 768, 1024, 2048])
def test_column_step_variants_are_bit_identical(gpu_ctx, kirkland, res):
    """Every column-step kernel the tuner may pick (the persistent TMA-fed passes, the one-block-per-tile kernel
    at other tile widths) and every launch mode of the row step, with the transmission rows loaded by the
    threads or staged by the copy engine, does the default kernel's arithmetic in the same order: identical
    detector values (the column kernel of the 16-element FFT plan at 1024² and 2048² agrees to FP32 rounding)
    over a batch large enough that every persistent block loops over many (wave, tile) items and reuses each
    shared-memory stage many times."""
    gpu_ctx.load_params(kirkland)
    s, st = small_stem(double_precision=False, res=res, n=(3, 3, 3), scan=12)
    s.cfg.probe_batch = 144
    conf = phonons(st, 1)[0]
    sim = Simulation(gpu_ctx, s.cfg)
    sim.set_atoms(conf)
    t = sim.tuning()
    nv = t["col_variants"]
    nr = t["row_variants"]
    # 4 prefetch / order modes; 4 more where the plain Stockham plan is the alternative row plan (wide default
    # plans), and 4 more with the transmission rows staged by the copy engine (FP32 wide and radix-24 plans)
    assert nr == (12 if res in (256, 384, 512, 768, 1024, 2048) else 4)
    assert nv >= (2 if res <= 512 else 1)   # the persistent passes where their stages and tables fit
    names = [sim.step_variant_name(0, v) for v in range(nv)]
    assert len(set(names)) == nv and all(names)
    assert len({sim.step_variant_name(1, v) for v in range(nr)}) == nr
    with pytest.raises(MsliceError):
        sim.step_variant_name(0, nv)
    pix = np.arange(144, dtype=np.int32)
    out = []
    same_plan = list(range(4)) + list(range(8, nr))   # the default row plan, T loaded or staged
    # column kernels of another FFT plan (the 16-element plan at 1024² and 2048²) round differently
    other_plan = [v for v in range(nv) if "16-element FFT plan" in names[v]]
    assert len(other_plan) == (1 if res in (1024, 2048) else 0)
    for v in [v for v in range(nv) if v not in other_plan]:
        for rv in same_plan:   # the row pass with and without its L2 prefetch, in wave-fastest order, T staged
            sim.set_step_variant(v, rv)
            assert sim.tuning()["col_variant"] == v and sim.tuning()["row_variant"] == rv
            out.append(sim.stem(pix))
            out.append(sim.stem(pix))   # a second run replays the batch's CUDA graph
    for r in out[1:]:
        assert np.array_equal(r, out[0])
    for v in other_plan:   # bit-identical across the row variants of the default plan, FP32 rounding of the rest
        other = []
        for rv in same_plan:
            sim.set_step_variant(v, rv)
            other.append(sim.stem(pix))
        for r in other[1:]:
            assert np.array_equal(r, other[0])
        assert np.linalg.norm(other[0] - out[0]) <= 1e-5 * np.linalg.norm(out[0])
    # the alternative row plan (variants 4-7): bit-identical among its four launch modes and with every column
    # kernel, within FP32 rounding of the default plan
    alt = []
    for v in (0, max(v for v in range(nv) if v not in other_plan)):
        for rv in range(4, min(nr, 8)):
            sim.set_step_variant(v, rv)
            alt.append(sim.stem(pix))
    for r in alt[1:]:
        assert np.array_equal(r, alt[0])
    if alt:
        assert np.linalg.norm(alt[0] - out[0]) <= 1e-5 * np.linalg.norm(out[0])
    with pytest.raises(MsliceError):
        sim.set_step_variant(nv, 0)
    with pytest.raises(MsliceError):
        sim.set_step_variant(0, nr)
    sim.close()


def test_tuner_reports_its_column_variant(gpu_ctx, kirkland):
    gpu_ctx.load_params(kirkland)
    s, st = small_stem(double_precision=False, res=512, scan=2)
    sim = Simulation(gpu_ctx, s.cfg)
    best, rate = sim.tune_batch([64, 256], reps=2)
    t = sim.tuning()
    assert t["batch"] == best and 0 <= t["col_variant"] < t["col_variants"] and 0 <= t["row_variant"] < t["row_variants"]
    sim.close()


@pytest.mark.parametrize("res", [384, 768])
def test_staged_transmission_rows_follow_each_waves_set(gpu_ctx, kirkland, res):
    """Mixed static potentials give every wave of a batch its own transmission set (the per-wave set index of
    the row pass): the staged-row kernels (row variants 8-11) fetch the rows of each wave's set and give the
    plain kernel's detector values bit for bit, in a staged run of three configurations over two iterations."""
    gpu_ctx.load_params(kirkland)
    s, st = small_stem(double_precision=False, res=res, n=(3, 3, 3), scan=4)
    s.cfg.mixed_static, s.cfg.iterations, s.cfg.seed = 3, 2, 11
    s.cfg.allow_any_resolution = 1   # 384 is not in the reference's resolution list
    sim = Simulation(gpu_ctx, s.cfg)
    sim.stage(phonons(st, 3, seed=21))
    t = sim.tuning()
    nr = t["row_variants"]
    assert nr == 12
    outs = []
    for rv in [0, 3] + list(range(8, nr)):
        sim.set_step_variant(t["col_variant"], rv)
        sim.run_staged()
        outs.append(sim.staged_result())
    for r in outs[1:]:
        assert np.array_equal(r, outs[0])
    sim.close()
