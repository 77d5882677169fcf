"""The N>1 merge on the engine's own images: two gloo ranks, each a process with its own context on cuda:0,
shard three frozen-phonon configurations (and, in the second case, the scan pixels), run the engine's staged
STEM, and merge with one all-reduce of (image sums, weights). The merged image equals the single-process
staged average. The ranks' kernels never wait on one another: the only exchange is the host-side gloo
all-reduce after each rank's work has finished.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_path, mode):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    from cltem_b200.distributed import merge_average, shard_configs, shard_pixels
    from cltem_b200.engine import Context, Simulation
    from cltem_b200.params import load_default
    from tests.cases import phonons, small_stem
    s, st = small_stem(double_precision=True, scan=4)
    confs = phonons(st, 3, seed=9)
    ctx = Context(0)
    ctx.load_params(load_default("kirkland"))
    sim = Simulation(ctx, s.cfg)
    if mode == "configs":
        mine = shard_configs(len(confs), rank, world)
        sim.stage([confs[c] for c in mine])
        sim.run_staged()
        avg = merge_average(sim.staged_result() * len(mine), len(mine))
    else:
        npx = s.cfg.stem_pixels_x * s.cfg.stem_pixels_y
        mine = np.array(shard_pixels(npx, rank, world), dtype=np.int32)
        acc = np.zeros((sim.n_outputs, s.cfg.n_detectors, npx))
        w = np.zeros_like(acc)
        for c in confs:
            sim.set_atoms(c)
            acc[..., mine] += sim.stem(mine)
            w[..., mine] += 1
        avg = merge_average(acc, w).reshape(sim.n_outputs, s.cfg.n_detectors, s.cfg.stem_pixels_y, -1)
    sim.close()
    ctx.close()
    if rank == 0:
        np.save(out_path, avg)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("mode", ["configs", "pixels"])
def test_two_rank_merge_of_engine_images(tmp_path, kirkland, mode):
    out = str(tmp_path / "avg.npy")
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out, mode)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = np.load(out)
    from cltem_b200.engine import Context, Simulation
    from tests.cases import phonons, small_stem
    s, st = small_stem(double_precision=True, scan=4)
    c = Context(0)
    c.load_params(kirkland)
    sim = Simulation(c, s.cfg)
    ref = sim.stem_simulate(phonons(st, 3, seed=9))
    sim.close()
    c.close()
    assert got.shape == ref.shape
    assert np.allclose(got, ref, rtol=1e-13, atol=0)
