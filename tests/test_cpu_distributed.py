"""The N>1 path on CPU: world-size-2 gloo processes shard frozen-phonon configurations (or scan pixels)
and merge the images with one all-reduce; the result equals the single-process average. (The images here
come from the CPU oracle so the test needs no GPU; tests/test_gpu_distributed.py merges the engine's own
images the same way.)"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from cltem_b200.distributed import merge_average, shard_configs, shard_pixels


def test_shards_cover_everything_once():
    for n, w in ((10, 2), (10, 4), (3, 8), (1, 2)):
        got = sorted(i for r in range(w) for i in shard_configs(n, r, w))
        assert got == list(range(n))
        px = sorted(i for r in range(w) for i in shard_pixels(n * 7, r, w))
        assert px == list(range(n * 7))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_path, mode="configs"):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from oracle import bind as ob
    from cltem_b200.params import load_default
    from tests.cases import phonons, small_stem
    ob.set_threads(2)
    s, st = small_stem(scan=2)
    confs = phonons(st, 3, seed=9)
    osim = ob.OracleSim(s.cfg, load_default("kirkland"))
    pix = np.arange(4, dtype=np.int32)
    acc = np.zeros((1, 2, 4))
    if mode == "configs":        # whole configurations per rank, one weight per rank
        mine = shard_configs(len(confs), rank, world)
        for c in mine:
            osim.set_atoms(confs[c])
            osim.build_transmission()
            acc += osim.stem(pix)
        avg = merge_average(acc, len(mine))
    else:                        # every configuration over this rank's scan pixels, per-pixel weights
        mine = np.array(shard_pixels(len(pix), rank, world), dtype=np.int32)
        w = np.zeros_like(acc)
        for c in confs:
            osim.set_atoms(c)
            osim.build_transmission()
            acc[..., mine] += osim.stem(pix[mine])
            w[..., mine] += 1
        avg = merge_average(acc, w)
    if rank == 0:
        np.save(out_path, avg)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("mode", ["configs", "pixels"])
def test_two_rank_gloo_merge_equals_single_process(tmp_path, mode):
    out = str(tmp_path / "avg.npy")
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out, mode)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    assert all(p.exitcode == 0 for p in procs)
    got = np.load(out)
    from oracle import bind as ob
    from cltem_b200.params import load_default
    from tests.cases import phonons, small_stem
    s, st = small_stem(scan=2)
    osim = ob.OracleSim(s.cfg, load_default("kirkland"))
    pix = np.arange(4, dtype=np.int32)
    ref = 0
    for c in phonons(st, 3, seed=9):
        osim.set_atoms(c)
        osim.build_transmission()
        ref = ref + osim.stem(pix)
    ref = ref / 3
    assert np.allclose(got, ref, rtol=1e-13, atol=0)
