"""Multi-GPU sharding of frozen-phonon configurations and the merge of the per-rank images.

One process per GPU (torch.distributed). The path shards without a data-path collective: every rank
propagates its own configurations (and, when there are fewer configurations than ranks, its own share
of the probes); the only exchange is the final merge of the weighted images, the counterpart of the
reference's SimulationManager::updateImages (src/simulation/simulationmanager.cpp:274-350), done as one
all-reduce of (sum of images, weights) in FP64.
"""
import numpy as np


def shard_configs(n_configs: int, rank: int, world: int):
    """Configuration indices of one rank: round-robin (the reference deals TDS jobs to its device
    threads from one queue, src/simulation/threading/simulationrunner.cpp:52-134)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank / world size")
    return list(range(rank, n_configs, world))


def shard_pixels(n_pixels: int, rank: int, world: int):
    """Contiguous block of scan pixels of one rank (used when configurations are fewer than ranks)."""
    base, extra = divmod(n_pixels, world)
    start = rank * base + min(rank, extra)
    return list(range(start, start + base + (1 if rank < extra else 0)))


def merge_average(image_sum: np.ndarray, weight: float, group=None, device=None):
    """All-reduce the per-rank image sums and weights; every rank gets sum / weight (FP64)."""
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(np.ascontiguousarray(image_sum, dtype=np.float64).ravel())
    w = torch.tensor([float(weight)], dtype=torch.float64)
    if device is not None:
        t, w = t.to(device), w.to(device)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, group=group)
        dist.all_reduce(w, group=group)
    out = (t / w).cpu().numpy().reshape(np.shape(image_sum))
    return out
