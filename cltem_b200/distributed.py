"""Multi-GPU sharding of frozen-phonon configurations and the merge of the per-rank images.

One process per GPU (torch.distributed). The path shards without a data-path collective: every rank
propagates its own configurations (shard_configs), or, when there are fewer configurations than ranks,
every configuration over its own block of scan pixels (shard_pixels). The only exchange is the final
merge of the weighted images, the counterpart of the reference's SimulationManager::updateImages
(src/simulation/simulationmanager.cpp:274-350), done as one all-reduce of (sum of images, weights) in
FP64; weights are per rank for configuration sharding and per pixel for pixel sharding.
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


def merge_average(image_sum: np.ndarray, weight, group=None, device=None):
    """All-reduce the per-rank image sums and weights; every rank gets sum / weight (FP64).

    `weight` is either one number (each rank ran whole configurations over every pixel: the count of
    configurations it ran) or an array of image_sum's shape (ranks that shard scan pixels: per pixel, the
    configurations this rank accumulated there, 0 for pixels of other ranks). The per-pixel form is the
    reference's Image weights (commonstructs.h:149-158, summed in SimulationManager::updateImages), so the
    average stays right whichever way the work was split. A pixel no rank covered is left at 0."""
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(np.ascontiguousarray(image_sum, dtype=np.float64).ravel())
    per_pixel = np.ndim(weight) > 0
    if per_pixel:
        if np.shape(weight) != np.shape(image_sum):
            raise ValueError("per-pixel weights must have the image's shape")
        w = torch.from_numpy(np.ascontiguousarray(weight, dtype=np.float64).ravel())
    else:
        w = torch.tensor([float(weight)], dtype=torch.float64)
    if device is not None:
        t, w = t.to(device), w.to(device)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, group=group)
        dist.all_reduce(w, group=group)
    out = torch.where(w > 0, t / torch.where(w > 0, w, torch.ones_like(w)), torch.zeros_like(t))
    return out.cpu().numpy().reshape(np.shape(image_sum))
