"""Trajectory shards across ranks (one process per GPU) and the one exchange step.

fTWA trajectories are independent, so a job of B trajectories splits into
contiguous ranges, one per rank, with the split of the reference's MPI solver
(src/FHfTWAMPISolver.cpp:89-100: B // ws each, the last B % ws ranks take one
more).  Each rank draws its own range of the seed's ensemble
(`Engine.sample(first=...)`), so the union is the single-GPU ensemble.  The only
collective is one FP64 sum of the observables at the end of the run; the
reference gathers them serially to rank 0 (src/FHfTWAMPISolver.cpp:345-558).

Observables normalised per shard are affine in the shard's sums (Niiu = S/B + 1/2,
NuNd = Sud/B + (Su+Sd)/(2B) + 1/4, E = S_E/B), so the ensemble value is the
trajectory-weighted mean of the shard values: sum_r B_r x_r / B.
"""
from __future__ import annotations

import numpy as np

OBS_KEYS = ("niiu", "niid", "n2iiu", "n2iid", "nund", "energies")


def shard_range(n_traj: int, rank: int, world_size: int) -> tuple[int, int]:
    """[first, end) of this rank's trajectories."""
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError("rank must be in [0, world_size)")
    per, extra = divmod(n_traj, world_size)
    first_big = world_size - extra          # ranks >= first_big take per + 1
    if rank < first_big:
        first = rank * per
        return first, first + per
    first = first_big * per + (rank - first_big) * (per + 1)
    return first, first + per + 1


def pack(obs: dict, count: int) -> np.ndarray:
    """Flattens a shard's normalised observables, weighted by its trajectory count."""
    parts = [np.asarray(obs[k], dtype=np.float64).ravel() * float(count) for k in OBS_KEYS]
    return np.concatenate(parts + [np.array([float(count)])])


def unpack(buf: np.ndarray, like: dict) -> dict:
    """Inverse of pack after the sum over ranks: divides by the total count."""
    total = float(buf[-1])
    out, o = {}, 0
    for k in OBS_KEYS:
        a = np.asarray(like[k])
        out[k] = (buf[o:o + a.size] / total).reshape(a.shape)
        o += a.size
    out["n_traj"] = int(round(total))
    return out


def combine(obs: dict, count: int, all_reduce_sum) -> dict:
    """Ensemble observables over all ranks.  `all_reduce_sum(np.ndarray) -> np.ndarray`
    is the collective (torch.distributed.all_reduce over NCCL on GPUs, gloo on CPU)."""
    return unpack(all_reduce_sum(pack(obs, count)), obs)


def torch_all_reduce_sum(device=None):
    """all_reduce_sum over the default torch.distributed process group, in FP64."""
    import torch
    import torch.distributed as dist

    def f(a: np.ndarray) -> np.ndarray:
        t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64))
        if device is not None:
            t = t.to(device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return t.cpu().numpy()
    return f
