"""Multi-GPU sharding of the fitness path, one process per GPU.

Two ways to split the work, both over ``torch.distributed`` process groups
(NCCL on GPUs; gloo works the same for the host-side logic):

* population sharding -- every rank scores a contiguous slice of the
  programs against its own resident copy of the dataset; there is no
  exchange on the data path, only a gather of the per-program fitness
  arrays at the end (``gather_population``);
* point sharding -- one large dataset split by 8-point batches, so the
  union of the shards is exactly the reference's padded batch list
  (src/engine/data/dataset.rs:96-154: zero padding only after the last
  point); every rank computes unscaled f64 sums over its shard, one
  all-reduce adds them, and the compute_mse / compute_mse_with_gradient
  epilogue (src/engine/eval/evaluator.rs:172-173, 211-223) runs on the
  totals with the whole dataset's num_samples.
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, Optional, Tuple

import numpy as np

from .dataset import Dataset


def shard_range(n: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous, balanced [lo, hi) of n units for rank (the first n % world
    ranks take one more)."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    q, r = divmod(n, world)
    lo = rank * q + min(rank, r)
    return lo, lo + q + (1 if rank < r else 0)


def shard_dataset(ds: Dataset, rank: int, world: int) -> Dataset:
    """The rank's slice of the AoSoA batches.  num_samples counts the real
    points inside the slice (the epilogue uses the whole dataset's)."""
    b0, b1 = shard_range(ds.num_batches, rank, world)
    nf = ds.num_features
    ff = np.ascontiguousarray(ds.feature_flat[b0 * nf * 8:b1 * nf * 8])
    tb = np.ascontiguousarray(ds.target_batches[b0 * 8:b1 * 8])
    real = max(0, min(ds.num_samples, b1 * 8) - b0 * 8)
    return Dataset(feature_flat=ff, target_batches=tb, num_features=nf, num_batches=b1 - b0, num_samples=real,
                   feature_means=ds.feature_means, feature_std_devs=ds.feature_std_devs,
                   target_mean=ds.target_mean, target_std_dev=ds.target_std_dev, is_normalized=ds.is_normalized,
                   feature_types=list(ds.feature_types))


def shard_population(programs, rank: int, world: int) -> Tuple[list, int, int]:
    progs = list(programs)
    lo, hi = shard_range(len(progs), rank, world)
    return progs[lo:hi], lo, hi


def finalize_sums(sums: np.ndarray, num_samples: int, gradient: bool) -> Tuple[np.ndarray, Optional[np.ndarray]]:
    """The evaluator epilogue on summed shards, through rsr_finalize_sums."""
    from . import _native as N
    stride = 33 if gradient else 1
    s = np.ascontiguousarray(sums, np.float64).reshape(-1)
    n = len(s) // stride
    mse = np.zeros(max(n, 1), np.float32)
    grad = np.zeros(max(n, 1) * 32, np.float32) if gradient else None
    N.check(N.lib().rsr_finalize_sums(n, int(gradient), s.ctypes.data, num_samples, mse.ctypes.data,
                                      grad.ctypes.data if grad is not None else None))
    return mse[:n], (grad[:n * 32].reshape(n, 32) if gradient else None)


def engine_sums(engine, programs, shard, gradient: bool = False) -> np.ndarray:
    """Unscaled per-program f64 sums of one shard on this rank's GPU
    (rsr_eval_sums_batch): (n,) or (n, 33)."""
    from . import _native as N
    from .evaluator import _as_population, _packed
    pk = _packed(programs)
    pop, keep = _as_population(pk)
    stride = 33 if gradient else 1
    out = np.zeros(max(pk.n, 1) * stride, np.float64)
    d = engine._ds(shard)
    N.check(N.lib().rsr_eval_sums_batch(engine.ctx, C.byref(pop), d.handle, None, int(gradient), out.ctypes.data))
    out = out[:pk.n * stride]
    return out.reshape(pk.n, 33) if gradient else out


def point_sharded_mse(programs, shard: Dataset, total_samples: int, sums_fn: Callable, group=None,
                      gradient: bool = False, device=None):
    """MSE (and gradients) of every program over a point-sharded dataset:
    local sums -> one all-reduce (sum, f64) -> epilogue.  ``sums_fn(programs,
    shard, gradient)`` computes the local sums (``engine_sums`` bound to an
    engine on GPU ranks)."""
    import torch
    import torch.distributed as dist
    local = np.asarray(sums_fn(programs, shard, gradient), np.float64)
    t = torch.from_numpy(local.copy())
    if device is not None:
        t = t.to(device)
    if dist.is_initialized():
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return finalize_sums(t.cpu().numpy(), total_samples, gradient)


def gather_population(values: np.ndarray, n_total: int, group=None, device=None) -> np.ndarray:
    """All-gather of per-program results of contiguous population shards
    (rank order = program order), padded to equal length for the collective."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    if world == 1:
        return np.asarray(values)
    width = max(shard_range(n_total, r, world)[1] - shard_range(n_total, r, world)[0] for r in range(world))
    v = np.asarray(values)
    pad = np.zeros((width,) + v.shape[1:], v.dtype)
    pad[:len(v)] = v
    t = torch.from_numpy(pad)
    if device is not None:
        t = t.to(device)
    outs = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(outs, t, group=group)
    parts = []
    for r in range(world):
        lo, hi = shard_range(n_total, r, world)
        parts.append(outs[r].cpu().numpy()[:hi - lo])
    return np.concatenate(parts, axis=0)
