"""Multi-rank paths on CPU: world_size-2 gloo process groups.

Population sharding (no data-path exchange, one gather) and point sharding
(one all-reduce of f64 sums, then the evaluator epilogue) checked against
the unsharded oracle; the per-shard sums come from the oracle here and from
the engine on the GPU (test_gpu_sharding.py)."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from rsr_b200 import sharding as S
from rsr_b200 import workloads as W

FMAX = float(np.finfo(np.float32).max)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_range_partitions():
    for n in (0, 1, 7, 8, 100, 12501):
        for world in (1, 2, 3, 8):
            spans = [S.shard_range(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [hi - lo for lo, hi in spans]
            assert max(sizes) - min(sizes) <= 1


def test_shard_dataset_union_is_dataset():
    ds = W.lorentz_dataset(1001, seed=3)   # 126 batches, the last one padded
    parts = [S.shard_dataset(ds, r, 3) for r in range(3)]
    assert np.array_equal(np.concatenate([p.feature_flat for p in parts]), ds.feature_flat)
    assert np.array_equal(np.concatenate([p.target_batches for p in parts]), ds.target_batches)
    assert sum(p.num_samples for p in parts) == ds.num_samples
    assert sum(p.num_batches for p in parts) == ds.num_batches


def _finalize_ref(sse, n):
    m = np.float32(sse / n)
    return FMAX if not (sse <= FMAX) or not np.isfinite(m) else float(m)


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    from oracle import binding as O
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        ds = W.scalar_dataset(997, seed=5)
        pop = W.scalar_population(40, seed=6)
        # point sharding: oracle sums of this rank's batches, all-reduced
        shard = S.shard_dataset(ds, rank, world)
        sums_fn = lambda progs, sh, grad: np.array([O.sse_f64(p, sh) for p in progs])
        mse, _ = S.point_sharded_mse(pop, shard, ds.num_samples, sums_fn)
        # population sharding: this rank's programs, gathered
        mine, lo, hi = S.shard_population(pop, rank, world)
        local = np.array([O.mse_f64(p, ds) for p in mine], np.float64)
        gathered = S.gather_population(local, len(pop))
        q.put((rank, mse.tolist(), gathered.tolist()))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_gloo_two_ranks():
    from oracle import binding as O
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ds = W.scalar_dataset(997, seed=5)
    pop = W.scalar_population(40, seed=6)
    want = np.array([_finalize_ref(O.sse_f64(p, ds), ds.num_samples) for p in pop])
    full64 = np.array([O.mse_f64(p, ds) for p in pop])
    for rank, mse, gathered in out:
        mse = np.asarray(mse)
        big = want >= FMAX
        assert np.array_equal(mse >= FMAX, big)
        np.testing.assert_allclose(mse[~big], want[~big], rtol=1e-6)
        np.testing.assert_array_equal(np.asarray(gathered), full64)
