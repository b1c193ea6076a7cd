"""Dataset construction and subsampling on the device (Dataset::new,
Dataset::subset) against the oracle restatement, bit for bit."""
import numpy as np
import pytest

from oracle import dataset_ref as DR
from rsr_b200 import workloads as W
from rsr_b200.dataset import Dataset
from rsr_b200.isa import FLOAT, VEC3

f32 = np.float32


def _rows(n, nf, seed):
    rng = np.random.default_rng(seed)
    x = (rng.standard_normal((n, nf)) * 3 + rng.uniform(-5, 5, nf)).astype(f32)
    y = (x.sum(axis=1) * f32(0.5) + rng.standard_normal(n).astype(f32)).astype(f32)
    x[:, -1] = f32(2.0)  # a constant column: variance below 1e-9, deviation 1
    return x, y


def test_oracle_new_matches_host_mirror():
    x, y = _rows(1003, 4, 1)
    ff, tb, n, means, stds = DR.new(x, y, True)
    ds = Dataset.new(x, y, [FLOAT] * 4, normalize=True)
    assert np.array_equal(ds.feature_flat, ff) and np.array_equal(ds.target_batches, tb)
    assert stds[3] == 1.0


def test_oracle_subset_whole_is_clone():
    x, y = _rows(100, 2, 2)
    ff, tb, n, _, _ = DR.new(x, y, False)
    sff, stb, m = DR.subset(ff, tb, 2, n, 1000)
    assert m == 100 and np.array_equal(sff, ff) and np.array_equal(stb, tb)


@pytest.mark.gpu
@pytest.mark.parametrize("n,nf,norm", [(1, 1, False), (1003, 4, True), (20_000, 9, True), (4096, 3, False)])
def test_device_new_bit_exact(engine, n, nf, norm):
    x, y = _rows(n, nf, 3 + n)
    d, stats = engine.upload_rows(x, y, normalize=norm)
    ff, tb = engine.download(d)
    rff, rtb, _, means, stds = DR.new(x, y, norm)
    assert np.array_equal(ff, rff) and np.array_equal(tb, rtb)
    if norm:
        assert np.array_equal(stats["means"], means) and np.array_equal(stats["stds"], stds)
    d.release()


@pytest.mark.gpu
@pytest.mark.parametrize("target", [1, 7, 64, 999, 1003, 5000])
def test_device_subset_bit_exact(engine, target):
    x, y = _rows(1003, 3, 9)
    d, _ = engine.upload_rows(x, y, normalize=True)
    s = engine.subset(d, target)
    ff, tb = engine.download(s)
    sff, stb, _ = DR.subset(*engine.download(d), 3, 1003, target)
    assert np.array_equal(ff, sff) and np.array_equal(tb, stb)
    assert s.num_samples == min(target, 1003)
    s.release()
    d.release()


@pytest.mark.gpu
def test_ingested_dataset_scores_like_uploaded(engine):
    """The mini-batch path: programs score the same on a device subset as on
    the same subset built on the host and uploaded."""
    ds = W.lorentz_dataset(10_000, seed=11)
    pop = W.lorentz_population(64, seed=12)
    xs = np.asarray(ds.feature_flat, f32).reshape(ds.num_batches, 9, 8).transpose(0, 2, 1).reshape(-1, 9)[:10_000]
    ys = np.asarray(ds.target_batches, f32)[:10_000]
    d, _ = engine.upload_rows(xs, ys)
    sub = engine.subset(d, 64)
    sff, stb, m = DR.subset(ds.feature_flat, ds.target_batches, 9, 10_000, 64)
    host = Dataset(feature_flat=sff, target_batches=stb, num_features=9, num_batches=m // 8 + (m % 8 > 0),
                   num_samples=m, feature_means=np.zeros(9, f32), feature_std_devs=np.ones(9, f32),
                   feature_types=[VEC3] * 3)
    assert np.array_equal(engine.compute_mse_batch(pop, sub), engine.compute_mse_batch(pop, host))
    sub.release()
    d.release()
