"""Point sharding on one GPU: the shards' f64 sums (rsr_eval_sums_batch),
added on the host as the all-reduce would add them, then rsr_finalize_sums,
against the unsharded engine (MSE 1e-6 relative; gradients 1e-5 of scale)."""
import numpy as np
import pytest

from rsr_b200 import sharding as S
from rsr_b200 import workloads as W

pytestmark = pytest.mark.gpu
FMAX = float(np.finfo(np.float32).max)


@pytest.mark.parametrize("world", [2, 3])
def test_point_shards_match_unsharded(engine, world):
    ds = W.transform_dataset(50_001, seed=91)
    pop = W.transform_population(48, seed=92)
    shards = [S.shard_dataset(ds, r, world) for r in range(world)]
    sums = sum(S.engine_sums(engine, pop, sh, gradient=False) for sh in shards)
    mse, _ = S.finalize_sums(sums, ds.num_samples, False)
    want = engine.compute_mse_batch(pop, ds)
    big = want >= FMAX
    assert np.array_equal(mse >= FMAX, big)
    np.testing.assert_allclose(mse[~big], want[~big], rtol=1e-6)

    gs = sum(S.engine_sums(engine, pop, sh, gradient=True) for sh in shards)
    gm, gg = S.finalize_sums(gs, ds.num_samples, True)
    wm, wg = engine.compute_mse_grad_batch(pop, ds)
    big = wm >= FMAX
    assert np.array_equal(gm >= FMAX, big)
    np.testing.assert_allclose(gm[~big], wm[~big], rtol=1e-6)
    # NaN / Inf gradients (the reference's sqrt and division rules) must match
    # in place; finite ones within 1e-5 of the program's largest finite entry
    g, w = gg[~big], wg[~big]
    assert np.array_equal(np.isnan(g), np.isnan(w)) and np.array_equal(np.isinf(g), np.isinf(w))
    fin = np.isfinite(w)
    scale = np.maximum(np.where(fin, np.abs(w), 0).max(axis=1, keepdims=True), 1e-12)
    assert np.all(np.abs(np.where(fin, g - w, 0)) <= 1e-5 * scale)
