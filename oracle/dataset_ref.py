"""CPU restatement of the reference's dataset construction and subsampling.

TEST INFRASTRUCTURE ONLY: the checker for ``rsr_dataset_upload_rows`` and
``rsr_dataset_subset``.  ``new`` follows Dataset::new
(src/engine/data/dataset.rs:37-169): sequential f32 sums for the z-score,
(value - mean) / std per point, AoSoA f32x8 batches with zero padding.
``subset`` follows Dataset::subset (dataset.rs:360-447).  Both return
(feature_flat, target_batches, num_samples).
"""
from __future__ import annotations

import numpy as np

f32 = np.float32


def _seq_sum(v):
    s = f32(0)
    for x in v:
        s = f32(s + x)
    return s


def new(x_rows, y, normalize: bool):
    x = np.asarray(x_rows, f32)
    y = np.asarray(y, f32)
    n, nf = len(y), x.shape[1]
    means = np.zeros(nf + 1, f32)
    stds = np.ones(nf + 1, f32)
    if normalize:
        cols = [x[:, f] for f in range(nf)] + [y]
        for c, col in enumerate(cols):
            m = f32(_seq_sum(col) / f32(n))
            d = (col - m).astype(f32)
            var = f32(_seq_sum((d * d).astype(f32)) / f32(n))
            means[c] = m
            stds[c] = f32(1) if var < f32(1e-9) else np.sqrt(var, dtype=f32)
    nb = (n + 7) // 8
    xs = np.zeros((nb * 8, nf), f32)
    ys = np.zeros(nb * 8, f32)
    xs[:n] = ((x - means[:nf]) / stds[:nf]).astype(f32)
    ys[:n] = ((y - means[nf]) / stds[nf]).astype(f32)
    ff = xs.reshape(nb, 8, nf).transpose(0, 2, 1).reshape(-1)
    return ff, ys, n, means, stds


def subset(feature_flat, target_batches, num_features: int, num_samples: int, target: int):
    m = min(target, num_samples)
    nb_src = len(target_batches) // 8
    if m == num_samples:
        return np.array(feature_flat, f32), np.array(target_batches, f32), m
    xs = np.asarray(feature_flat, f32).reshape(nb_src, num_features, 8).transpose(0, 2, 1).reshape(nb_src * 8, num_features)
    ys = np.asarray(target_batches, f32)
    nb = (m + 7) // 8
    step = (float(num_samples) - 1.0) / max(float(m) - 1.0, 1.0)
    ox = np.zeros((nb * 8, num_features), f32)
    oy = np.zeros(nb * 8, f32)
    for j in range(nb * 8):
        v = float(j) * step               # f64 product, then round half away from zero
        o = int(v)
        if v - o >= 0.5:
            o += 1
        if o < num_samples:
            ox[j] = xs[o]
            oy[j] = ys[o]
    return ox.reshape(nb, 8, num_features).transpose(0, 2, 1).reshape(-1), oy, m
