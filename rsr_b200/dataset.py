"""Host-side ``Dataset``: the reference's AoSoA layout built from rows.

Restates ``Dataset::new`` (src/engine/data/dataset.rs:37-169): optional z-score
normalisation with sequential f32 sums (dataset.rs:63-94), padding to a
multiple of 8 with zeros (dataset.rs:96-104) and the f32x8 batch layout
``feature_flat[b*F + f]`` / ``target_batches[b]`` (dataset.rs:125-154).  The
engine uploads these arrays unchanged (``rsr_dataset_upload``) and transposes
them to structure-of-arrays on the device.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Sequence

import numpy as np

from .isa import FLOAT, TYPE_WIDTH


def _seq_sum_f32(v: np.ndarray) -> np.float32:
    """Left-to-right f32 sum, as Iterator::sum over f32 does."""
    if len(v) == 0:
        return np.float32(0.0)
    return np.cumsum(v.astype(np.float32), dtype=np.float32)[-1]


@dataclass
class Dataset:
    feature_flat: np.ndarray          # float32 [num_batches * num_features * 8]
    target_batches: np.ndarray        # float32 [num_batches * 8]
    num_features: int
    num_batches: int
    num_samples: int
    feature_means: np.ndarray
    feature_std_devs: np.ndarray
    target_mean: float = 0.0
    target_std_dev: float = 1.0
    is_normalized: bool = False
    feature_types: List[int] = field(default_factory=list)

    @staticmethod
    def new(data_x: Sequence[Sequence[float]] | np.ndarray, data_y: Sequence[float] | np.ndarray,
            feature_types: Sequence[int], normalize: bool = False) -> "Dataset":
        x = np.asarray(data_x, dtype=np.float32)
        y = np.asarray(data_y, dtype=np.float32)
        n = len(y)
        nf = sum(TYPE_WIDTH[t] for t in feature_types)
        if x.ndim != 2 or x.shape != (n, nf):
            raise ValueError(f"data_x must be ({n}, {nf})")
        means = np.zeros(nf, np.float32)
        stds = np.ones(nf, np.float32)
        tmean, tstd = np.float32(0.0), np.float32(1.0)
        if normalize:
            nn = np.float32(n)
            for f in range(nf):
                m = _seq_sum_f32(x[:, f]) / nn
                d = (x[:, f] - m).astype(np.float32)
                var = _seq_sum_f32(d * d) / nn
                means[f] = m
                stds[f] = np.float32(1.0) if var < np.float32(1e-9) else np.sqrt(var, dtype=np.float32)
            tmean = _seq_sum_f32(y) / nn
            d = (y - tmean).astype(np.float32)
            tvar = _seq_sum_f32(d * d) / nn
            tstd = np.float32(1.0) if tvar < np.float32(1e-9) else np.sqrt(tvar, dtype=np.float32)
            x = ((x - means) / stds).astype(np.float32)
            y = ((y - tmean) / tstd).astype(np.float32)
        nb = (n + 7) // 8
        xp = np.zeros((nb * 8, nf), np.float32)
        yp = np.zeros(nb * 8, np.float32)
        xp[:n] = x
        yp[:n] = y
        ff = np.ascontiguousarray(xp.reshape(nb, 8, nf).transpose(0, 2, 1)).reshape(-1)
        return Dataset(ff, yp, nf, nb, n, means, stds, float(tmean), float(tstd), normalize, list(feature_types))

    @staticmethod
    def from_columns(features: np.ndarray, targets: np.ndarray, feature_types: Sequence[int] | None = None) -> "Dataset":
        """features: (num_features, n) columns."""
        features = np.asarray(features, np.float32)
        nf = features.shape[0]
        ft = list(feature_types) if feature_types is not None else [FLOAT] * nf
        return Dataset.new(features.T, targets, ft, False)

    def point_features(self) -> np.ndarray:
        """(num_batches*8, num_features) view back in row order."""
        return self.feature_flat.reshape(self.num_batches, self.num_features, 8).transpose(0, 2, 1).reshape(
            -1, self.num_features)

    def variable_registry(self):
        """get_variable_registry (dataset.rs:200-222): (type, offset) of each
        variable, plus Float views of vector/matrix components."""
        reg, cur = [], 0
        for t in self.feature_types:
            reg.append((t, cur))
            w = TYPE_WIDTH[t]
            if w > 1:
                reg.extend((FLOAT, cur + o) for o in range(w))
            cur += w
        return reg

    def denormalize_target(self, v: float) -> float:
        return v * self.target_std_dev + self.target_mean if self.is_normalized else v
