"""Tournament selection over (fitness, age) Pareto ranks -- the consumer of
the engine's fitness arrays.

Restates src/engine/search/operators/selection.rs:5-134 in f32 arithmetic:
dominance on (fitness, age) (`dominates`, :5-11), NSGA-II front ranks and
crowding distances (`assign_rank_and_crowding_distance`, :40-134), the
comparison (`nsga2_compare`, :29-38) and the k-way tournament
(`tournament_selection_pareto`, :13-27).  The random draws are inputs here:
the reference draws them from rand 0.10's xoshiro streams, which are not
restated, so callers pass the indices their generator produced.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple

import numpy as np

f32 = np.float32
FMAX = np.finfo(np.float32).max


def _dominates(fa, aa, fb, ab) -> bool:
    return (fa <= fb and aa <= ab) and (fa < fb or aa < ab)


def assign_rank_and_crowding(fitness: Sequence[float], age: Sequence[int]) -> Tuple[np.ndarray, np.ndarray]:
    """Front rank (u32) and crowding distance (f32) of every individual."""
    fit = np.asarray(fitness, f32)
    age = np.asarray(age, np.int64)
    n = len(fit)
    rank = np.zeros(n, np.uint32)
    crowd = np.zeros(n, f32)
    count = [0] * n
    dominated: List[List[int]] = [[] for _ in range(n)]
    fronts: List[List[int]] = [[]]
    for i in range(n):
        for j in range(n):
            if i == j:
                continue
            if _dominates(fit[i], age[i], fit[j], age[j]):
                dominated[i].append(j)
            elif _dominates(fit[j], age[j], fit[i], age[i]):
                count[i] += 1
        if count[i] == 0:
            rank[i] = 0
            fronts[0].append(i)
    i = 0
    while i < len(fronts):
        nxt = []
        for p in fronts[i]:
            for q in dominated[p]:
                count[q] -= 1
                if count[q] == 0:
                    rank[q] = i + 1
                    nxt.append(q)
        if not nxt:
            break
        fronts.append(nxt)
        i += 1
    for front in fronts:
        if not front:
            continue
        for idx in front:
            crowd[idx] = f32(0)
        if len(front) < 3:
            for idx in front:
                crowd[idx] = FMAX
            continue
        s = sorted(front, key=lambda a: fit[a])          # stable, like sort_by
        crowd[s[0]] = FMAX
        crowd[s[-1]] = FMAX
        rng = f32(fit[s[-1]] - fit[s[0]])
        if rng > f32(1e-9):
            for k in range(1, len(s) - 1):
                d = f32(f32(fit[s[k + 1]] - fit[s[k - 1]]) / rng)
                if crowd[s[k]] != FMAX:
                    crowd[s[k]] = f32(crowd[s[k]] + d)
        s = sorted(s, key=lambda a: age[a])              # stable, like sort_by_key
        crowd[s[0]] = FMAX
        crowd[s[-1]] = FMAX
        amin, amax = f32(age[s[0]]), f32(age[s[-1]])
        arng = f32(amax - amin)
        if arng > f32(1e-9):
            for k in range(1, len(s) - 1):
                d = f32(f32(f32(age[s[k + 1]]) - f32(age[s[k - 1]])) / arng)
                if crowd[s[k]] != FMAX:
                    crowd[s[k]] = f32(crowd[s[k]] + d)
    return rank, crowd


def nsga2_less(rank, crowd, a: int, b: int) -> bool:
    """nsga2_compare(a, b) == Less: lower rank, else larger crowding."""
    if rank[a] != rank[b]:
        return rank[a] < rank[b]
    return crowd[b] < crowd[a]


def tournament(rank, crowd, draws: Sequence[int]) -> int:
    """Winner of one k-way tournament given its k drawn indices."""
    best = int(draws[0])
    for c in draws[1:]:
        if nsga2_less(rank, crowd, int(c), best):
            best = int(c)
    return best


def select(fitness, age, draws: np.ndarray) -> np.ndarray:
    """Indices chosen by len(draws) tournaments (draws: [t, k] indices)."""
    rank, crowd = assign_rank_and_crowding(fitness, age)
    return np.array([tournament(rank, crowd, d) for d in np.asarray(draws)], np.int64)
