"""Tournament selection on (fitness, age) Pareto ranks
(src/engine/search/operators/selection.rs), and the bit-exact indices check:
selection driven by the engine's fitness picks the same individuals as
selection driven by the oracle's restatement of the reference's f32 MSE."""
import numpy as np
import pytest

from rsr_b200 import selection as SEL
from rsr_b200 import workloads as W

f32 = np.float32
FMAX = np.finfo(np.float32).max


def _fronts_bruteforce(fit, age):
    """Front index by repeatedly peeling the non-dominated set."""
    n = len(fit)
    left = set(range(n))
    rank = np.zeros(n, np.uint32)
    r = 0
    while left:
        front = [i for i in left if not any(
            (fit[j] <= fit[i] and age[j] <= age[i]) and (fit[j] < fit[i] or age[j] < age[i]) for j in left if j != i)]
        for i in front:
            rank[i] = r
        left -= set(front)
        r += 1
    return rank


def test_ranks_match_front_peeling():
    rng = np.random.default_rng(1)
    for _ in range(50):
        n = int(rng.integers(1, 30))
        fit = rng.choice(np.array([0.5, 1.0, 2.0, 3.0, FMAX], f32), n) if rng.random() < 0.5 else \
            rng.uniform(0, 10, n).astype(f32)
        age = rng.integers(0, 6, n)
        rank, crowd = SEL.assign_rank_and_crowding(fit, age)
        assert np.array_equal(rank, _fronts_bruteforce(fit, age))
        assert crowd.dtype == np.float32 and np.all(crowd >= 0)


def test_crowding_hand_case():
    # four mutually non-dominated individuals: fitness up, age down
    fit = np.array([1, 2, 3, 4], f32)
    age = np.array([3, 2, 1, 0])
    rank, crowd = SEL.assign_rank_and_crowding(fit, age)
    assert list(rank) == [0, 0, 0, 0]
    inner = f32(f32(f32(3) - f32(1)) / f32(3))                     # fitness term of 1 and 2
    age_term = f32(f32(f32(2) - f32(0)) / f32(3))
    assert crowd[0] == FMAX and crowd[3] == FMAX
    assert crowd[1] == f32(inner + age_term) and crowd[2] == f32(inner + age_term)
    # fronts of fewer than three get f32::MAX
    r2, c2 = SEL.assign_rank_and_crowding(np.array([1, 2], f32), np.array([0, 0]))
    assert list(r2) == [0, 1] and c2[0] == FMAX and c2[1] == FMAX


def test_tournament_prefers_rank_then_crowding():
    rank = np.array([1, 0, 0], np.uint32)
    crowd = np.array([5.0, 1.0, 2.0], f32)
    assert SEL.tournament(rank, crowd, [0, 1]) == 1      # lower rank wins
    assert SEL.tournament(rank, crowd, [1, 2]) == 2      # larger crowding wins
    assert SEL.tournament(rank, crowd, [2, 2]) == 2      # a tie keeps the incumbent


@pytest.mark.gpu
def test_indices_bit_exact_engine_vs_oracle(engine):
    from oracle import binding as O
    ds = W.scalar_dataset(400, seed=21)
    pop = W.scalar_population(8 * 25, seed=22)
    gpu = engine.compute_mse_batch(pop, ds)
    ref = np.array([O.mse_ref32(p, ds) for p in pop], f32)
    rng = np.random.default_rng(23)
    for isl in range(8):
        sl = slice(25 * isl, 25 * (isl + 1))
        age = rng.integers(0, 10, 25)
        draws = rng.integers(0, 25, (25, 2))                       # 25 tournaments, k = 2
        a = SEL.select(gpu[sl], age, draws)
        b = SEL.select(ref[sl], age, draws)
        assert np.array_equal(a, b), (isl, a, b)
