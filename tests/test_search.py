"""The genetic search over the engine and the batched CMA-ES fit.

CPU: the expression rules (simplify_ast, Program::from_nodes, the forbidden
patterns, subtree bounds), the variation operators' invariants, the
oracle's CMA-ES restatement, and a whole search on the scalar workload
(y = 2.5 x^2 - 1.2, config C1) scored by the oracle.  GPU: ``rsr_fit_cma_es``
takes exactly the steps of the one-program-at-a-time restatement when both see
the same evaluations, and SymbolicRegressor.fit reaches MSE < 1e-7 on C1
through the engine.
"""
import numpy as np
import pytest

from oracle import binding as B
from oracle import cmaes as OC
from oracle import dataset_ref as DR
from oracle import lbfgs as OL
from oracle import nelder_mead as ON
from rsr_b200 import isa as I
from rsr_b200 import workloads as W
from rsr_b200.dataset import Dataset
from rsr_b200.search import engine as S
from rsr_b200.search import expr as E
from rsr_b200.search import operators as OPS

f32 = np.float32
X = (E.VAR, 0, I.FLOAT)


def C(i, t=I.FLOAT):
    return (E.CONST, i, t)


def O(name):
    return (E.OPER, I.OP[name], E.return_type(I.OP[name]))


# ------------------------------------------------------------ expressions
def test_simplify_folds_constants_and_renumbers():
    nodes = [C(0), C(1), O("AddF"), X, O("MulF")]
    out, oc = E.simplify(nodes, [I.Scalar.float(2.5), I.Scalar.float(-1.2)])
    # (2.5 + -1.2) * x -> c2 * x; the consumed constants stay in the list
    assert out == [C(2), X, O("MulF")]
    assert f32(oc[2].values[0]) == f32(f32(2.5) + f32(-1.2))


@pytest.mark.parametrize("nodes,consts,expect", [
    ([X, C(0), O("AddF")], [0.0], [X]),                       # x + 0
    ([C(0), X, O("AddF")], [0.0], [X]),                       # 0 + x
    ([X, C(0), O("MulF")], [1.0], [X]),                       # x * 1
    ([X, C(0), O("MulF")], [0.0], [C(1)]),                    # x * 0 -> 0
    ([X, X, O("SubF")], [], [C(0)]),                          # x - x -> 0
    ([X, X, O("DivF")], [], [C(0)]),                          # x / x -> 1
    ([X, O("ExpF"), O("LnF")], [], [X]),                      # ln(exp(x))
    ([X, O("SqrF"), O("SqrtF")], [], [X]),                    # sqrt(x^2), as the reference drops it
    ([X, C(0), O("DivF")], [1.0], [X]),
])
def test_simplify_identities(nodes, consts, expect):
    out, oc = E.simplify(nodes, [I.Scalar.float(v) for v in consts])
    assert out == expect
    if out == [C(0)] and nodes[-1] == O("DivF"):
        assert oc[0].values[0] == 1.0


def test_simplify_keeps_non_finite_folds():
    # 1 / 0 is not finite: the division stays
    out, _ = E.simplify([C(0), C(1), O("DivF")], [I.Scalar.float(1.0), I.Scalar.float(0.0)])
    assert out[-1] == O("DivF")


def test_simplify_linalg_rules():
    v = I.Scalar(I.VEC3, (1.0, 2.0, 3.0))
    z = I.Scalar(I.VEC3, (0.0, 0.0, 0.0))
    V = (E.VAR, 0, I.VEC3)
    out, oc = E.simplify([V, C(0, I.VEC3), O("CrossV3")], [z])
    assert out == [C(1, I.VEC3)] and oc[1].values == (0.0, 0.0, 0.0)
    out, oc = E.simplify([C(0, I.VEC3), C(1, I.VEC3), O("DotV3")], [v, v])
    assert out == [C(2)] and oc[2].values[0] == 14.0
    ident = I.Scalar(I.MAT2, (1.0, 0.0, 0.0, 1.0))
    M = (E.VAR, 0, I.MAT2)
    out, _ = E.simplify([C(0, I.MAT2), M, O("MulM2")], [ident])
    assert out == [M]


def test_simplified_programs_evaluate_alike():
    """simplify keeps the value of random expressions.  Folding rounds a
    constant subexpression once, where the VM rounds each step (and uses its
    own transcendental approximations), so a program that cancels can differ
    in a few points; a rule that changed the value would differ nearly
    everywhere."""
    rng = np.random.default_rng(3)
    ds = W.scalar_dataset(64, seed=4)
    allowed = S.Config().allowed_operators()
    checked = 0
    for _ in range(200):
        nodes, consts = OPS.generate_random_tree(I.FLOAT, 4, rng, [(I.FLOAT, 0)], allowed)
        a = B.eval_points(E.compile_program(nodes, consts), ds)
        sn, sc = E.simplify(nodes, consts)
        b = B.eval_points(E.compile_program(sn, sc), ds)
        ok = np.isfinite(a) & np.isfinite(b)
        if not ok.any():
            continue
        close = np.isclose(b[ok], a[ok], rtol=1e-4, atol=1e-4)
        assert close.mean() >= 0.9, (nodes, consts)
        np.testing.assert_allclose(b[ok], a[ok], rtol=1e-2, atol=1e-2)
        checked += 1
    assert checked > 100


def test_compile_and_bounds():
    nodes = [X, X, O("MulF"), C(0), O("MulF"), C(1), O("AddF")]
    p = E.compile_program(nodes, [I.Scalar.float(2.5), I.Scalar.float(-1.2)])
    assert p.code == [I.load_var(I.FLOAT, 0), I.load_var(I.FLOAT, 0), I.op("MulF"), I.load_const(I.FLOAT, 0),
                      I.op("MulF"), I.load_const(I.FLOAT, 1), I.op("AddF")]
    assert E.subtree_bounds(nodes, 4) == (0, 4)
    assert E.subtree_bounds(nodes, 5) == (5, 5)
    assert E.subtree_bounds(nodes, 6) == (0, 6)
    assert E.complexity(nodes) == 7


def test_forbidden_patterns():
    assert E.has_forbidden_patterns([X, O("SinF"), O("CosF")])
    assert E.has_forbidden_patterns([X, O("ExpF"), O("SqrF")])
    assert not E.has_forbidden_patterns([X, O("SinF"), X, O("AddF")])
    assert E.has_forbidden_patterns([O("AddF")])  # stack underflow


# ------------------------------------------------------------- operators
def _valid(nodes, consts, nf):
    p = E.compile_program(nodes, consts)
    return B.validate(p, nf) == 0


def test_operators_keep_programs_valid():
    rng = np.random.default_rng(11)
    cfg = S.Config(allowed_modules=[S.BASIC, S.LINALG])
    allowed = cfg.allowed_operators()
    reg = S.variable_registry([I.VEC3, I.VEC3, I.FLOAT])
    nf = 7
    pop = [OPS.generate_random_tree(I.FLOAT, 5, rng, reg, allowed) for _ in range(60)]
    for nodes, consts in pop:
        assert _valid(nodes, consts, nf)
    for k in range(300):
        a = pop[k % len(pop)]
        b = pop[(7 * k + 3) % len(pop)]
        nodes, consts = list(a[0]), list(a[1])
        r = k % 4
        if r == 0:
            OPS.point_mutation(nodes, consts, rng, reg, allowed)
        elif r == 1:
            OPS.constant_perturbation(nodes, consts, rng)
        elif r == 2:
            nodes = OPS.subtree_mutation(nodes, consts, rng, reg, 32, 4, allowed)
        else:
            c = OPS.crossover(a[0], a[1], b[0], b[1], rng, 32)
            if c is None:
                continue
            nodes, consts = c
            assert len(nodes) <= 32
        assert _valid(nodes, consts, nf), (r, nodes)
        sn, sc = E.simplify(nodes, consts)
        assert _valid(sn, sc, nf)


def test_selection_matches_restated_tournament():
    ind = []
    for f, a in [(0.5, 3), (0.1, 9), (0.3, 1), (0.3, 2), (2.0, 0)]:
        i = S.Individual([X], [])
        i.fitness, i.age = f, a
        ind.append(i)
    isl = S.Island.__new__(S.Island)
    isl.individuals = ind
    isl.cfg = S.Config()
    isl.rank_population()
    from rsr_b200 import selection as SEL
    rank, crowd = SEL.assign_rank_and_crowding([i.fitness for i in ind], [i.age for i in ind])
    assert [i.rank for i in ind] == list(rank)


# ------------------------------------------------------------------ CMA-ES
def _quadratic(n=200, seed=5):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-3.0, 3.0, n).astype(f32)
    y = (f32(2.5) * x * x - f32(1.2)).astype(f32)
    ds = Dataset.new(x[:, None], y, [I.FLOAT])
    prog = I.Program([I.load_const(I.FLOAT, 0), I.load_var(I.FLOAT, 0), I.op("MulF"), I.load_var(I.FLOAT, 0),
                      I.op("MulF"), I.load_const(I.FLOAT, 1), I.op("SubF")],
                     [I.Scalar.float(2.0), I.Scalar.float(1.0)])
    return prog, ds


def test_oracle_cma_es_reduces_error():
    prog, ds = _quadratic()
    m0 = B.mse_ref32(prog, ds)
    x, m, st = OC.run_cma_es(prog, ds, 60, seed=9)
    assert m < 0.05 * m0 and st["iterations"] > 5


def _cma_population():
    """Programs with Float, Vec2 and Mat2 constants and one without any, on
    the uneven-batch features (A, B Mat2)."""
    ds = W.inverse_dataset(300, seed=41)
    M = lambda i: I.load_var(I.MAT2, i)
    progs = [
        I.Program([M(0), I.op("InverseM2"), I.load_const(I.MAT2, 0), I.op("AddM2"), I.op("TraceM2")],
                  [I.Scalar(I.MAT2, (0.5, -0.2, 0.1, 0.4))]),
        I.Program([M(0), I.op("DetM2"), I.load_const(I.FLOAT, 0), I.op("MulF"), M(4), I.op("TraceM2"),
                   I.op("AddF")], [I.Scalar.float(0.7)]),
        I.Program([M(4), I.load_const(I.VEC2, 0), I.op("MulM2V2"), I.op("NormV2")],
                  [I.Scalar(I.VEC2, (1.0, -1.0))]),
        I.Program([M(0), I.op("InverseM2"), M(4), I.op("MulM2"), I.op("TraceM2")], []),
    ]
    return progs, ds


@pytest.mark.gpu
def test_cma_es_matches_sequential_restatement():
    """Same evaluations in -> same steps out: the batched fit against
    run_cma_es driven by single-program calls of the same engine."""
    from rsr_b200.evaluator import Engine
    progs, ds = _cma_population()
    with Engine() as eng:
        d = eng.upload(ds)
        params, mse, st = eng.fit_cma_es(progs, d, 6, seed=1234)
        pk = I.pack(progs)
        for i, p in enumerate(progs):
            q = I.Program(list(p.code), [I.Scalar(c.kind, c.values) for c in p.constants])
            x, m, _ = OC.run_cma_es(q, ds, 6, seed=1234, index=i, mse_fn=lambda pr: eng.compute_mse(pr, d))
            got = params[pk.param_off[i]:pk.param_off[i + 1]]
            np.testing.assert_array_equal(got, x[:len(got)], err_msg=f"program {i}")
            assert f32(mse[i]) == f32(m), i
        assert st["iterations"] >= 1


@pytest.mark.gpu
def test_cma_es_per_program_datasets_match_restatement():
    """Programs fitted against different resident datasets in one call take
    the steps of the restatement run on each program's own dataset."""
    from rsr_b200.evaluator import Engine
    progs, _ = _cma_population()
    sets = [W.inverse_dataset(n, seed=90 + k) for k, n in enumerate((300, 1700, 5000))]
    with Engine() as eng:
        dev = [eng.upload(ds) for ds in sets]
        which = [0, 2, 1, 2]
        params, mse, _ = eng.fit_cma_es(progs, datasets=[dev[k] for k in which], max_iterations=4, seed=77)
        pk = I.pack(progs)
        for i, p in enumerate(progs):
            q = I.Program(list(p.code), [I.Scalar(c.kind, c.values) for c in p.constants])
            d = dev[which[i]]
            x, m, _ = OC.run_cma_es(q, sets[which[i]], 4, seed=77, index=i,
                                    mse_fn=lambda pr: eng.compute_mse(pr, d))
            got = params[pk.param_off[i]:pk.param_off[i + 1]]
            np.testing.assert_array_equal(got, x[:len(got)], err_msg=f"program {i}")
            assert f32(mse[i]) == f32(m), i


@pytest.mark.gpu
def test_cma_es_quadratic(engine):
    prog, ds = _quadratic()
    m0 = B.mse_ref32(prog, ds)
    x, m, _ = engine.fit_cma_es([prog], ds, 60, seed=9)
    assert m[0] < 0.05 * m0


# ------------------------------------------------------------------ search
class OracleBackend(S.Backend):
    """Scores with the oracle's f32 compute_mse and fits with the oracle's
    restated optimisers (CPU)."""

    def __init__(self, train, mini):
        self.data = {"train": train, "mini": mini}

    def mse(self, programs, which):
        if not programs:
            return np.zeros(0, f32)
        return B.mse_batch(I.pack(list(programs)), self.data[which], threads=4)[1]

    def fit(self, programs, method, iterations):
        out = []
        for i, p in enumerate(programs):
            q = I.Program(list(p.code), [I.Scalar(c.kind, c.values) for c in p.constants])
            if method == "lbfgs":
                flat, _, _ = OL.run_lbfgs(q, self.data["train"], 15)
            elif method == "nelder_mead":
                flat, _, _ = ON.run_nelder_mead(q, self.data["train"], iterations)
            else:
                flat, _, _ = OC.run_cma_es(q, self.data["train"], max(iterations // 16, 2), index=i)
            out.append(np.asarray(flat, f32))
        return out


def _subset(ds, m):
    ff, tb, n = DR.subset(ds.feature_flat, ds.target_batches, ds.num_features, ds.num_samples, m)
    return Dataset(ff, tb, ds.num_features, len(tb) // 8, n, ds.feature_means, ds.feature_std_devs,
                   feature_types=ds.feature_types)


def _c1_config(**kw):
    # C1's operator set: {+, -, *, /, sin, cos, exp} (neg is written 0 - x)
    return S.Config(excluded_ops=["SqrF", "SqrtF", "LnF"], **kw)


def test_search_reaches_target_on_scalar_workload():
    ds = W.scalar_dataset(400)
    train = _subset(ds, 400)
    mini = _subset(train, 64)
    cfg = _c1_config(num_islands=8, max_generations=60, migration_interval=10)
    search = S.SearchEngine(cfg, S.variable_registry([I.FLOAT]), OracleBackend(train, mini))
    best = search.run()
    mse = B.mse_ref32(best.compile(), ds)
    assert mse <= 1e-7, (str(best), mse, search.generations)
    assert search.generations < 60
    front = search.pareto_front()
    assert front and all(front[k][1] > front[k + 1][1] for k in range(len(front) - 1))


@pytest.mark.gpu
def test_regressor_reaches_target_on_device(engine):
    """Config C1 end to end: 1024 random programs scored, then the search to
    MSE < 1e-7 with every score and fit on the engine."""
    ds = W.scalar_dataset(400)
    d = engine.upload(ds)
    pop = W.scalar_population(1024)
    m = engine.compute_mse_batch(pop, d)
    assert len(m) == 1024
    res = S.SymbolicRegressor(_c1_config()).fit(engine, d, [I.FLOAT])
    assert res.mse <= 1e-7, res
    assert res.generations < 3000
