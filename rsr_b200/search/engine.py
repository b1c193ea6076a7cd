"""The island search, driven through batched engine calls.

Restates the reference's genetic search -- Config (src/engine/search/config.rs:10-69),
StaticStrategy's operator lists (strategy.rs:122-195), Individual
(individual.rs:14-110), Island (island.rs:21-262), Engine (engine.rs:11-156)
and SymbolicRegressor::fit (src/api.rs:104-132) -- with one change of
structure: the reference steps each island on its own rayon thread and
scores one individual per call; here all islands step in lockstep and every
evaluation phase of a generation is one batched call for the whole
archipelago (mini-batch scores of the offspring, their full-data scores, the
constant fits, the re-scores), so the device sees hundreds of programs per
launch.

The decisions that the reference takes one individual at a time against a
running best (which offspring get their constants fitted) are replayed in
the reference's order after the batched calls: the fits run for every
offspring that could qualify against the generation's starting best, and the
replay keeps a fit only where the reference's sequential rule would have made
it.  Random draws come from one numpy Generator per island (seeded 42 + i
like the reference's islands); the reference's xoshiro streams are not
restated, so runs follow the reference's rules but not its exact sequences.

The optimiser choice follows optimize_individual_constants
(src/engine/optimize/mod.rs:10-59): L-BFGS with 15 iterations for
differentiable programs, CMA-ES with max(iterations / 16, 2) generations for
non-differentiable programs with vector or matrix constants, Nelder-Mead
otherwise.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from .. import isa as I
from .. import selection as SEL
from . import expr as E
from . import operators as OPS

f32 = np.float32
FMAX = float(np.finfo(np.float32).max)

BASIC, LINALG, LOGIC = "basic", "linalg", "logic"

# strategy.rs:131-185, in the reference's order
_MODULE_OPS = {
    BASIC: ["AddF", "SubF", "MulF", "DivF", "SinF", "CosF", "ExpF", "SqrF", "LnF", "SqrtF"],
    LINALG: ["MakeVec2", "MakeVec3", "GetXV2", "GetYV2", "GetXV3", "GetYV3", "GetZV3", "AddV2", "SubV2",
             "ScaleV2", "DotV2", "NormV2", "AddV3", "SubV3", "ScaleV3", "DotV3", "NormV3", "CrossV3",
             "MakeMat2", "AddM2", "SubM2", "ScaleM2", "MulM2", "MulM2V2", "DetM2", "TraceM2", "TransposeM2",
             "InverseM2", "MakeMat3", "AddM3", "SubM3", "ScaleM3", "MulM3", "MulM3V3", "DetM3", "TraceM3",
             "TransposeM3", "InverseM3"],
    LOGIC: [],
}


@dataclass
class Config:
    """Search parameters with the reference's defaults (config.rs:41-69)."""
    allowed_modules: List[str] = field(default_factory=lambda: [BASIC])
    num_islands: int = 24
    island_size: int = 25
    max_generations: int = 3000
    crossover_rate: float = 0.10
    tournament_size: int = 2
    migration_interval: int = 25
    parsimony_penalty: float = 0.000005
    opt_prob: float = 0.01
    opt_iterations: int = 100
    final_opt_iterations: int = 4000
    stagnation_threshold: int = 1000
    target_mse: float = 1e-7
    min_improvement: float = 1e-6
    random_injection_rate: float = 0.10
    min_random_injection: int = 2
    max_tree_size: int = 32
    mutation_max_depth: int = 4
    mutation_cycles: int = 2
    verbose: bool = False
    custom_ops: List[str] = field(default_factory=list)
    excluded_ops: List[str] = field(default_factory=list)
    subset_size: Optional[int] = 400
    mini_batch_size: int = 64

    def allowed_operators(self) -> List[int]:
        """get_allowed_operators (strategy.rs:122-195): the modules' operators,
        then the custom ones, without the excluded ones or repeats."""
        names = [n for m in self.allowed_modules for n in _MODULE_OPS[m]] + list(self.custom_ops)
        out: List[int] = []
        for n in names:
            op = I.OP[n]
            if n not in self.excluded_ops and op not in out:
                out.append(op)
        return out


def variable_registry(feature_types: Sequence[int]) -> List[Tuple[int, int]]:
    """get_variable_registry (dataset.rs:200-222): each feature at its flat
    offset, and every component of a vector or matrix feature as a Float."""
    reg: List[Tuple[int, int]] = []
    off = 0
    for t in feature_types:
        reg.append((t, off))
        w = I.TYPE_WIDTH[t]
        if w > 1:
            reg.extend((I.FLOAT, off + k) for k in range(w))
        off += w
    return reg


class Individual:
    """individual.rs:14-110: an expression, its constants and its scores."""
    __slots__ = ("nodes", "consts", "fitness", "age", "program", "rank", "crowd")

    def __init__(self, nodes: List[E.Node], consts: List[I.Scalar]):
        self.nodes = nodes
        self.consts = consts
        self.fitness = FMAX
        self.age = 0
        self.program: Optional[I.Program] = None
        self.rank = 0
        self.crowd = 0.0

    def clone(self) -> "Individual":
        c = Individual(list(self.nodes), list(self.consts))
        c.fitness, c.age, c.program, c.rank, c.crowd = self.fitness, self.age, self.program, self.rank, self.crowd
        return c

    def compile(self) -> I.Program:
        if self.program is None:
            self.program = E.compile_program(self.nodes, self.consts)
        return self.program

    def invalidate(self) -> None:
        self.program = None
        self.fitness = FMAX

    def simplify(self) -> None:
        if self.nodes:
            self.nodes, self.consts = E.simplify(self.nodes, self.consts)
        self.invalidate()

    def complexity(self) -> int:
        return E.complexity(self.nodes)

    def forbidden(self) -> bool:
        return E.has_forbidden_patterns(self.nodes)

    def set_fitted(self, flat: np.ndarray) -> None:
        """Writes a fitted program's flat parameters back into the constants
        in node order (lbfgs.rs:154-164), zeroes components below 0.05,
        simplifies and recompiles (individual.rs:58-68)."""
        prog = self.compile()
        fitted = I.Program(prog.code, [I.Scalar(c.kind, c.values) for c in prog.constants])
        fitted.unflatten_params(flat)
        k = 0
        consts = list(self.consts)
        for n in self.nodes:
            if n[0] == E.CONST and k < len(fitted.constants):
                consts[n[1]] = fitted.constants[k]
                k += 1
        self.consts = [E.apply_threshold(c, 0.05) for c in consts]
        self.simplify()
        self.compile()

    def method(self) -> str:
        """optimize_individual_constants' choice (optimize/mod.rs:24-58)."""
        if all(E.is_differentiable(n[1]) for n in self.nodes if n[0] == E.OPER):
            return "lbfgs"
        prog = self.compile()
        if any(c.kind in (I.VEC2, I.VEC3, I.MAT2, I.MAT3) for c in prog.constants):
            return "cmaes"
        return "nelder_mead"

    def __str__(self) -> str:
        return E.format_expr(self.nodes, self.consts)


class Backend:
    """Batched scoring and constant fitting on the two resident datasets of a
    search: the training data ("train") and its mini-batch ("mini")."""

    def mse(self, programs: Sequence[I.Program], which: str) -> np.ndarray:
        raise NotImplementedError

    def fit(self, programs: Sequence[I.Program], method: str, iterations: int) -> List[np.ndarray]:
        """Fitted flat parameters of each program on the training data."""
        raise NotImplementedError


class EngineBackend(Backend):
    """The device engine (rsr_b200.evaluator.Engine) with resident datasets."""

    def __init__(self, engine, train, mini, seed: int = 0):
        self.engine, self.data = engine, {"train": train, "mini": mini}
        self.rng = np.random.default_rng(seed)
        self.calls = 0

    def mse(self, programs, which):
        if not programs:
            return np.zeros(0, f32)
        self.calls += 1
        return np.asarray(self.engine.compute_mse_batch(I.pack(list(programs)), self.data[which]), f32)

    def fit(self, programs, method, iterations):
        if not programs:
            return []
        self.calls += 1
        pk = I.pack(list(programs))
        if method == "lbfgs":
            params, _, _ = self.engine.fit_lbfgs(pk, self.data["train"], 15)
        elif method == "nelder_mead":
            params, _, _ = self.engine.fit_nelder_mead(pk, self.data["train"], iterations)
        else:
            params, _, _ = self.engine.fit_cma_es(pk, self.data["train"], max(iterations // 16, 2), rng=self.rng)
        return [np.asarray(params[pk.param_off[i]:pk.param_off[i + 1]], f32) for i in range(pk.n)]


class Island:
    """Population state of one island (island.rs:21-68)."""

    def __init__(self, seed: int, registry, cfg: Config, allowed: List[int]):
        self.rng = np.random.default_rng(seed)
        self.registry, self.cfg, self.allowed = registry, cfg, allowed
        self.individuals = [self.random_individual() for _ in range(cfg.island_size)]
        self.best = self.individuals[0].clone()
        self.stagnation = 0
        self.hof: Dict[int, Tuple[float, Individual]] = {}

    def random_individual(self) -> Individual:
        nodes, consts = OPS.generate_random_tree(I.FLOAT, 5, self.rng, self.registry, self.allowed)
        ind = Individual(nodes, consts)
        ind.simplify()
        return ind

    def tournament(self) -> Individual:
        """tournament_selection_pareto (selection.rs:13-27)."""
        pop = self.individuals
        best = int(self.rng.integers(0, len(pop)))
        for _ in range(1, self.cfg.tournament_size):
            c = int(self.rng.integers(0, len(pop)))
            a, b = pop[c], pop[best]
            if a.rank < b.rank or (a.rank == b.rank and b.crowd < a.crowd):
                best = c
        return pop[best]

    def rank_population(self) -> None:
        rank, crowd = SEL.assign_rank_and_crowding([i.fitness for i in self.individuals],
                                                   [i.age for i in self.individuals])
        for ind, r, c in zip(self.individuals, rank, crowd):
            ind.rank, ind.crowd = int(r), float(c)


def _penalised(mse: float, complexity: int, penalty: float) -> float:
    return float(f32(f32(mse) + f32(f32(complexity) * f32(penalty))))


class SearchEngine:
    """engine.rs:11-156 over lockstep islands (see the module docstring)."""

    def __init__(self, cfg: Config, registry, backend: Backend):
        self.cfg, self.backend = cfg, backend
        self.allowed = cfg.allowed_operators()
        self.islands = [Island(42 + i, registry, cfg, self.allowed) for i in range(cfg.num_islands)]
        self.global_hof: Dict[int, Tuple[float, Individual]] = {}
        self.generations = 0
        self._train_mse: Optional[Tuple[Individual, float]] = None

    # ------------------------------------------------------------ a generation
    def _fill(self) -> List[List[Individual]]:
        """fill_next_generation (island.rs:98-182) for every island: elitism,
        random injection, crossover, and mutation candidates whose hill-climb
        cycles are scored on the mini-batch in one call per cycle."""
        cfg = self.cfg
        buffers: List[List[Individual]] = []
        slots: List[Tuple[Island, List[Individual], int]] = []  # mutation candidates
        for isl in self.islands:
            pop_size = cfg.island_size
            buf = [isl.best.clone()]
            n_random = int(f32(max(f32(pop_size) * f32(cfg.random_injection_rate), f32(cfg.min_random_injection))))
            for _ in range(n_random):
                if len(buf) >= pop_size:
                    break
                buf.append(isl.random_individual())
            while len(buf) < pop_size:
                if isl.rng.random() < cfg.crossover_rate:
                    p1, p2 = isl.tournament(), isl.tournament()
                    r = OPS.crossover(p1.nodes, p1.consts, p2.nodes, p2.consts, isl.rng, cfg.max_tree_size)
                    child = Individual(*r) if r is not None else p1.clone()
                    if child.forbidden():
                        child = p1.clone()
                    child.age = max(p1.age, p2.age)
                    child.simplify()
                    buf.append(child)
                else:
                    slots.append((isl, buf, len(buf)))
                    buf.append(isl.tournament().clone())
            buffers.append(buf)
        # candidates never scored get their mini-batch score first
        unscored = [(b, k) for _, b, k in slots if b[k].fitness == FMAX]
        if unscored:
            scores = self.backend.mse([b[k].compile() for b, k in unscored], "mini")
            for (b, k), s in zip(unscored, scores):
                b[k].fitness = float(s)
        for _ in range(cfg.mutation_cycles):
            trial: List[Tuple[List[Individual], int, Individual]] = []
            for isl, b, k in slots:
                m = b[k].clone()
                kind = int(isl.rng.integers(0, 3))
                if kind == 0:
                    OPS.point_mutation(m.nodes, m.consts, isl.rng, isl.registry, self.allowed)
                elif kind == 1:
                    OPS.constant_perturbation(m.nodes, m.consts, isl.rng)
                else:
                    m.nodes = OPS.subtree_mutation(m.nodes, m.consts, isl.rng, isl.registry, cfg.max_tree_size,
                                                   cfg.mutation_max_depth, self.allowed)
                m.simplify()
                if not m.forbidden():
                    trial.append((b, k, m))
            scores = self.backend.mse([m.compile() for _, _, m in trial], "mini")
            for (b, k, m), s in zip(trial, scores):
                if f32(s) < f32(b[k].fitness):
                    m.fitness = float(s)
                    b[k] = m
        return buffers

    def _fit_all(self, inds: List[Individual], iterations: int) -> List[Individual]:
        """Constant fitting of copies of `inds`, one batched call per method."""
        out = [i.clone() for i in inds]
        by_method: Dict[str, List[int]] = {}
        for j, ind in enumerate(out):
            by_method.setdefault(ind.method(), []).append(j)
        for method, idx in by_method.items():
            fitted = self.backend.fit([out[j].compile() for j in idx], method, iterations)
            for j, flat in zip(idx, fitted):
                out[j].set_fitted(flat)
        return out

    def _evaluate(self, buffers: List[List[Individual]]) -> None:
        """evaluate_buffer (island.rs:218-261) for every island."""
        cfg = self.cfg
        bests = [isl.best.clone() for isl in self.islands]
        flat = [ind for buf in buffers for ind in buf]
        mini = self.backend.mse([b.compile() for b in bests] + [i.compile() for i in flat], "mini")
        base, mini = mini[:len(bests)], mini[len(bests):]
        # promising offspring and the fit lottery, drawn in the reference's order
        promising, lottery, pos = [], [], 0
        for isl, buf, b0 in zip(self.islands, buffers, base):
            for _ in buf:
                p = bool(f32(mini[pos]) < f32(f32(b0) * f32(2.0)))
                if not p and isl.rng.random() < 0.05:
                    p = True
                promising.append(p)
                lottery.append(p and isl.rng.random() < cfg.opt_prob)
                pos += 1
        full = np.full(len(flat), np.nan, f32)
        pi = [j for j, p in enumerate(promising) if p]
        full[pi] = self.backend.mse([flat[j].compile() for j in pi], "train")
        # fit every offspring that could qualify against its island's starting best
        start_best, pos = [], 0
        for isl, buf in zip(self.islands, buffers):
            start_best += [isl.best.fitness] * len(buf)
        cand = [j for j in pi if math.isfinite(full[j]) and (lottery[j] or f32(full[j]) < f32(start_best[j]))]
        fitted = dict(zip(cand, self._fit_all([flat[j] for j in cand], cfg.opt_iterations)))
        fitted_mse = dict(zip(cand, self.backend.mse([fitted[j].compile() for j in cand], "train")))
        # replay in order against the running best
        pos = 0
        for isl, buf in zip(self.islands, buffers):
            for k in range(len(buf)):
                j = pos + k
                ind, final = buf[k], float(mini[j])
                if promising[j]:
                    final = float(full[j])
                    elite = f32(final) < f32(isl.best.fitness)
                    if (elite or lottery[j]) and math.isfinite(final):
                        ind = fitted[j]
                        final = float(fitted_mse[j])
                if math.isfinite(final):
                    c = ind.complexity()
                    if c not in isl.hof or f32(final) < f32(isl.hof[c][0]):
                        isl.hof[c] = (final, ind.clone())
                    ind.fitness = _penalised(final, c, cfg.parsimony_penalty)
                else:
                    ind.fitness = FMAX
                buf[k] = ind
                if f32(ind.fitness) < f32(isl.best.fitness):
                    isl.best = ind.clone()
            pos += len(buf)

    def _nuke(self, islands: List[Island]) -> None:
        """island.rs:184-216: the best survives; the rest are new random
        individuals scored on the training data."""
        cfg = self.cfg
        fresh: List[Tuple[Island, List[Individual]]] = []
        for isl in islands:
            new = [isl.random_individual() for _ in range(1, cfg.island_size)]
            fresh.append((isl, new))
        allnew = [i for _, new in fresh for i in new]
        scores = self.backend.mse([i.compile() for i in allnew], "train")
        pos = 0
        for isl, new in fresh:
            for ind in new:
                s = float(scores[pos])
                pos += 1
                if math.isfinite(s):
                    ind.fitness = _penalised(s, ind.complexity(), cfg.parsimony_penalty)
            isl.individuals = [isl.best.clone()] + new
            isl.stagnation = 0

    def step(self) -> None:
        """Island::step_generation (island.rs:70-96) for every island."""
        cfg = self.cfg
        old = [isl.best.fitness for isl in self.islands]
        for isl in self.islands:
            for ind in isl.individuals:
                ind.age += 1
            isl.rank_population()
        buffers = self._fill()
        self._evaluate(buffers)
        nuke = []
        for isl, buf, o in zip(self.islands, buffers, old):
            isl.individuals = buf
            if f32(f32(o) - f32(isl.best.fitness)) > f32(cfg.min_improvement):
                isl.stagnation = 0
            else:
                isl.stagnation += 1
            if isl.stagnation >= cfg.stagnation_threshold * 4:
                nuke.append(isl)
        if nuke:
            self._nuke(nuke)
        self.generations += 1

    # --------------------------------------------------------------- the run
    def global_best(self) -> Individual:
        return min((isl.best for isl in self.islands), key=lambda i: i.fitness)

    def train_mse(self, ind: Individual) -> float:
        """MSE on the training data (calculate_mse), remembered for the last
        individual asked about: the global best rarely changes."""
        if self._train_mse is None or self._train_mse[0] is not ind:
            self._train_mse = (ind, float(self.backend.mse([ind.compile()], "train")[0]))
        return self._train_mse[1]

    def migrate(self) -> None:
        """engine.rs:116-136: each island's best replaces the last individual
        of the next island."""
        if len(self.islands) < 2:
            return
        migrants = [isl.best.clone() for isl in self.islands]
        migrants = migrants[-1:] + migrants[:-1]
        for isl, m in zip(self.islands, migrants):
            isl.individuals[-1] = m

    def run(self) -> Individual:
        """engine.rs:39-113: generations until the target MSE, with migration;
        then a final constant fit of the global best."""
        cfg = self.cfg
        for gen in range(cfg.max_generations):
            self.step()
            for isl in self.islands:
                for c, (mse, ind) in isl.hof.items():
                    if c not in self.global_hof or f32(mse) < f32(self.global_hof[c][0]):
                        self.global_hof[c] = (mse, ind.clone())
            pure = self.train_mse(self.global_best())
            if f32(pure) <= f32(cfg.target_mse):
                if cfg.verbose:
                    print(f">>> target reached in generation {gen}: {self.global_best()}")
                break
            if gen > 0 and gen % cfg.migration_interval == 0:
                self.migrate()
                if cfg.verbose:
                    print(f"generation {gen}, best MSE {pure}, {self.global_best()}")
        best = self._fit_all([self.global_best()], cfg.final_opt_iterations)[0]
        best.fitness = _penalised(self.backend.mse([best.compile()], "train")[0], best.complexity(),
                                  cfg.parsimony_penalty)
        self.islands[0].best = best
        return best

    def pareto_front(self) -> List[Tuple[int, float, Individual]]:
        """get_pareto_front (engine.rs:157-179)."""
        front = sorted(((c, m, i) for c, (m, i) in self.global_hof.items()), key=lambda t: t[0])
        out, best = [], FMAX
        for c, m, i in front:
            if m < best:
                best = m
                out.append((c, m, i))
        return out


@dataclass
class FitResult:
    """api.rs:29-37."""
    equation: str
    mse: float
    complexity: int
    generations: int


class SymbolicRegressor:
    """SymbolicRegressor (api.rs:20-132) on the device engine: the training
    subset and the mini-batch are built on the device from the resident
    dataset (Dataset::subset), and every score and fit of the search runs
    through batched engine calls."""

    def __init__(self, config: Optional[Config] = None):
        self.config = config or Config()

    def fit(self, engine, dataset, feature_types: Sequence[int]) -> FitResult:
        cfg = self.config
        train = engine.subset(dataset, cfg.subset_size) if cfg.subset_size else dataset
        mini = engine.subset(train, cfg.mini_batch_size)
        try:
            search = SearchEngine(cfg, variable_registry(feature_types), EngineBackend(engine, train, mini))
            best = search.run()
            full = float(engine.compute_mse_batch(I.pack([best.compile()]), dataset)[0])
        finally:
            mini.release()
            if train is not dataset:
                train.release()
        return FitResult(str(best), full, best.complexity(), search.generations)
