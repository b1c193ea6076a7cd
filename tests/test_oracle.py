"""The CPU oracle against the golden fixtures, the known-answer targets of the
reference's tests, IEEE-754, libm (error bounds) and its own dual-number and
finite-difference gradients.  CPU only."""
from pathlib import Path

import numpy as np
import pytest

import npvm
import programs as PR
from oracle import binding as O
from rsr_b200 import isa as I
from rsr_b200.dataset import Dataset
from rsr_b200.isa import FLOAT, Program, Scalar

GOLDEN = np.load(Path(__file__).parent / "golden" / "golden.npz")
f32 = np.float32


def _golden_program(prefix):
    code = [int(w) for w in GOLDEN[prefix + "_code"]]
    kinds = GOLDEN[prefix + "_kinds"]
    params = GOLDEN[prefix + "_params"]
    consts, p = [], 0
    for k in kinds:
        w = I.KIND_WIDTH[int(k)]
        consts.append(Scalar(int(k), tuple(params[p:p + w])))
        p += w
    return Program(code, consts)


def ulp_err(y, ref):
    ref = np.asarray(ref, np.float64)
    ulp = np.spacing(np.abs(ref).astype(np.float32)).astype(np.float64)
    return np.abs(y.astype(np.float64) - ref) / ulp


@pytest.mark.parametrize("name,fn,lo,hi", [("sin", np.sin, -100, 100), ("cos", np.cos, -100, 100),
                                           ("exp", np.exp, -87, 88), ("log", np.log, 1e-30, 1e30)])
def test_transcendentals_within_2ulp_of_libm(name, fn, lo, hi):
    rng = np.random.default_rng(0)
    x = (np.exp(rng.uniform(np.log(lo), np.log(hi), 4000)) if name == "log" else rng.uniform(lo, hi, 4000)).astype(f32)
    y = O.transcendental(name, x)
    assert ulp_err(y, fn(x.astype(np.float64))).max() <= 2.0


def test_transcendental_special_values():
    inf, nan = np.inf, np.nan
    x = np.array([0.0, -0.0, inf, -inf, nan, -1.0, 1e-40, 200.0, -200.0, 1e30], f32)
    s, c, e, l = (O.transcendental(n, x) for n in ("sin", "cos", "exp", "log"))
    assert np.isnan(s[2:5]).all() and np.isnan(c[2:5]).all()
    assert s[0] == 0 and c[0] == 1 and e[0] == 1 and l[0] == -inf and l[1] == -inf
    assert e[2] == inf and e[3] == 0 and np.isnan(e[4]) and e[7] == inf and e[8] == 0
    assert np.isnan(l[5]) and l[2] == inf and np.isfinite(l[6])


def test_simd_transcendentals_bit_identical_to_scalar():
    rng = np.random.default_rng(1)
    x = np.concatenate([rng.uniform(-50, 50, 1000), rng.uniform(-90, 90, 1000), [0, -0.0, np.inf, -np.inf, np.nan,
                                                                              1e-40, -1, 2e30]]).astype(f32)
    x = x[:len(x) // 8 * 8]
    for name in ("sin", "cos", "exp", "log"):
        a, b = O.transcendental(name, x), O.transcendental(name, x, simd=True)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)) or \
            np.array_equal(np.isnan(a), np.isnan(b)) and np.array_equal(a[~np.isnan(a)], b[~np.isnan(b)]), name


def test_n_opcodes():
    assert O.lib().orc_n_opcodes() == I.N_OPCODES == 62


@pytest.mark.parametrize("name", I.BASIC_NAMES + I.LINALG_NAMES)
def test_each_op_matches_golden(name):
    p = _golden_program(f"op_{name}")
    X = GOLDEN["op_X"]
    ds = Dataset.new(X, np.zeros(len(X), f32), [FLOAT] * X.shape[1])
    got = O.eval_points(p, ds)[:len(X)]
    want = GOLDEN[f"op_{name}_pred"]
    assert np.array_equal(np.isnan(got), np.isnan(want))
    m = ~np.isnan(want)
    assert np.array_equal(got[m].view(np.uint32), want[m].view(np.uint32))


@pytest.mark.parametrize("name", sorted(PR.kat_cases().keys()))
def test_known_answer_targets(name):
    p = _golden_program(f"kat_{name}")
    X, y = GOLDEN[f"kat_{name}_X"], GOLDEN[f"kat_{name}_y"]
    exact = bool(GOLDEN[f"kat_{name}_exact"])
    ds = Dataset.new(X, y, [FLOAT] * X.shape[1])
    pred = O.eval_points(p, ds)[:len(y)]
    m64 = O.mse_f64(p, ds)
    if exact:
        assert np.array_equal(pred, y)
        assert m64 == 0.0 and O.mse_ref32(p, ds) == 0.0
    else:
        assert m64 <= 1e-10 * max(1.0, float(np.mean(y.astype(np.float64) ** 2)))


def test_oracle_matches_numpy_vm_on_random_programs():
    from rsr_b200 import workloads as W
    ds = W.lorentz_dataset(300, seed=5)
    X = ds.point_features()
    for p in W.lorentz_population(60, seed=6):
        with np.errstate(all="ignore"):
            want = npvm.eval_points(p, X)
        got = O.eval_points(p, ds)
        assert np.array_equal(np.isnan(got), np.isnan(want))
        m = ~np.isnan(want)
        assert np.array_equal(got[m], want[m])


def test_padding_semantics():
    # 10 points -> 2 batches; padded lanes have x = 0, y = 0 and their squared
    # error is counted with divisor num_samples (evaluator.rs:159-173).
    x = np.arange(1, 11, dtype=f32)
    ds = Dataset.new(x[:, None], np.zeros(10, f32), [FLOAT])
    p = Program([I.load_const(FLOAT, 0)], [Scalar.float(2.0)])  # prediction 2 everywhere
    assert ds.num_batches == 2 and ds.num_samples == 10
    assert O.mse_f64(p, ds) == pytest.approx(16 * 4.0 / 10)
    assert O.mse_ref32(p, ds) == pytest.approx(16 * 4.0 / 10)


def test_result_is_stack_f0_not_top():
    # x, 3 -> two floats on the stack; the result is stack_f[0] = x
    p = Program([I.load_var(FLOAT, 0), I.load_const(FLOAT, 0)], [Scalar.float(3.0)])
    ds = Dataset.new(np.array([[5.0]], f32), np.array([0.0], f32), [FLOAT])
    assert O.eval_points(p, ds)[0] == 5.0


def test_nonfinite_mse_maps_to_f32_max():
    p = Program([I.load_var(FLOAT, 0), I.load_const(FLOAT, 0), I.op("DivF")], [Scalar.float(0.0)])
    ds = Dataset.new(np.array([[1.0], [2.0]], f32), np.zeros(2, f32), [FLOAT])
    assert O.mse_ref32(p, ds) == np.finfo(f32).max


def test_validation():
    assert O.validate(Program([I.op("AddF")]), 1) == -2                       # underflow
    assert O.validate(Program([I.load_var(FLOAT, 3)]), 2) == -3               # feature out of range
    assert O.validate(Program([I.load_const(FLOAT, 0)]), 1) == -4             # constant out of range
    assert O.validate(Program([I.load_var(FLOAT, 0)] * 33), 1) == -7          # > 32 slots
    assert O.validate(Program([I.load_var(FLOAT, 0)] * 32), 1) == 0


def test_dual_gradient_matches_finite_differences():
    from rsr_b200 import workloads as W
    ds = W.transform_dataset(512, seed=8)
    checked = 0
    for p in W.transform_population(30, seed=9):
        m, g = O.mse_grad_dual(p, ds)
        if not np.isfinite(m) or m == np.finfo(f32).max or m > 1e4 or not np.isfinite(g).all():
            continue  # sqrt/norm at 0 gives the reference's own inf/NaN derivative
        fd = O.grad_fd(p, ds, 1e-3)
        n = min(32, p.param_count())
        scale = max(np.abs(fd[:n]).max(), 1e-3)
        assert np.abs(g[:n] - fd[:n]).max() <= 2e-2 * scale
        checked += 1
    assert checked >= 10


def test_simd_baseline_matches_oracle_mse():
    from rsr_b200 import workloads as W
    ds = W.lorentz_dataset(1000, seed=10)
    pk = I.pack(W.lorentz_population(50, seed=11))
    m64, m32 = O.mse_batch(pk, ds, threads=4)
    simd = O.simd_mse_batch(pk, ds, threads=4)
    assert np.array_equal(simd, m32)


def test_dual_gradient_with_f64_sums_and_l1_scale():
    """orc_grad_dual_f64 applies the same per-point dual rules as
    orc_mse_grad_dual and differs only in summing over points in f64; its L1
    scale bounds the gradient's magnitude."""
    from rsr_b200 import workloads as W
    ds = W.transform_dataset(4000, seed=91)
    checked = 0
    for p in W.transform_population(40, seed=92):
        md, gd = O.mse_grad_dual(p, ds)
        m64, g64, l1 = O.grad_dual_f64(p, ds)
        n = min(32, p.param_count())
        if not (np.isfinite(gd[:n]).all() and np.isfinite(m64) and m64 < 1e4):
            continue
        # the value of the dual pass may differ from the plain pass by an ulp
        # in a few points (as the reference's does)
        assert abs(m64 - O.mse_f64(p, ds)) <= 1e-7 * max(1e-3, m64)
        assert np.all(np.abs(g64[:n]) <= l1[:n] * (1 + 1e-12))
        assert np.all(np.abs(gd[:n] - g64[:n]) <= 1e-5 * l1[:n] + 1e-30)
        assert np.all(g64[n:] == 0) and np.all(l1[n:] == 0)
        checked += 1
    assert checked >= 10
