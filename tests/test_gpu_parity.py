"""Parity of the CUDA engine (through the C ABI) with the CPU oracle.

Bars: per-point predictions bit-identical to the oracle's restatement of
eval_simd (so NaN/Inf patterns are identical and the 1e-5 relative bound holds
with margin); MSE within 1e-6 relative of the FP64 oracle, with the
f32::MAX class identical; gradients within 1e-3 relative of central finite
differences (h = 1e-3) and of the reference's dual-number gradient.
"""
import numpy as np
import pytest

import programs as PR
from oracle import binding as O
from rsr_b200 import _native as N
from rsr_b200 import isa as I
from rsr_b200 import workloads as W
from rsr_b200.dataset import Dataset
from rsr_b200.evaluator import Engine
from rsr_b200.isa import FLOAT, VEC2, Program, Scalar

pytestmark = pytest.mark.gpu
f32 = np.float32
FMAX = np.finfo(f32).max

WORKLOADS = {
    "scalar": (lambda: W.scalar_dataset(1000, seed=21), lambda: W.scalar_population(96, seed=22)),
    "lorentz": (lambda: W.lorentz_dataset(1500, seed=23), lambda: W.lorentz_population(96, seed=24)),
    "transform": (lambda: W.transform_dataset(1200, seed=25), lambda: W.transform_population(64, seed=26)),
    "inverse": (lambda: W.inverse_dataset(1100, seed=27), lambda: W.inverse_population(96, seed=28)),
}


def same_bits(a, b):
    a, b = np.asarray(a, f32), np.asarray(b, f32)
    na, nb = np.isnan(a), np.isnan(b)
    return np.array_equal(na, nb) and np.array_equal(a[~na], b[~nb])


def oracle_points(pop, ds):
    return np.stack([O.eval_points(p, ds) for p in pop])


@pytest.mark.parametrize("kernel", [N.KERNEL_PLAIN, N.KERNEL_AUTO])
@pytest.mark.parametrize("wl", sorted(WORKLOADS))
def test_points_bit_identical(engine, wl, kernel):
    ds, pop = WORKLOADS[wl][0](), WORKLOADS[wl][1]()
    got = engine.eval_points_batch(pop, ds, kernel=kernel)
    want = oracle_points(pop, ds)
    for i in range(len(pop)):
        assert same_bits(got[i], want[i]), (wl, i, [I.OP_NAMES[w & 255] for w in pop[i].code])


@pytest.mark.parametrize("ppt,ppw", [(1, 1), (2, 3), (4, 8), (8, 2)])
def test_points_bit_identical_all_tile_shapes(ppt, ppw):
    with Engine(points_per_thread=ppt, programs_per_warp=ppw) as e:
        for wl in ("scalar", "lorentz", "inverse"):
            ds, pop = WORKLOADS[wl][0](), WORKLOADS[wl][1]()[:40]
            got = e.eval_points_batch(pop, ds)
            want = oracle_points(pop, ds)
            for i in range(len(pop)):
                assert same_bits(got[i], want[i]), (wl, ppt, ppw, i)


def check_mse(got, m64, num_samples):
    # the reference accumulates in f32: a sum of squared errors above f32::MAX
    # overflows there and the fitness becomes f32::MAX (evaluator.rs:172-173)
    bad = ~np.isfinite(m64) | (m64 * float(num_samples) > FMAX)
    assert np.array_equal(got[bad], np.full(bad.sum(), FMAX, f32))
    ok = ~bad
    rel = np.abs(got[ok].astype(np.float64) - m64[ok]) / np.maximum(np.abs(m64[ok]), 1e-30)
    assert (rel <= 1e-6).all(), rel.max()


@pytest.mark.parametrize("kernel", [N.KERNEL_PLAIN, N.KERNEL_AUTO])
@pytest.mark.parametrize("wl", sorted(WORKLOADS))
def test_mse_within_1e6_of_fp64_oracle(engine, wl, kernel):
    ds, pop = WORKLOADS[wl][0](), WORKLOADS[wl][1]()
    got = engine.compute_mse_batch(pop, ds, kernel=kernel)
    m64, _ = O.mse_batch(I.pack(pop), ds)
    check_mse(got, m64, ds.num_samples)


@pytest.mark.parametrize("name", sorted(PR.kat_cases().keys()))
def test_known_answer_targets_gpu(engine, name):
    p, ds, exact = PR.kat_cases()[name]
    pred = engine.eval_points(p, ds)[:ds.num_samples]
    m = engine.compute_mse(p, ds)
    if exact:
        assert np.array_equal(pred, ds.target_batches[:ds.num_samples])
        assert m == 0.0
    else:
        assert m <= 1e-10 * max(1.0, float(np.mean(ds.target_batches.astype(np.float64) ** 2)))
    assert same_bits(pred, O.eval_points(p, ds)[:ds.num_samples])


def test_single_op_programs(engine):
    ds = PR.op_dataset()
    for name, p in PR.single_op_programs().items():
        for k in (N.KERNEL_PLAIN, N.KERNEL_AUTO):
            got = engine.eval_points_batch([p], ds, kernel=k)[0]
            assert same_bits(got, O.eval_points(p, ds)), (name, k)


def test_edge_programs(engine):
    ds = Dataset.new(np.array([[1.5, -2.0, 0.0, 3.0]] * 13, f32) * np.arange(1, 14, dtype=f32)[:, None],
                     np.linspace(-1, 1, 13).astype(f32), [FLOAT] * 4)
    progs = [
        Program([]),                                                         # result 0
        Program([I.load_var(FLOAT, 1), I.load_const(FLOAT, 0)], [Scalar.float(3.0)]),  # stack_f[0], not top
        Program([I.word(2, 0), I.word(4, 1), I.load_var(FLOAT, 0)]),        # B/I loads are no-ops
        Program([I.load_var(FLOAT, 0), I.load_var(FLOAT, 1), I.op("MakeVec2")]),  # F[0] holds a consumed value
        Program([I.load_var(FLOAT, 3), I.load_const(FLOAT, 0), I.op("AddF")],  # stale: Vec2 constant as Float
                [Scalar(VEC2, (5.0, 6.0))]),
        Program([I.load_var(FLOAT, 0), I.load_var(FLOAT, 2), I.op("DivF")]),  # inf / nan
        Program([I.load_var(FLOAT, 0)] * 32 + [I.op("AddF")] * 31),           # 32 slots deep
        Program([I.load_var(FLOAT, 2), I.op("LnF"), I.op("SqrtF"), I.op("ExpF")]),
    ]
    want = oracle_points(progs, ds)
    for k in (N.KERNEL_PLAIN, N.KERNEL_AUTO):
        got = engine.eval_points_batch(progs, ds, kernel=k)
        for i in range(len(progs)):
            assert same_bits(got[i], want[i]), (k, i)
        m64, _ = O.mse_batch(I.pack(progs), ds)
        check_mse(engine.compute_mse_batch(progs, ds, kernel=k), m64, ds.num_samples)


def test_tiny_and_ragged_datasets(engine):
    pop = W.scalar_population(20, seed=31)
    for n in (1, 7, 8, 9, 4095, 4097, 10007):
        ds = W.scalar_dataset(n, seed=n)
        m64, _ = O.mse_batch(I.pack(pop), ds)
        for k in (N.KERNEL_PLAIN, N.KERNEL_AUTO):
            check_mse(engine.compute_mse_batch(pop, ds, kernel=k), m64, ds.num_samples)


def test_empty_population(engine):
    ds = W.scalar_dataset(64)
    assert engine.compute_mse_batch([], ds).shape == (0,)


def test_reference_drop_ins(engine):
    ds = W.lorentz_dataset(2000, seed=41)
    for p in W.lorentz_population(10, seed=42):
        m = engine.compute_mse(p, ds)
        m64 = O.mse_f64(p, ds)
        check_mse(np.array([m], f32), np.array([m64]), ds.num_samples)
        assert same_bits(engine.eval_points(p, ds), O.eval_points(p, ds))


def grad_ok(g, ref, mse, tol=1e-3, noise=0.0):
    """|g - ref| <= tol * scale + noise.  scale = max(|ref|_inf, 1e-4 sqrt(MSE)):
    a gradient far below the loss's own scale is rounding noise (e.g. the
    derivative of a cross product of parallel vectors), where relative error
    means nothing."""
    scale = max(float(np.abs(ref).max()), 1e-4 * float(np.sqrt(max(mse, 0.0))), 1e-12)
    return float(np.abs(g - ref).max()) <= tol * scale + noise


def fd_noise(p, ds, h=1e-3):
    """Noise and truncation estimate of the central difference: how far the
    estimates at steps h and 2h disagree (large where cancellation inside
    the program makes the f32 loss noisy in a parameter)."""
    return 2.0 * float(np.abs(O.grad_fd(p, ds, h) - O.grad_fd(p, ds, 2 * h)).max())


def components_ok(g, ref, l1, mse, noise=0.0):
    """Per component: |g_k - r_k| <= 1e-3 |r_k| + 1e-4 L_k + 1e-6 max_j L_j
    + 1e-7 sqrt(MSE) (+ noise_k), L_k the L1 scale of the sum behind
    component k (the sum of |2 diff dpred/dtheta_k| over points / n, from the
    oracle): 1.1e-3 relative where the per-point terms do not cancel, f32
    resolution where they do; a derivative the dual rules give as exactly
    zero in every point (a cross product of parallel vectors) is rounding
    noise of the loss's own scale in reverse mode (the last term)."""
    g, ref, l1 = (np.asarray(x, np.float64) for x in (g, ref, l1))
    floor = 1e-4 * l1 + 1e-6 * l1.max() + 1e-7 * np.sqrt(max(mse, 0.0)) + noise + 1e-30
    return bool((np.abs(g - ref) <= 1e-3 * np.abs(ref) + floor).all())


def test_gradient_vs_finite_differences_and_dual():
    ds = W.transform_dataset(3000, seed=51)
    pop = W.transform_population(60, seed=52)
    with Engine() as e:
        mse, grad = e.compute_mse_grad_batch(pop, ds)
    checked = 0
    for i, p in enumerate(pop):
        n = min(32, p.param_count())
        m64 = O.mse_f64(p, ds)
        check_mse(mse[i:i + 1], np.array([m64]), ds.num_samples)
        md, gd = O.mse_grad_dual(p, ds)
        if not (np.isfinite(gd).all() and md < 1e4):
            continue
        _, g64, l1 = O.grad_dual_f64(p, ds)
        fd, fd2 = O.grad_fd(p, ds, 1e-3), O.grad_fd(p, ds, 2e-3)
        assert components_ok(grad[i, :n], g64[:n], l1[:n], m64), (i, grad[i, :n], g64[:n])
        assert components_ok(grad[i, :n], gd[:n], l1[:n], m64), (i, grad[i, :n], gd[:n])
        assert components_ok(grad[i, :n], fd[:n], l1[:n], m64, noise=2 * np.abs(fd[:n] - fd2[:n])), \
            (i, grad[i, :n], fd[:n])
        assert np.all(grad[i, n:] == 0)
        checked += 1
    assert checked >= 25


def test_gradient_all_op_kinds():
    # every differentiable op, with constants as operands, against the dual restatement
    ds = PR.op_dataset(300, seed=3, scale=1.0)
    with Engine() as e:
        for name, p in PR.single_op_programs().items():
            if not p.constants:
                continue
            m, g = e.compute_mse_with_gradient(p, ds)
            md, gd = O.mse_grad_dual(p, ds)
            n = min(32, p.param_count())
            m64 = O.mse_f64(p, ds)
            if name in ("InverseM2", "InverseM3"):
                fd = O.grad_fd(p, ds, 1e-3)   # the reference's dual skips inverses
                assert grad_ok(g[:n], fd[:n], m64, noise=fd_noise(p, ds)), (name, g[:n], fd[:n])
                continue
            if not np.isfinite(gd[:n]).all():
                assert not np.isfinite(g[:n]).all(), name
                continue
            assert grad_ok(g[:n], gd[:n], m64), (name, g[:n], gd[:n])
            _, g64, l1 = O.grad_dual_f64(p, ds)
            assert components_ok(g[:n], g64[:n], l1[:n], m64), (name, g[:n], g64[:n])


def test_alone_and_in_the_mix_identical(engine):
    dsa, popa = WORKLOADS["lorentz"][0](), WORKLOADS["lorentz"][1]()
    dsb, popb = WORKLOADS["inverse"][0](), WORKLOADS["inverse"][1]()
    alone = engine.compute_mse_batch(popa, dsa)
    mix = engine.compute_mse_batch(popb[:30] + popa + popb[30:],
                                   datasets=[dsb] * 30 + [dsa] * len(popa) + [dsb] * (len(popb) - 30))
    assert np.array_equal(alone, mix[30:30 + len(popa)])


def test_gradient_alone_and_in_a_large_batch_identical(engine):
    """A large batch's register-adjoint items cover several 4096-point parts
    and a small batch's one part each; every part is summed on its own, so a
    program's MSE and gradient are the same bits either way."""
    ds = engine.upload(W.lorentz_dataset(100_000, seed=2))
    pop = W.lorentz_population(2048, seed=12)
    mse_all, g_all = engine.compute_mse_grad_batch(pop, ds)
    mse_sub, g_sub = engine.compute_mse_grad_batch(pop[100:116], ds)
    assert same_bits(mse_sub, mse_all[100:116])
    assert same_bits(g_sub, g_all[100:116])


def test_multi_dataset_batch(engine):
    sizes = [400, 1000, 2500, 7000]
    dss = [W.inverse_dataset(n, seed=60 + i) for i, n in enumerate(sizes)]
    pop = W.inverse_population(80, seed=65)
    which = [dss[i % len(dss)] for i in range(len(pop))]
    got = engine.compute_mse_batch(pop, datasets=which)
    for i, p in enumerate(pop):
        check_mse(got[i:i + 1], np.array([O.mse_f64(p, which[i])]), which[i].num_samples)


def test_prepared_batch_graph_replay(engine):
    ds, pop = WORKLOADS["lorentz"][0](), WORKLOADS["lorentz"][1]()
    b = engine.prepare(pop, ds)
    try:
        outs = []
        for _ in range(3):
            b.run()
            outs.append(b.results())
        assert all(np.array_equal(outs[0], o) for o in outs)
        assert np.array_equal(outs[0], engine.compute_mse_batch(pop, ds))
        e_ms, t_ms = b.timing()
        assert t_ms > 0
        d = b.describe()
        assert d["programs"] == len(pop) and d["register_kernel_programs"] + d["slot_kernel_programs"] == len(pop)
        # the vector workload uses no unary Float op: its register launches
        # run on the instances built without those handlers
        assert all(g["no_unary"] for g in d["groups"] if g["kernel"] == "register")
    finally:
        b.close()


def test_unary_and_plain_programs_split_and_agree(engine):
    """A scalar population mixes programs with and without sin/cos/exp:
    they launch on different kernel instances, and every result matches the
    FP64 oracle as in the single-kind calls."""
    ds, pop = W.scalar_dataset(1000, seed=21), W.scalar_population(600, seed=22)
    uses = [any(I.OP_NAMES[w & 0xFF] in ("SinF", "CosF", "ExpF") for w in p.code) for p in pop]
    assert 0 < sum(uses) < len(pop)
    b = engine.prepare(pop, ds)
    try:
        b.run()
        got = b.results()
        flags = {g["no_unary"] for g in b.describe()["groups"] if g["kernel"] == "register"}
        assert flags == {True, False}
    finally:
        b.close()
    m64, _ = O.mse_batch(I.pack(pop), ds)
    fin = np.isfinite(m64) & (m64 < 1e30)
    np.testing.assert_allclose(got[fin], m64[fin], rtol=1e-6)
    alone = np.concatenate([engine.compute_mse_batch([p for p, u in zip(pop, uses) if u], ds),
                            engine.compute_mse_batch([p for p, u in zip(pop, uses) if not u], ds)])
    order = [i for i, u in enumerate(uses) if u] + [i for i, u in enumerate(uses) if not u]
    np.testing.assert_array_equal(alone, got[order])


def test_dataset_handles(engine):
    ds = W.scalar_dataset(100)
    d = engine.upload(ds)
    b = engine.prepare(W.scalar_population(4), d)
    with pytest.raises(N.RsrError) as ei:
        d.release()          # referenced by a prepared batch
    assert ei.value.code == N.RSR_EBUSY
    b.close()
    d.release()
    with pytest.raises(N.RsrError):
        engine.compute_mse_batch(W.scalar_population(2), d)


def test_full_size_vector_workload_properties():
    # 4096 programs x 100k points: plain and batched kernels agree within
    # 1e-6, a sample agrees with the FP64 oracle
    ds = W.lorentz_dataset(100_000)
    pop = W.lorentz_population(4096)
    with Engine() as e:
        fast = e.compute_mse_batch(pop, ds, kernel=N.KERNEL_AUTO)
        plain = e.compute_mse_batch(pop, ds, kernel=N.KERNEL_PLAIN)
    finite = fast < FMAX
    assert np.array_equal(finite, plain < FMAX)
    rel = np.abs(fast[finite].astype(np.float64) - plain[finite]) / np.maximum(plain[finite], 1e-30)
    assert rel.max() <= 2e-6
    idx = np.arange(0, 4096, 64)
    m64, _ = O.mse_batch(I.pack([pop[i] for i in idx]), ds)
    check_mse(fast[idx], m64, ds.num_samples)


@pytest.mark.parametrize("wl", ["scalar", "lorentz", "transform", "inverse"])
def test_register_and_slot_adjoints_agree(wl):
    """Gradients of the register adjoint (the default where a program fits
    it) against the slot-file adjoint (RSR_OPT_SLOT_ADJOINT): both reverse
    sweeps of the same programs, within 1e-3 relative per component plus
    f32 resolution against the gradient's scale; MSEs within 1e-6."""
    ds, pop = WORKLOADS[wl][0](), WORKLOADS[wl][1]()
    with Engine() as e, Engine(flags=N.OPT_SLOT_ADJOINT) as s:
        m1, g1 = e.compute_mse_grad_batch(pop, ds)
        m2, g2 = s.compute_mse_grad_batch(pop, ds)
        b = e.prepare(pop, ds, gradient=True)
        kinds = {g["kernel"] for g in b.describe()["groups"]}
        b.close()
    assert "register_adjoint" in kinds, kinds
    fin = (m2 < FMAX) & np.isfinite(g2).all(1) & np.isfinite(g1).all(1)
    assert np.array_equal(m1 < FMAX, m2 < FMAX)
    np.testing.assert_allclose(m1[fin], m2[fin], rtol=1e-6)
    for i in np.nonzero(fin)[0]:
        n = min(32, pop[i].param_count())
        if n == 0:
            continue
        scale = np.abs(g2[i, :n]).max()
        assert (np.abs(g1[i, :n] - g2[i, :n]) <= 1e-3 * np.abs(g2[i, :n]) + 1e-5 * scale + 1e-30).all(), \
            (wl, i, g1[i, :n], g2[i, :n])
