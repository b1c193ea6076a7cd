"""Serving loop: continuous batching, memory admission, failures on the host.

The determinism test is the one the serving design promises: each job's
result is the same alone and in the mix (MSE within the engine's 1e-6
relative tolerance, gradients within 1e-4 of their scale, fits identical).
"""
import threading

import numpy as np
import pytest

from rsr_b200 import _native as N
from rsr_b200 import isa as I
from rsr_b200 import workloads as W
from rsr_b200.evaluator import Engine
from rsr_b200.isa import Program
from rsr_b200.serving import Server

pytestmark = pytest.mark.gpu

MSE_RTOL = 1e-6


def _close_mse(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    big = (a >= 3.0e38) | (b >= 3.0e38)
    assert np.array_equal(a >= 3.0e38, b >= 3.0e38)
    np.testing.assert_allclose(a[~big], b[~big], rtol=MSE_RTOL, atol=1e-30)


@pytest.fixture(scope="module")
def setup():
    eng = Engine()
    data = {
        "scalar": W.scalar_dataset(400, seed=81),
        "lorentz": W.lorentz_dataset(30_000, seed=82),
        "inverse": W.inverse_dataset(5_000, seed=83),
    }
    pops = {
        "scalar": W.scalar_population(256, seed=84),
        "lorentz": W.lorentz_population(300, seed=85),
        "inverse": W.inverse_population(200, seed=86),
    }
    dev = {k: eng.upload(v) for k, v in data.items()}
    yield eng, data, pops, dev
    eng.close()


def _jobs(pops):
    rng = np.random.default_rng(87)
    jobs = []
    for i in range(24):
        name = ["scalar", "lorentz", "inverse"][i % 3]
        pop = pops[name]
        lo = int(rng.integers(0, len(pop) - 40))
        hi = lo + int(rng.integers(16, 40))
        kind = ["mse", "grad", "mse", "fit"][i % 4]
        jobs.append((name, pop[lo:hi], kind))
    return jobs


def _alone(eng, dev, name, progs, kind):
    if kind == "mse":
        return {"mse": eng.compute_mse_batch(progs, dev[name])}
    if kind == "grad":
        m, g = eng.compute_mse_grad_batch(progs, dev[name])
        return {"mse": m, "grad": g}
    p, m, _ = eng.fit_lbfgs(progs, dev[name], 10)
    return {"mse": m, "params": p}


def _compare(kind, got, want):
    _close_mse(got["mse"], want["mse"])
    if kind == "grad":
        g, w = np.asarray(got["grad"], np.float64), np.asarray(want["grad"], np.float64)
        ok = np.asarray(want["mse"]) < 3.0e38
        g, w = g[ok], w[ok]
        assert np.array_equal(np.isnan(g), np.isnan(w)) and np.array_equal(np.isinf(g), np.isinf(w))
        fin = np.isfinite(w)
        scale = np.maximum(np.where(fin, np.abs(w), 0).max(axis=1, keepdims=True), 1e-12)
        assert np.all(np.abs(np.where(fin, g - w, 0)) <= 1e-4 * scale)
    if kind == "fit":
        np.testing.assert_array_equal(np.asarray(got["params"]), np.asarray(want["params"]))


def test_alone_equals_mix(setup):
    eng, data, pops, dev = setup
    jobs = _jobs(pops)
    alone = [_alone(eng, dev, n, p, k) for n, p, k in jobs]
    results = [None] * len(jobs)
    with Server(eng, slots=4) as srv:
        def island(idx):
            for i in idx:
                n, p, k = jobs[i]
                t = srv.submit(p, dev[n], kind=k, fit_iterations=10)
                results[i] = srv.wait(t)
        threads = [threading.Thread(target=island, args=(list(range(s, len(jobs), 8)),)) for s in range(8)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        st = srv.stats()
    assert st["completed"] == len(jobs) and st["failed"] == 0
    for (n, p, k), got, want in zip(jobs, results, alone):
        _compare(k, got, want)


def test_continuous_batching_merges(setup):
    eng, data, pops, dev = setup
    with Server(eng, slots=1) as srv:
        # a long job occupies the only slot; the small ones queue behind it
        big = srv.submit(pops["lorentz"], dev["lorentz"], kind="grad")
        small = [srv.submit(pops["scalar"][i * 8:(i + 1) * 8], dev["scalar"]) for i in range(20)]
        srv.wait(big)
        infos = [srv.wait(t)["info"] for t in small]
        st = srv.stats()
    assert max(i["batch_jobs"] for i in infos) > 1
    assert st["launches"] < st["completed"]
    assert st["p99_ms"] >= st["p50_ms"] > 0


def test_merged_batch_isolates_bad_program(setup):
    eng, data, pops, dev = setup
    bad = Program([I.op("AddF")], [])  # stack underflow
    with Server(eng, slots=1) as srv:
        big = srv.submit(pops["lorentz"], dev["lorentz"], kind="grad")
        good1 = srv.submit(pops["scalar"][:10], dev["scalar"])
        broken = srv.submit([pops["scalar"][0], bad], dev["scalar"])
        good2 = srv.submit(pops["scalar"][10:20], dev["scalar"])
        srv.wait(big)
        m1 = srv.wait(good1)["mse"]
        with pytest.raises(N.RsrError) as e:
            srv.wait(broken)
        assert e.value.code == N.RSR_EPROGRAM
        m2 = srv.wait(good2)["mse"]
    _close_mse(m1, eng.compute_mse_batch(pops["scalar"][:10], dev["scalar"]))
    _close_mse(m2, eng.compute_mse_batch(pops["scalar"][10:20], dev["scalar"]))


def test_memory_admission(setup):
    eng, data, pops, dev = setup
    with Server(eng, slots=2, mem_budget_bytes=256 * 1024) as srv:
        with pytest.raises(N.RsrError) as e:
            srv.submit(pops["lorentz"], dev["lorentz"], kind="grad")
        assert e.value.code == N.RSR_ENOMEM
        t = srv.submit(pops["scalar"][:16], dev["scalar"])
        _close_mse(srv.wait(t)["mse"], eng.compute_mse_batch(pops["scalar"][:16], dev["scalar"]))
        assert srv.stats()["refused"] == 1


def test_cancel_queued_and_timeout(setup):
    eng, data, pops, dev = setup
    with Server(eng, slots=1) as srv:
        big = srv.submit(pops["lorentz"], dev["lorentz"], kind="fit", fit_iterations=10)
        queued = [srv.submit(pops["scalar"][:8], dev["scalar"]) for _ in range(4)]
        with pytest.raises(N.RsrError) as e:
            srv.wait(big, timeout=1e-6)
        assert e.value.code == N.RSR_ETIMEDOUT
        for t in queued:
            srv.cancel(t)
        n_cancelled = 0
        for t in queued:
            try:
                srv.wait(t)  # it had started before the cancel
            except N.RsrError as e:
                assert e.code == N.RSR_ECANCELED
                n_cancelled += 1
        srv.wait(big)
        assert n_cancelled >= 1 and srv.stats()["cancelled"] == n_cancelled


@pytest.mark.filterwarnings("ignore::pytest.PytestUnhandledThreadExceptionWarning")
def test_dataset_pinned_by_job_and_dead_submitter(setup):
    eng, data, pops, dev = setup
    ds = W.scalar_dataset(2000, seed=88)
    d = eng.upload(ds)
    with Server(eng, slots=1) as srv:
        big = srv.submit(pops["lorentz"], dev["lorentz"], kind="grad")
        holder = {}

        def island_that_dies():
            holder["t"] = srv.submit(pops["scalar"][:32], d)
            raise RuntimeError("island thread dies before waiting")

        th = threading.Thread(target=island_that_dies)
        th.start()
        th.join()
        t = holder["t"]
        # the dataset is referenced by the orphaned job
        if srv.poll(t) != "done":
            with pytest.raises(N.RsrError) as e:
                d.release()
            assert e.value.code == N.RSR_EBUSY
        srv.wait(big)
        # the other islands keep being served
        ok = srv.submit(pops["scalar"][:8], dev["scalar"])
        srv.wait(ok)
        for _ in range(1000):
            if srv.poll(t) == "done":
                break
            threading.Event().wait(0.01)
        assert srv.poll(t) == "done"
        srv.wait(t)
    d.release()


def _method(p):
    """optimize_individual_constants' choice (src/engine/optimize/mod.rs:24-58)."""
    ops = {w & 0xFF for w in p.code}
    if not ops & {I.OP["InverseM2"], I.OP["InverseM3"]}:
        return "lbfgs"
    return "cmaes" if any(c.kind in (I.VEC2, I.VEC3, I.MAT2, I.MAT3) for c in p.constants) else "nelder_mead"


def test_fit_auto_picks_the_reference_optimiser(setup):
    """A "fit_auto" job fits each program with the optimiser the reference
    would pick, and each group's results are exactly those of the batched
    driver called on that group alone."""
    eng, data, pops, dev = setup
    M = lambda i: I.load_var(I.MAT2, i)
    extra = [
        Program([M(0), I.op("InverseM2"), I.load_const(I.MAT2, 0), I.op("AddM2"), I.op("TraceM2")],
                [I.Scalar(I.MAT2, (0.5, -0.2, 0.1, 0.4))]),
        Program([M(4), I.load_const(I.VEC2, 0), I.op("MulM2V2"), I.op("NormV2"), M(0), I.op("InverseM2"),
                 I.op("DetM2"), I.op("AddF")], [I.Scalar(I.VEC2, (1.0, -1.0))]),
    ]
    progs = [p for p in pops["inverse"][:60] if p.param_count() > 0] + extra
    kinds = [_method(p) for p in progs]
    assert {"lbfgs", "nelder_mead", "cmaes"} <= set(kinds)
    iters, seed = 40, 4242
    srv = Server(eng, slots=2)
    try:
        out = srv.wait(srv.submit(progs, dev["inverse"], kind="fit_auto", fit_iterations=iters, seed=seed))
    finally:
        srv.close()
    pk = I.pack(progs)
    for method in ("lbfgs", "nelder_mead", "cmaes"):
        idx = [i for i, k in enumerate(kinds) if k == method]
        sub = [progs[i] for i in idx]
        if method == "lbfgs":
            p, m, _ = eng.fit_lbfgs(sub, dev["inverse"], 15)
        elif method == "nelder_mead":
            p, m, _ = eng.fit_nelder_mead(sub, dev["inverse"], iters)
        else:
            p, m, _ = eng.fit_cma_es(sub, dev["inverse"], max(iters // 16, 2), seed=seed)
        spk = I.pack(sub)
        for k, i in enumerate(idx):
            got = out["params"][pk.param_off[i]:pk.param_off[i + 1]]
            np.testing.assert_array_equal(got, p[spk.param_off[k]:spk.param_off[k + 1]], err_msg=f"{method} {i}")
            assert np.float32(out["mse"][i]) == np.float32(m[k]), (method, i)
