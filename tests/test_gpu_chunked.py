"""One-shot calls large enough to run in chunks.

A one-shot MSE (or MSE + gradient) call of 1024 programs or more is planned
and launched in chunks that double in size, on two streams, with the host
encoding a chunk while the device runs the ones before it.  Every program's
result must be the one the unchunked path (a prepared batch of the whole
population) gives, bit for bit, in the caller's order, and an invalid
program in a later chunk must be reported by its index in the caller's
population.
"""
import numpy as np
import pytest

from oracle import binding as B
from rsr_b200 import _native as N
from rsr_b200 import isa as I
from rsr_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _prepared(eng, pop, d=None, datasets=None, gradient=False):
    b = eng.prepare(pop, d, datasets=datasets, gradient=gradient)
    try:
        b.run()
        return b.results()
    finally:
        b.close()


@pytest.mark.parametrize("n", [1024, 1500, 3333])
def test_chunked_mse_equals_unchunked(engine, n):
    ds = W.lorentz_dataset(20_000, seed=5)
    pop = W.lorentz_population(n, seed=50 + n)
    d = engine.upload(ds)
    got = engine.compute_mse_batch(pop, d)
    want = _prepared(engine, pop, d)
    np.testing.assert_array_equal(got, want)
    m64, _ = B.mse_batch(I.pack(pop[:64]), ds)
    fin = np.isfinite(m64) & (m64 < 1e30)
    np.testing.assert_allclose(got[:64][fin], m64[fin], rtol=1e-5)


def test_chunked_gradient_equals_unchunked(engine):
    ds = W.scalar_dataset(2000, seed=6)
    pop = [p for p in W.scalar_population(1400, seed=61) if p.param_count() > 0][:1100]
    d = engine.upload(ds)
    mse, grad = engine.compute_mse_grad_batch(pop, d)
    want_mse, want_grad = _prepared(engine, pop, d, gradient=True)
    np.testing.assert_array_equal(mse, want_mse)
    np.testing.assert_array_equal(grad, want_grad)


def test_chunked_per_program_datasets(engine):
    sizes = W.uneven_sizes(6, hi=20_000, seed=8)
    dss = [engine.upload(W.inverse_dataset(n, seed=70 + i)) for i, n in enumerate(sizes)]
    pop = W.inverse_population(1200, seed=71)
    rng = np.random.default_rng(9)
    per = [dss[int(k)] for k in rng.integers(0, len(dss), len(pop))]
    got = engine.compute_mse_batch(pop, datasets=per)
    want = _prepared(engine, pop, datasets=per)
    np.testing.assert_array_equal(got, want)


def test_chunked_error_names_caller_index(engine):
    ds = W.lorentz_dataset(5_000, seed=5)
    pop = W.lorentz_population(2000, seed=77)
    bad = 1789  # inside the last chunk (256 + 512 + 1232)
    p = pop[bad]
    pop[bad] = I.Program([I.op("AddF")] + list(p.code), p.constants)  # stack underflow
    d = engine.upload(ds)
    with pytest.raises(N.RsrError, match=f"program {bad}:"):
        engine.compute_mse_batch(pop, d)
    # the context stays usable
    ok = engine.compute_mse_batch(pop[:1500], d)
    assert len(ok) == 1500
