"""rsr_compute_mse_noalloc against rsr_compute_mse, through the C ABI.

Named so that pytest collects it last; it passes alone and after the rest of
the suite (the static scratch array is set up by whichever call comes first).
"""
import ctypes as C

import numpy as np
import pytest

from rsr_b200 import _native as N
from rsr_b200 import isa as I
from rsr_b200 import workloads as W
from rsr_b200.evaluator import Engine, _as_program
from rsr_b200.isa import FLOAT, Program, Scalar

from programs import kat_cases

FMAX = float(np.finfo(np.float32).max)
MSE_RTOL = 1e-6   # MSE bar of the engine against the FP64 oracle


def _cases():
    out = []
    for name, (p, ds, _exact) in kat_cases(300, seed=71).items():
        out.append((name, p, ds))
    lds = W.lorentz_dataset(20_000, seed=72)
    for i, p in enumerate(W.lorentz_population(24, seed=73)):
        out.append((f"lorentz{i}", p, lds))
    sds = W.scalar_dataset(5000, seed=74)
    for i, p in enumerate(W.scalar_population(16, seed=75)):
        out.append((f"scalar{i}", p, sds))
    # a constant load of the wrong kind leaves its slot unwritten (stale)
    stale = Program([I.load_const(FLOAT, 0), I.load_var(FLOAT, 0), I.op("AddF")],
                    [Scalar(I.VEC3, (1.0, 2.0, 3.0))])
    out.append(("stale", stale, sds))
    out.append(("empty", Program([], []), sds))
    return out


def _noalloc(eng, p, d):
    s, keep = _as_program(p)
    out = C.c_float()
    rc = N.lib().rsr_compute_mse_noalloc(eng.ctx, C.byref(s), d.handle, C.byref(out))
    return rc, float(out.value)


def _same(a, b):
    if a >= FMAX or b >= FMAX:
        return a == b
    return abs(a - b) <= MSE_RTOL * max(abs(a), abs(b)) + 1e-30


@pytest.fixture(scope="module")
def eng():
    e = Engine()
    yield e
    e.close()


@pytest.mark.gpu
def test_noalloc_matches_compute_mse(eng):
    bad = []
    for name, p, ds in _cases():
        d = eng.upload(ds)
        want = eng.compute_mse(p, d)
        for call in range(2):  # two calls in a row reuse the scratch array
            rc, got = _noalloc(eng, p, d)
            assert rc == N.RSR_OK, (name, N.lib().rsr_last_error())
            if not _same(got, want):
                bad.append((name, call, got, want))
    assert not bad, bad[:5]


@pytest.mark.gpu
def test_noalloc_rejects_oversize_program(eng):
    ds = W.scalar_dataset(100, seed=76)
    d = eng.upload(ds)
    code = [I.load_var(FLOAT, 0)] + [I.load_var(FLOAT, 0), I.op("AddF")] * 256  # 513 instructions
    rc, _ = _noalloc(eng, Program(code, []), d)
    assert rc == N.RSR_EINVAL
    # a rejected call leaves the entry point usable
    p = Program([I.load_var(FLOAT, 0), I.op("SinF")])
    rc, got = _noalloc(eng, p, d)
    assert rc == N.RSR_OK and _same(got, eng.compute_mse(p, d))
