"""rsr_compute_mse_noalloc through the C ABI.

Its callers cannot allocate device memory per call: a serving process whose
device memory is all handed to a fixed pool (a cudaMalloc there fails), or a
host thread that shares the GPU with running streams (a cudaFree would
synchronise the whole device).  The tests check its MSE against the FP64
oracle and against rsr_compute_mse on two calls in a row, that calls after
the first leave the device's free memory unchanged, and that inputs beyond
its stated limits are refused.

Named so that pytest collects it last; it passes alone and after the rest of
the suite (the static scratch array is set up by whichever call comes first).
"""
import ctypes as C

import numpy as np
import pytest

from oracle import binding as O
from rsr_b200 import _native as N
from rsr_b200 import isa as I
from rsr_b200 import workloads as W
from rsr_b200.evaluator import Engine, _as_program
from rsr_b200.isa import FLOAT, MAT2, MAT3, VEC3, Program, Scalar

from programs import kat_cases

FMAX = float(np.finfo(np.float32).max)
MSE_RTOL = 1e-6          # MSE bar of the engine against the FP64 oracle
MAX_POINTS = 16_777_216  # the entry point's dataset limit


def _deep_program(m3: int, m2: int = 0, v3: int = 0) -> Program:
    """Sums of m3 Mat3, m2 Mat2 and v3 Vec3 constants, all pushed before the
    first add, so the slot file is deep enough to force fewer points per lane
    (more than 220 slots: 2 points per lane; more than 440: 1)."""
    consts = [Scalar(MAT3, tuple(0.1 * (i + 1) for i in range(9)))]
    code = [I.load_const(MAT3, 0)] * m3 + [I.op("AddM3")] * (m3 - 1) + [I.op("TraceM3")]
    if m2:
        consts.append(Scalar(MAT2, (0.5, -0.25, 0.125, 1.0)))
        code += [I.load_const(MAT2, 1)] * m2 + [I.op("AddM2")] * (m2 - 1) + [I.op("TraceM2"), I.op("AddF")]
    if v3:
        consts.append(Scalar(VEC3, (0.3, -0.2, 0.7)))
        code += [I.load_const(VEC3, len(consts) - 1)] * v3 + [I.op("AddV3")] * (v3 - 1) + [I.op("NormV3"),
                                                                                         I.op("AddF")]
    code += [I.load_var(FLOAT, 0), I.op("MulF")]
    return Program(code, consts)


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
    out.append(("deep_p2", _deep_program(25), sds))           # 226 slots: 2 points per lane
    out.append(("deep_p1", _deep_program(32, 32, 10), sds))   # 449 slots: 1 point per lane
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


def _oracle_ok(got, p, ds):
    """MSE within 1e-6 of the FP64 oracle, or f32::MAX where the reference's
    f32 accumulation overflows or the result is not finite."""
    m64 = O.mse_f64(p, ds)
    if not np.isfinite(m64) or m64 * ds.num_samples > FMAX:
        return got == FMAX
    return abs(got - m64) <= MSE_RTOL * abs(m64) + 1e-30


def _free_bytes() -> int:
    from cuda.bindings import runtime as rt
    err, free, _total = rt.cudaMemGetInfo()
    assert err == rt.cudaError_t.cudaSuccess, err
    return int(free)


@pytest.fixture(scope="module")
def eng():
    e = Engine()
    yield e
    e.close()


@pytest.mark.gpu
def test_noalloc_matches_oracle_and_compute_mse(eng):
    bad = []
    for name, p, ds in _cases():
        d = eng.upload(ds)
        want = eng.compute_mse(p, d)
        for call in range(2):  # two calls in a row reuse the scratch array
            rc, got = _noalloc(eng, p, d)
            assert rc == N.RSR_OK, (name, N.lib().rsr_last_error())
            if not _oracle_ok(got, p, ds):
                bad.append(("oracle", name, call, got, O.mse_f64(p, ds)))
            if not _same(got, want):
                bad.append(("compute_mse", name, call, got, want))
    assert not bad, bad[:5]


@pytest.mark.gpu
def test_noalloc_allocates_nothing_after_the_first_call(eng):
    sds = W.scalar_dataset(50_000, seed=77)
    lds = W.lorentz_dataset(30_000, seed=78)
    progs = [(W.scalar_population(1, seed=79)[0], eng.upload(sds)),     # 4 points per lane
             (W.lorentz_population(1, seed=80)[0], eng.upload(lds)),
             (_deep_program(25), eng.upload(sds)),                      # 2 points per lane
             (_deep_program(32, 32, 10), eng.upload(sds))]              # 1 point per lane
    first = []
    for p, d in progs:  # the first call on the device sets up; each variant runs once
        rc, m = _noalloc(eng, p, d)
        assert rc == N.RSR_OK, N.lib().rsr_last_error()
        first.append(m)
    free0 = _free_bytes()
    for i in range(100):
        p, d = progs[i % len(progs)]
        rc, m = _noalloc(eng, p, d)
        assert rc == N.RSR_OK, N.lib().rsr_last_error()
        assert m == first[i % len(progs)], i
    assert _free_bytes() == free0


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
    assert rc == N.RSR_OK and _same(got, eng.compute_mse(p, d)) and _oracle_ok(got, p, ds)


@pytest.mark.gpu
def test_noalloc_rejects_dataset_over_the_point_limit(eng):
    n = MAX_POINTS + 8
    x = np.linspace(-1.0, 1.0, n, dtype=np.float32)[:, None]
    big, _ = eng.upload_rows(x, np.zeros(n, np.float32))
    p = Program([I.load_var(FLOAT, 0), I.op("SqrF")])
    rc, _ = _noalloc(eng, p, big)
    assert rc == N.RSR_EINVAL
    big.release()
    # exactly at the limit it runs
    n = MAX_POINTS
    x = np.full((n, 1), 0.5, np.float32)
    edge, _ = eng.upload_rows(x, np.zeros(n, np.float32))
    rc, got = _noalloc(eng, p, edge)
    assert rc == N.RSR_OK, N.lib().rsr_last_error()
    assert abs(got - 0.0625) <= MSE_RTOL * 0.0625
    edge.release()
