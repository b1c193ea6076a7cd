"""The register adjoint's code (encoder.cpp AdjEmitter), run on the CPU by a
numpy emulator of its forward and reverse sweeps (tests/accvm.py): the
gradients it gives are the dual-number oracle's (evaluator.rs:177-388) on
random programs of every workload, within the per-component bound of the
GPU tests; programs with an inverse, whose dual rule in the reference is a
no-op, are held against central differences instead."""
import warnings

import numpy as np

import accvm
from oracle import binding as O
from rsr_b200 import evaluator as E
from rsr_b200 import isa as I
from rsr_b200 import workloads as W

CASES = [("scalar", lambda: W.scalar_dataset(300, seed=3), lambda: W.scalar_population(40, seed=4)),
         ("vector", lambda: W.lorentz_dataset(240, seed=5), lambda: W.lorentz_population(40, seed=6)),
         ("matrix", lambda: W.transform_dataset(240, seed=7), lambda: W.transform_population(40, seed=8)),
         ("uneven", lambda: W.inverse_dataset(240, seed=9), lambda: W.inverse_population(40, seed=10))]


def test_register_adjoint_code_gives_the_dual_gradients():
    checked = {}
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)  # random programs divide by zero
        for name, dsf, popf in CASES:
            ds, pop = dsf(), popf()
            checked[name] = 0
            for i, p in enumerate(pop):
                n = min(32, p.param_count())
                if n == 0:
                    continue
                m64, gd, l1 = O.grad_dual_f64(p, ds)
                if not (np.isfinite(gd[:n]).all() and np.isfinite(m64) and m64 < 1e4):
                    continue
                m, g = accvm.run(p, ds)
                inverse = any(I.OP_NAMES[w & 255].startswith("Inverse") for w in p.code)
                # the reference's dual pass skips inverses in its value too
                m_ref = O.mse_f64(p, ds) if inverse else m64
                assert abs(m - m_ref) <= 1e-5 * max(m_ref, 1e-6), (name, i, m, m_ref)
                floor = 1e-4 * l1[:n] + 1e-6 * l1[:n].max() + 1e-12
                if inverse:
                    # an inverse near a singular matrix somewhere in the data
                    # makes central differences unstable: such programs are
                    # skipped, the others must agree within the noise
                    fd, fd4 = O.grad_fd(p, ds, 1e-3)[:n], O.grad_fd(p, ds, 1e-4)[:n]
                    if not (np.abs(fd - fd4) <= 1e-2 * np.abs(fd) + floor).all():
                        continue
                    noise = 2 * np.abs(fd - O.grad_fd(p, ds, 2e-3)[:n]) + 2 * np.abs(fd - fd4)
                    ok = np.abs(g[:n] - fd) <= 1e-3 * np.abs(fd) + floor + noise
                    checked["inverse"] = checked.get("inverse", 0) + 1
                else:
                    ok = np.abs(g[:n] - gd[:n]) <= 1e-3 * np.abs(gd[:n]) + floor
                assert ok.all(), (name, i, g[:n], gd[:n])
                checked[name] += 1
    assert all(checked[name] >= 10 for name, _, _ in CASES) and checked.get("inverse", 0) >= 3, checked


def test_accumulator_form_mse_matches_the_oracle():
    """The register kernel's code (accumulator form, form 1): loads fused
    into unary ops and PUSHes.  Emulated on the CPU, every program's MSE
    agrees with the FP64 oracle, and the fused forms occur."""
    unary = fused = 0
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        for name, dsf, popf in CASES:
            ds, pop = dsf(), popf()
            n = 0
            for p in pop:
                words = E.encoding(p, ds.num_features, 1)
                if len(words) == 0:
                    continue
                for w in (int(x) for x in words):
                    t = accvm.block(w & 255)
                    if (w & 255) - accvm.BASE[t] == 2:
                        fused += ((w >> 12) & 7) != 0
                    elif accvm._is_unary(t, (w & 255) - accvm.BASE[t]):
                        unary += ((w >> 20) & 3) != 0
                m = accvm.run(p, ds, form=1)
                m64 = O.mse_f64(p, ds)
                if not (np.isfinite(m64) and m64 < 1e30):
                    continue
                assert abs(m - m64) <= 1e-5 * max(abs(m64), 1e-6), (name, m, m64)
                n += 1
            assert n >= 10, name
    assert unary > 0 and fused > 0, (unary, fused)


def test_adjoint_stacks_can_share_the_forward_slots():
    """The kernel keeps a spilled value's adjoint in the value's own stack
    slot.  That is sound when the one micro-op that pops a value is the last
    reader of its forward slot and the first writer of its adjoint: the
    emulator with shared slots gives bit for bit the gradients of the one
    with separate adjoint stacks."""
    n = 0
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        for name, dsf, popf in CASES:
            ds, pop = dsf(), popf()
            for p in pop:
                try:
                    m1, g1 = accvm.run(p, ds, alias_stacks=True)
                except ValueError:  # no register adjoint form
                    continue
                m2, g2 = accvm.run(p, ds, alias_stacks=False)
                assert np.array_equal(g1, g2, equal_nan=True) and (m1 == m2 or (np.isnan(m1) and np.isnan(m2))), name
                n += 1
    assert n >= 100


def test_register_adjoint_code_layout():
    """Header words, one reverse entry per non-TAPE forward entry, PUSH
    slots all distinct, tape slots inside the reported tape."""
    for p in W.lorentz_population(30, seed=11) + W.inverse_population(30, seed=12):
        enc = E.encoding(p, 9, 5)
        if enc[0] == 0xFFFFFFFF:
            continue
        tape, depth, code = int(enc[1]), [int(x) for x in enc[2:7]], enc[7:]
        nf, nr = int(code[0]), int(code[1])
        assert len(code) == 2 + 2 * nf + 2 * nr
        fwd = [int(w) for w in code[2:2 + 2 * nf:2]]
        stores = [int(w) for w in code[3:3 + 2 * nf:2]]
        tapes = [w for w in fwd if (w & 255) in accvm.TAPE]
        assert nr == nf - len(tapes)
        assert all((w >> 8) < tape for w in tapes)
        # stores an entry carries: tape slots inside the tape, none on TAPE entries
        for w, st in zip(fwd, stores):
            for s in (st & 0xFFFF, st >> 16):
                assert s == 0xFFFF or (s < tape and (w & 255) not in accvm.TAPE)
        # reverse references: tape slots inside the tape, or features /
        # constants (values the reverse sweep reads again instead of a tape)
        r0 = 2 + 2 * nf
        refs = [r for i in range(nr) for r in (int(code[r0 + 1 + 2 * i]) & 0xFFFF, int(code[r0 + 1 + 2 * i]) >> 16)]
        assert all(r < tape or r & 0xC000 for r in refs if r)
        pushes = {}
        for w in fwd:
            t = accvm.block(w & 255)
            if (w & 255) - accvm.BASE[t] == 2:
                pushes.setdefault(t, []).append((w >> 8) & 15)  # the slot; a fused load sits above it
        for t, slots in pushes.items():
            assert sorted(slots) == list(range(len(slots))) and len(slots) == depth[t]
