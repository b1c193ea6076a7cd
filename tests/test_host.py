"""Host-side logic of the engine, no GPU needed: the C ABI library loads and
exports every symbol include/rsr_gpu.h declares, the ISA numbering agrees
across the Python mirror, the C oracle and the device header, and the
encoder validates and analyses programs (rsr_validate_program /
rsr_program_analyze touch no device)."""
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from rsr_b200 import _native as N
from rsr_b200 import evaluator as E
from rsr_b200 import isa as I
from rsr_b200 import workloads as W
from rsr_b200.dataset import Dataset
from rsr_b200.isa import FLOAT, VEC2, VEC3, Program, Scalar

ROOT = Path(__file__).resolve().parent.parent
f32 = np.float32


def test_library_exports_every_declared_symbol():
    header = (ROOT / "include" / "rsr_gpu.h").read_text()
    declared = set(re.findall(r"RSR_API [^;]*?\b(rsr_\w+)\(", header))
    assert len(declared) >= 26
    out = subprocess.run(["nm", "-D", "--defined-only", str(N.LIB_PATH)], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if l.strip()}
    assert declared <= exported, sorted(declared - exported)
    L = N.lib()  # loads without a GPU
    for s in declared:
        assert hasattr(L, s)
    assert set(N.exported_symbols()) <= declared


_C_SCALAR = {"int": "c_int", "uint32_t": "u32", "int32_t": "i32", "uint64_t": "u64", "double": "f64",
             "float": "f32", "size_t": "usize", "char": "c_char", "uint8_t": "u8", "rsr_dataset": "RsrDataset"}


def _rust_type(c: str) -> str:
    """The Rust spelling of a C parameter or field type of the header."""
    c = " ".join(c.replace("*", " * ").split())
    stars = c.count("*")
    base = c.replace("*", "").replace("const", "").strip()
    rust = _C_SCALAR.get(base) or "Rsr" + "".join(w.capitalize() for w in base[len("rsr_"):].split("_"))
    if stars == 0:
        return rust
    first = "*const " if c.startswith("const") else "*mut "
    return first + "*mut " * (stars - 1) + rust


def _c_functions():
    header = (ROOT / "include" / "rsr_gpu.h").read_text()
    out = {}
    for ret, name, args in re.findall(r"RSR_API ([^;]*?)\b(rsr_\w+)\(([^;]*?)\);", header, re.S):
        params = [] if args.strip() == "void" else [" ".join(a.split()) for a in args.split(",")]
        types = []
        for a in params:
            m = re.match(r"(.*?)(\w+)$", a)
            types.append(_rust_type(m.group(1)))
        r = " ".join(ret.split())
        out[name] = (types, None if r == "void" else _rust_type(r))
    return out


def _rust_functions():
    text = (ROOT / "integration" / "rust" / "gpu.rs").read_text()
    out = {}
    for name, args, ret in re.findall(r"pub fn (rsr_\w+)\(([^)]*)\)\s*(?:->\s*([^;{]+?))?\s*;", text, re.S):
        types = [" ".join(a.split(":", 1)[1].split()) for a in args.split(",") if a.strip()]
        out[name] = (types, " ".join(ret.split()) if ret else None)
    return out


def test_rust_bindings_cover_the_header():
    """The Rust binding a maintainer adds (integration/rust/gpu.rs) declares
    every entry point of the header under the same name, with the same
    parameter and return types, and nothing the header lacks."""
    c, rust = _c_functions(), _rust_functions()
    assert set(rust) == set(c), (sorted(set(c) - set(rust)), sorted(set(rust) - set(c)))
    for name in c:
        assert rust[name] == c[name], (name, rust[name], c[name])


def test_rust_structs_mirror_the_header():
    """Every struct of the header has a #[repr(C)] Rust mirror with the same
    fields, in order, of the same types."""
    header = (ROOT / "include" / "rsr_gpu.h").read_text()
    text = (ROOT / "integration" / "rust" / "gpu.rs").read_text()
    structs = re.findall(r"typedef struct (rsr_\w+) \{(.*?)\} \1;", header, re.S)
    assert len(structs) >= 9
    for cname, body in structs:
        fields = []
        for decl in re.sub(r"/\*.*?\*/", "", body, flags=re.S).split(";"):
            decl = " ".join(decl.split())
            if not decl:
                continue
            m = re.match(r"((?:const )?\w+ \**)\s*(.*)$", decl)
            ctype, names = m.group(1), m.group(2)
            for n in names.split(","):
                n = n.strip()
                arr = re.match(r"(\w+)\[(\d+)\]", n)
                if arr:
                    fields.append((arr.group(1), f"[{_rust_type(ctype)}; {arr.group(2)}]"))
                else:
                    stars = n.count("*")
                    fields.append((n.strip("* "), _rust_type(ctype + "*" * stars)))
        rname = _rust_type(cname)
        m = re.search(r"#\[repr\(C\)\]\s*pub struct " + rname + r" \{(.*?)\}", text, re.S)
        assert m, rname
        rfields = [(f.split(":")[0].replace("pub", "").strip(), " ".join(f.split(":", 1)[1].split()))
                   for f in m.group(1).split(",") if ":" in f]
        assert rfields == fields, (cname, rfields, fields)


def test_opcode_numbering_matches_device_header():
    text = (ROOT / "rsr_b200" / "csrc" / "uops.h").read_text()
    body = text[text.index("enum Opcode"):text.index("N_OPCODES,")]
    names = re.findall(r"\b([A-Z][A-Z0-9_]+)\b", body.split("{", 1)[1])
    assert [n.replace("_", "") for n in names] == [n.upper() for n in I.OP_NAMES]


def test_version_and_errors():
    assert b"sm_100a" in N.lib().rsr_version()
    with pytest.raises(N.RsrError) as ei:
        E.validate(Program([I.op("AddF")]), 1)
    assert ei.value.code == N.RSR_EPROGRAM and "underflow" in str(ei.value)


@pytest.mark.parametrize("prog,nf,code,msg", [
    (Program([I.op("AddF")]), 1, N.RSR_EPROGRAM, "underflow"),
    (Program([I.load_var(FLOAT, 3)]), 2, N.RSR_EPROGRAM, "feature offset"),
    (Program([I.load_var(VEC3, 0)]), 2, N.RSR_EPROGRAM, "feature offset"),
    (Program([I.load_const(FLOAT, 0)]), 1, N.RSR_EPROGRAM, "constant index"),
    (Program([I.load_var(FLOAT, 0)] * 33), 1, N.RSR_EPROGRAM, "32 values"),
    (Program([250]), 1, N.RSR_EPROGRAM, "unknown opcode"),
])
def test_validation_errors(prog, nf, code, msg):
    with pytest.raises(N.RsrError) as ei:
        E.validate(prog, nf)
    assert ei.value.code == code and msg in str(ei.value)


def test_validation_accepts_edge_programs():
    E.validate(Program([I.load_var(FLOAT, 0)] * 32), 1)
    E.validate(Program([]), 1)                                            # empty program: result 0
    E.validate(Program([I.word(2, 0), I.word(4, 0), I.load_var(FLOAT, 0)]), 1)  # B/I loads are no-ops
    # LoadConstF on a Vec2 constant: slot left unwritten, not an error
    E.validate(Program([I.load_const(FLOAT, 0)], [Scalar(VEC2, (1.0, 2.0))]), 1)


def test_param_count_mismatch_rejected():
    p = Program([I.load_const(FLOAT, 0)], [Scalar.float(1.0)])
    s, keep = E._as_program(p)
    s.n_params = 2
    import ctypes as C
    rc = N.lib().rsr_validate_program(C.byref(s), 1)
    assert rc == N.RSR_EPROGRAM


def test_reordering_reduces_depth_and_keeps_semantics_profile():
    # right-deep chain x + (x + (x + ...)) needs one F slot per level in the
    # reference's order, 2 after reordering with fused leaves
    code = [I.load_var(FLOAT, 0)] * 12 + [I.op("AddF")] * 11
    info = E.analyze(Program(code), 1)
    assert info["depth_ref"][0] == 12
    assert info["depth_fast"][0] <= 2 and info["fast_profile"] == 0


def test_analysis_of_workloads():
    for fn, nf, prof in [(W.scalar_population, 1, {0}), (W.lorentz_population, 9, {0, 1}),
                         (W.transform_population, 15, {0, 1, 3}), (W.inverse_population, 8, {0, 2, -1})]:
        infos = [E.analyze(p, nf) for p in fn(200)]
        profiles = {i["fast_profile"] for i in infos}
        assert profiles <= prof, (fn.__name__, profiles)
        assert np.mean([i["fast_profile"] >= 0 for i in infos]) > 0.9


def test_flop_count_matches_python_table():
    for p in W.lorentz_population(50):
        assert E.analyze(p, 9)["flops_per_point"] == p.flops_per_point()


def test_dataset_layout_and_padding():
    x = np.arange(30, dtype=f32).reshape(10, 3)
    y = np.arange(10, dtype=f32)
    ds = Dataset.new(x, y, [FLOAT, VEC2])
    assert ds.num_batches == 2 and ds.num_samples == 10 and ds.num_features == 3
    ff = ds.feature_flat.reshape(2, 3, 8)
    assert np.array_equal(ff[0, 1], x[:8, 1]) and np.array_equal(ff[1, 2, :2], x[8:, 2])
    assert np.all(ff[1, :, 2:] == 0) and np.all(ds.target_batches[10:] == 0)
    assert np.array_equal(ds.point_features()[:10], x)


def test_dataset_normalisation_matches_reference_formula():
    rng = np.random.default_rng(0)
    x = rng.normal(3, 2, (50, 2)).astype(f32)
    y = rng.normal(-1, 4, 50).astype(f32)
    ds = Dataset.new(x, y, [FLOAT, FLOAT], normalize=True)
    # sequential f32 sums (dataset.rs:63-94)
    s = f32(0)
    for v in x[:, 0]:
        s = f32(s + v)
    mean = f32(s / f32(50))
    assert ds.feature_means[0] == mean
    assert ds.variable_registry() == [(FLOAT, 0), (FLOAT, 1)]
    assert abs(float(np.mean(ds.target_batches[:50]))) < 1e-5


def test_generator_is_seeded_and_in_range():
    a = W.lorentz_population(20, seed=3)
    b = W.lorentz_population(20, seed=3)
    assert [p.code for p in a] == [p.code for p in b]
    assert all(4 <= len(p.code) <= 48 for p in a)
    t = W.transform_population(50, seed=4)
    assert all(1 <= len(p.constants) <= 8 and 8 <= len(p.code) <= 40 for p in t)


def test_noalloc_slot_encoder_matches_encode_program():
    """rsr_compute_mse_noalloc encodes the slot form into fixed arrays by its
    own pass; it must give the words, slot count and flags of the engine's
    encoder on every program it accepts: random programs of every workload,
    stale constant loads, B/I loads, empty programs and 32-deep stacks."""
    pops = [(W.scalar_population(150, seed=61), 1), (W.lorentz_population(150, seed=62), 9),
            (W.transform_population(100, seed=63), 15), (W.inverse_population(150, seed=64), 8)]
    edge = [Program([]), Program([I.word(2, 0), I.word(4, 1), I.load_var(FLOAT, 0)]),
            Program([I.load_const(FLOAT, 0), I.load_var(FLOAT, 0), I.op("AddF")], [Scalar(VEC3, (1.0, 2.0, 3.0))]),
            Program([I.load_var(FLOAT, 1), I.load_const(FLOAT, 0)], [Scalar(VEC2, (5.0, 6.0))]),
            Program([I.load_var(FLOAT, 0)] * 32 + [I.op("AddF")] * 31),
            Program([I.load_var(FLOAT, 0), I.load_var(FLOAT, 1), I.op("MakeVec2")])]
    pops.append((edge, 4))
    checked = 0
    for pop, nf in pops:
        for p in pop:
            a = E.encoding(p, nf, 3)
            b = E.encoding(p, nf, 4)
            np.testing.assert_array_equal(a, b)
            checked += 1
    assert checked >= 550
    # beyond the fixed arrays' limit the fixed encoder refuses
    long = Program([I.load_var(FLOAT, 0)] + [I.load_var(FLOAT, 0), I.op("AddF")] * 256)
    with pytest.raises(N.RsrError) as ei:
        E.encoding(long, 1, 4)
    assert ei.value.code == N.RSR_EINVAL
