"""Regenerates tests/golden/golden.npz.

The reference (Rust, src/ + tests/) cannot be built or run in this image and
its tests hold no golden vectors, so the fixtures are built from the
reference's own test targets instead:

* kat_*: inputs drawn (seeded) from the ranges of tests/basic.rs and
  tests/linalg.rs and the targets those tests compute, in f32, in the tests'
  operation order (tests/programs.py restates each expression), together with
  the program that encodes the same expression;
* op_*: every operator applied to seeded inputs (zero vectors and singular
  matrices included), evaluated by the numpy restatement of the op kernels
  (tests/npvm.py, src/domains/*/eval.rs) -- a second, independent restatement
  against which the C oracle and the GPU are checked bit for bit.

Run: python tests/golden/make_golden.py
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))
sys.path.insert(0, str(HERE.parent))

import npvm  # noqa: E402
import programs as PR  # noqa: E402


def main():
    out = {}
    for name, (p, ds, exact) in PR.kat_cases().items():
        out[f"kat_{name}_X"] = ds.point_features()[:ds.num_samples]
        out[f"kat_{name}_y"] = ds.target_batches[:ds.num_samples]
        out[f"kat_{name}_code"] = p.code_array()
        out[f"kat_{name}_kinds"] = p.kinds()
        out[f"kat_{name}_params"] = p.flatten_params()
        out[f"kat_{name}_exact"] = np.array(exact)
    ds = PR.op_dataset()
    X = ds.point_features()
    out["op_X"] = X
    with np.errstate(all="ignore"):
        for name, p in PR.single_op_programs().items():
            out[f"op_{name}_code"] = p.code_array()
            out[f"op_{name}_kinds"] = p.kinds()
            out[f"op_{name}_params"] = p.flatten_params()
            out[f"op_{name}_pred"] = npvm.eval_points(p, X)
    np.savez_compressed(HERE / "golden.npz", **out)
    print(HERE / "golden.npz", len(out), "arrays")


if __name__ == "__main__":
    main()
