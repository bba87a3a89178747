"""Regenerates the golden fixtures in tests/golden/ from the reference's own CPU solver.

    make -C oracle ref && python tests/golden/make_golden.py

Runs oracle/_ref/feat_oracle (the reference built from its sources by oracle/Makefile) and packs
its dumps into compressed .npz files: every level's A, P, R, unit filter and vertex coordinates,
the fine right-hand side, the V-cycle applied to it, every PCG iterate, the recursive defect
norms, the final solution, and the reference's summary line.  Indices are stored as u32 to keep
the files small (loaders widen them back to the reference's u64).
"""
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "feat3.doxytest_b200"))

import oracle as O  # noqa: E402
from featb200 import assembly as AS  # noqa: E402


def pack(name, out_dir, summary, extra=None):
    arrays = {}
    for f in sorted(os.listdir(out_dir)):
        if not f.endswith(".npy"):
            continue
        a = np.load(os.path.join(out_dir, f))
        if a.dtype == np.uint64 and a.size and a.max() < 2 ** 32:
            a = a.astype(np.uint32)
        arrays[f[:-4]] = a
    arrays["summary_json"] = np.frombuffer(json.dumps(summary).encode(), dtype=np.uint8)
    if extra:
        arrays.update(extra)
    np.savez_compressed(os.path.join(HERE, name), **arrays)
    print(name, summary)


def case(name, **kw):
    with tempfile.TemporaryDirectory() as d:
        extra = {}
        if kw.get("gauss") is not None:
            p = os.path.join(d, "gauss.txt")
            AS.write_params(p, gauss=kw["gauss"])
            kw["params"] = p
            extra["gauss_params"] = kw["gauss"]
        if kw.get("field") is not None:
            p = os.path.join(d, "field.txt")
            AS.write_params(p, field=kw["field"])
            kw["kappa"] = p
            kx, ky, xi, eta, s = kw["field"]
            extra.update(field_kx=kx, field_ky=ky, field_xi=xi, field_eta=eta, field_s=np.array([s]))
        kw.pop("gauss", None)
        kw.pop("field", None)
        summary = O.feat_solve(d, dump_levels=True, vcycle=True, **kw)
        # dump every iterate up to convergence
        summary = O.feat_solve(d, dump_levels=True, vcycle=True, iterates=summary["iters"], **kw)
        pack(name, d, summary, extra)


def fd_case():
    import subprocess
    with tempfile.TemporaryDirectory() as d:
        res = subprocess.run([O.FEAT_BIN, "fd", "17", "2", d], check=True, capture_output=True, text=True)
        pack("fd17.npz", d, json.loads(res.stdout.strip().splitlines()[-1]))


if __name__ == "__main__":
    if not O.feat_available():
        sys.exit("oracle/_ref/feat_oracle is missing: run `make -C oracle ref` where the reference tree exists")
    case("c1_L4.npz", dim=2, level=4, rhs="sine")
    case("c1_L5.npz", dim=2, level=5, rhs="sine")
    case("gauss2d_L5.npz", dim=2, level=5, rhs="gauss", gauss=AS.gauss_params(2, dim=2))
    case("c3d_L3.npz", dim=3, level=3, rhs="sine")
    case("gauss3d_L3.npz", dim=3, level=3, rhs="gauss", gauss=AS.gauss_params(3, dim=3, width=(0.03, 0.12)))
    case("kappa2d_L4.npz", dim=2, level=4, rhs="gauss", gauss=AS.gauss_params(4, dim=2),
         field=AS.field_params(5))
    fd_case()
