"""Regenerates the golden fixtures in this directory from the reference.

Run in a container where the reference sources are present:

    python tests/golden/make_golden.py --reference <reference checkout>

(or with TAPP_REFERENCE_DIR set instead of --reference)

What it does:
  1. builds the reference from its own C sources (oracle/Makefile, target
     `ref`) into oracle/_ref/;
  2. compiles recorder.c, and the reference's example programs
     (test/demo.c, test/test.c, test/exercise.c, examples/driver/driver.c,
     examples/exercise_contraction/answers/exercise_contraction_answers.c)
     against this repository's include/ headers, linked to the recorder,
     which forwards to the reference and logs every TAPP_execute_product;
  3. writes
       reference_programs.jsonl  one record per execute call (inputs, D before
                                 and after, returned code)
       reference_stdout.json     each program's standard output
       explain_error.json        TAPP_explain_error text of codes 0..14
       error_cases.json          seeded invalid products with the code the
                                 reference returns for each
Nothing here is needed at test time except the files it writes.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "reference-implementation_b200"))
sys.path.insert(0, os.path.join(REPO, "tests"))

PROGRAMS = {
    "demo": ["test/demo.c", "test/helpers.c"],
    "test": ["test/test.c"],
    "exercise": ["test/exercise.c", "test/helpers.c"],
    "driver": ["examples/driver/driver.c", "test/helpers.c"],
    "exercise_contraction_answers": ["examples/exercise_contraction/answers/exercise_contraction_answers.c",
                                     "test/helpers.c"],
}


def sh(cmd, **kw):
    print("+", " ".join(cmd) if isinstance(cmd, list) else cmd)
    return subprocess.run(cmd, check=True, **kw)


def build_and_record(ref_dir: str) -> None:
    sh(["make", "-s", "-C", os.path.join(REPO, "oracle"), "ref", f"REF={ref_dir}"])
    ref_so = os.path.join(REPO, "oracle", "_ref", "libtapp-reference.so")
    tmp = tempfile.mkdtemp(prefix="tapp_golden_")
    rec_so = os.path.join(tmp, "libtapp.so")
    sh(["gcc", "-O1", "-fPIC", "-shared", "-o", rec_so, os.path.join(HERE, "recorder.c"), "-ldl"])
    records = os.path.join(tmp, "records.jsonl")
    stdout = {}
    for name, srcs in PROGRAMS.items():
        exe = os.path.join(tmp, name)
        sh(["gcc", "-O1", "-std=gnu11", "-w", "-I", os.path.join(REPO, "include"),
            "-I", os.path.join(ref_dir, "test"), "-o", exe] +
           [os.path.join(ref_dir, s) for s in srcs] + ["-L", tmp, "-ltapp", f"-Wl,-rpath,{tmp}", "-lm"])
        env = dict(os.environ, TAPP_RECORD_TARGET=ref_so, TAPP_RECORD_OUT=records, TAPP_RECORD_PROGRAM=name)
        r = subprocess.run([exe], env=env, capture_output=True, text=True, check=True)
        stdout[name] = r.stdout
    with open(records) as f, open(os.path.join(HERE, "reference_programs.jsonl"), "w") as g:
        n = 0
        for line in f:
            json.loads(line)  # well-formed
            g.write(line)
            n += 1
    print(f"{n} execute records")
    with open(os.path.join(HERE, "reference_stdout.json"), "w") as g:
        json.dump(stdout, g, indent=1, sort_keys=True)


def explain_strings() -> None:
    from oracle import reference_lib
    ref = reference_lib()
    out = {str(c): ref.explain(c) for c in range(0, 15)}
    with open(os.path.join(HERE, "explain_error.json"), "w") as g:
        json.dump(out, g, indent=1)


def error_cases(seed: int = 20241001, n: int = 400) -> None:
    """Invalid products in the classes the reference's error tests use
    (test/test.cpp:3032-3356) plus the remaining codes; the expected code is
    what the reference itself returns."""
    from oracle import reference_lib
    from families import random_case
    ref = reference_lib()
    rng = np.random.default_rng(seed)
    cases = []
    kinds = ["extent_AB", "extent_A_D", "extent_B_D", "C_structure", "aliasing", "missing_label",
             "repeated_extent_A", "repeated_extent_B", "repeated_extent_D", "C_null_beta", "valid"]
    for i in range(n):
        kind = kinds[i % len(kinds)]
        case = random_case(rng, dtype=0, n_contracted=int(rng.integers(0, 3)), n_hadamard=int(rng.integers(0, 2)),
                           n_freeA=int(rng.integers(0, 3)), n_freeB=int(rng.integers(0, 3)),
                           min_ext=1, max_ext=4)
        A, B, Cc, D = case.A, case.B, case.C, case.D
        bump = int(rng.integers(1, 5))
        if kind == "extent_AB" and A.nmode:
            j = int(rng.integers(0, A.nmode)); A.extents[j] += bump
        elif kind == "extent_A_D" and D.nmode:
            j = int(rng.integers(0, D.nmode)); D.extents[j] += bump; Cc.extents[j] += bump
        elif kind == "extent_B_D" and B.nmode:
            j = int(rng.integers(0, B.nmode)); B.extents[j] += bump
        elif kind == "C_structure":
            sub = int(rng.integers(0, 3))
            if sub == 0:
                Cc.extents.append(2); Cc.strides.append(1); Cc.idx.append(10**15)
            elif sub == 1 and Cc.nmode > 1:
                Cc.idx[1] = Cc.idx[0]
            elif Cc.nmode:
                Cc.extents[int(rng.integers(0, Cc.nmode))] += bump
        elif kind == "aliasing" and D.nmode >= 2:
            j = int(rng.integers(1, D.nmode))
            D.strides[j] = int(rng.choice([-1, 1])) * max(1, abs(D.strides[j - 1]) * D.extents[j - 1] - 1)
            if rng.random() < 0.3:
                D.strides[j] = 0
        elif kind == "missing_label":
            D.idx.append(10**15 + 1); D.extents.append(2); D.strides.append(10**6)
            Cc.idx.append(10**15 + 1); Cc.extents.append(2); Cc.strides.append(10**6)
        elif kind.startswith("repeated_extent"):
            T = {"A": A, "B": B, "D": D}[kind[-1]]
            if T.nmode:
                j = int(rng.integers(0, T.nmode))
                T.idx.append(T.idx[j]); T.extents.append(T.extents[j] + bump); T.strides.append(1)
                if kind[-1] == "D":
                    Cc.idx.append(Cc.idx[j]); Cc.extents.append(Cc.extents[j] + bump); Cc.strides.append(1)
        elif kind == "C_null_beta":
            case.C_is_null = True
            case.beta[0] = 0.0 if rng.random() < 0.3 else 0.5
        # execute only validates on the reference when it fails; give it no data
        # beyond what a valid product would touch by pointing at large buffers
        rec = {"kind": kind, "beta": float(case.beta[0]), "C_null": bool(case.C_is_null),
               "tensors": [{"extents": list(map(int, t.extents)), "strides": list(map(int, t.strides)),
                            "idx": list(map(int, t.idx))} for t in (A, B, Cc, D)]}
        code = _ref_code(ref, rec)
        rec["expected"] = code
        cases.append(rec)
    with open(os.path.join(HERE, "error_cases.json"), "w") as g:
        json.dump(cases, g)
    print("error codes:", sorted({c["expected"] for c in cases}))


def _ref_code(ref, rec) -> int:
    """Runs the product on the reference with buffers large enough for any
    layout in `rec` and returns its code."""
    from tapp_b200.case import alloc, scalar, Case
    ts = []
    for t in rec["tensors"]:
        ts.append(alloc(0, t["extents"], t["strides"], t["idx"]))
    case = Case(*ts, scalar(0, 1.0), scalar(0, rec["beta"]), -1, rec["C_null"])
    return case.run(ref)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("TAPP_REFERENCE_DIR"),
                    help="checkout of the reference (default: $TAPP_REFERENCE_DIR)")
    a = ap.parse_args()
    if not a.reference:
        ap.error("give --reference <reference checkout> or set TAPP_REFERENCE_DIR")
    build_and_record(a.reference)
    explain_strings()
    error_cases()


if __name__ == "__main__":
    main()
