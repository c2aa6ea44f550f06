"""Reference energies of the larger synthetic precision cases.  TEST
INFRASTRUCTURE ONLY (fixture generator).

Runs the reference library built from its own sources (oracle/_ref/
libpt_ref.so: src/pt.c, src/ptmp.c, src/misc.c with OpenBLAS) on the seeded
host-generated inputs of libpt_b200.synth and writes
tests/golden/reference_energies.json:

  rpt  o=8 v=64                   (the CPU-runnable restricted (T) case)
  upt  oa=20 va=180 ob=18 vb=182  (unrestricted (T))
  uft  o=15 v=150 per spin        (unrestricted (fT))

each in FP64 (libpt_*) and FP32 (libpt_*_mp, src/ptmp.c), with OpenMP over
triples on every host core and one BLAS thread (the reference's own layout,
src/pt.c:227-230), plus the wall time and core count of each run and a
SHA-256 of the FP64 input bytes so that a consumer can check it generated
the same inputs.  The GPU-side consumers (bench.py's precision table and the
slow GPU parity tests) regenerate the inputs with the same generator and
seed and compare against these values; the reference itself does not travel.

    OMP_NUM_THREADS=$(nproc) OPENBLAS_NUM_THREADS=1 \
        python tests/golden/make_reference_energies.py [--only KIND]

Restricted (fT) at o=30, v=300 is not here: the reference would need about
seven hours on eight cores; that case is pinned on the GPU through the
rft = uft(closed shell) identity instead.
"""
import argparse
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

OUT = os.path.join(HERE, "reference_energies.json")

# (name, kind, sizes, seed): the precision cases of bench.py and the tests
CASES = [
    ("rpt_8_64", "rpt", (8, 64), 7),
    ("upt_20_180_18_182", "upt", (20, 180, 18, 182), 7),
    ("uft_15_150", "uft", (15, 150, 15, 150), 7),
]


def input_digest(case):
    """SHA-256 over the FP64 bytes of the pt.h arrays, in argument order."""
    from oracle import oracle
    h = hashlib.sha256()
    for n in oracle.args_of(case["kind"]):
        h.update(np.ascontiguousarray(case[n], dtype=np.float64).tobytes())
    return h.hexdigest()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", default=None)
    a = ap.parse_args()
    from libpt_b200 import synth
    from oracle import oracle
    ref = oracle.reference()
    data = {}
    if os.path.exists(OUT):
        with open(OUT) as fp:
            data = json.load(fp)
    threads = dict(omp=os.environ.get("OMP_NUM_THREADS"),
                   blas=os.environ.get("OPENBLAS_NUM_THREADS"))
    for name, kind, sz, seed in CASES:
        if a.only and a.only not in (name, kind):
            continue
        case = synth.make(kind, *sz, seed=seed)
        row = dict(kind=kind, sizes=list(sz), seed=seed,
                   generator="libpt_b200.synth.make (numpy PCG64)",
                   input_sha256=input_digest(case), threads=threads,
                   cores=os.cpu_count())
        for mp in (False, True):
            t0 = time.perf_counter()
            e = oracle.solve(ref, case, mp=mp)
            dt = time.perf_counter() - t0
            key = "fp32_mp" if mp else "fp64"
            row[key] = dict(energy=e, seconds=dt)
            print(f"{name} {key}: E = {e!r} ({dt:.1f} s)", flush=True)
        data[name] = row
        with open(OUT, "w") as fp:
            json.dump(data, fp, indent=1, sort_keys=True)
            fp.write("\n")


if __name__ == "__main__":
    main()
