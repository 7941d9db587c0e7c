#!/usr/bin/env python3
"""Generates tests/golden/ref_c1.json from the reference's own CPU driver.

Runs the reference (RIKEN-RCCS/hpl-ai) built by oracle/build_ref.sh from its
sources with the thread-rank MPI runtime (oracle/tmpi/): 4 ranks (a 2 x 2
grid, P = 2) and one OpenMP thread each, the commands of the C1 case

    driver.out 1200 60 2 -not -r        (FP16 Schur update, FP32 accumulation)
    driver.out 1200 60 2 -not -d -r     (the C1 command: lazy init, FP16 deck)

once with the netlib-order BLAS build (ref_driver_netlib.out, whose LU is
deterministic) and once with OpenBLAS (ref_driver.out).  It records, per run,
the printed refinement steps and report line, the solution vector x (the
reference's refinement result, collected through TMPI_XDUMP) and, for the
netlib build, the SHA-256 of the FP32 factors the LU left in memory
(TMPI_LUDUMP), so that a test can pin a restatement of the LU bit for bit
without a 5.8 MB fixture.  Two more netlib runs cover the driver's other
factor paths: `--l1est` (approximate factors without a decomposition) and
`-w` (the benchmark warm-up: the first P + 2 = 4 block steps, one
refinement step).  The `-d` runs also record the factors' digest: with lazy
initialisation the LU runs through the FP16-accumulating Schur update
(hgemm_opt), which the oracle restates in oracle/hplai_oracle_deck.c; one more
`-d` run at n = 2400, b = 120 covers its k-chunks of 100 (two per panel).

Needs oracle/_ref (built from the reference tree on this machine); the
fixture it writes is what the tests read.
"""
import hashlib
import json
import os
import re
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, "oracle", "_ref")
N, B, P = 1200, 60, 2
STEP = re.compile(r"# iterative refinement: step=\s*(\d+), residual=(\S+) hpl-harness=(\S+)")
REPORT = re.compile(r"^(\S+) sec\. (\S+) GFlop/s resid = (\S+) hpl-harness = (\S+)$", re.M)


def run(exe, flags, ludump, n=N, b=B, keep_x=True):
    with tempfile.TemporaryDirectory() as td:
        xf, lf = os.path.join(td, "x.bin"), os.path.join(td, "lu.bin")
        env = dict(os.environ, TMPI_NP="4", OMP_NUM_THREADS="1", OPENBLAS_NUM_THREADS="1", TMPI_XDUMP=xf)
        if ludump:
            env["TMPI_LUDUMP"] = lf
        out = subprocess.run([os.path.join(REF, exe), str(n), str(b), str(P)] + flags, capture_output=True, text=True,
                             env=env, cwd=td, timeout=600, check=True).stdout
        x = np.fromfile(xf, dtype=np.float64)
        digest = None
        if ludump:
            lu = np.fromfile(lf, dtype=np.float32)
            assert lu.size == n * n
            digest = hashlib.sha256(lu.tobytes()).hexdigest()
    steps = [{"residual": float(r), "hpl_harness": float(h)} for _, r, h in STEP.findall(out)]
    m = REPORT.search(out)
    assert (x.size == n or "-w" in flags) and steps and m, out[-2000:]
    rec = {"command": f"driver.out {n} {b} {P} " + " ".join(flags), "build": exe,
           "steps": steps, "resid": float(m.group(3)), "hpl_harness": float(m.group(4)),
           "gflops": float(m.group(2)), "seconds": float(m.group(1))}
    if "-w" not in flags and keep_x:
        rec["x"] = [float(v).hex() for v in x]
    if digest:
        rec["lu_sha256"] = digest
    return rec


def main():
    runs = {
        "netlib_not_r": run("ref_driver_netlib.out", ["-not", "-r"], True),
        "netlib_l1est": run("ref_driver_netlib.out", ["-not", "-r", "--l1est"], True),
        "netlib_warmup": run("ref_driver_netlib.out", ["-not", "-r", "-w"], True),
        "netlib_not_d_r": run("ref_driver_netlib.out", ["-not", "-d", "-r"], True),
        "netlib_not_d_r_2400": run("ref_driver_netlib.out", ["-not", "-d", "-r"], True, n=2400, b=120, keep_x=False),
        "openblas_not_r": run("ref_driver.out", ["-not", "-r"], False),
        "openblas_not_d_r": run("ref_driver.out", ["-not", "-d", "-r"], False),
    }
    doc = {"n": N, "b": B, "seed": 42, "ranks": "4 threads (2 x 2 grid), OMP_NUM_THREADS=1",
           "generator": "tests/golden/make_ref_fixtures.py (reference built by oracle/build_ref.sh)",
           "x_format": "float.hex() per entry", "runs": runs}
    with open(os.path.join(HERE, "ref_c1.json"), "w") as f:
        json.dump(doc, f, indent=1)
        f.write("\n")
    for k, v in runs.items():
        print(k, v["command"], [(s["residual"], s["hpl_harness"]) for s in v["steps"]])


if __name__ == "__main__":
    main()
