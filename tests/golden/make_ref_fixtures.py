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
Two `--back_buffer` runs (n = 2400 and 4800, b = 60: one and two write-backs
of the deck into the back buffer, at steps 32 and 64) record the factors'
digest of that form too.

Higham's matrix (`--highammat`): the alpha and beta that the reference's
higham_mat_comp_beta returns for a list of orders (oracle/_ref/libref_higham.so,
its higham_mat_impl.cpp compiled alone), and the first refinement steps of
its driver with `--highammat` (with and without `-d`), which diverge: its
pmatgen drops the signs of Higham's matrix (matgen.hpp:25-77; the lazy
initialisation keeps them, lazy_init.hpp:331-440) and its FP64 GEMV swaps
alpha and beta inside the diagonal blocks (hmg_gemv_diag,
otf_gemv.cpp:296-314), so the residual it refines against is of neither
matrix.  The tests use the step-0 numbers to pin alpha, beta, the diagonal
and the right-hand side through the reference's own residual evaluation.

Needs oracle/_ref (built from the reference tree on this machine); the
fixture it writes is what the tests read.
"""
import ctypes
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


def higham():
    lib = ctypes.CDLL(os.path.join(REF, "libref_higham.so"))
    lib.higham_mat_comp_beta.restype = ctypes.c_double
    lib.higham_mat_comp_beta.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double]
    betas = []
    for n in [64, 120, 1200, 2400, 4096, 8192, 16384, 46340, 46341, 50000, 65536, 98304, 131072, 196608]:
        for cond, rho in [(1000.0, 0.5), (100.0, 0.5), (1.0e4, 0.25)]:
            betas.append({"n": n, "cond": cond, "rho": rho, "beta": lib.higham_mat_comp_beta(n, cond, rho).hex()})
    runs = {}
    for key, flags in [("not_r", ["-not", "-r", "--highammat"]), ("not_d_r", ["-not", "-d", "-r", "--highammat"])]:
        with tempfile.TemporaryDirectory() as td:
            env = dict(os.environ, TMPI_NP="4", OMP_NUM_THREADS="1", OPENBLAS_NUM_THREADS="1")
            out = subprocess.run([os.path.join(REF, "ref_driver_netlib.out"), str(N), str(B), str(P)] + flags,
                                 capture_output=True, text=True, env=env, cwd=td, timeout=600, check=True).stdout
        steps = [{"residual": float(r), "hpl_harness": float(h)} for _, r, h in STEP.findall(out)]
        m = REPORT.search(out)
        runs[key] = {"command": f"driver.out {N} {B} {P} " + " ".join(flags), "build": "ref_driver_netlib.out",
                     "first_steps": steps[:3], "steps": len(steps), "resid": float(m.group(3)),
                     "hpl_harness": float(m.group(4))}
    return {"betas": betas, "runs": runs,
            "note": "the reference's --highammat refinement diverges (IRErrors {-1,-1}); see make_ref_fixtures.py"}


def main():
    runs = {
        "netlib_not_r": run("ref_driver_netlib.out", ["-not", "-r"], True),
        "netlib_l1est": run("ref_driver_netlib.out", ["-not", "-r", "--l1est"], True),
        "netlib_warmup": run("ref_driver_netlib.out", ["-not", "-r", "-w"], True),
        "netlib_not_d_r": run("ref_driver_netlib.out", ["-not", "-d", "-r"], True),
        "netlib_not_d_r_2400": run("ref_driver_netlib.out", ["-not", "-d", "-r"], True, n=2400, b=120, keep_x=False),
        "netlib_not_r_bb_2400": run("ref_driver_netlib.out", ["-not", "-r", "--back_buffer"], True, n=2400, b=60,
                                    keep_x=False),
        "netlib_not_r_bb_4800": run("ref_driver_netlib.out", ["-not", "-r", "--back_buffer"], True, n=4800, b=60,
                                    keep_x=False),
        "openblas_not_r": run("ref_driver.out", ["-not", "-r"], False),
        "openblas_not_d_r": run("ref_driver.out", ["-not", "-d", "-r"], False),
    }
    doc = {"n": N, "b": B, "seed": 42, "ranks": "4 threads (2 x 2 grid), OMP_NUM_THREADS=1",
           "generator": "tests/golden/make_ref_fixtures.py (reference built by oracle/build_ref.sh)",
           "x_format": "float.hex() per entry", "runs": runs, "higham": higham()}
    with open(os.path.join(HERE, "ref_c1.json"), "w") as f:
        json.dump(doc, f, indent=1)
        f.write("\n")
    for k, v in runs.items():
        print(k, v["command"], [(s["residual"], s["hpl_harness"]) for s in v["steps"]])


if __name__ == "__main__":
    main()
