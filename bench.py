#!/usr/bin/env python3
"""HPL-AI GFLOP/s of the single-GPU B200 solver (one JSON line on rank 0).

One step = one solve of the HPL-AI system on the GPU: the blocked no-pivot
LU followed by FP64 refinement to hpl-harness < 16 -- the reference's timed
region (main.cpp:283-441).  The matrix is regenerated on the device before
every step, outside the timed window, as the reference generates it before
its timer starts (the LU overwrites A).  Work per step: 2/3 n^3 + 3/2 n^2
flops (main.cpp:441).

By default the workload is n = 131072, b = 1024 in two forms, timed back to
back on the same GPU:
  * the precision form (the headline `value`): e4m3 Schur update with
    per-128 power-of-two factors and FP32 accumulation into the FP16
    trailing-update deck, FP32 panels, FP64 GMRES-IR;
  * the plain form (`plain`): FP16 Schur update with FP32 accumulation into
    the FP32 trailing matrix, FP32 panels, FP64 iterative refinement;
and `speedup_vs_plain` is the plain form's time per solve over the
precision form's.  `--n 65536 --b 512` gives the smaller plain-scale case.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 (under torchrun, one rank per GPU) runs N independent replicas: a
single solve does not shard on this build ("replicas only").  `value` is
the flops of all ranks over the slowest rank's time.

--impl reference times the reference algorithm on the host cores: the
reference's own code built from its sources (oracle/_ref) when present,
else the CPU restatement in oracle/ -- on a bounded sample of the workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "hpl-ai_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

METRIC = "HPL-AI GFLOP/s to hpl-harness<16: FP8-Schur+GMRES-IR vs plain; % tensor peak"
UNIT = "GFLOP/s"
DEFAULT_N, DEFAULT_B = 131072, 1024   # the precision-vs-plain configuration (C3)
ADJOINT_N, ADJOINT_B = 8192, 256
CPU_SAMPLE = (4800, 120)           # bounded CPU sample of the same workload (seconds per solve)


def hpl_flops(n):
    return 2.0 / 3.0 * n * n * n + 3.0 / 2.0 * n * n


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), d.get("bf16_tflops_sustained", 1400.0), "measured"
    return 6650.0, 1590.0, 1400.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, ValueError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        load = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(load), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def replica_value(total_ms, units, world, device=None):
    """Whole-job throughput over `world` replicas: the units of all ranks over
    the slowest rank's time (max over ranks), in units/s / 1e9.  Every rank
    takes the same two collectives."""
    import torch
    t = torch.tensor([float(total_ms)], dtype=torch.float64, device=device)
    u = torch.tensor([float(units)], dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(u, op=dist.ReduceOp.SUM)
    max_ms = float(t.item())
    return float(u.item()) / (max_ms * 1e-3) / 1e9, max_ms


def batch_seeds(rank, count):
    """Seeds of rank `rank`'s systems: replicas solve disjoint systems."""
    return [rank * count + s for s in range(count)]


REF_FLAGS = ["-not", "-d", "-r"]   # the reference command of the north star: mpirun -n 4 driver.out n b 2 -not -d -r


def cpu_solve_gflops(n, b, threads):
    """One CPU solve of the sample by the reference's own driver (built from
    its sources by oracle/build_ref.sh: 4 ranks as threads of one process, a
    2 x 2 grid, threads // 4 OpenMP threads each, OpenBLAS single-threaded
    per rank), timed by the driver itself (LU + refinement, main.cpp:283-452);
    the oracle restatement when that build is absent."""
    ref_bin = os.path.join(ROOT, "oracle", "_ref", "ref_driver.out")
    if os.path.exists(ref_bin):
        per_rank = max(1, threads // 4)
        env = dict(os.environ, OMP_NUM_THREADS=str(per_rank), OPENBLAS_NUM_THREADS="1", TMPI_NP="4")
        out = subprocess.run([ref_bin, str(n), str(b), "2"] + REF_FLAGS, capture_output=True, text=True, env=env,
                             timeout=600)
        for ln in out.stdout.splitlines():
            if "GFlop/s" in ln and "sec." in ln:
                f = ln.split()
                secs, harness = float(f[0]), float(f[-1])
                if not harness < 16:
                    raise RuntimeError(f"reference solve did not reach hpl-harness < 16: {ln}")
                return hpl_flops(n) / secs / 1e9, secs, harness, "reference", 4 * per_rank
        raise RuntimeError(f"reference build printed no report line (rc {out.returncode}): {out.stdout[-400:]}")
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    import oracle
    t0 = time.perf_counter()
    rc, x, res, har, steps = oracle.solve(n, b, q=1)
    secs = time.perf_counter() - t0
    if rc != 0:
        raise RuntimeError("oracle solve did not converge")
    return hpl_flops(n) / secs / 1e9, secs, har, "port", threads


def cpu_sample_note(kind, cores, n, b):
    if kind == "reference":
        return (f"the reference's driver.out {n} {b} 2 {' '.join(REF_FLAGS)} built from its sources "
                f"(oracle/build_ref.sh; 4 ranks as threads, {cores // 4} OpenMP threads each, OpenBLAS 0.3.15 "
                f"single-threaded per rank), its own LU + IR timer")
    return f"the oracle's CPU restatement, full solve (LU + IR) at n={n} b={b}"


def run_reference(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    n, b = CPU_SAMPLE
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_solve_gflops(n, b, threads)
    vals, secs = [], []
    for _ in range(args.steps):
        g, s, har, kind, cores = cpu_solve_gflops(n, b, threads)
        vals.append(g)
        secs.append(s)
    sample = cpu_sample_note(kind, cores, n, b)
    value = len(vals) * hpl_flops(n) / sum(secs) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(secs) / len(secs),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp16/fp32/fp64",
        "data": "synthetic (the reference's own LCG matrix, seed 42)",
        "config": {"workload": f"HPL-AI solve, bounded CPU sample n={n} b={b} of the n={args.n} b={args.b} "
                               f"workload", "n": n, "b": b,
                   "command": f"driver.out {n} {b} 2 {' '.join(REF_FLAGS)}" if kind == "reference" else None},
        "hpl_harness": har,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": f"{sample}; {args.steps} steps"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def schur_algorithmic(n, b, panel_bytes=2, c_bytes=8, group=1):
    """Flops, bytes and launches of all Schur updates of one factorisation,
    in the order hplai_factor issues them.  The update by a group of `group`
    panels (K = group * b) of the trailing matrix from block e on is split
    into the next group's block columns, its block rows and the rest; with
    panel groups a group's block e + j first receives the updates of the
    group's panels e .. e + j - 1, each alone (K = b).  A region of m x n C
    elements with panel width K
    does 2 m n K flops and moves c_bytes per C element (8: FP32 read +
    write; 4: the FP16 deck) plus (m + n) K panel elements of panel_bytes
    (2 for FP16, 1 for e4m3)."""
    acc = {"flops": 0.0, "bytes": 0.0, "launches": 0}
    nb = n // b

    def region(m, nn, k):
        if m <= 0 or nn <= 0:
            return
        acc["flops"] += 2.0 * m * nn * k
        acc["bytes"] += float(c_bytes) * m * nn + float(panel_bytes) * (m + nn) * k
        acc["launches"] += 1

    def panel_updates(j, first):
        for _ in range(j - first):
            region(n - j * b, b, b)
            region(b, n - (j + 1) * b, b)

    for j in range(1, min(group, nb)):
        panel_updates(j, 0)
    s = 0
    while s + group < nb:
        e = s + group
        ne = min(group, nb - e)
        r1, r2, k = e * b, (e + ne) * b, group * b
        region(n - r1, r2 - r1, k)
        region(r2 - r1, n - r2, k)
        for j in range(e + 1, e + ne):
            panel_updates(j, e)
        region(n - r2, n - r2, k)
        s += group
    return acc["flops"], acc["bytes"], acc["launches"]


def schur_traffic_per_launch(n, b, group=1, kind="fp16_fp32c"):
    """DRAM bytes per average launch from the committed ncu summaries (DRAM
    bytes per updated C element of the kernel at the group's K: 2048 or 4096),
    times the C elements of one factorisation's launches (traffic grows with
    the C area), per launch."""
    p = os.path.join(ROOT, "profiles", "schur_kernel_traffic.json")
    if not os.path.exists(p):
        return None
    kernels = json.load(open(p)).get("kernels", {})
    d = kernels.get(kind + "_k4096") if group * b >= 4096 else None
    d = d or kernels.get(kind)
    if not d:
        return None
    _, byts, launches = schur_algorithmic(n, b, 0, 1, group)   # bytes = C elements
    return d["dram_bytes_per_c_element"] * byts / launches


FORMS = {
    # the precision form: e4m3 Schur update (per-128 power-of-two factors, FP32
    # accumulation) into the FP16 trailing-update deck, FP64 GMRES-IR
    "precision": {"precision": "f8", "deck": True, "refine": "gmres",
                  "label": "precision: e4m3 Schur into the FP16 deck + FP64 GMRES-IR(30)"},
    # the plain form: FP16 Schur update with FP32 accumulation into the FP32
    # trailing matrix, FP64 iterative refinement (the reference's no -d form)
    "plain": {"precision": "f16", "deck": False, "refine": "ir",
              "label": "plain: FP16 Schur into the FP32 trailing matrix + FP64 IR"},
}


def schur_roofline(hplai, n, b, fp8, deck, gemm_ms, group=1):
    """Roofline of the Schur GEMM over one factorisation: algorithmic flops
    and bytes per launch (schur_algorithmic) over the average launch time
    (CUDA events around each launch on its stream, summed by the library)."""
    hbm, tc_burst, tc_sus, peak_kind = load_peaks()
    peak_note = f"{peak_kind} (MEASURED_PEAKS.json: hbm_gbs, bf16_tflops_sustained)"
    if fp8:
        e4 = load_e4m3_peak()
        if e4:
            tc_sus = e4["sustained_tflops"]
            peak_note = f"measured e4m3 dense (cuBLAS e4m3 8192^3 back to back, {e4['source']})"
        else:
            tc_sus *= 2.0
            peak_note += " x 2 for e4m3 (nominal e4m3:bf16 ratio; no measured e4m3 peak)"
    sflops, sbytes, slaunch = schur_algorithmic(n, b, 1 if fp8 else 2, 4 if deck else 8, group)
    avg_launch_s = gemm_ms * 1e-3 / slaunch
    ach_gbs = sbytes / slaunch / avg_launch_s / 1e9
    ach_tf = sflops / slaunch / avg_launch_s / 1e12
    ridge = tc_sus * 1e12 / (hbm * 1e9)
    intensity = sflops / sbytes
    bound = "tensor" if intensity >= ridge else "hbm"
    if bound == "hbm":
        roof = {"bound": "hbm", "achieved": ach_gbs, "peak": hbm, "unit": "GB/s", "frac": ach_gbs / hbm}
    else:
        roof = {"bound": "tensor", "achieved": ach_tf, "peak": tc_sus, "unit": "TFLOP/s", "frac": ach_tf / tc_sus}
    cdesc = "FP16 deck, deck -= s*L*U" if deck else "FP32 C, C -= L*U"
    kname = f"schur_kernel (tcgen05 {'e4m3 x e4m3' if fp8 else 'FP16 x FP16'} -> FP32 accumulator; {cdesc})"
    kind = "e4m3_deck" if (fp8 and deck) else ("fp16_fp32c" if (not fp8 and not deck) else None)
    traffic = schur_traffic_per_launch(n, b, group, kind) if kind else None
    roof.update({"traffic": traffic, "kernel": kname,
                 "launches_per_step": slaunch, "avg_launch_ms": avg_launch_s * 1e3,
                 "algorithmic_bytes_per_launch": sbytes / slaunch, "algorithmic_flops_per_launch": sflops / slaunch,
                 "algorithmic_bytes_note": ("per C element 4 B (FP16 deck read + write)" if deck else
                                            "per C element 8 B (FP32 read + write)") +
                 f" + panels {1 if fp8 else 2} B per element",
                 "intensity_flop_per_byte": intensity, "ridge_flop_per_byte": ridge,
                 "tensor_achieved_tflops": ach_tf, "tensor_peak_tflops": tc_sus,
                 "tensor_frac": ach_tf / tc_sus, "hbm_achieved_gbs": ach_gbs, "hbm_frac": ach_gbs / hbm,
                 "panels_per_update": group,
                 "peak_source": peak_note})
    return roof


def load_e4m3_peak():
    """Measured dense e4m3 rate of this GPU type (bench.py --workload peak),
    committed as a figure under profiles/."""
    p = os.path.join(ROOT, "profiles", "tensor_peaks_cublas_8192.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p))
    e4 = d.get("e4m3")
    if not e4:
        return None
    return {"sustained_tflops": e4["sustained_tflops"], "burst_tflops": e4["burst_tflops"],
            "source": "profiles/tensor_peaks_cublas_8192.json"}


class FormRun:
    """One solver form timed over `steps` solves (factor + refinement to
    hpl-harness < 16) after `warmup` untimed ones, the matrix regenerated on
    the device before each solve outside the timed window."""

    def __init__(self, hplai, torch, form, n, b, seed, maxit, autotune, lookahead, barrier, group=1, side_sms=32,
                 matrix="lcg", lazy_a=False):
        self.hplai, self.torch, self.form = hplai, torch, form
        self.n, self.b, self.seed, self.maxit = n, b, seed, maxit
        self.fp8 = form["precision"] == "f8"
        self.deck = form["deck"]
        self.mode = hplai.GMRES if form["refine"] == "gmres" else hplai.IR
        flags = hplai.FLAG_LOOKAHEAD if lookahead else 0
        if self.deck:
            flags |= hplai.FLAG_FP16_DECK
        self.lazy_a = bool(lazy_a and self.deck and self.fp8)
        if self.lazy_a:
            flags |= hplai.FLAG_LAZY_A
        if group == 2:
            flags |= hplai.FLAG_GROUP2
        elif group == 4:
            flags |= hplai.FLAG_GROUP4
        prec = hplai.F32_F8 if self.fp8 else hplai.F32_F16
        self.s = None
        if autotune and b % 128 == 0 and group != 4:
            # buffers for four-panel groups, so that the tuner can choose them
            # (skipped when they do not fit)
            try:
                self.s = hplai.Solver(n, b, precision=prec, flags=flags | hplai.FLAG_GROUP4)
                self.s.set_schedule(flags & (hplai.FLAG_LOOKAHEAD | hplai.FLAG_GROUP2), side_sms)
            except hplai.HplaiError:
                self.s = None
        if self.s is None:
            self.s = hplai.Solver(n, b, precision=prec, flags=flags)
        if matrix == "higham":
            self.s.set_matrix(hplai.MATRIX_HIGHAM, 1000.0, 0.5)
        self.ext = torch.cuda.ExternalStream(self.s.stream())
        self.barrier = barrier
        self.tuned = None
        def group_of(f):
            return 4 if (f & hplai.FLAG_GROUP4) else 2 if (f & hplai.FLAG_GROUP2) else 1
        self.group = group_of(flags)
        sched_bits = hplai.FLAG_LOOKAHEAD | hplai.FLAG_GROUP2 | hplai.FLAG_GROUP4
        if lookahead:
            self.s.set_schedule(flags & sched_bits, side_sms)
        self.schedule = {"lookahead": bool(lookahead), "side_sms": side_sms if lookahead else None,
                         "panels_per_update": self.group, "source": "flags"}
        if autotune:
            # outside the timed region: time the factorisation under each schedule, keep the fastest
            tflags, tside, tms = self.s.autotune(seed)
            la = bool(tflags & hplai.FLAG_LOOKAHEAD)
            self.group = group_of(tflags)
            def side_desc(f, sd):
                if not (f & hplai.FLAG_LOOKAHEAD):
                    return None
                return sd if sd > 0 else f"share sms*c/(r+c), c={-sd} panels, r = trailing block columns"
            trials = [{"panels_per_update": group_of(f), "cta_pairs": bool(f & hplai.TRIAL_CTA_PAIRS),
                       "lookahead": bool(f & hplai.FLAG_LOOKAHEAD), "side_sms": side_desc(f, sd),
                       "tile_group": tg, "factor_ms": round(ms, 2)} for f, sd, tg, ms in self.s.autotune_trials()]
            self.tuned = {"factor_ms": tms, "trials_warmup_first": trials}
            self.schedule = {"lookahead": la, "side_sms": side_desc(tflags, tside), "panels_per_update": self.group,
                             "tile_group": self.s.tile_group(), "cta_pairs": self.s.cta_pairs() == 1,
                             "source": "hplai_autotune"}
        self.results = []

    def step(self, timed):
        s, torch = self.s, self.torch
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(self.ext)
        s.generate(self.seed)   # outside the timed window, as the reference's (main.cpp:255-327)
        g1.record(self.ext)
        self.barrier()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(self.ext)
        s.factor()
        r = s.iterative_refinement(self.maxit, mode=self.mode)
        ev1.record(self.ext)
        ev1.synchronize()
        self.barrier()
        if r.status != self.hplai.HPLAI_OK:
            raise RuntimeError(f"solve did not converge: {r}")
        if timed:
            self.results.append((ev0.elapsed_time(ev1), r, s.phase_ms(), s.refine_counts(), g0.elapsed_time(g1)))

    def run(self, steps, warmup):
        for _ in range(warmup):
            self.step(False)
        for _ in range(steps):
            self.step(True)
        return self

    def summary(self, world):
        hplai = self.hplai
        total_ms = sum(r[0] for r in self.results)
        steps = len(self.results)
        value, max_ms = replica_value(total_ms, steps * hpl_flops(self.n), world, device="cuda")
        phases = {k: statistics.mean(r[2][k] for r in self.results) for k in self.results[0][2]}
        roof = schur_roofline(hplai, self.n, self.b, self.fp8, self.deck, phases["GEMM_UPDATE"], self.group)
        last = self.results[-1]
        return {
            "form": self.form["label"], "value": value, "unit": UNIT, "steps": steps,
            "ms_per_step": max_ms / steps, "ms_min": min(r[0] for r in self.results),
            "ms_max": max(r[0] for r in self.results),
            "schedule": self.schedule, "autotuned": self.tuned,
            "trailing_matrix": ("FP16 deck (updates rounded to FP16 once per step, folded in per panel)"
                                + ("; A not stored: each block regenerated from the LCG when it joins a panel, "
                                   "the deck in the upper half of each FP32 column" if self.lazy_a else ""))
            if self.deck else "FP32",
            "hpl_harness": last[1].hpl_harness, "resid": last[1].residual,
            "residual_evaluations": last[1].iters,
            "gmres_inner_steps": last[3][1] if self.mode == hplai.GMRES else None,
            "phases_ms": phases, "roofline": roof,
            "generation_ms": statistics.median(r[4] for r in self.results),
        }

    def close(self):
        self.s.close()


def e2e_run(hplai, torch, fr, steps, warmup, world, barrier):
    """The same solve through the public C API with host buffers: pinned FP32
    A, FP64 rhs and diagonal copied in, x copied out, every step
    (hplai_solve_host)."""
    s, n, seed = fr.s, fr.n, fr.seed
    s.generate(seed)
    torch.cuda.synchronize()
    try:
        a_h = torch.empty(n * n, dtype=torch.float32, pin_memory=True)
        pinned = True
    except RuntimeError:
        a_h = torch.empty(n * n, dtype=torch.float32)
        pinned = False
    hplai.check(hplai._get_lu(s._h, a_h.data_ptr(), n), "hplai_get_lu")
    rhs_h = torch.from_numpy(s.rhs())
    d_h = torch.from_numpy(s.diag())
    if pinned:
        rhs_h, d_h = rhs_h.pin_memory(), d_h.pin_memory()
    x_h = torch.empty(n, dtype=torch.float64, pin_memory=pinned)
    ets = []
    for i in range(warmup + steps):
        barrier()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(fr.ext)
        r = s.solve_host_ptrs(a_h.data_ptr(), n, rhs_h.data_ptr(), d_h.data_ptr(), seed, fr.maxit, x_h.data_ptr())
        ev1.record(fr.ext)
        ev1.synchronize()
        barrier()
        if r.status != hplai.HPLAI_OK:
            raise RuntimeError(f"e2e solve did not converge: {r}")
        if i >= warmup:
            ets.append(ev0.elapsed_time(ev1))
    del a_h
    te = torch.tensor([sum(ets)], dtype=torch.float64, device="cuda")
    if world > 1:
        torch.distributed.all_reduce(te, op=torch.distributed.ReduceOp.MAX)
    return {"value": world * len(ets) * hpl_flops(n) / (float(te.item()) * 1e-3) / 1e9, "unit": UNIT,
            "h2d_bytes_per_step": n * n * 4 + 2 * n * 8, "d2h_bytes_per_step": n * 8,
            "host_memory": "pinned" if pinned else "pageable", "ms_per_step": float(te.item()) / len(ets),
            "steps": len(ets), "warmup": warmup, "call": "hplai_solve_host (" + fr.form["label"] + ")"}


def run_ours(args):
    import torch
    world, rank, local = dist_setup()
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    import hplai
    hplai.set_cta_pairs_default(args.pairs != "off")

    n, b, seed, maxit = args.n, args.b, 42, 50
    dev = torch.cuda.current_device()

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()

    if args.forms == "both":
        head_key, other_key = "precision", "plain"
    else:
        head_key, other_key = args.forms, None
    head_form = dict(FORMS[head_key])
    if args.precision:
        head_form["precision"] = args.precision
    if args.deck:
        head_form["deck"] = args.deck == "on"
    if args.refine:
        head_form["refine"] = args.refine
    if head_form != FORMS[head_key]:
        head_form["label"] = (f"{'e4m3' if head_form['precision'] == 'f8' else 'FP16'} Schur into the "
                              f"{'FP16 deck' if head_form['deck'] else 'FP32 trailing matrix'} + FP64 "
                              f"{'GMRES-IR' if head_form['refine'] == 'gmres' else 'IR'}")

    # the headline form: exactly `steps` timed solves after `warmup`
    if args.lazy_a and not (head_form["precision"] == "f8" and head_form["deck"] and args.matrix == "lcg"):
        raise SystemExit("--lazy-a needs the e4m3 form with the FP16 deck and the LCG matrix")
    fr = FormRun(hplai, torch, head_form, n, b, seed, maxit, args.autotune, args.lookahead, barrier, args.group,
                 args.side_sms, args.matrix, args.lazy_a)
    fr.run(0, args.warmup)
    sampler = ClockSampler(dev)
    sampler.start()
    l0 = hplai.launch_count()
    fr.run(args.steps, 0)
    launches = hplai.launch_count() - l0
    clocks = sampler.stop()
    head = fr.summary(world)
    e2e = None
    if args.lazy_a:
        e2e = {"unavailable": "HPLAI_FLAG_LAZY_A takes no host matrix: A is regenerated from its seed on the device"}
    elif not args.no_e2e:
        e2e = e2e_run(hplai, torch, fr, min(args.steps, args.e2e_steps), args.e2e_warmup, world, barrier)
    fr.close()

    # the comparison form, on the same GPU right after (its own context)
    other = None
    if other_key:
        fo = FormRun(hplai, torch, FORMS[other_key], n, b, seed, maxit, args.autotune, args.lookahead, barrier,
                     args.group, args.side_sms, args.matrix)
        fo.run(min(args.steps, args.compare_steps), min(args.warmup, args.compare_warmup))
        other = fo.summary(world)
        fo.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        nb_, bb_ = CPU_SAMPLE
        threads = os.cpu_count() or 1
        reps, tot = 0, 0.0
        kind, cores = "port", threads
        while tot < 10.0 and reps < 8:
            g, secs, har, kind, cores = cpu_solve_gflops(nb_, bb_, threads)
            reps += 1
            tot += secs
        cpu = {"value": reps * hpl_flops(nb_) / tot / 1e9, "unit": UNIT, "cores": cores, "kind": kind,
               "sample": f"{reps} solve(s) by {cpu_sample_note(kind, cores, nb_, bb_)}, {tot:.1f} s"}

    if rank == 0:
        cfg = "C3" if (n, b) == (131072, 1024) else ("C2" if (n, b) == (65536, 512) else "custom")
        wl = f"HPL-AI solve n={n} b={b} ({cfg}), {head['form']}"
        if other:
            wl += f"; compared with the {other['form']}"
        line = {
            "metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "e4m3/fp16/fp32/fp64" if head_form["precision"] == "f8" else "fp16/fp32/fp64",
            "data": ("synthetic (the reference's own LCG matrix, seed 42, regenerated on the device before each step)"
                     if args.matrix == "lcg" else
                     "synthetic (Higham's HPL-AI matrix, cond 1000, rho 0.5, as --highammat; LCG right-hand side, "
                     "seed 42; regenerated on the device before each step)"),
            "config": {"workload": wl, "n": n, "b": b, "matrix": args.matrix, "form": head["form"],
                       "schedule": head["schedule"],
                       "autotuned": head["autotuned"],
                       "trailing_matrix": head["trailing_matrix"],
                       "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                       "l2": f"inputs {n * n * 4 / 1e9:.1f} GB FP32 > 126 MB L2, rewritten between steps"},
            "hpl_harness": head["hpl_harness"], "resid": head["resid"],
            "residual_evaluations": head["residual_evaluations"], "gmres_inner_steps": head["gmres_inner_steps"],
            "phases_ms": head["phases_ms"], "generation_ms_untimed": head["generation_ms"], "roofline": head["roofline"], "gpu_launches": int(launches),
            "clocks": clocks, "e2e": e2e, "cpu_baseline": cpu,
        }
        if other:
            line["plain" if other_key == "plain" else other_key] = other
            line["speedup_vs_" + other_key] = other["ms_per_step"] / head["ms_per_step"]
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def run_batch(args):
    """Many independent systems on one GPU (log-uniform orders 256..4096,
    1..8 right-hand sides, system s seeded with s), through the batched C API."""
    import torch
    world, rank, local = dist_setup()
    torch.cuda.set_device(local if world > 1 else 0)
    import hplai
    count = args.batch_count
    n, nrhs = hplai.batch_sizes(count, rng_seed=args.batch_seed)
    seeds = batch_seeds(rank, count)
    flops = float(sum(2.0 / 3.0 * float(v) ** 3 + 1.5 * float(v) ** 2 * int(r) for v, r in zip(n, nrhs)))
    dev = torch.cuda.current_device()
    t0 = time.perf_counter()
    bt = hplai.Batch(n, nrhs, seeds, workers=args.batch_workers)
    create_s = time.perf_counter() - t0
    stream = torch.cuda.Stream()
    for _ in range(args.warmup):
        if bt.solve() != hplai.HPLAI_OK:
            raise RuntimeError("batch did not converge")
    sampler = ClockSampler(dev)
    sampler.start()
    l0 = hplai.launch_count()
    times = []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rc = bt.solve()
        e1.record(stream)
        e1.synchronize()
        if rc != hplai.HPLAI_OK:
            raise RuntimeError("batch did not converge")
        times.append(e0.elapsed_time(e1))
    launches = hplai.launch_count() - l0
    clocks = sampler.stop()
    worst = max(bt.result(s).hpl_harness for s in range(count))
    graph_launches = bt.launches()
    bt.close()
    total_ms = sum(times)
    value, max_ms = replica_value(total_ms, args.steps * flops, world, device="cuda")
    if rank == 0:
        xbytes = int(sum(int(v) * int(r) * 8 for v, r in zip(n, nrhs)))
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp16/fp32/fp64",
            "data": f"synthetic (LCG matrices, system s seeded with s; sizes from host generator seed {args.batch_seed})",
            "config": {"workload": f"batched: {count} systems, n log-uniform 256..4096 (round 64), 1..8 "
                                   f"right-hand sides each, plain form + IR", "systems": count,
                       "n_total": int(n.sum()), "rhs_total": int(nrhs.sum()),
                       "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"},
            "systems_per_s": world * count * args.steps / (max_ms / 1e3),
            "worst_hpl_harness": worst, "create_s": create_s, "gpu_launches": int(launches),
            "launches_per_solve": int(launches) // max(args.steps, 1),
            "graph_kernel_nodes": graph_launches,
            "engine": "batched engine: every kernel over all systems (128-wide panels, identity padding), generation "
                      "+ factorisation one CUDA graph, refinement steps until every right-hand side is below 16"
            if graph_launches else "per-system contexts fed by host worker threads",
            "clocks": clocks,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": int(count * 16),
                    "d2h_bytes_per_step": xbytes,
                    "note": "the batched call itself: sizes and seeds in, every solution vector out"},
        }), flush=True)
    return 0


def run_adjoint(args):
    """Forward solve and adjoint (transposed) solve of one system, n = 8192,
    b = 256 by default: factor + A x = b + A^T lambda = x - x_t, the adjoint
    of L = 0.5 ||x - x_t||^2 with x_t ~ U[-1, 1)."""
    import torch
    import numpy as np
    torch.cuda.set_device(0)
    import hplai
    n, b = args.n, args.b
    rng = np.random.default_rng(2024)
    bvec = rng.uniform(-1, 1, n)
    xt = rng.uniform(-1, 1, n)
    s = hplai.Solver(n, b)
    ext = torch.cuda.ExternalStream(s.stream())
    res = []
    for i in range(args.warmup + args.steps):
        s.generate(42)
        torch.cuda.synchronize()
        e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        e[0].record(ext)
        s.factor()
        e[1].record(ext)
        x, r1 = s.solve_rhs(bvec)
        e[2].record(ext)
        lam, r2 = s.solve_transpose(x - xt)
        e[3].record(ext)
        e[3].synchronize()
        if r1.status != hplai.HPLAI_OK or r2.status != hplai.HPLAI_OK:
            raise RuntimeError("adjoint solve did not converge")
        if i >= args.warmup:
            res.append([e[0].elapsed_time(e[1]), e[1].elapsed_time(e[2]), e[2].elapsed_time(e[3]), r2.hpl_harness])
    s.close()
    arr = np.array(res)
    fl = hpl_flops(n)
    print(json.dumps({
        "metric": METRIC, "value": fl / (arr[:, 0].sum() + arr[:, 1].sum()) * len(res) * 1e-6, "unit": UNIT,
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": float(arr[:, :3].sum(1).mean()), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp16/fp32/fp64", "data": "synthetic (LCG matrix seed 42; b, x_t ~ U[-1,1) seed 2024)",
        "config": {"workload": f"adjoint of 0.5|x - x_t|^2: factor, A x = b and A^T lambda = x - x_t at n={n} b={b}",
                   "n": n, "b": b},
        "factor_ms": float(arr[:, 0].mean()), "forward_solve_ms": float(arr[:, 1].mean()),
        "adjoint_solve_ms": float(arr[:, 2].mean()), "adjoint_hpl_harness": float(arr[-1, 3]),
    }), flush=True)
    return 0


def run_gemm(args):
    """The Schur GEMM alone through its leaf entry point: C (m x n FP32) -= L U
    with FP16 (or e4m3) panels of width k, C larger than L2; with --deck on,
    the FP16 deck form deck -= dscale L U."""
    import torch
    torch.cuda.set_device(0)
    import hplai
    m, n, k = args.m, args.n_cols, args.k
    fp8 = args.precision == "f8"
    hplai.set_cta_pairs_default(args.pairs != "off")
    torch.manual_seed(0)
    ldc = (m + 63) // 64 * 64 + 64   # the solver's padded leading dimension (no power-of-two stride)
    deck = args.deck == "on"
    # FP32 C, or the FP16 deck of the lazy form (updated as deck - dscale * L U)
    c = torch.zeros(n, ldc, dtype=torch.float16 if deck else torch.float32, device="cuda")
    dscale = 2.0 ** -8
    if fp8:
        ld = (k + 127) // 128 * 128
        lp = (torch.rand(m, ld, device="cuda") * 4).to(torch.float8_e4m3fn).view(torch.uint8)
        up = (torch.rand(n, ld, device="cuda") * 4).to(torch.float8_e4m3fn).view(torch.uint8)
        sl = torch.ones((m + 127) // 128, device="cuda")
        su = torch.ones((n + 127) // 128, device="cuda")

        def call():
            if deck:
                hplai.check(hplai.f8gemm_deck_minus(m, n, k, lp.data_ptr(), ld, sl.data_ptr(), up.data_ptr(), ld,
                                                    su.data_ptr(), c.data_ptr(), ldc, dscale, None))
            else:
                hplai.check(hplai.f8gemm_minus(m, n, k, lp.data_ptr(), ld, sl.data_ptr(), up.data_ptr(), ld,
                                               su.data_ptr(), c.data_ptr(), ldc, None))
    else:
        ld = (k + 63) // 64 * 64
        lp = torch.rand(m, ld, device="cuda").half()
        up = torch.rand(n, ld, device="cuda").half()

        def call():
            if deck:
                hplai.check(hplai.shgemm_deck_minus(m, n, k, lp.data_ptr(), ld, up.data_ptr(), ld, c.data_ptr(), ldc,
                                                    dscale, None))
            else:
                hplai.check(hplai.shgemm_minus(m, n, k, lp.data_ptr(), ld, up.data_ptr(), ld, c.data_ptr(), ldc,
                                               None))
    for _ in range(args.warmup):
        call()
    torch.cuda.synchronize()
    sampler = ClockSampler(0)
    sampler.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        call()
    e1.record()
    e1.synchronize()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1) / args.steps
    flops = 2.0 * m * n * k
    byts = (4.0 if deck else 8.0) * m * n + (m + n) * k * (1 if fp8 else 2)
    cform = "FP16 deck" if deck else "FP32 C"
    if deck:
        cform += ", CTA pairs" if args.pairs != "off" else ", single CTAs"
    print(json.dumps({"workload": f"schur GEMM leaf m={m} n={n} k={k} {'e4m3' if fp8 else 'fp16'} {cform}",
                      "ms_per_launch": ms, "tflops": flops / ms / 1e9, "gbs": byts / ms / 1e6,
                      "algorithmic_bytes": byts, "flops": flops, "clocks": clocks}), flush=True)
    return 0


def run_check(args):
    """The factored-matrix checksum (panel_check.hpp:9-65) alone through its
    leaf entry point: one read of an n x n FP32 matrix (4 n^2 bytes, larger
    than L2 at the default n) into three FP64 sums; reports GB/s of that read."""
    import torch
    torch.cuda.set_device(0)
    import hplai
    n = args.n
    lda = (n + 63) // 64 * 64 + 64   # the solver's padded leading dimension
    torch.manual_seed(0)
    a = torch.rand(n, lda, device="cuda") - 0.5
    ws = hplai.panel_check_workspace(n)
    work = torch.empty(ws // 8 + 1, dtype=torch.float64, device="cuda")
    sig = torch.empty(3, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()

    def call():
        hplai.check(hplai.panel_check(n, a.data_ptr(), lda, sig.data_ptr(), work.data_ptr(), ws, stream.cuda_stream))
    for _ in range(args.warmup):
        call()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        call()
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    byts = 4.0 * n * n
    print(json.dumps({"workload": f"panel_check leaf n={n} lda={lda} FP32", "ms_per_launch": ms,
                      "gbs": byts / ms / 1e6, "algorithmic_bytes": byts}), flush=True)
    return 0


def run_peak(args):
    """Dense tensor-core peaks of this GPU as cuBLAS reaches them (torch
    matmul in bf16, torch._scaled_mm in e4m3 with FP32 scales, bf16 out),
    M = N = K = 8192: the best of 10 launches (burst) and the mean over 4 s
    back to back (sustained, under the power cap).  A measurement of the
    denominator only: no product path calls these."""
    import torch
    torch.cuda.set_device(0)
    m = 8192
    fl = 2.0 * m * m * m
    a = torch.randn(m, m, device="cuda").to(torch.bfloat16)
    bm = torch.randn(m, m, device="cuda").to(torch.bfloat16)
    a8 = a.to(torch.float8_e4m3fn)
    b8 = bm.to(torch.float8_e4m3fn).t()   # column-major operand
    one = torch.ones((), device="cuda")
    kinds = {"bf16": lambda: torch.matmul(a, bm),
             "e4m3": lambda: torch._scaled_mm(a8, b8, scale_a=one, scale_b=one, out_dtype=torch.bfloat16)}
    out = {"gpu": torch.cuda.get_device_name(0), "m": m, "n": m, "k": m}
    sampler = ClockSampler(0)
    sampler.start()
    for name, fn in kinds.items():
        for _ in range(5):
            fn()
        torch.cuda.synchronize()
        best = float("inf")
        for _ in range(10):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        reps, t_end = 0, time.perf_counter() + 4.0
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        while time.perf_counter() < t_end:
            for _ in range(20):
                fn()
            reps += 20
            torch.cuda.synchronize()
        e1.record()
        e1.synchronize()
        out[name] = {"burst_tflops": fl / best / 1e9, "sustained_tflops": fl * reps / e0.elapsed_time(e1) / 1e9,
                     "sustained_launches": reps}
    out["clocks"] = sampler.stop()
    print(json.dumps(out), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--n", type=int, default=None, help="order (default 131072; 8192 for the adjoint workload)")
    ap.add_argument("--b", type=int, default=None, help="block size (default 1024; 256 for the adjoint workload)")
    ap.add_argument("--e2e-warmup", type=int, default=1)
    ap.add_argument("--e2e-steps", type=int, default=5, help="end-to-end solves timed (at most --steps)")
    ap.add_argument("--forms", choices=("both", "precision", "plain"), default="both",
                    help="solve workload: the precision form (headline) and the plain form back to back, or one")
    ap.add_argument("--compare-steps", type=int, default=8, help="timed solves of the comparison form (at most --steps)")
    ap.add_argument("--compare-warmup", type=int, default=2)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--precision", choices=("f16", "f8"), default=None,
                    help="override the headline form's Schur operands: FP16 or e4m3 with per-128 factors")
    ap.add_argument("--workload", choices=("solve", "batch", "adjoint", "gemm", "check", "peak"), default="solve",
                    help="solve: one system (default n=131072 b=1024, precision and plain forms); batch: many "
                         "systems; adjoint: forward + transposed solves; gemm / check: the Schur GEMM or the "
                         "factor checksum leaf alone; peak: cuBLAS bf16/e4m3 dense rates (the roofline denominators)")
    ap.add_argument("--pairs", choices=("on", "off"), default="off",
                    help="deck updates on CTA pairs (tcgen05 cta_group::2) or single CTAs")
    ap.add_argument("--lazy-a", action="store_true",
                    help="headline form without a stored A (HPLAI_FLAG_LAZY_A; e4m3 + FP16 deck, LCG matrix)")
    ap.add_argument("--matrix", choices=("lcg", "higham"), default="lcg",
                    help="solve workload: the benchmark's LCG matrix or Higham's (the reference's --highammat)")
    ap.add_argument("--m", type=int, default=16384, help="gemm workload: rows of C")
    ap.add_argument("--n-cols", type=int, default=16384, help="gemm workload: columns of C")
    ap.add_argument("--k", type=int, default=512, help="gemm workload: panel width")
    ap.add_argument("--batch-count", type=int, default=512)
    ap.add_argument("--batch-seed", type=int, default=20240611)
    ap.add_argument("--batch-workers", type=int, default=8)
    ap.add_argument("--deck", choices=("on", "off"), default=None,
                    help="override the headline form's trailing matrix: FP16 deck (HPLAI_FLAG_FP16_DECK) or FP32")
    ap.add_argument("--autotune", action="store_true",
                    help="choose the schedule (serial or look-ahead, side-stream SMs) with hplai_autotune first "
                         "(the default for the solve workload unless --lookahead or --no-autotune is given)")
    ap.add_argument("--no-autotune", action="store_true", help="keep the serial schedule (or --lookahead's)")
    ap.add_argument("--side-sms", type=int, default=32, help="SMs of the side stream with --lookahead (no autotune)")
    ap.add_argument("--group", type=int, choices=(1, 2, 4), default=1,
                    help="panels per trailing update without autotuning (2 = HPLAI_FLAG_GROUP2, 4 = HPLAI_FLAG_GROUP4; "
                         "b %% 128 == 0)")
    ap.add_argument("--lookahead", action="store_true",
                    help="form the next step's diagonal block and panels on a side stream (HPLAI_FLAG_LOOKAHEAD)")
    ap.add_argument("--refine", choices=("ir", "gmres"), default=None,
                    help="override the headline form's correction: classical IR or GMRES")
    args = ap.parse_args()
    if not args.lookahead and not args.no_autotune and args.group == 1:
        args.autotune = True
    if args.n is None:
        args.n = ADJOINT_N if args.workload == "adjoint" else DEFAULT_N
    if args.b is None:
        args.b = ADJOINT_B if args.workload == "adjoint" else DEFAULT_B
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "adjoint":
        return run_adjoint(args)
    if args.workload == "gemm":
        return run_gemm(args)
    if args.workload == "check":
        return run_check(args)
    if args.workload == "peak":
        return run_peak(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
