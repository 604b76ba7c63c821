"""Benchmark of the DF J/K path: one line of JSON on rank 0.

A step is one complete density-fitting J/K build of a seeded water cluster
(default (H2O)_16: 480 spherical AOs, 2256 spherical auxiliary functions, 80
occupied orbitals): the (P|Q) metric and its factor, the 3-center integrals,
B = (ij|P) L, then J and K of D = C C^T. Inputs (basis arrays, C) are resident
before the timed region; the fitted 3-center tensor (1.9 GB for (H2O)_16) is
larger than L2, so no explicit flush is needed between steps.

The headline (``--precision both``, the default) is the mixed-precision form
(int8 tensor-core products with exact accumulation; integrals, metric and J
in float64); the float64 form of the same step is timed in the same run and
reported under ``fp64``, with |dE|, max|dJ| and max|dK| of the mixed result
against it under ``accuracy_vs_fp64``.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--workload water16] [--precision both|mixed|fp64]

N > 1 runs under torchrun, one rank per GPU; each rank builds its own cluster
(seeded by rank): the path has no exchange between molecules, so the ranks are
independent replicas and ``value`` sums their builds ("scaling": "weak").
``--impl reference`` times full builds of the same workload by the compiled
CPU restatement of dftax's DF path (oracle/cpu.py: C++ integrals on all host
threads, then dftax's metric pseudo-inverse and J/K contractions with numpy),
W untimed and K timed, on rank 0.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "DF J/K builds/s"
UNIT = "builds/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="water16")
    ap.add_argument("--precision", default="both", choices=["both", "fp64", "mixed"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--scf-steps", type=int, default=2,
                    help="timed SCF solves per precision (0: no SCF measurement)")
    ap.add_argument("--serve-requests", type=int, default=16,
                    help="requests of the seeded Poisson serving stream (0: none)")
    ap.add_argument("--serve-rate", type=float, default=4.0, help="arrivals per second")
    ap.add_argument("--serve-sweep", default="16",
                    help="further arrival rates (comma separated) replayed after --serve-rate; "
                         "empty for none")
    ap.add_argument("--serve-max-water", type=int, default=12,
                    help="largest water cluster of the stream (log-uniform from 3)")
    ap.add_argument("--serve-max-alkane", type=int, default=8,
                    help="largest alkane of the stream (log-uniform from 4)")
    ap.add_argument("--batch", type=int, default=0,
                    help="also solve a batch of this many water clusters (64: the 64-cluster "
                         "batch, n log-uniform in [3, 40])")
    ap.add_argument("--workers", type=int, default=4, help="concurrent solves of the engine")
    ap.add_argument("--build-batch", type=int, default=64,
                    help="water clusters of the batched-build measurement (0: off)")
    ap.add_argument("--guess", default="sad", choices=["sad", "core"],
                    help="SCF starting density of the SCF, serving and batch measurements")
    ap.add_argument("--screen", type=float, default=0.0,
                    help="relative Schwarz screen of shell pairs (0: none, the default)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# CPU baseline: full builds by the compiled CPU restatement of dftax's path
# ---------------------------------------------------------------------------

def cpu_full_builds(workload: str, nbuild: int, nwarm: int = 0, seed: int = 0):
    """Seconds of each of ``nbuild`` complete DF J/K builds of the workload by
    oracle/cpu.py (after ``nwarm`` untimed ones), and the parts of the last.

    Each build computes the metric, its pseudo-inverse, the dense 3-center
    tensor and J, K of D = C C^T as dftax's materialized path does, on all host
    threads (C++ integrals; numpy/OpenBLAS eigh and GEMMs)."""
    from threadpoolctl import threadpool_limits

    from dftax_b200 import systems
    from oracle import cpu as ocpu

    sym, xyz, orb, aux, nocc = systems.workload(workload, seed=seed)
    C = systems.random_occupied(orb.nao, nocc, seed=100 + seed)
    n = ocpu.threads()
    secs, parts = [], {}
    with threadpool_limits(n):
        for i in range(nwarm + nbuild):
            t0 = time.perf_counter()
            r = ocpu.df_build_jk(orb, aux, C, nthreads=n)
            dt = time.perf_counter() - t0
            if i >= nwarm:
                secs.append(dt)
                parts = r["seconds"]
    return secs, parts, n


def cpu_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------

class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                c = [x.strip() for x in line.split(",")]
                if len(c) >= 9 and c[0] == str(self.index):
                    rows.append(c)
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------

def measured_peaks():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


def measured_sustained_bf16():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            return json.load(fh).get("bf16_tflops_sustained")
    return 1400.0


def fp64_gemm_peak(torch):
    """Burst FP64 GEMM rate (cuBLAS DGEMM 8192^3, best of 5) in TFLOP/s."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        a @ b
    best = 1e30
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        a @ b
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e))
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def load_traffic(key: str, nrows: int, naux: int, ldb: int, digits: int):
    """DRAM bytes of the dominant kernel's launches in this step, from one ncu
    capture (profiles/traffic.json) by its measured-over-algorithmic ratio
    (digit planes of the raw rows read, float64 B written); the ratio is
    scaled to this workload's rows and row size when the capture was of
    another workload."""
    p = os.path.join(HERE, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as fh:
        d = json.load(fh).get(key)
    if d is None:
        return None
    naux16 = (naux + 15) // 16 * 16
    alg = nrows * (digits * naux16 + 8 * ldb)
    return {"bytes": round(d["ratio"] * alg), "algorithmic_bytes": alg,
            "source": f"ncu capture of {d['kernel']} on {d['workload']}: dram read+write "
                      f"{d['dram_bytes'] / 1e9:.3f} GB = {d['ratio']:.4f} x algorithmic; "
                      f"scaled to this workload's rows and row size"}


def int8_gemm_peak(torch):
    """Burst int8 tensor-core GEMM rate (torch._int_mm, cuBLASLt, 8192^3, best of 5) in TOP/s."""
    n = 8192
    try:
        a = torch.randint(-64, 64, (n, n), dtype=torch.int8, device="cuda")
        b = torch.randint(-64, 64, (n, n), dtype=torch.int8, device="cuda")
        for _ in range(2):
            torch._int_mm(a, b)
        best = 1e30
        for _ in range(5):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            torch._int_mm(a, b)
            e.record()
            torch.cuda.synchronize()
            best = min(best, s.elapsed_time(e))
        del a, b
        torch.cuda.empty_cache()
        return 2.0 * n ** 3 / (best * 1e-3) / 1e12, "in-bench cuBLASLt int8 GEMM 8192^3 burst"
    except Exception as ex:  # pragma: no cover - depends on the cuBLASLt build
        _, bf16, src = measured_peaks()
        return 2.0 * bf16, f"2 x {src} bf16 (int8 GEMM unavailable: {type(ex).__name__})"


def timed_steps(torch, step, steps, warmup, stream, barrier, lib):
    """W untimed steps, then K steps between CUDA events on the launching stream."""
    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    l0 = lib.dfjk_kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    return e0.elapsed_time(e1), (lib.dfjk_kernel_launches() - l0) // max(steps, 1)


def rank_sync(world, backend="nccl", device="cuda", local_rank=0):
    """(barrier, max_over_ranks, dist) for a run of `world` ranks, one per GPU
    (replicas: no collective in the measured work; the ranks only line up
    their timed regions and take the slowest one). `backend="gloo"` with
    `device="cpu"` serves the CPU test of this plumbing."""
    import datetime

    import torch

    dist = None
    if world > 1:
        import torch.distributed as dist

        kw = {"device_id": torch.device(f"cuda:{local_rank}")} if backend == "nccl" else {}
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=900), **kw)

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    return barrier, max_over_ranks, dist


def run_ours(args, rank, world, local_rank):
    import torch

    from dftax_b200 import Plan, _lib, systems

    torch.cuda.set_device(local_rank)
    barrier, max_over_ranks, dist = rank_sync(world, local_rank=local_rank)

    head = "mixed" if args.precision in ("both", "mixed") else "fp64"
    precs = [head] + (["fp64"] if args.precision == "both" else [])
    sym, xyz, orb, aux, nocc = systems.workload(args.workload, seed=rank)
    C = systems.random_occupied(orb.nao, nocc, seed=100 + rank)
    Cd = torch.as_tensor(C, device="cuda")
    stream = torch.cuda.current_stream()
    lib = _lib.load()
    res = {}
    for prec in precs:
        plan = Plan(orb, aux, precision=prec, screen=args.screen or None)
        J = torch.empty((orb.nao, orb.nao), dtype=torch.float64, device="cuda")
        K = torch.empty_like(J)

        def step():
            plan.build(stream)
            plan.jk(Cd, out=(J, K), stream=stream)

        clocks = Clocks(local_rank)
        clocks.start()
        ms, launches = timed_steps(torch, step, args.steps, args.warmup, stream, barrier, lib)
        clk = clocks.stop()
        ms = max_over_ranks(ms)
        phases = plan.phase_times()
        # per-iteration J/K with B resident (the SCF inner loop)
        jk_ms, _ = timed_steps(torch, lambda: plan.jk(Cd, out=(J, K), stream=stream), 5, 1, stream,
                               barrier, lib)
        jk_phases = plan.phase_times()
        P = 2.0 * Cd @ Cd.T
        e, _ = plan.energy(P, 0.25, want_grad=False, stream=stream)
        res[prec] = {"ms": ms, "launches": launches, "clocks": clk, "phases": phases,
                     "jk_ms": max_over_ranks(jk_ms / 5), "jk_phases": jk_phases, "info": plan.info(),
                     "J": J.cpu().numpy(), "K": K.cpu().numpy(), "E": e}
        plan.close()
        del plan, J, K
        torch.cuda.empty_cache()

    r = res[head]
    info = r["info"]
    value = world * args.steps / (r["ms"] / 1e3)

    # end to end through the public host API: host basis arrays and C in,
    # host J and K out, copies inside the timed region
    Jh = np.empty((orb.nao, orb.nao))
    Kh = np.empty_like(Jh)
    h2d = sum(a.nbytes for b in (orb, aux) for a in (b.centers, b.exponents, b.coefficients,
                                                      b.angular, b.cart2sph)) + C.nbytes
    d2h = Jh.nbytes + Kh.nbytes
    # one untimed step first, like the warm-up of the device-resident step (the
    # other precision's plans left differently sized buffers in the cache)
    p2 = Plan(orb, aux, precision=head, screen=args.screen or None)
    p2.build(stream)
    p2.jk_host(C, J=Jh, K=Kh, stream=stream)
    p2.close()
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.e2e_steps):
        p2 = Plan(orb, aux, precision=head, screen=args.screen or None)
        p2.build(stream)
        p2.jk_host(C, J=Jh, K=Kh, stream=stream)
        p2.close()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1))
    e2e_value = world * args.e2e_steps / (e2e_ms / 1e3)

    # roofline of the dominant phase of the headline precision
    hbm, bf16, src = measured_peaks()
    bf16_sus = measured_sustained_bf16()
    fp64 = fp64_gemm_peak(torch) if rank == 0 else None
    i8_bench, i8_src = int8_gemm_peak(torch) if rank == 0 else (None, "")
    i8 = 2.0 * bf16   # dense int8 tensor rate = 2 x dense bf16 on B200
    i8_src_line = f"2 x {src} bf16_tflops (burst): dense int8 = 2 x dense bf16"
    nrows, naux, nfit, nao = info["nrows"], info["naux"], info["nfit"], info["nao"]
    ldb = (nfit + 7) // 8 * 8
    nao_p = (nao + 15) // 16 * 16
    mixed = head == "mixed"
    dgemm = ("in-bench cuBLAS DGEMM 8192^3 burst (MEASURED_PEAKS.json has no float64 figure)")
    units = {
        "metric": ("tensor", (4.0 / 3.0 + 2.0) * naux ** 3 / 1e12, "TFLOP/s", fp64, dgemm,
                   "float64 FLOP of the eigensolver: 4/3 naux^3 (tridiagonalization) + "
                   "2 naux^3 (back-transformation), divide and conquer not counted"),
        "eri3c": ("hbm", 8.0 * nrows * naux / 1e9, "GB/s", hbm, f"{src} hbm_gbs",
                  "bytes of (ij|P) rows written"),
        "j": ("hbm", 2.0 * 8.0 * nrows * ldb / 1e9, "GB/s", hbm, f"{src} hbm_gbs",
              "B streamed twice"),
    }
    digits = 5 if mixed else 7
    products = digits * (digits + 1) // 2
    units["bgemm"] = ("tensor", products * 2.0 * nrows * naux * nfit / 1e12, "TOP/s", i8,
                      i8_src_line, f"int8 ops: {products} digit products x 2 nrows naux nfit "
                      f"({digits} digits per value)")
    if mixed:
        # tiles of 128 rows x 96 columns that reach the lower triangle (the others are skipped)
        elems = sum(min(128, nao - m0) * min(96, nao - n0)
                    for m0 in range(0, nao, 128) for n0 in range(0, nao, 96) if n0 <= m0 + 127)
        units["khalf"] = ("tensor", 10 * 2.0 * nfit * nao * nao * nocc / 1e12, "TOP/s", i8,
                          i8_src_line, "int8 ops: 10 digit products x 2 nfit nao^2 nocc")
        units["ksyrk"] = ("tensor", 15 * 2.0 * elems * nfit * nocc / 1e12, "TOP/s", i8,
                          i8_src_line, "int8 ops: 15 digit products x 2 nfit nocc x the "
                          "elements of the tiles that reach the lower triangle")
        units["kplanes"] = ("hbm", (2 * 8.0 * (2 * nrows - nao) * nfit + 4.0 * nfit * nao * nao_p) / 1e9,
                            "GB/s", hbm, f"{src} hbm_gbs",
                            "B gathered twice per AO list + 4 int8 digit planes written")
    else:
        units["khalf"] = ("tensor", 2.0 * (2 * nrows - nao) * nfit * nocc / 1e12, "TFLOP/s", fp64,
                          dgemm, "2 sum_m |list(m)| nfit nocc")
        units["ksyrk"] = ("tensor", 1.0 * nao * (nao + 1) * nfit * nocc / 1e12, "TFLOP/s", fp64,
                          dgemm, "nao (nao+1) nfit nocc (lower tiles)")
    phases = {k: v for k, v in r["phases"].items() if k not in ("j", "khalf", "ksyrk")}
    phases |= {k: r["jk_phases"][k] for k in ("j", "khalf", "ksyrk")}
    total = sum(phases.values())
    dom = max(units, key=lambda k: phases.get(k, 0.0))
    bound, amount, unit, peak, peak_src, what = units[dom]
    achieved = amount / (phases[dom] / 1e3) if phases[dom] > 0 else 0.0
    roof = {"kernel": dom, "bound": bound,
            "achieved": round(achieved, 3), "peak": round(peak, 3) if peak else None, "unit": unit,
            "frac": round(achieved / peak, 4) if peak else None, "peak_source": peak_src,
            "algorithmic": what, "ms_per_launch_group": round(phases[dom], 3),
            "share_of_step": round(phases[dom] / total, 4) if total > 0 else None,
            "traffic": None}
    if unit == "TOP/s":
        roof["frac_vs_sustained"] = round(achieved / (2.0 * bf16_sus), 4) if bf16_sus else None
        roof["frac_vs_in_bench_int8"] = round(achieved / i8_bench, 4) if i8_bench else None
        roof["in_bench_int8_peak"] = round(i8_bench, 3) if i8_bench else None
        roof["in_bench_int8_source"] = i8_src
    if dom == "bgemm":
        roof["fp64_equivalent_tflops"] = round(2.0 * nrows * naux * nfit / (phases[dom] / 1e3) / 1e12, 3)
    tr = load_traffic(f"bgemm@{head}", nrows, naux, ldb, digits) if dom == "bgemm" else None
    if tr is not None:
        # bytes of the phase's int8 GEMM launches (all raw-row chunks), like `achieved`
        roof["traffic"] = tr["bytes"]
        roof["traffic_algorithmic"] = tr["algorithmic_bytes"]
        roof["traffic_source"] = tr["source"]
    # every phase against its own roofline, largest first
    per_phase = {}
    for k in sorted(units, key=lambda k: -phases.get(k, 0.0)):
        if phases.get(k, 0.0) <= 0:
            continue
        b_, amt, u_, pk, _, _ = units[k]
        ach = amt / (phases[k] / 1e3)
        per_phase[k] = {"ms": round(phases[k], 3), "achieved": round(ach, 3), "unit": u_,
                        "frac": round(ach / pk, 4) if pk else None}

    line = {
        "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(r["ms"] / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64+i8" if mixed else "f64", "data": "synthetic",
        "config": workload_config(args, orb, aux, nocc, world),
        "precision": head, "nfit": nfit, "nrows": nrows,
        "phases_ms": {k: round(v, 3) for k, v in phases.items()},
        "phase_share": {k: round(v / total, 4) for k, v in phases.items()} if total > 0 else {},
        "jk_iteration": {"value": round(1e3 / r["jk_ms"], 3), "unit": "J/K builds/s with B resident",
                         "ms": round(r["jk_ms"], 3)},
        "e2e": {"value": round(e2e_value, 4), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(r["launches"]),
        "roofline": roof,
        "roofline_by_phase": per_phase,
        "clocks": r["clocks"],
    }
    if "fp64" in res and head != "fp64":
        f = res["fp64"]
        line["fp64"] = {"value": round(world * args.steps / (f["ms"] / 1e3), 4), "unit": UNIT,
                        "ms_per_step": round(f["ms"] / args.steps, 3),
                        "jk_iteration_ms": round(f["jk_ms"], 3),
                        "phases_ms": {k: round(v, 3) for k, v in f["phases"].items()
                                      if k not in ("j", "khalf", "ksyrk", "kplanes")}
                        | {k: round(f["jk_phases"][k], 3) for k in ("j", "khalf", "ksyrk")},
                        "clocks": f["clocks"], "gpu_launches": int(f["launches"])}
        line["speedup_vs_fp64"] = {"build_and_jk": round(f["ms"] / r["ms"], 3),
                                   "jk_iteration": round(f["jk_ms"] / r["jk_ms"], 3)}
        line["accuracy_vs_fp64"] = {
            "abs_dE_Ha": abs(r["E"] - f["E"]), "E_fp64_Ha": f["E"],
            "max_abs_dJ": float(np.abs(r["J"] - f["J"]).max()),
            "max_abs_dK": float(np.abs(r["K"] - f["K"]).max()),
            "rel_dJ": float(np.linalg.norm(r["J"] - f["J"]) / np.linalg.norm(f["J"])),
            "rel_dK": float(np.linalg.norm(r["K"] - f["K"]) / np.linalg.norm(f["K"])),
            "energy": "DFCoulomb energy of P = 2 C C^T with a_x = 0.25 (PBE0 exchange share)"}
    if args.scf_steps > 0:
        line["scf"] = scf_measure(args, torch, precs, sym, xyz, orb, aux, world, max_over_ranks)
    if args.serve_requests > 0:
        line["serve"] = serve_measure(args, precs, rank)
        sweep = []
        for rate in [float(x) for x in args.serve_sweep.split(",") if x.strip()]:
            r = serve_measure(args, precs, rank, rate=rate)
            sweep.append({"rate_per_s": rate,
                          **{k: r[k] for k in ("value", "p50_latency_s", "p99_latency_s",
                                               "failed", "max_concurrent")},
                          "fp64": {k: r["fp64"][k] for k in ("value", "p50_latency_s",
                                                             "p99_latency_s", "failed")}
                          if "fp64" in r else None})
        if sweep:
            line["serve"]["sweep"] = sweep
    if args.batch > 0:
        line["batch"] = batch_measure(args, precs, rank)
    if args.build_batch > 0:
        line["build_batch"] = build_batch_measure(args, precs, rank)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        secs, parts, n = cpu_full_builds(args.workload, 1)
        line["cpu_baseline"] = {"value": round(1.0 / secs[0], 6), "unit": UNIT, "cores": n,
                                "kind": "port",
                                "sample": "one complete build of the same workload (same geometry "
                                          "and C) by the compiled CPU restatement: C++ integrals, "
                                          "numpy eigh and dftax's J/K contractions",
                                "parts_s": {k: round(v, 3) for k, v in parts.items()}}
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def scf_measure(args, torch, precs, sym, xyz, orb, aux, world, max_over_ranks):
    """SCF solves/s of the workload from geometry, per precision: the DF plan
    and build, the Becke grid (75 radial shells, 302-point Lebedev, NWChem
    pruning), one-electron integrals and the DIIS iterations of a closed-shell
    DF-PBE0 SCF from the --guess density (``sad``: superposition of atomic
    densities, the per-element atomic solves cached by the untimed first
    solve, their assembly timed; ``core``: the core Hamiltonian), to
    |dE| < 1e-8 Ha and a commutator below 1e-6 (dftax's defaults)."""
    from dftax_b200 import df
    from dftax_b200.ks import KS, scf

    out = {}
    res = {}
    for prec in precs:
        def solve():
            ks = KS(sym, xyz, orb, coulomb=df(aux, precision=prec))
            r = scf(ks, guess=args.guess)
            ks.close()
            ks.plan.close()
            return r

        solve()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rs = [solve() for _ in range(args.scf_steps)]
        torch.cuda.synchronize()
        sec = max_over_ranks(time.perf_counter() - t0)
        r = rs[-1]
        res[prec] = r
        it_ms = sum(r.timings_ms.values())
        out[prec] = {"value": round(world * args.scf_steps / sec, 4), "unit": "SCF solves/s",
                     "ms_per_solve": round(1e3 * sec / args.scf_steps, 2),
                     "n_iter": r.n_iter, "converged": r.converged, "e_tot_Ha": r.e_tot,
                     "iteration_parts_ms": {k: round(v, 2) for k, v in r.timings_ms.items()},
                     "xc_chunk_points": r.xc_chunk, "xc_cuda_graph": r.xc_graph,
                     # the two float64 DGEMMs per XC chunk, over the whole XC time
                     # (which also holds the AO, density and functional kernels)
                     "xc_dgemm": {"tflop_per_evaluation": round(r.xc_gemm_flop / 1e12, 4),
                                  "evaluations": r.n_iter + 1,
                                  "tflop_s_over_xc_time": round(
                                      r.xc_gemm_flop * (r.n_iter + 1)
                                      / max(r.timings_ms["xc"], 1e-9) / 1e9, 2)},
                     "eigensolver_densities": r.n_eig,
                     "setup_ms": round(1e3 * sec / args.scf_steps - it_ms, 2)}
    head = precs[0]
    line = dict(out[head])
    line["precision"] = head
    line["guess"] = args.guess
    line["what"] = ("one closed-shell DF-PBE0 SCF from geometry: plan and DF build, Becke grid "
                    f"(75 x 302, NWChem pruning), one-electron integrals, {args.guess} guess, "
                    "DIIS to |dE| < 1e-8 Ha and commutator < 1e-6")
    if "fp64" in out and head != "fp64":
        line["fp64"] = out["fp64"]
        line["speedup_vs_fp64"] = round(out["fp64"]["ms_per_solve"] / out[head]["ms_per_solve"], 3)
        line["abs_dE_vs_fp64_Ha"] = abs(res[head].e_tot - res["fp64"].e_tot)
    return line


def _loguniform_ints(rng, lo, hi, n):
    return np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi + 1), n))).astype(int)


def _requests(eng, mols, grids, prec, guess=None):
    return [eng.request(s, x, o, a, grid=g, precision=prec, guess=guess)
            for (s, x, o, a), g in zip(mols, grids)]


def serve_measure(args, precs, rank, rate=None):
    """A seeded Poisson stream of SCF requests (water clusters, n log-uniform
    in [3, serve-max-water], and alkanes, n log-uniform in [4, serve-max-alkane],
    half each) through the batch engine: each request is submitted at its
    arrival time while earlier ones run, admitted FIFO as device memory frees
    up. Solves/s = requests / (last completion - first arrival); latency =
    completion - arrival. Grids (Becke 75 x 302) are built before the stream
    starts; one untimed pass of the requests warms the engine first. The same
    stream is replayed per precision."""
    from dftax_b200 import systems
    from dftax_b200.batch import BatchEngine
    from dftax_b200.grid import becke_grid

    rng = np.random.default_rng(50 + rank)
    n = args.serve_requests
    kinds = rng.integers(0, 2, n)
    wn = _loguniform_ints(rng, 3, args.serve_max_water, n)
    an = _loguniform_ints(rng, 4, args.serve_max_alkane, n)
    rate = rate or args.serve_rate
    gaps = rng.exponential(1.0 / rate, n)
    mols, names = [], []
    for i in range(n):
        name = f"water{wn[i]}" if kinds[i] == 0 else f"alkane{an[i]}"
        sym, xyz, orb, aux, _ = systems.workload(name, seed=1000 + i)
        mols.append((sym, xyz, orb, aux))
        names.append(name)
    grids = [becke_grid(m[0], m[1]) for m in mols]
    out, energies, ok_mask = {}, {}, {}
    for prec in precs:
        with BatchEngine(workers=args.workers) as eng:
            reqs = _requests(eng, mols, grids, prec, args.guess)
            # one untimed pass, all at once: the XC chunk autotuner settles its
            # per-size choices and the device-memory cache fills, as in a
            # server that has been running
            for i in [eng.submit_request(r) for r in reqs]:
                eng.wait(i)
            ids = []
            t0 = time.perf_counter()
            for i, req in enumerate(reqs):
                due = t0 + float(np.sum(gaps[:i]))
                time.sleep(max(0.0, due - time.perf_counter()))
                ids.append(eng.submit_request(req))
            res = [eng.wait(i) for i in ids]
        ok = [r for r in res if r.status == 0]
        lat = np.array([r.latency for r in ok])
        span = max(r.t_end for r in ok) - min(r.t_submit for r in ok)
        energies[prec] = [r.e_tot for r in res]
        ok_mask[prec] = [r.status == 0 for r in res]
        out[prec] = {"value": round(len(ok) / span, 4), "unit": "SCF solves/s",
                     "p50_latency_s": round(float(np.percentile(lat, 50)), 3),
                     "p99_latency_s": round(float(np.percentile(lat, 99)), 3),
                     "failed": len(res) - len(ok),
                     "failures": [{"molecule": names[i], "status": r.status,
                                   "message": r.message[:160]}
                                  for i, r in enumerate(res) if r.status != 0][:4],
                     "converged": int(sum(r.converged for r in ok)),
                     "max_concurrent": max(sum(1 for q in res if q.t_start <= r.t_start < q.t_end)
                                           for r in res)}
    head = precs[0]
    line = dict(out[head])
    line["precision"] = head
    line["stream"] = {"requests": n, "rate_per_s": rate, "workers": args.workers,
                      "water_n": [3, args.serve_max_water], "alkane_n": [4, args.serve_max_alkane],
                      "molecules": names, "seed": 50 + rank,
                      "guess": args.guess,
                      "what": "closed-shell DF-PBE0 SCF per request, Becke 75 x 302 grid"}
    if "fp64" in out and head != "fp64":
        line["fp64"] = out["fp64"]
        both = [i for i in range(n) if ok_mask[head][i] and ok_mask["fp64"][i]]
        line["max_abs_dE_vs_fp64_Ha"] = (float(np.max(np.abs(
            np.array(energies[head])[both] - np.array(energies["fp64"])[both]))) if both else None)
    return line


def build_batch_measure(args, precs, rank):
    """DF builds of many small molecules: water clusters, n log-uniform in
    [3, 12] (seeded), plans made up front (untimed); the same builds timed one
    plan after another (dfjk_build each) and all together (dfjk_build_batch:
    one launch per light integral class for every molecule). CUDA events on
    the stream around each way, after one untimed round."""
    import torch

    from dftax_b200 import Plan, systems
    from dftax_b200._lib import load

    lib = load()
    rng = np.random.default_rng(12 + rank)
    ns = _loguniform_ints(rng, 3, 12, args.build_batch)
    out = {}
    for prec in precs:
        plans = []
        for i, n in enumerate(ns):
            _, _, orb, aux, _ = systems.workload(f"water{n}", seed=3000 + i)
            plans.append(Plan(orb, aux, precision=prec))
        res = {}
        for way in ("single", "batched"):
            def run():
                if way == "single":
                    for p in plans:
                        p.build()
                else:
                    Plan.build_many(plans)
            run()
            torch.cuda.synchronize()
            k0 = lib.dfjk_kernel_launches()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            run()
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            res[way] = {"value": round(len(plans) / (ms / 1e3), 3), "unit": "builds/s",
                        "ms": round(ms, 2),
                        "kernel_launches": int(lib.dfjk_kernel_launches() - k0)}
        res["speedup"] = round(res["single"]["ms"] / res["batched"]["ms"], 3)
        for p in plans:
            p.close()
        out[prec] = res
    head = precs[0]
    line = dict(out[head])
    line["precision"] = head
    line["molecules"] = {"count": int(args.build_batch), "n": ns.tolist(), "seed": 12 + rank,
                         "what": "one DF build (metric, 3-center rows, B) per water cluster"}
    if "fp64" in out and head != "fp64":
        line["fp64"] = out["fp64"]
    return line


def batch_measure(args, precs, rank):
    """A batch of water clusters, n log-uniform in [3, 40] (seeded), all
    submitted at once to the batch engine: solves/s = clusters / (last
    completion - first submission), per-molecule |dE| of the headline precision
    against float64."""
    from dftax_b200 import systems
    from dftax_b200.batch import BatchEngine
    from dftax_b200.grid import becke_grid

    rng = np.random.default_rng(64 + rank)
    ns = _loguniform_ints(rng, 3, 40, args.batch)
    mols = []
    for i, n in enumerate(ns):
        sym, xyz, orb, aux, _ = systems.workload(f"water{n}", seed=2000 + i)
        mols.append((sym, xyz, orb, aux))
    grids = [becke_grid(m[0], m[1]) for m in mols]
    out, energies = {}, {}
    for prec in precs:
        with BatchEngine(workers=args.workers) as eng:
            t0 = time.perf_counter()
            ids = [eng.submit(*m, grid=g, precision=prec, guess=args.guess)
                   for m, g in zip(mols, grids)]
            res = [eng.wait(i) for i in ids]
            sec = time.perf_counter() - t0
        energies[prec] = np.array([r.e_tot for r in res])
        out[prec] = {"value": round(len(res) / sec, 4), "unit": "SCF solves/s",
                     "seconds": round(sec, 2),
                     "failed": int(sum(r.status != 0 for r in res)),
                     "failures": [{"n": int(ns[i]), "status": r.status, "message": r.message[:160]}
                                  for i, r in enumerate(res) if r.status != 0][:4],
                     "converged": int(sum(r.converged for r in res))}
    head = precs[0]
    line = dict(out[head])
    line["precision"] = head
    line["clusters"] = {"count": int(args.batch), "n": ns.tolist(), "seed": 64 + rank,
                        "workers": args.workers, "guess": args.guess}
    if "fp64" in out and head != "fp64":
        line["fp64"] = out["fp64"]
        d = np.abs(energies[head] - energies["fp64"])
        line["abs_dE_vs_fp64_Ha"] = {"max": float(d.max()), "median": float(np.median(d)),
                                     "all_below_1uHa": bool(np.all(d < 1e-6))}
    return line


def workload_config(args, orb, aux, nocc, world):
    """The workload as both arms name it (identical dicts)."""
    nao, naux = orb.nao, aux.nao
    gb = 8.0 * nao * (nao + 1) / 2 * naux / 1e9
    return {"workload": f"{args.workload} one DF J/K build from geometry (seeded)",
            "nao": nao, "naux": naux, "nocc": nocc, "screen": args.screen,
            "parallelism": f"replicas x{world}",
            "l2": f"inputs larger than L2 (the fitted 3-center tensor, ~{gb:.1f} GB, is "
                  f"rebuilt and streamed every step)"}


def run_reference(args, rank):
    if rank != 0:
        return
    from dftax_b200 import systems

    sym, xyz, orb, aux, nocc = systems.workload(args.workload, seed=0)
    secs, parts, n = cpu_full_builds(args.workload, args.steps, nwarm=args.warmup)
    total = float(np.sum(secs))
    value = len(secs) / total
    sample = ("complete builds of the same workload (geometry seed 0, C seed 100): C++ "
              "3-center and 2-center integrals on all host threads, numpy eigh for the metric "
              "pseudo-inverse, J and K by dftax's einsum contractions (OpenBLAS, all threads); "
              f"{args.warmup} untimed, {args.steps} timed")
    line = {
        "metric": METRIC, "value": round(value, 6), "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * total / len(secs), 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "impl": "reference",
        "config": workload_config(args, orb, aux, nocc, 1),
        "precision": "fp64",
        "cpu_baseline": {"value": round(value, 6), "unit": UNIT, "cores": n, "kind": "port",
                         "sample": sample, "parts_s": {k: round(v, 3) for k, v in parts.items()}},
        "e2e": {"value": round(value, 6), "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "step_s": {"min": round(min(secs), 3), "max": round(max(secs), 3)},
        "note": "dftax (JAX) is not installable here; the compiled CPU restatement of its DF "
                "path is timed on full builds",
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
