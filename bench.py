"""Benchmark: heat-bath VCI + Epstein-Nesbet PT2 solve of the workload-1 synthetic PES.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--precision 0|1]

Workload (one "step" = one full solve): seeded synthetic PES with Nm = 15 modes (cubic keep
p = 0.5, values +-10^U(0,2.5); quartic keep p = 0.3, values +-10^U(-1,1.5), diagonal positive),
HCI_Eps = 0.5, Nstate = 200, PT2 on with PT2_Eps = 0.01, Max_quanta = 2.  The solve runs the
reference procedure: dense first step, heat-bath iterations with a sparse eigensolve each, then
PT2 over the screened perturber space.

Our arm (default): the library (libvhci_gpu.so, sm_100a) through its C ABI.
  value  = seconds per solve over the whole job (max over ranks of the timed region, divided by the
           solves all ranks completed), device-timed with CUDA events on the library's stream with
           the problem tables resident on the device;
  e2e    = the same through the public call a user makes (`vhci_b200.solve(path)`: parse, upload,
           solve, read the energies back), wall-clocked around synchronised steps.
  N > 1 GPUs run independent replicas (requests do not share data): weak scaling, no collective
  on the data path; ranks meet only at the timing barriers.
Reference arm (--impl reference): the reference algorithm on the host cores, as the CPU oracle's
literal restatement of its pair loop (src/Ham.cpp:237-323, the same body as src/PT2.cpp:70-118),
timed on a bounded sample of rows and extrapolated to the workload's pair count (the basis sizes
per iteration and |P| below, which any implementation of the algorithm reproduces).  Selection
and eigensolver time are not added, so it is a lower bound on the reference's time per solve.

--workload 0 (Nm = 12, HCI_Eps = 1.0, Nstate = 50, no PT2; small enough for the host cores to
finish): both arms run complete solves.  The reference arm times the oracle's literal restatement
of the whole procedure (pair-loop Hamiltonian builds, selection, LAPACK/ARPACK eigen-steps) per
step, nothing extrapolated, and our arm's cpu_baseline is one such solve.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = 1
WORKLOAD_DESCS = {
    0: ("VHCI, synthetic PES Nm=12 (cubic p=0.5 +-10^U(0,2.5), quartic p=0.3 +-10^U(-1,1.5)), "
        "HCI_Eps=1.0, Nstate=50, PT2=0, Max_quanta=2"),
    1: ("VHCI+PT2, synthetic PES Nm=15 (cubic p=0.5 +-10^U(0,2.5), quartic p=0.3 "
        "+-10^U(-1,1.5)), HCI_Eps=0.5, Nstate=200, PT2_Eps=0.01, Max_quanta=2"),
}
WORKLOAD_DESC = WORKLOAD_DESCS[WORKLOAD]
# The benchmark's L2 statement (timed solves stream matrices far larger than the 126 MB L2).
L2_NOTE = "working set larger than L2 (Hamiltonian of 0.2-3 GB), no flush needed"


def bench_config(workload: int, batch: int) -> dict:
    """The `config` object both arms print: the workload and the solves per step."""
    return {"workload": WORKLOAD_DESCS[workload], "global_batch": batch, "l2": L2_NOTE}


# Basis size after each heat-bath iteration and |P| of the workload-1 solve (FP64 path).
WORKLOAD_COUNTS = {"sizes": [38934, 215006, 336950, 372333, 380418], "n_pert": 6583465}
# DRAM traffic of one k_spmm_pairs launch over its algorithmic bytes, from an ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum = 4.186e9 + 0.051e9 bytes) of a 16-column product
# on the final workload-1 basis (380,418 rows, 255,052,558 entries; algorithmic 3.164e9 bytes) by
# `python bench.py --spmm-sweep --sweep-eigs --sweep-reps 2 --checkpoint <file>` on B200.  The
# bench's launches run on every basis of the solve, so their traffic is this ratio times their
# algorithmic bytes (the excess is vector-block gathers that miss L2, which scales with the entries).
NCU_SPMM_TRAFFIC_RATIO = (4.186275e9 + 0.051259e9) / 3.1641044e9


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Clocks:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["active", "hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names[1:], p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def write_workload(path: str, workload: int = WORKLOAD) -> None:
    from vhci_b200 import pes
    pes.write_workload(path, workload)


# ------------------------------------------------------------------------------ reference arm

def reference_sample(budget_s: float = 15.0) -> dict:
    """Time the reference pair loop on rows of the workload's first-iteration basis with all host
    threads; return seconds per solve extrapolated to the workload's pair count."""
    import numpy as np
    from oracle import oracle as O
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "workload.inp")
        write_workload(path)
        o = O.Oracle(path)
        w, C = np.linalg.eigh(o.dense_h())
        o.append_basis(o.select(C, min(o.neig, o.n), o.eps1))
        n = o.n
        threads = int(O.lib().orc_num_threads())
        # grow the row sample until it takes about budget_s
        stride = max(1, n // 64)
        pairs, dt = 0, 0.0
        while True:
            t0 = time.perf_counter()
            p, _ = O.pair_rows(o, 0, n, stride)
            d = time.perf_counter() - t0
            pairs += p
            dt += d
            if dt >= budget_s or stride == 1:
                break
            stride = max(1, int(stride * d / max(budget_s - dt, 1e-3) / 2) or 1)
    per_pair = dt / pairs
    sizes, npert = WORKLOAD_COUNTS["sizes"], WORKLOAD_COUNTS["n_pert"]
    total_pairs = sum(s * (s + 1) / 2 for s in sizes) + npert * sizes[-1]
    return {"s_per_solve": per_pair * total_pairs, "threads": threads, "pairs_timed": pairs,
            "seconds_timed": dt, "sample_basis": n, "ns_per_pair": per_pair * 1e9,
            "total_pairs": total_pairs}


def reference_full_solve(workload: int) -> dict:
    """One complete solve of the workload by the oracle's literal restatement of the reference:
    pair-loop Hamiltonian builds (src/Ham.cpp:228-344) and, with PT2, the pair-loop PT2
    (src/PT2.cpp:66-149); heat-bath selection as src/HB.cpp:24-223; LAPACK / ARPACK eigen-steps
    with Spectra's settings.  Timed end to end on the host cores, nothing extrapolated."""
    from oracle import oracle as O
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "workload.inp")
        write_workload(path, workload)
        t0 = time.perf_counter()
        r = O.solve(path, h_mode="pairs", pt2_mode="pairs")
        dt = time.perf_counter() - t0
    return {"s_per_solve": dt, "threads": int(O.lib().orc_num_threads()),
            "n_basis": int(len(r.basis)), "n_pert": int(r.n_pert), "E0": float(r.E[0])}


def run_reference(args):
    ws, rank, _ = _dist()
    if rank != 0:
        return
    if args.workload != WORKLOAD:
        return run_reference_full(args)
    vals = []
    info = None
    for i in range(args.warmup + args.steps):
        info = reference_sample(args.ref_budget)
        if i >= args.warmup:
            vals.append(info["s_per_solve"])
    v = statistics.median(vals)
    line = {
        "impl": "reference", "metric": "s/solve", "value": v, "unit": "s/solve",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": bench_config(WORKLOAD, 1),
        "run": {"parallelism": "host threads"},
        "cpu_baseline": {"value": v, "unit": "s/solve", "cores": info["threads"], "kind": "port",
                         "sample": (f"literal reference pair loop, {info['pairs_timed']:.3g} pairs on "
                                    f"the first-iteration basis ({info['sample_basis']} states) in "
                                    f"{info['seconds_timed']:.1f} s, extrapolated to "
                                    f"{info['total_pairs']:.3g} pairs (H builds + PT2); "
                                    "selection and eigensolver time not included")},
        "e2e": {"value": v, "unit": "s/solve", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_reference_full(args):
    vals, info = [], None
    for i in range(args.warmup + args.steps):
        info = reference_full_solve(args.workload)
        if i >= args.warmup:
            vals.append(info["s_per_solve"])
    v = statistics.median(vals)
    sample = (f"complete solves (median of {args.steps}) by the oracle's literal restatement "
              f"of the reference (pair-loop H builds, ARPACK eigen-steps): {info['n_basis']} "
              f"states, |P| {info['n_pert']}")
    line = {
        "impl": "reference", "metric": "s/solve", "value": v, "unit": "s/solve",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": bench_config(args.workload, 1),
        "run": {"parallelism": "host threads", "n_basis": info["n_basis"], "E0": info["E0"]},
        "cpu_baseline": {"value": v, "unit": "s/solve", "cores": info["threads"], "kind": "port",
                         "sample": sample},
        "e2e": {"value": v, "unit": "s/solve", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------ our arm

def run_ours(args):
    import numpy as np
    import torch
    from vhci_b200 import api

    from vhci_b200.replicas import Replicas, job_seconds_per_solve

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    rep = Replicas()            # NCCL process group of the replica ranks (none at N = 1)
    barrier, allmax = rep.barrier, rep.allmax

    td = tempfile.mkdtemp(prefix="vhci_bench_")
    path = os.path.join(td, "workload.inp")
    write_workload(path, args.workload)

    ctx = api.VHCI(path, device=local, precision=args.precision)
    q0 = ctx.basis()
    npert = [0]

    def solve_resident():
        ctx.set_basis(q0)
        s0 = ctx.stats()
        ctx.hci()
        if ctx.info.pt2:
            npert[0] = ctx.pt2()[1]
        s1 = ctx.stats()
        return (s1["ms_total"] - s0["ms_total"]) + (s1["ms_pt2"] - s0["ms_pt2"])

    for _ in range(args.warmup):
        solve_resident()
    ctx.reset_stats()
    clocks = Clocks(local)
    barrier()
    clocks.start()
    l0 = ctx.stats()["kernel_launches"]
    t0 = time.perf_counter()
    dev_ms = [solve_resident() for _ in range(args.steps)]
    barrier()
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    st = ctx.stats()
    launches = st["kernel_launches"] - l0
    info = ctx.info
    E = ctx.energies()
    ctx.close()

    dev_s = allmax(sum(dev_ms) / 1e3)
    wall_s = allmax(wall)
    value = job_seconds_per_solve(dev_s, args.steps, ws)

    # end to end through the public call, host inputs and outputs
    barrier()
    e2e_t, h2d, d2h = 0.0, 0, 0
    for _ in range(args.steps):
        t1 = time.perf_counter()
        r = api.solve(path, device=local, precision=args.precision)
        torch.cuda.synchronize()
        e2e_t += time.perf_counter() - t1
        h2d += r["stats"]["h2d_bytes"]
        d2h += r["stats"]["d2h_bytes"]
    barrier()
    e2e_s = job_seconds_per_solve(allmax(e2e_t), args.steps, ws)

    hbm, peak_kind = measured_peaks()
    spmm_gbs = st["spmm_bytes"] / (st["ms_spmm"] / 1e3) / 1e9 if st["ms_spmm"] else None
    en_gbs = (st["pt2_reduce_bytes"] / (st["ms_pt2_reduce"] / 1e3) / 1e9
              if st["ms_pt2_reduce"] else None)
    alg_per_launch = st["spmm_bytes"] / st["spmm_calls"] if st["spmm_calls"] else None
    roof = {"bound": "hbm", "kernel": "k_spmm_pairs (eigensolver H*X)", "achieved": spmm_gbs,
            "peak": hbm, "unit": "GB/s", "frac": (spmm_gbs / hbm) if spmm_gbs else None,
            "traffic": (args.traffic if args.traffic else
                        NCU_SPMM_TRAFFIC_RATIO * alg_per_launch if alg_per_launch else None),
            "traffic_note": ("ncu DRAM bytes of a captured final-basis launch, scaled to the "
                             "average launch by algorithmic bytes"),
            "algorithmic_bytes_per_launch": alg_per_launch, "peak_kind": peak_kind,
            "other": {"k_pt2_en GB/s": en_gbs,
                      # the product's bound: each of the nnz entries gathers one b-column vector
                      # row (b * 8 bytes), mostly served from L2
                      "spmm_gathered_bytes_per_launch": (st["spmm_gather_bytes"] / st["spmm_calls"]
                                                         if st["spmm_calls"] else None),
                      "spmm_gather GB/s": (st["spmm_gather_bytes"] / (st["ms_spmm"] / 1e3) / 1e9
                                           if st["ms_spmm"] else None)}}

    line = {
        "metric": "s/solve", "value": value, "unit": "s/solve", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_s * 1e3 / args.steps,
        "wall_s_timed": wall_s, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.precision == 0 else "f32-storage/f64-accum",
        "data": "synthetic",
        "config": bench_config(args.workload, ws),
        "run": {"n_basis": int(info.n_basis), "n_pert": int(npert[0]),
                "parallelism": f"replicas x{ws}", "E0": float(E[0])},
        "clocks": clk,
        "e2e": {"value": e2e_s, "unit": "s/solve", "h2d_bytes_per_step": h2d // args.steps,
                "d2h_bytes_per_step": d2h // args.steps},
        "gpu_launches": launches,
        "roofline": roof,
        "phase_ms": {k: round(st[k] / args.steps, 2) for k in
                     ("ms_select", "ms_hbuild", "ms_eigs", "ms_spmm", "ms_pt2", "ms_pt2_reduce")},
    }
    if rank == 0 and ws == 1 and not args.no_cpu_baseline and args.workload != WORKLOAD:
        ref = reference_full_solve(args.workload)
        line["cpu_baseline"] = {
            "value": ref["s_per_solve"], "unit": "s/solve", "cores": ref["threads"],
            "kind": "port",
            "sample": ("one complete solve by the oracle's literal restatement of the reference "
                       f"(pair-loop H builds, ARPACK eigen-steps): {ref['n_basis']} states")}
    elif rank == 0 and ws == 1 and not args.no_cpu_baseline:
        ref = reference_sample(args.ref_budget)
        line["cpu_baseline"] = {
            "value": ref["s_per_solve"], "unit": "s/solve", "cores": ref["threads"],
            "kind": "port",
            "sample": (f"literal reference pair loop, {ref['pairs_timed']:.3g} pairs in "
                       f"{ref['seconds_timed']:.1f} s, extrapolated to {ref['total_pairs']:.3g} "
                       "pairs (H builds + PT2); selection and eigensolver time not included")}
    if rank == 0:
        print(json.dumps(line), flush=True)
    rep.close()


def run_spmm_sweep(args):
    """Time the sparse product H X on the workload's final variational basis for block widths
    4-32 (CUDA events around the product only), then one eigensolve of the Nstate lowest pairs on
    that basis.  With --checkpoint PATH the basis is read from PATH when the file exists, so that
    nothing but the H build runs before the timed products (a profiler capture of them then starts
    after a handful of launches and holds only H and the blocks on the device); otherwise the
    workload is solved variationally and its basis written to PATH."""
    import numpy as np
    from vhci_b200 import api
    td = tempfile.mkdtemp(prefix="vhci_sweep_")
    path = os.path.join(td, "workload.inp")
    write_workload(path, args.workload)
    with api.VHCI(path) as v:
        if args.checkpoint and os.path.exists(args.checkpoint):
            v.read_checkpoint(args.checkpoint)
        else:
            v.hci()
            if args.checkpoint:
                v.write_checkpoint(args.checkpoint)
        nnz = v.build_h()
        rng = np.random.default_rng(0)
        print(json.dumps({"n": v.n, "nnz": int(nnz)}), flush=True)
        for b in (4, 8, 16, 32):
            X = rng.standard_normal((v.n, b))
            v.apply_h(X)
            s0 = v.stats()
            for _ in range(args.sweep_reps):
                v.apply_h(X)
            s1 = v.stats()
            ms = (s1["ms_spmm"] - s0["ms_spmm"]) / args.sweep_reps
            gbs = (s1["spmm_bytes"] - s0["spmm_bytes"]) / args.sweep_reps / (ms / 1e3) / 1e9
            print(json.dumps({"b": b, "ms": round(ms, 3), "ms_per_column": round(ms / b, 4),
                              "algorithmic_GBs": round(gbs, 1)}), flush=True)
        if args.sweep_eigs:
            k = min(int(v.info.nstate), v.n)
            s0 = v.stats()
            v.eigs(k)
            s1 = v.stats()
            print(json.dumps({"eigs_k": k, "ms_eigs": round(s1["ms_eigs"] - s0["ms_eigs"], 1),
                              "ms_spmm": round(s1["ms_spmm"] - s0["ms_spmm"], 1)}), flush=True)


def _write_serving_request(r, path):
    from vhci_b200 import pes as P
    spec, run = P.serving_request(r)
    P.write_input(path, spec, run)
    return {"nm": len(spec.freqs), "nstate": run.nstate, "eps1": run.eps1}


def _pct(x, p):
    import numpy as np
    return float(np.percentile(np.asarray(x), p)) if len(x) else None


def run_serving(args):
    """Serving stream: R requests (fresh admissible PES each, Nm 6..24, Nstate 10..100, eps1
    log-uniform in [0.3, 3], PT2 with eps2 = 0.1 eps1) with Poisson arrivals, under per-request size
    limits (basis and perturber space; a request past them is rejected with E_LIMIT by both paths).
    The one-at-a-time path is the same server with one slot and every request queued at t = 0: its
    service times s_i give its latencies under the Poisson arrivals (c_i = max(a_i, c_{i-1}) + s_i).
    The server (continuous batching over `slots` concurrent contexts) then replays the arrivals in
    real time.  The arrival rate defaults to 1.5x the one-at-a-time throughput."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor

    import numpy as np
    td = tempfile.mkdtemp(prefix="vhci_serve_")
    paths = [os.path.join(td, f"req{r:03d}.inp") for r in range(args.requests)]
    # request generation (PES draws + admissibility screen) on host processes, before any GPU call
    with ProcessPoolExecutor(max_workers=min(32, os.cpu_count() or 1),
                             mp_context=mp.get_context("spawn")) as ex:
        meta = list(ex.map(_write_serving_request, range(args.requests), paths))
    from vhci_b200 import api
    lim = {"max_basis": args.max_basis, "max_pert": args.max_pert}
    small = min(range(len(paths)), key=lambda i: meta[i]["nm"])
    api.serve([(paths[small], 0.0)], slots=1, **lim)      # warm-up: module load, handles, pool
    _, seq = api.serve([(p, 0.0) for p in paths], slots=1, **lim)
    service = [r["t_done"] - r["t_admit"] for r in seq]
    if args.verbose_requests:
        for i, (m, r, s) in enumerate(zip(meta, seq, service)):
            print(json.dumps({"request": i, **m, "status": r["status"], "n_basis": r["n_basis"],
                              "n_pert": r["n_pert"], "service_s": round(s, 4),
                              "message": r["message"]}), file=sys.stderr, flush=True)
    ok = [r["status"] == 0 for r in seq]
    seq_tput = sum(ok) / sum(service)
    rate = args.rate if args.rate else 1.5 * len(paths) / sum(service)
    rng = np.random.default_rng(12345)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, len(paths)))
    arrivals -= arrivals[0]
    c, seq_lat = 0.0, []
    for a, s, g in zip(arrivals, service, ok):
        c = max(a, c) + s
        if g:
            seq_lat.append(c - a)
    seq_wall = c
    summ, res = api.serve(list(zip(paths, arrivals)), slots=args.slots, reserve_bytes=8e9, **lim)
    lat = [r["t_done"] - r["arrival"] for r in res if r["status"] == 0]
    worst, mismatched = 0.0, 0
    for a, r in zip(seq, res):
        if a["status"] != r["status"]:
            mismatched += 1
        elif r["status"] == 0:
            if (r["n_basis"], r["n_pert"]) != (a["n_basis"], a["n_pert"]):
                mismatched += 1
            worst = max(worst, float(np.abs(r["E"] - a["E"]).max()))
    done = [r for r in seq if r["status"] == 0]
    line = {
        "metric": "serving_throughput", "value": round(summ["completed"] / summ["wall_s"], 4),
        "unit": "req/s", "higher_is_better": True, "n_gpus": 1, "requests": len(paths),
        "completed": summ["completed"],
        "rejected_limit": sum(r["status"] == api.E_LIMIT for r in res),
        "failed_other": sum(r["status"] not in (0, api.E_LIMIT) for r in res),
        "slots": args.slots, "arrival_rate": round(rate, 4),
        "p50_s": round(_pct(lat, 50), 4) if lat else None,
        "p99_s": round(_pct(lat, 99), 4) if lat else None,
        "wall_s": round(summ["wall_s"], 3), "peak_in_flight": summ["peak_in_flight"],
        "oom_retries": int(sum(r["retries"] for r in res)),
        "mix_vs_alone": {"max_abs_dE_cm1": worst, "mismatched_requests": mismatched},
        "one_at_a_time": {"value": round(seq_tput, 4), "unit": "req/s",
                          "service_s_total": round(sum(service), 3),
                          "p50_s": round(_pct(seq_lat, 50), 4) if seq_lat else None,
                          "p99_s": round(_pct(seq_lat, 99), 4) if seq_lat else None,
                          "wall_s_under_arrivals": round(seq_wall, 3)},
        "sizes": {"nm_max": max(m["nm"] for m in meta),
                  "n_basis_p50": int(_pct([r["n_basis"] for r in done], 50)) if done else 0,
                  "n_basis_max": int(max([r["n_basis"] for r in done] or [0])),
                  "n_pert_max": int(max([r["n_pert"] for r in done] or [0])),
                  "service_s_p50": round(_pct(service, 50), 4),
                  "service_s_max": round(max(service), 4)},
        "data": "synthetic", "dtype": "f64",
        "config": {"workload": "serving stream, Poisson arrivals, Nm 6..24, Nstate 10..100, "
                               "eps1 log-uniform [0.3,3], PT2 eps2=0.1*eps1",
                   "max_basis": args.max_basis, "max_pert": args.max_pert},
    }
    print(json.dumps(line), flush=True)


def run_mixed_check(args):
    """Mixed precision (FP32 Hamiltonian values and FP32 vector gathers in the eigensolver's
    products, FP64 accumulation, orthogonalisation, Ritz values, final Rayleigh-Ritz sweep and PT2)
    against the FP64 path on one workload: device time of each (median of --mixed-reps alternating
    solves after one warm-up pair) with its phases, basis and perturber counts, and the per-state
    error of the variational and PT2-corrected energies."""
    import numpy as np
    from vhci_b200 import api, pes
    td = tempfile.mkdtemp(prefix="vhci_mixed_")
    path = os.path.join(td, "workload.inp")
    pes.write_workload(path, args.workload)
    res, times, phases = {}, {0: [], 1: []}, {0: [], 1: []}
    keys = ("ms_select", "ms_hbuild", "ms_eigs", "ms_spmm", "ms_pt2")
    for rep in range(args.mixed_reps + 1):
        for prec in (0, 1):
            r = api.solve(path, precision=prec)
            s = r["stats"]
            res[prec] = r
            if rep > 0:     # the first pair warms up
                times[prec].append((s["ms_total"] + s["ms_pt2"]) / 1e3)
                phases[prec].append([s[q] for q in keys])
    a, b = res[0], res[1]
    ta, tb = statistics.median(times[0]), statistics.median(times[1])
    k = min(len(a["E"]), len(b["E"]))
    line = {
        "metric": "mixed_vs_fp64", "workload": args.workload,
        "fp64_s": round(ta, 3), "mixed_s": round(tb, 3), "speedup": round(ta / tb, 3),
        "solves_each": args.mixed_reps, "fp64_s_all": [round(t, 3) for t in times[0]],
        "mixed_s_all": [round(t, 3) for t in times[1]],
        "phase_ms_median": {q: [round(statistics.median(p[i] for p in phases[prec]), 1)
                                for prec in (0, 1)] for i, q in enumerate(keys)},
        "n_basis": [a["n_basis"], b["n_basis"]], "n_pert": [a["n_pert"], b["n_pert"]],
        "max_abs_dE_variational_cm1": float(np.abs(a["E_var"][:k] - b["E_var"][:k]).max()),
        "max_abs_dE_cm1": float(np.abs(a["E"][:k] - b["E"][:k]).max()),
        "per_state_abs_dE_cm1": [float(x) for x in np.abs(a["E"][:k] - b["E"][:k])],
        "target_cm1": 0.01,
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", type=int, default=0)
    ap.add_argument("--ref-budget", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--traffic", type=float, default=None,
                    help="ncu dram bytes per SpMM launch, if captured")
    ap.add_argument("--spmm-sweep", action="store_true",
                    help="time the sparse product on the workload's final basis and exit")
    ap.add_argument("--checkpoint", default=None,
                    help="with --spmm-sweep: basis file read if present, written otherwise")
    ap.add_argument("--sweep-reps", type=int, default=8)
    ap.add_argument("--sweep-eigs", action="store_true",
                    help="with --spmm-sweep: also time one eigensolve on the basis")
    ap.add_argument("--serving", action="store_true",
                    help="run the request-serving stream (one GPU) and exit")
    ap.add_argument("--requests", type=int, default=64)
    ap.add_argument("--slots", type=int, default=8)
    ap.add_argument("--rate", type=float, default=None, help="Poisson arrival rate, req/s")
    ap.add_argument("--max-basis", type=int, default=500_000)
    ap.add_argument("--max-pert", type=int, default=100_000_000)
    ap.add_argument("--verbose-requests", action="store_true")
    ap.add_argument("--mixed-check", action="store_true",
                    help="solve a workload in FP64 and in mixed precision, report per-state errors")
    ap.add_argument("--mixed-reps", type=int, default=3)
    ap.add_argument("--workload", type=int, default=WORKLOAD)
    args = ap.parse_args()
    if args.spmm_sweep:
        run_spmm_sweep(args)
        return
    if args.serving:
        run_serving(args)
        return
    if args.mixed_check:
        run_mixed_check(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
