"""Throughput benchmark of the batched ionic-model hot path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload cipa_pop|ord_pop] [--seg STEPS]

One bench step = one launch of SEG fixed time steps (dt = 0.005 ms) over the
whole population resident in HBM, with the biomarker state machine fused.
The population keeps advancing from step to step, so consecutive steps walk
through the action potential exactly as a long screening run does.

value  : mixed-precision cell-steps/s over the whole job (all ranks), device
         time (CUDA events), inputs resident in HBM.
fp64   : the plain FP64 path on the same workload (same timing rules).
e2e    : the same metric through the C ABI with host buffers: every step
         uploads the population state from pinned host memory, runs, and
         downloads state + biomarkers.
Multi-GPU (torchrun): every rank owns an independent population (weak
scaling); no data-path collective, only a barrier and a max-reduction of
the timings.
"""
from __future__ import annotations

import argparse
import ctypes
import importlib
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "ORd cell-steps/s mixed vs FP64 (APD90 err≤0.1 ms); screen-job p50/p99 latency"
DT = 0.005


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="ord_pop", choices=["ord_pop"])
    ap.add_argument("--seg", type=int, default=10000, help="time steps per bench step")
    ap.add_argument("--samples", type=int, default=2000)
    ap.add_argument("--concs", type=int, default=5)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    return ap.parse_args()


# ------------------------------------------------------------ inputs
def population(n_samples: int, n_conc: int, seed: int):
    """Seeded population: 2,000 IC50/Hill samples lognormal (sigma 0.5 in
    ln-space) around a nominal drug drawn from the single-cell ranges
    (IC50 log-U[0.1,100] uM, h U[0.6,1.8]), Cmax log-U[0.01,10] uM,
    concentrations 0..(n_conc-1) x Cmax. Returns (conc[n], hill[n,20])."""
    rng = np.random.default_rng(seed)
    nom_ic50 = 10 ** rng.uniform(-1, 2, 7)
    nom_h = rng.uniform(0.6, 1.8, 7)
    cmax = 10 ** rng.uniform(-2, 1)
    ic50 = nom_ic50 * np.exp(0.5 * rng.standard_normal((n_samples, 7)))
    h = nom_h * np.exp(0.5 * rng.standard_normal((n_samples, 7)))
    hill = np.zeros((n_samples, 20))
    hill[:, 0:14:2] = ic50
    hill[:, 1:14:2] = h
    hill = np.repeat(hill, n_conc, axis=0)
    conc = np.tile(np.arange(n_conc) * cmax, n_samples)
    return conc, hill


# ------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            p = [x.strip() for x in l.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------ distributed
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        import torch
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(x: float, pg) -> float:
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


# ------------------------------------------------------------ our arm
def run_ours(args, world, rank, local, pg):
    import torch
    cep = importlib.import_module("2ddrugsimulation_b200")
    torch.cuda.set_device(local)
    conc, hill = population(args.samples, args.concs, seed=1234 + rank)
    n = len(conc)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")  # > L2 (126 MB)
    res = {}
    launches = 0
    for prec in ("mixed", "fp64"):
        b = cep.Batch("ord2011", n, prec)
        b.init(conc=conc, hill=hill, dutta=False, quirks=True)
        b.set_pacing(2000.0)
        b.set_protocol(DT, 1000, 750, dt_write=1.0)
        for _ in range(args.warmup):
            b.run(args.seg)
            flush.zero_()
        torch.cuda.synchronize()
        barrier(pg)
        torch.cuda.synchronize()
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        kst = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        ken = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        with ClockSampler(local) as clk:
            start.record()
            for k in range(args.steps):
                kst[k].record()
                b.run(args.seg)
                ken[k].record()
                flush.zero_()
            stop.record()
            torch.cuda.synchronize()
        barrier(pg)
        ms = start.elapsed_time(stop)
        kms = [kst[k].elapsed_time(ken[k]) for k in range(args.steps)]
        ms_max = max_over_ranks(ms, pg)
        kernel_ms = statistics.mean(kms)
        cell_steps = n * args.seg * args.steps * world
        res[prec] = dict(value=cell_steps / (ms_max / 1e3), ms_per_step=ms_max / args.steps, kernel_ms=kernel_ms,
                         clocks=clk.summary(), status=b.status())
        launches += args.steps
        if prec == "mixed" and not args.no_e2e:
            res["e2e"] = run_e2e(args, b, n, world, pg, cep)
        b.close()
    return res, n, launches


def run_e2e(args, b, n, world, pg, cep):
    """Same workload through the C ABI with host buffers: per step, upload
    the population state from pinned host memory, run, download state and
    biomarkers."""
    import torch
    ns = cep.N_STATES["ord2011"]
    pinned_in = torch.empty(ns * n, dtype=torch.float64, pin_memory=True).numpy()
    pinned_out = torch.empty(ns * n, dtype=torch.float64, pin_memory=True).numpy()
    pinned_in[:] = b.get_states(cep.LAYOUT_SOA).ravel()
    lib = cep.lib()
    dp = ctypes.POINTER(ctypes.c_double)
    bm = (cep.Biomarkers * n)()
    torch.cuda.synchronize()
    barrier(pg)
    t0 = time.perf_counter()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(args.steps):
        lib.cep_batch_set_states(b._h, pinned_in.ctypes.data_as(dp), cep.LAYOUT_SOA)
        lib.cep_batch_run(b._h, args.seg)
        lib.cep_batch_get_states(b._h, pinned_out.ctypes.data_as(dp), cep.LAYOUT_SOA)
        lib.cep_batch_get_biomarkers(b._h, bm)
        pinned_in[:] = pinned_out
    stop.record()
    torch.cuda.synchronize()
    ms = max_over_ranks(start.elapsed_time(stop), pg)
    cell_steps = n * args.seg * args.steps * world
    return {"value": cell_steps / (ms / 1e3), "unit": "cell-steps/s", "h2d_bytes_per_step": ns * n * 8,
            "d2h_bytes_per_step": ns * n * 8 + n * ctypes.sizeof(cep.Biomarkers), "ms_per_step": ms / args.steps}


# ------------------------------------------------------------ CPU baseline / reference arm
def cpu_reference_rate(conc, hill, n_inst: int, n_steps: int, threads: int):
    """The reference's own ORd implementation (compiled from its sources by
    oracle/Makefile) or, where that build is absent, the oracle port; run
    over n_inst instances x n_steps on `threads` host threads."""
    from oracle import oracle as O
    kind = "reference" if O.ref_available("ord2011") else "port"
    per = [None] * threads
    idx = np.array_split(np.arange(n_inst), threads)

    def work(k):
        for i in idx[k]:
            if kind == "reference":
                c = O.RefCell("ord2011", 0.0, conc[i], hill[i, :14])
                c.consts[140] = 2000.0
            else:
                c = O.Cell("ord2011", 0.0, conc[i], hill[i, :14])
                c.set_pacing(2000.0)
            c.run(0.0, DT, n_steps)

    th = [threading.Thread(target=work, args=(k,)) for k in range(threads)]
    t0 = time.perf_counter()
    for t in th:
        t.start()
    for t in th:
        t.join()
    dt = time.perf_counter() - t0
    return n_inst * n_steps / dt, kind, dt


def main():
    args = parse()
    world, rank, local, pg = dist_setup(args)
    conc, hill = population(args.samples, args.concs, seed=1234)
    threads = os.cpu_count() or 1
    if args.impl == "reference":
        if rank != 0:
            return
        rates = []
        for _ in range(args.warmup + args.steps):
            n_inst = max(threads, 16)
            r, kind, _ = cpu_reference_rate(conc, hill, n_inst, 4000, threads)
            rates.append(r)
        v = statistics.mean(rates[args.warmup:])
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "cell-steps/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": "ORd-2011 population, 10,000 instances (2,000 IC50/Hill samples x 5 concs), "
                                       "BCL 2000 ms, dt 0.005 ms", "sample": f"{max(threads,16)} instances x 4000 steps per step"},
                "cpu_baseline": {"value": v, "unit": "cell-steps/s", "cores": threads, "kind": kind,
                                 "sample": f"{max(threads,16)} instances x 4000 fixed steps per bench step"},
                "e2e": {"value": v, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return
    res, n, launches = run_ours(args, world, rank, local, pg)
    if rank != 0:
        if pg is not None:
            pg.destroy_process_group()
        return
    cpu = None
    if not args.no_cpu:
        r, kind, secs = cpu_reference_rate(conc, hill, max(threads, 16), 20000, threads)
        cpu = {"value": r, "unit": "cell-steps/s", "cores": threads, "kind": kind,
               "sample": f"{max(threads,16)} instances x 20000 fixed steps ({secs:.1f} s)"}
    mixed, fp64 = res["mixed"], res["fp64"]
    line = {
        "metric": METRIC, "value": mixed["value"], "unit": "cell-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": mixed["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64 (mixed)", "data": "synthetic",
        "config": {"workload": f"ORd-2011 population, {n} instances per GPU ({args.samples} IC50/Hill samples x "
                               f"{args.concs} concs), BCL 2000 ms, dt 0.005 ms, {args.seg} steps per bench step, "
                               f"biomarkers fused", "l2": "flushed between timed steps (256 MiB write)",
                   "parallelism": f"instance sharding x{world}"},
        "fp64": {"value": fp64["value"], "ms_per_step": fp64["ms_per_step"], "kernel_ms": fp64["kernel_ms"]},
        "mixed_over_fp64": mixed["value"] / fp64["value"],
        "kernel_ms": mixed["kernel_ms"],
        "gpu_launches": launches,
        "clocks": mixed["clocks"],
        "cpu_baseline": cpu,
        "e2e": res.get("e2e"),
        "roofline": None,
    }
    print(json.dumps(line))
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
