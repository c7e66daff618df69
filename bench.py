"""Throughput benchmark of the batched ionic-model hot path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload cipa_pop|ord_pop] [--seg STEPS]

Workload (default, the population configuration): CiPA-ORd v1 2017 with the
dynamic hERG Markov IKr and drug trapping, 10,000 instances per GPU =
2,000 seeded IC50/Hill samples (lognormal around a nominal drug, sigma 0.5
in ln-space) x 5 concentrations, BCL 2000 ms, dt 0.005 ms, biomarkers
(steepest of the last 250 paces of a 1000-pace protocol) fused.

One bench step = one launch advancing the whole population resident in HBM
by SEG fixed time steps (default 10,000 = 50 ms of simulated time); the
population keeps advancing from step to step, walking through the action
potential exactly as the long screening run does.

value : mixed-precision cell-steps/s over the whole job (all ranks), device
        time (CUDA events around the timed region, max over ranks).
fp64  : the plain FP64 path on the same workload, same rules.
e2e   : the same metric through the C ABI with host buffers: every step
        uploads the population state from pinned host memory, runs, and
        downloads the state and the biomarker records.
Multi-GPU (torchrun): every rank owns an independent population (weak
scaling); no data-path collective, only barriers and a max of the timings.
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
BCL = 2000.0

# Algorithmic operations per cell-step, counted by running the oracle's
# restatement with an operation-counting scalar (operations on instance
# constants are folded and not counted): `make -C oracle opcount &&
# oracle/_build/opcount <model> 1 1000` (profiles/opcount_ionic_models.txt).
# flop = one add/sub, mul, div or elementary-function evaluation.
OPS = {
    "cipa2017": dict(add=520.97, mul=561.99, div=269.99, exp=123.0, log=3.0, pow=1.0),
    "ord2011": dict(add=474.97, mul=435.99, div=281.99, exp=100.0, log=3.0, pow=1.0),
    "tt2006": dict(add=220.89, mul=161.24, div=136.71, exp=62.62, log=4.0, pow=0.0, sqrt=1.0),
    "tt2004": dict(add=184.95, mul=140.90, div=122.73, exp=57.71, log=4.0, pow=1.0, sqrt=1.0),
    "tomek2019": dict(add=547.02, mul=560.61, div=275.99, exp=112.81, log=3.0, pow=1.0, sqrt=2.0),
}
# DRAM bytes per launch per instance measured by ncu on the run kernel
# (profiles/run_kernel_cipa2017_pop10k.md): the state and biomarker records
# are read and written once per launch; everything else stays on chip.
TRAFFIC_PER_INSTANCE = {"cipa2017": 705.0, "ord2011": None}


def flops_per_step(model: str) -> float:
    o = OPS[model]
    return o["add"] + o["mul"] + o["div"] + o["exp"] + o["log"] + o["pow"]


def sfu_ops_per_step(model: str) -> float:
    """Operations that need the special-function unit in the mixed path
    (exp2/log2/reciprocal for every division and elementary function)."""
    o = OPS[model]
    return o["div"] + o["exp"] + o["log"] + o["pow"] + o.get("sqrt", 0.0)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cipa_pop",
                    choices=["cipa_pop", "ord_pop", "tt06_sheet", "ord_slab", "serve"])
    ap.add_argument("--jobs", type=int, default=40, help="serving trace length")
    ap.add_argument("--seg", type=int, default=None,
                    help="time steps per bench step (default 10000 for populations, 200 for tissue)")
    ap.add_argument("--nx", type=int, default=512, help="tissue sheet edge in nodes")
    ap.add_argument("--format", default="auto", choices=["auto", "csr", "ell", "stencil", "classed"],
                    help="sparse format of the tissue operators (auto: timed on the first operator)")
    ap.add_argument("--samples", type=int, default=2000)
    ap.add_argument("--concs", type=int, default=5)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-sub", action="store_true", help="skip the other configurations' sub-results")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU-baseline sample length")
    ap.add_argument("--kernel", default="auto", choices=["auto", "cell", "roles", "pairs"],
                    help="one thread per cell, 4 warps per 32 cells, or the library's default for the size")
    a = ap.parse_args()
    if a.seg is None:
        a.seg = {"tt06_sheet": 200, "ord_slab": 20}.get(a.workload, 10000)
    return a


def model_of(workload: str) -> str:
    return {"cipa_pop": "cipa2017", "ord_pop": "ord2011", "tt06_sheet": "tt2006", "serve": "cipa2017",
            "ord_slab": "ord2011"}[workload]


# ------------------------------------------------------------ inputs
def population(model: str, n_samples: int, n_conc: int, seed: int):
    """Seeded population: a nominal drug (IC50 log-U[0.1,100] uM, h
    U[0.6,1.8]; for CiPA the static hERG block is off and the dynamic hERG
    set Kmax, Ku, n, halfmax, Vhalf is seeded, Kt = 3.5e-5), n_samples
    lognormal around it (sigma 0.5 in ln-space), Cmax log-U[0.01,10] uM,
    concentrations 0..n_conc-1 x Cmax. Returns (conc[n], hill[n, 20])."""
    rng = np.random.default_rng(seed)
    nom = np.zeros(20)
    nom[0:14:2] = 10 ** rng.uniform(-1, 2, 7)
    nom[1:14:2] = rng.uniform(0.6, 1.8, 7)
    halfmax = 10 ** rng.uniform(3, 6)
    dyn = [halfmax * 10 ** rng.uniform(-1, 1), 10 ** rng.uniform(-4, -2), rng.uniform(0.8, 1.0), halfmax,
           rng.uniform(-100, -10), 3.5e-5]
    if model == "cipa2017":
        nom[14:20] = dyn
        nom[12] = nom[13] = 0.0
    cmax = 10 ** rng.uniform(-2, 1)
    pert = np.exp(0.5 * rng.standard_normal((n_samples, 20)))
    pert[:, 18:20] = 1.0
    hill = nom[None, :] * pert
    hill = np.repeat(hill, n_conc, axis=0)
    conc = np.tile(np.arange(n_conc) * cmax, n_samples)
    return conc, hill


# ------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            time.sleep(0.3)
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.15)
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
def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180))
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
def measured_peaks():
    """FP32/FP64 FMA throughput of this GPU (probe kernels) and the
    driver-measured HBM/bf16 peaks."""
    out = {}
    try:
        L = ctypes.CDLL(str(ROOT / "2ddrugsimulation_b200" / "lib" / "libcep_probe.so"))
        L.cep_probe_fp32_fma_flops.restype = ctypes.c_double
        L.cep_probe_fp64_fma_flops.restype = ctypes.c_double
        out["fp32_tflops"] = max(L.cep_probe_fp32_fma_flops() for _ in range(3)) / 1e12
        out["fp64_tflops"] = max(L.cep_probe_fp64_fma_flops() for _ in range(3)) / 1e12
        L.cep_probe_sfu_ops.restype = ctypes.c_double
        L.cep_probe_warp_slots.restype = ctypes.c_double
        L.cep_probe_warp_slots.argtypes = [ctypes.c_int]
        out["sfu_tops"] = max(L.cep_probe_sfu_ops() for _ in range(3)) / 1e12
        L.cep_probe_l2_copy_bytes.restype = ctypes.c_double
        out["l2_gbs"] = max(L.cep_probe_l2_copy_bytes() for _ in range(3)) / 1e9
        out["role_blocks_on_distinct_smsp"] = L.cep_probe_warp_slots(313)
    except OSError:
        pass
    mp = ROOT / "MEASURED_PEAKS.json"
    if mp.exists():
        out["measured_peaks_json"] = json.loads(mp.read_text())
    return out


def beat_launches(args) -> int:
    """Launches of --seg time steps that make one BCL (at least one)."""
    return max(1, int(round(BCL / DT / args.seg)))


def run_ours(args, world, rank, local, pg, model):
    import torch
    cep = importlib.import_module("2ddrugsimulation_b200")
    torch.cuda.set_device(local)
    # one screening job of samples x world, sharded by whole samples
    shard = importlib.import_module("2ddrugsimulation_b200.shard")
    conc_all, hill_all = population(model, args.samples * world, args.concs, seed=1234)
    i0, i1 = shard.instance_range(args.samples * world, args.concs, world, rank)
    conc, hill = conc_all[i0:i1], hill_all[i0:i1]
    n = len(conc)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")  # > L2 (126 MB)
    res = {}
    launches = 0
    # One bench step is one whole beat (BCL / dt time steps as launches of
    # --seg steps): a step's cost varies within a beat (stiff Markov-chain
    # phases of drugged instances in diastole), so the timed window covers
    # whole beats, after whole warm-up beats.
    per_beat = beat_launches(args)
    for prec in ("mixed", "fp64"):
        b = cep.Batch(model, n, prec)
        if args.kernel != "auto":
            b.set_kernel(args.kernel)
        b.init(conc=conc, hill=hill, quirks=True)
        b.set_pacing(BCL)
        # every beat evaluated (the state machine of the last 250 paces runs
        # on every step, as it does in the biomarker window)
        b.set_protocol(DT, 1000, 0, dt_write=1.0)
        for _ in range(args.warmup):
            for _ in range(per_beat):
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
                for _ in range(per_beat):
                    b.run(args.seg)
                ken[k].record()
                flush.zero_()
            stop.record()
            torch.cuda.synchronize()
        barrier(pg)
        ms = start.elapsed_time(stop)
        kms = [kst[k].elapsed_time(ken[k]) for k in range(args.steps)]
        ms_max = max_over_ranks(ms, pg)
        kernel_ms = max_over_ranks(statistics.mean(kms), pg)
        cell_steps = n * args.seg * per_beat * args.steps * world
        st = b.status()
        res[prec] = dict(value=cell_steps / (ms_max / 1e3), ms_per_step=ms_max / args.steps, kernel_ms=kernel_ms,
                         clocks=clk.summary(), n_running=int((st == cep.INST_RUNNING).sum()),
                         n_nonfinite=int((st == cep.INST_NONFINITE).sum()))
        launches += args.steps * per_beat
        if prec == "mixed" and not args.no_e2e:
            res["e2e"] = run_e2e(args, b, n, world, pg, cep, model)
        b.close()
    res["compliant"] = run_compliant(args, world, rank, local, pg, model, conc, hill, flush)
    launches += res["compliant"]["launches"]
    return res, n, launches


def run_compliant(args, world, rank, local, pg, model, conc, hill, flush, refine_above_vm=-80.0):
    """The headline path: the mixed population on one stream and, on a
    second stream concurrently, the FP64 batch of the instances whose
    diastolic Vm after the first (screening) beat is above refine_above_vm
    (drug-depolarised cells that do not repolarise; FP32 gates cannot hold
    their APD90 to 0.1 ms, so their records come from FP64). The same split
    as cep_population_run. One bench step = one beat of both batches."""
    import torch
    cep = importlib.import_module("2ddrugsimulation_b200")
    n = len(conc)
    per_beat = beat_launches(args)
    sa, sb = torch.cuda.Stream(), torch.cuda.Stream()
    a = cep.Batch(model, n, "mixed", stream=sa.cuda_stream)
    if args.kernel != "auto":
        a.set_kernel(args.kernel)
    a.init(conc=conc, hill=hill, quirks=True)
    a.set_pacing(BCL)
    a.set_protocol(DT, 1000, 0, dt_write=1.0)

    def beat(bs):
        for _ in range(per_beat):
            for b in bs:
                b.run(args.seg)

    beat([a])  # screening beat
    a.sync()
    cand = np.flatnonzero(~(a.get_states()[:, 0] < refine_above_vm))
    bs = [a]
    if len(cand):
        b = cep.Batch(model, len(cand), "fp64", stream=sb.cuda_stream)
        b.init(conc=conc[cand], hill=hill[cand], quirks=True)
        b.set_pacing(BCL)
        b.set_protocol(DT, 1000, 0, dt_write=1.0)
        beat([b])  # the candidates' first beat, from their initial state
        bs.append(b)
    for _ in range(max(0, args.warmup - 1)):
        beat(bs)
        torch.cuda.synchronize()
        flush.zero_()
    torch.cuda.synchronize()
    barrier(pg)
    torch.cuda.synchronize()

    def ev():
        return torch.cuda.Event(enable_timing=True)

    start, stop = ev(), ev()
    ka = [(ev(), ev()) for _ in range(args.steps)]
    kb = [(ev(), ev()) for _ in range(args.steps)]
    main = torch.cuda.current_stream()
    with ClockSampler(local) as clk:
        start.record(main)
        for k in range(args.steps):
            go = ev()
            go.record(main)
            for st, (e0, _) in ((sa, ka[k]), (sb, kb[k])):
                st.wait_event(go)
                e0.record(st)
            beat(bs)
            ka[k][1].record(sa)
            kb[k][1].record(sb)
            main.wait_event(ka[k][1])
            main.wait_event(kb[k][1])
            flush.zero_()
        stop.record(main)
        torch.cuda.synchronize()
    barrier(pg)
    ms = max_over_ranks(start.elapsed_time(stop), pg)
    ms_a = max_over_ranks(statistics.mean(e0.elapsed_time(e1) for e0, e1 in ka), pg)
    ms_b = max_over_ranks(statistics.mean(e0.elapsed_time(e1) for e0, e1 in kb), pg) if len(cand) else 0.0
    cell_steps = n * args.seg * per_beat * args.steps * world
    st = a.status()
    out = dict(value=cell_steps / (ms / 1e3), ms_per_step=ms / args.steps, kernel_ms_mixed=ms_a,
               kernel_ms_fp64_candidates=ms_b, n_candidates=int(len(cand)), candidate_fraction=len(cand) / n,
               refine_above_vm=refine_above_vm, clocks=clk.summary(),
               n_nonfinite=int((st == cep.INST_NONFINITE).sum()), launches=args.steps * per_beat * len(bs))
    if not args.no_e2e:
        out["e2e"] = compliant_e2e(args, bs, n, world, pg, cep, model, sa, sb)
    for b in bs:
        b.close()
    return out


def compliant_e2e(args, bs, n, world, pg, cep, model, sa, sb):
    """The headline path through the C ABI with host buffers: every step
    uploads both batches' states from pinned host memory, runs the beat on
    both streams, and downloads the states and the biomarker records."""
    import torch
    ns = cep.N_STATES[model]
    lib = cep.lib()
    dp = ctypes.POINTER(ctypes.c_double)
    per_beat = beat_launches(args)
    bufs = []
    for b in bs:
        pin_in = torch.empty(ns * b.n, dtype=torch.float64, pin_memory=True).numpy()
        pin_out = torch.empty(ns * b.n, dtype=torch.float64, pin_memory=True).numpy()
        pin_in[:] = b.get_states(cep.LAYOUT_SOA).ravel()
        bufs.append((b, pin_in, pin_out, (cep.Biomarkers * b.n)()))

    def step():
        rc = 0
        for b, pin_in, _, _ in bufs:
            rc |= lib.cep_batch_set_states(b._h, pin_in.ctypes.data_as(dp), cep.LAYOUT_SOA)
        for _ in range(per_beat):
            for b, _, _, _ in bufs:
                rc |= lib.cep_batch_run(b._h, args.seg)
        for b, pin_in, pin_out, bm in bufs:
            rc |= lib.cep_batch_get_states(b._h, pin_out.ctypes.data_as(dp), cep.LAYOUT_SOA)
            rc |= lib.cep_batch_get_biomarkers(b._h, bm)
            pin_in[:] = pin_out
        if rc:
            raise RuntimeError(lib.cep_last_error().decode())

    step()  # untimed
    torch.cuda.synchronize()
    barrier(pg)
    t0 = time.perf_counter()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(args.steps):
        step()
    sa.synchronize()
    sb.synchronize()
    stop.record()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    ms = max_over_ranks(max(start.elapsed_time(stop), wall * 1e3), pg)
    cell_steps = n * args.seg * per_beat * args.steps * world
    h2d = sum(ns * b.n * 8 for b in bs)
    d2h = h2d + sum(b.n * ctypes.sizeof(cep.Biomarkers) for b in bs)
    return {"value": cell_steps / (ms / 1e3), "unit": "cell-steps/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "ms_per_step": ms / args.steps}


def run_e2e(args, b, n, world, pg, cep, model):
    """The same workload through the C ABI with host buffers."""
    import torch
    ns = cep.N_STATES[model]
    pinned_in = torch.empty(ns * n, dtype=torch.float64, pin_memory=True).numpy()
    pinned_out = torch.empty(ns * n, dtype=torch.float64, pin_memory=True).numpy()
    pinned_in[:] = b.get_states(cep.LAYOUT_SOA).ravel()
    lib = cep.lib()
    dp = ctypes.POINTER(ctypes.c_double)
    bm = (cep.Biomarkers * n)()
    torch.cuda.synchronize()
    barrier(pg)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    per_beat = beat_launches(args)
    steps_per_beat = args.seg * per_beat

    def run_beat():  # the beat as the same launches the device-timed path makes
        r = 0
        for _ in range(per_beat):
            r |= lib.cep_batch_run(b._h, args.seg)
        return r

    # one untimed beat through the same calls first
    rc = lib.cep_batch_set_states(b._h, pinned_in.ctypes.data_as(dp), cep.LAYOUT_SOA)
    rc |= run_beat()
    rc |= lib.cep_batch_get_states(b._h, pinned_out.ctypes.data_as(dp), cep.LAYOUT_SOA)
    rc |= lib.cep_batch_get_biomarkers(b._h, bm)
    if rc:
        raise RuntimeError(lib.cep_last_error().decode())
    pinned_in[:] = pinned_out
    torch.cuda.synchronize()
    barrier(pg)
    start.record()
    for _ in range(args.steps):
        rc = lib.cep_batch_set_states(b._h, pinned_in.ctypes.data_as(dp), cep.LAYOUT_SOA)
        rc |= run_beat()
        rc |= lib.cep_batch_get_states(b._h, pinned_out.ctypes.data_as(dp), cep.LAYOUT_SOA)
        rc |= lib.cep_batch_get_biomarkers(b._h, bm)
        if rc:
            raise RuntimeError(lib.cep_last_error().decode())
        pinned_in[:] = pinned_out
    stop.record()
    torch.cuda.synchronize()
    ms = max_over_ranks(start.elapsed_time(stop), pg)
    cell_steps = n * steps_per_beat * args.steps * world
    return {"value": cell_steps / (ms / 1e3), "unit": "cell-steps/s", "h2d_bytes_per_step": ns * n * 8,
            "d2h_bytes_per_step": ns * n * 8 + n * ctypes.sizeof(cep.Biomarkers), "ms_per_step": ms / args.steps}


# ------------------------------------------------------------ CPU baseline / reference arm
def cpu_rate(model: str, conc, hill, threads: int, steps_per_thread: int):
    """The reference's CPU implementation of the path on `threads` host
    threads, one instance per thread: for ORd the reference compiled from
    its own sources (oracle/_ref); for CiPA-ORd, whose reference integrates
    only with CVODE (not buildable here), the oracle port (the reference's
    computeRates restated bit-exact plus the fixed-step scheme)."""
    from oracle import oracle as O
    kind = "reference" if (model == "ord2011" and O.ref_available("ord2011")) else "port"

    def work(k):
        i = (k * len(conc)) // threads  # instances spread over the whole population
        if kind == "reference":
            c = O.RefCell("ord2011", 0.0, conc[i], hill[i, :14])
            c.consts[140] = BCL
        else:
            c = O.Cell(model, 0.0, conc[i], hill[i], quirks=True)
            c.set_pacing(BCL)
        c.run(0.0, DT, steps_per_thread)

    th = [threading.Thread(target=work, args=(k,)) for k in range(threads)]
    t0 = time.perf_counter()
    for t in th:
        t.start()
    for t in th:
        t.join()
    secs = time.perf_counter() - t0
    return threads * steps_per_thread / secs, kind, secs


def calibrate_cpu(model, conc, hill, threads, target_s):
    r, _, _ = cpu_rate(model, conc, hill, 1, 20000)
    return max(20000, int(r * target_s))


def config_of(args, model, n, world):
    name = {"cipa2017": "CiPA-ORd v1 2017 (dynamic hERG, drug trapping)", "ord2011": "ORd 2011"}[model]
    per_beat = beat_launches(args)
    return {"workload": f"{name} population, {n} instances per GPU ({args.samples} IC50/Hill samples x "
                        f"{args.concs} concs), BCL 2000 ms, dt 0.005 ms, 1000-pace protocol with steepest-of-last-"
                        f"250 biomarkers fused; one bench step = one whole beat ({args.seg * per_beat} time steps "
                        f"as {per_beat} launches of {args.seg})",
            "instances_per_gpu": n, "time_steps_per_bench_step": args.seg * per_beat,
            "launches_per_bench_step": per_beat, "kernel": args.kernel,
            "l2": "flushed between timed steps (256 MiB write)", "parallelism": f"instance sharding x{world}"}


# ------------------------------------------------------------ single-cell configuration
def config1_run(args):
    """ORd 2011 single cells as the single-cell configuration runs them: one
    seeded drug (IC50 log-U[0.1,100] uM, h U[0.6,1.8], Cmax log-U[0.01,10]
    uM) at 0..4 x Cmax, BCL 1000 ms, dt 0.005 ms, 100 paces, last-beat
    biomarkers. Five instances are latency-bound: each precision is timed
    over 2 paces after a warm-up pace (CUDA events) and the 100-pace time is
    projected from it; the compiled reference on 5 host threads beside it."""
    import torch
    cep = importlib.import_module("2ddrugsimulation_b200")
    rng = np.random.default_rng(7)
    h = np.zeros(14)
    h[0::2] = 10 ** rng.uniform(-1, 2, 7)
    h[1::2] = rng.uniform(0.6, 1.8, 7)
    cmax = 10 ** rng.uniform(-2, 1)
    conc = np.arange(5) * cmax
    hill = np.repeat(h[None, :], 5, axis=0)
    spp = int(round(1000.0 / DT))
    out = {"workload": "ORd 2011, 5 concentrations of one drug, BCL 1000 ms, dt 0.005 ms, 100 paces; timed over "
                       "2 paces after 1 warm-up pace, 100-pace time projected"}
    for prec in ("fp64", "mixed"):
        b = cep.Batch("ord2011", 5, prec)
        b.init(conc=conc, hill=hill, quirks=True)
        b.set_pacing(1000.0)
        b.set_protocol(DT, 100, 99, dt_write=1.0)
        for _ in range(spp // 50000):
            b.run(50000)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(2 * spp // 50000):
            b.run(50000)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 2
        out[prec] = {"ms_per_pace": ms, "s_per_100_paces": ms * 100 / 1e3, "us_per_step": ms * 1e3 / spp,
                     "cell_steps_per_s": 5 * spp / (ms / 1e3)}
        b.close()
    if not args.no_cpu:
        r, kind, secs = cpu_rate("ord2011", conc, hill, 5, spp // 2)
        out["cpu_baseline"] = {"cell_steps_per_s": r, "kind": kind, "cores": 5,
                               "s_per_100_paces": 5 * 100 * spp / r / 5,
                               "sample": f"5 instances x {spp // 2} steps, one per thread ({secs:.1f} s)"}
    return out


def sub_results(args):
    """The other configurations, each bounded to seconds of GPU time, as
    extra keys of the default line: the single-cell configuration, the
    TT2006 sheets, the ORd slab and the serving trace."""
    import copy
    subs = {}
    jobs = [("config1", lambda a: config1_run(a), {}),
            ("tt06_sheet_512x512x3", lambda a: tissue_main(a, 1, 0, 0, None),
             dict(workload="tt06_sheet", nx=512, seg=200, steps=2, warmup=1)),
            ("ord_slab_256x256x48x2", lambda a: slab_main(a, 1, 0, 0, None),
             dict(workload="ord_slab", nx=512, seg=20, steps=2, warmup=1)),
            ("serve", lambda a: serve_main(a), dict(workload="serve", jobs=20))]
    for name, fn, over in jobs:
        a = copy.copy(args)
        for k, v in over.items():
            setattr(a, k, v)
        t0 = time.perf_counter()
        try:
            r = fn(a)
        except Exception as e:  # a failing sub-configuration must not hide the headline
            r = {"error": f"{type(e).__name__}: {e}"}
        if isinstance(r, dict):
            r.pop("peaks", None)
            r["wall_s"] = time.perf_counter() - t0
        subs[name] = r
    return subs


# ------------------------------------------------------------ tissue workload
TISSUE_DT, TISSUE_H, TISSUE_D, TISSUE_RTOL = 0.01, 0.025, 0.0013, 1e-8
def pcg_bytes_per_row(fmt: int, slots: int, iters: float) -> float:
    """Algorithmic bytes one row moves in one solve of the batched
    Jacobi-PCG kernel, each vector element and matrix entry counted once per
    pass. Setup: B v (the format's B entries, v), the Jacobi inverse, and
    r, z, p_0 written (40 B + matrix). Each iteration: the product pass
    reads p, z, x and A's entries and writes p, q, x (the previous
    iteration's x update rides on it); the update pass reads q, r and the
    Jacobi inverse and writes r, z (88 B + matrix). A last pass applies the
    final x update (24 B). Matrix bytes per row: CSR 12 per entry + 4 (row
    pointer), ELL 12 per slot, stencil 8 per slot (implicit columns),
    classed 4 (the class index; the per-class table stays in cache)."""
    mat = {0: 12 * slots + 4, 1: 12 * slots, 2: 8 * slots, 3: 4}[fmt]
    return (40 + mat) + iters * (88 + mat) + 24


# DRAM bytes (read + write) per unit measured by ncu on one launch of the
# tissue kernels (profiles/pcg_many_kernel_tissue_groups.md,
# profiles/tissue_kernel_ionic_step.md): PCG per row and solve (the sheets
# stay L2-resident; the slab figure is the 192x192x48 capture, which scales
# with rows), ionic step per cell.
PCG_TRAFFIC_PER_ROW_SOLVE = {"tt2006": 37.95e6 / 786432, "ord2011": 4.328e9 / 3538944}
IONIC_TRAFFIC_PER_CELL = {"tt2006": 61.63e6 / 262144, "ord2011": 1.4896e9 / 1769472}


def hbm_peak(peaks: dict):
    """The driver-measured HBM copy bandwidth, else the pool's fallback."""
    mp = peaks.get("measured_peaks_json") or {}
    for k in ("hbm_gbs", "hbm_GBs", "hbm_gb_s"):
        if k in mp:
            return float(mp[k]), "MEASURED_PEAKS.json hbm_gbs (measured)"
    return 6650.0, "fallback 6650 GB/s"


def phase_rooflines(model: str, prec: str, cells: int, steps: int, timing: dict, fmt: int, slots: int,
                    iters: float, n_states: int, peaks: dict, hbm: float, hbm_src: str) -> dict:
    """Live per-phase device time of a tissue group (CUDA events around each
    step's ionic launches and its batched PCG launch) against each phase's
    roofline. `cells` = nodes of all tissues in the group, `steps` = Godunov
    steps timed. Ionic: every cell reads and writes its state vector once
    per step (16 B per state + 1 B stimulus mask) and, in the mixed path,
    issues the model's special-function operations; the binding bound is
    the slower of the two. Diffusion: pcg_bytes_per_row per row per solve."""
    ion_ms, dif_ms = timing["ionic_ms"] / steps, timing["diffusion_ms"] / steps
    ion_bytes = cells * (16 * n_states + 1)
    ion_hbm_ms = ion_bytes / (hbm * 1e9) * 1e3
    sfu = peaks.get("sfu_tops")
    ion_sfu_ms = (sfu_ops_per_step(model) * cells / (sfu * 1e12) * 1e3) if (sfu and prec == "mixed") else 0.0
    if ion_sfu_ms > ion_hbm_ms:
        ion = {"bound": "sfu", "achieved": sfu_ops_per_step(model) * cells / (ion_ms * 1e-3) / 1e12, "peak": sfu,
               "unit": "TFLOP/s", "peak_source": "bench.py ex2.approx throughput probe on this GPU (1 op/MUFU)",
               "ops_per_cell_step": sfu_ops_per_step(model)}
    else:
        ion = {"bound": "hbm", "achieved": ion_bytes / (ion_ms * 1e-3) / 1e9, "peak": hbm, "unit": "GB/s",
               "peak_source": hbm_src, "bytes_per_cell_step": 16 * n_states + 1}
    tr = IONIC_TRAFFIC_PER_CELL.get(model) if prec == "mixed" else None
    ion.update(kernel="tissue_kernel (ionic step + stimulus, one launch per tissue; figures cover a step's "
                      "launches for all tissues of the group)", ms_per_step=ion_ms,
               frac=ion["achieved"] / ion["peak"], traffic=tr * cells if tr else None,
               other_bound_ms={"hbm": ion_hbm_ms, "sfu": ion_sfu_ms or None})
    dif_bytes = cells * pcg_bytes_per_row(fmt, slots, iters)
    # An operator whose ncu DRAM traffic is far below its algorithmic bytes
    # runs out of the L2 (the 512^2 sheets): its bound is the L2 bandwidth
    # (the bench's L2 copy probe), not HBM.
    meas = PCG_TRAFFIC_PER_ROW_SOLVE.get(model) if fmt == 3 else None
    l2 = peaks.get("l2_gbs")
    if meas is not None and l2 and meas < 0.25 * pcg_bytes_per_row(fmt, slots, iters):
        dif_bound, dif_peak, dif_src = "l2", l2, "bench.py L2 copy probe on this GPU (2 x 24 MiB working set)"
    else:
        dif_bound, dif_peak, dif_src = "hbm", hbm, hbm_src
    dif = {"bound": dif_bound, "kernel": "pcg_many_kernel (one cooperative launch per step for the group)",
           "achieved": dif_bytes / (dif_ms * 1e-3) / 1e9, "peak": dif_peak, "unit": "GB/s", "peak_source": dif_src,
           "ms_per_step": dif_ms,
           "traffic": PCG_TRAFFIC_PER_ROW_SOLVE[model] * cells if (fmt == 3 and model in PCG_TRAFFIC_PER_ROW_SOLVE) else None,
           "bytes_per_row_per_solve": pcg_bytes_per_row(fmt, slots, iters),
           "cg_iters_per_solve": iters}
    dif["frac"] = dif["achieved"] / dif_peak
    return {"ionic": ion, "diffusion": dif, "ionic_share": ion_ms / (ion_ms + dif_ms)}


def tissue_inputs(seed: int, n_conc: int = 3):
    """IKr block of one seeded drug: IC50 log-U[0.1,100] uM, h U[0.6,1.8],
    Cmax log-U[0.01,10] uM; concentrations 0, 1x, 3x Cmax."""
    rng = np.random.default_rng(seed)
    hill = np.zeros(14)
    hill[12] = 10 ** rng.uniform(-1, 2)
    hill[13] = rng.uniform(0.6, 1.8)
    cmax = 10 ** rng.uniform(-2, 1)
    return [0.0, cmax, 3 * cmax][:n_conc], hill


def format_arg(cep, args):
    """The --format choice as a format id (None: autotune)."""
    return {"auto": None, "csr": cep.FEM_CSR, "ell": cep.FEM_ELL, "stencil": cep.FEM_STENCIL,
            "classed": cep.FEM_CLASSED}[args.format]


def make_sheet(cep, nx, prec, conc, hill, fmt=None):
    n = nx * nx
    cells = cep.Batch("tt2006", n, prec)
    cells.init(conc=np.full(n, conc), hill=hill)
    fem = cep.Fem.grid(2, nx, nx, 1, TISSUE_H, TISSUE_DT, TISSUE_D,
                       fmt=cep.FEM_AUTO if fmt is None else fmt).set_solver(TISSUE_RTOL)
    t = cep.Tissue(cells, fem, TISSUE_DT)
    mask = np.zeros((nx, nx), np.uint8)
    c = max(2, nx // 64)
    mask[:c, :c] = 1  # corner S1
    t.set_stimulus(mask.ravel(), 1000.0, 0.0, 1.0, 2)
    return t


def run_tissue(args, world, rank, local, pg):
    import torch
    cep = importlib.import_module("2ddrugsimulation_b200")
    torch.cuda.set_device(local)
    concs, hill = tissue_inputs(4321 + rank)
    nx = args.nx
    n = nx * nx
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    res = {}
    launches = 0
    fmt = format_arg(cep, args)
    for prec in ("mixed", "fp64"):
        sheets = [make_sheet(cep, nx, prec, concs[0], hill, fmt)]  # auto: timed on the first sheet
        fmt = sheets[0].fem.format
        sheets += [make_sheet(cep, nx, prec, c, hill, fmt) for c in concs[1:]]
        group = cep.TissueGroup(sheets)  # one batched diffusion solve per step for all sheets
        for _ in range(args.warmup):
            group.run(args.seg)
            flush.zero_()
        for t in sheets:
            t.sync()
        it0 = [t.stats()["cg_iters"] for t in sheets]
        torch.cuda.synchronize()
        group.set_timing(True)
        barrier(pg)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clk:
            start.record()
            for _ in range(args.steps):
                group.run(args.seg)
                flush.zero_()
            stop.record()
            torch.cuda.synchronize()
        barrier(pg)
        timing = group.timing()
        ms = max_over_ranks(start.elapsed_time(stop), pg)
        st = [t.stats() for t in sheets]
        cg = sum(s["cg_iters"] for s in st) - sum(it0)
        node_steps = n * len(sheets) * args.seg * args.steps * world
        res[prec] = dict(value=node_steps / (ms / 1e3), ms_per_step=ms / args.steps, clocks=clk.summary(),
                         cg_iters_per_solve=cg / (len(sheets) * args.seg * args.steps),
                         not_converged=sum(s["not_converged"] for s in st), fmt=sheets[0].fem.format,
                         ell_width=sheets[0].fem.ell_width, timing=timing)
        if prec == "mixed":
            launches = args.steps * (len(sheets) + 1) * args.seg  # ionic per sheet + one batched PCG, per step
            if not args.no_e2e:
                res["e2e"] = tissue_e2e(args, sheets, n, world, pg, cep)
        group.close()
        for t in sheets:
            t.close()
    return res, n, launches


def tissue_e2e(args, sheets, n, world, pg, cep):
    """Each step through the C ABI with host buffers: upload every sheet's
    state from pinned memory, run SEG Godunov steps, download V."""
    import torch
    ns = cep.N_STATES["tt2006"]
    lib = cep.lib()
    dp = ctypes.POINTER(ctypes.c_double)
    pin = [torch.empty(ns * n, dtype=torch.float64, pin_memory=True).numpy() for _ in sheets]
    vout = [torch.empty(n, dtype=torch.float64, pin_memory=True).numpy() for _ in sheets]
    for p, t in zip(pin, sheets):
        p[:] = t.cells.get_states(cep.LAYOUT_SOA).ravel()
    torch.cuda.synchronize()
    barrier(pg)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(args.steps):
        for p, v, t in zip(pin, vout, sheets):
            rc = lib.cep_batch_set_states(t.cells._h, p.ctypes.data_as(dp), cep.LAYOUT_SOA)
            rc |= lib.cep_tissue_run(t._h, args.seg)
            rc |= lib.cep_tissue_get_v(t._h, v.ctypes.data_as(dp))
            if rc:
                raise RuntimeError(lib.cep_last_error().decode())
    stop.record()
    torch.cuda.synchronize()
    ms = max_over_ranks(start.elapsed_time(stop), pg)
    node_steps = n * len(sheets) * args.seg * args.steps * world
    return {"value": node_steps / (ms / 1e3), "unit": "node-steps/s", "h2d_bytes_per_step": ns * n * 8 * len(sheets),
            "d2h_bytes_per_step": n * 8 * len(sheets), "ms_per_step": ms / args.steps}


def tissue_cpu(args):
    """The oracle's tissue loop (TT2006 step + CSR Jacobi-PCG, one core) on
    a 128x128 sheet, 400 Godunov steps (about 10 s)."""
    from oracle import oracle as O
    concs, hill = tissue_inputs(4321)
    nx, steps = 128, 400
    mask = np.zeros((nx, nx), np.uint8)
    mask[:2, :2] = 1
    t0 = time.perf_counter()
    O.tissue_run("tt2006", 2, nx, nx, 1, TISSUE_H, TISSUE_D, TISSUE_DT, steps, mask.ravel(), 1000.0, 0.0, 1.0, 2,
                 conc=concs[1], hill=hill, rtol=TISSUE_RTOL)
    secs = time.perf_counter() - t0
    return {"value": nx * nx * steps / secs, "unit": "node-steps/s", "cores": 1, "kind": "port",
            "sample": f"{nx}x{nx} sheet, {steps} Godunov steps ({secs:.1f} s)"}


def tissue_main(args, world, rank, local, pg):
    peaks = measured_peaks() if rank == 0 else {}
    res, n, launches = run_tissue(args, world, rank, local, pg)
    if rank != 0:
        return
    mixed, fp64 = res["mixed"], res["fp64"]
    hbm, src = hbm_peak(peaks)
    ns = importlib.import_module("2ddrugsimulation_b200").N_STATES["tt2006"]
    roofs = {prec: phase_rooflines("tt2006", prec, 3 * n, args.steps * args.seg, res[prec]["timing"],
                                   res[prec]["fmt"], res[prec]["ell_width"], res[prec]["cg_iters_per_solve"], ns,
                                   peaks, hbm, src) for prec in ("mixed", "fp64")}
    rm = roofs["mixed"]
    dominant = rm["ionic"] if rm["ionic_share"] >= 0.5 else rm["diffusion"]
    line = {
        "metric": "TT2006 monodomain node-steps/s (Godunov: ionic + Jacobi-PCG), mixed vs FP64",
        "value": mixed["value"], "unit": "node-steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": mixed["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64 (mixed ionic), f64 PCG", "data": "synthetic",
        "config": {"workload": f"2D TT2006 epi sheet {args.nx}x{args.nx} Q1 nodes, dx 0.025 cm, D 0.0013 cm^2/ms, "
                               f"dt 0.01 ms, Jacobi-PCG rtol 1e-8, corner S1 at BCL 1000 ms, IKr Hill block at 3 "
                               f"concentrations (3 sheets per GPU stepped as one group: one batched PCG launch per "
                               f"step); {args.seg} Godunov steps per sheet per bench step",
                   "nodes_per_sheet": n, "sheets_per_gpu": 3, "sparse_format": ["csr", "ell", "stencil", "classed"][mixed["fmt"]],
                   "l2": "flushed between timed steps (256 MiB write)", "parallelism": f"sheet sharding x{world}"},
        "fp64": {"value": fp64["value"], "ms_per_step": fp64["ms_per_step"], "clocks": fp64["clocks"],
                 "cg_iters_per_solve": fp64["cg_iters_per_solve"], "phases": roofs["fp64"]},
        "mixed_over_fp64": mixed["value"] / fp64["value"],
        "cg_iters_per_solve": mixed["cg_iters_per_solve"], "not_converged": mixed["not_converged"] + fp64["not_converged"],
        "roofline": dominant, "phases": rm,
        "gpu_launches": launches, "clocks": mixed["clocks"],
        "cpu_baseline": None if args.no_cpu else tissue_cpu(args),
        "e2e": res.get("e2e"),
    }
    return line


# ------------------------------------------------------------ serving workload
SERVE_BCL, SERVE_DT = 1000.0, 0.005


def serve_trace(n_jobs: int, seed: int):
    """Seeded screening jobs: four in five are CiPA populations of
    log-U[20, 500] samples x 1-4 concentrations, 1-2 paces at BCL 1000 ms
    (biomarkers on the last pace), each around its own nominal drug; one in
    five is a 2D TT2006 patch of log-U[64, 192]^2 nodes for U[50, 200] ms
    (dt 0.01 ms, corner S1) with an IKr Hill block."""
    rng = np.random.default_rng(seed)
    jobs = []
    for k in range(n_jobs):
        if rng.uniform() < 0.2:
            nx = int(round(10 ** rng.uniform(np.log10(64), np.log10(192))))
            hill = np.zeros(14)
            hill[12], hill[13] = 10 ** rng.uniform(-1, 2), rng.uniform(0.6, 1.8)
            jobs.append(dict(kind="tissue", nx=nx, duration=float(rng.uniform(50, 200)),
                             conc=float(10 ** rng.uniform(-2, 1)), hill=hill))
            continue
        ns = int(round(10 ** rng.uniform(np.log10(20), np.log10(500))))
        nc = int(rng.integers(1, 5))
        paces = int(rng.integers(1, 3))
        conc, hill = population("cipa2017", ns, nc, seed=seed * 1000 + k)
        jobs.append(dict(kind="pop", conc=conc, hill=hill, n_pace=paces, first_pace=paces - 1))
    return jobs


def submit_job(srv, j):
    if j["kind"] == "tissue":
        return srv.submit_tissue(j["nx"], j["nx"], j["duration"], conc=j["conc"], hill=j["hill"],
                                 stim=(max(2, j["nx"] // 32),) * 2)
    return srv.submit(j["conc"], j["hill"], bcl=SERVE_BCL, n_pace=j["n_pace"], first_pace=j["first_pace"])


def job_steps(j) -> int:
    if j["kind"] == "tissue":
        return j["nx"] * j["nx"] * int(round(j["duration"] / 0.01))
    return len(j["conc"]) * int(j["n_pace"] * SERVE_BCL / SERVE_DT)


def run_serving(cep, jobs, arrivals, mode: str, capacity: int, k_steps: int):
    """Replay the trace: 'batched' submits every job at its arrival time
    (continuous batching); 'serial' runs one job at a time in arrival order.
    Returns per-job latencies (ms from arrival to completion), the makespan
    and the server's counters."""
    srv = cep.Server("cipa2017", "mixed", capacity=capacity, dt=SERVE_DT, max_bcl=SERVE_BCL, steps_per_launch=k_steps)
    try:
        t0 = time.perf_counter()
        lat = [0.0] * len(jobs)
        if mode == "batched":
            ids = []
            for j, ta in zip(jobs, arrivals):
                d = t0 + ta - time.perf_counter()
                if d > 0:
                    time.sleep(d)
                ids.append(submit_job(srv, j))
            for k, (j, jid) in enumerate(zip(jobs, ids)):
                srv.wait(jid, 0)
                tm = srv.tissue_result(jid)[2] if j["kind"] == "tissue" else srv.result(jid)[1]
                lat[k] = tm["latency_ms"]
        else:
            for k, (j, ta) in enumerate(zip(jobs, arrivals)):
                d = t0 + ta - time.perf_counter()
                if d > 0:
                    time.sleep(d)
                jid = submit_job(srv, j)
                srv.wait(jid, 0)
                lat[k] = (time.perf_counter() - (t0 + ta)) * 1e3
        makespan = time.perf_counter() - t0
        st = srv.stats()
    finally:
        srv.close()
    return np.array(lat), makespan, st


def serve_main(args):
    cep = importlib.import_module("2ddrugsimulation_b200")
    jobs = serve_trace(args.jobs, 777)
    steps = [job_steps(j) for j in jobs]
    capacity, k_steps = 16384, 10000
    # calibration: every job once, back to back and one at a time, gives
    # each job's service time; arrivals are then Poisson at 1.2x the rate
    # one-at-a-time service sustains
    lat0, _, _ = run_serving(cep, jobs, np.zeros(len(jobs)), "serial", capacity, k_steps)
    service = np.diff(np.concatenate([[0.0], lat0])) / 1e3  # s
    mean_service = float(service.mean())
    rng = np.random.default_rng(778)
    gaps = rng.exponential(mean_service / 1.2, len(jobs))
    arrivals = np.cumsum(gaps) - gaps[0]
    res = {}
    for mode in ("batched", "serial"):
        lat, span, st = run_serving(cep, jobs, arrivals, mode, capacity, k_steps)
        res[mode] = {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                     "mean_ms": float(lat.mean()), "makespan_s": span,
                     "cell_steps_per_s": float(sum(steps)) / span, "launches": int(st["launches"])}
    b, s_ = res["batched"], res["serial"]
    line = {
        "metric": "screen-job p50/p99 latency (continuous batching vs one at a time), CiPA-ORd populations and TT2006 patches, mixed",
        "value": b["p99_ms"], "unit": "ms (p99 latency)", "n_gpus": 1, "steps": len(jobs), "warmup": 3,
        "ms_per_step": b["mean_ms"], "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64 (mixed)", "data": "synthetic",
        "config": {"workload": f"{len(jobs)} Poisson-arriving screening jobs: CiPA-ORd populations (log-U[20,500] "
                               f"samples x 1-4 concs, 1-2 paces at BCL 1000 ms, dt 0.005 ms, biomarkers on the last "
                               f"pace) and, one in five, 2D TT2006 patches (log-U[64,192]^2 nodes, U[50,200] ms, dt "
                               f"0.01 ms, IKr block); offered load 1.2x one-at-a-time capacity; pool of {capacity} "
                               f"slots, {k_steps} steps per launch (scaled down from 2,000 jobs of 100-5,000 samples "
                               f"x 200-1,000 paces and 64^2-384^2 patches for 500-2,000 ms)",
                   "n_tissue_jobs": sum(j["kind"] == "tissue" for j in jobs), "total_cell_steps": int(sum(steps)),
                   "mean_service_s_one_at_a_time": mean_service},
        "latency_ms": {"p50": b["p50_ms"], "p99": b["p99_ms"]},
        "serial": s_, "batched": b,
        "p99_speedup_vs_serial": s_["p99_ms"] / b["p99_ms"],
        "throughput_speedup_vs_serial": b["cell_steps_per_s"] / s_["cell_steps_per_s"],
        "gpu_launches": b["launches"], "cpu_baseline": None, "e2e": None,
    }
    return line


# ------------------------------------------------------------ 3D ORd slab workload
SLAB_NZ, SLAB_DL, SLAB_DT_ = 48, 0.0013, 0.00045


def slab_fields(nx: int, ny: int, nz: int):
    """Transmural layers (endo 30 % / M 40 % / epi 30 % of the depth, ORd
    celltypes 0 / 2 / 1), fibre angle rotating linearly from -60 to +60 deg
    from the endocardial (z = 0) to the epicardial face, conductivity
    D = Dt I + (Dl - Dt) f f^T per element at its centroid depth, and the
    endocardial surface (the first two node planes, 0.025 cm: one plane
    alone does not excite the slab against its electrotonic load) as the S1
    region, stimulated for 1 ms."""
    z = np.arange(nz) / (nz - 1)
    ct_z = np.where(z < 0.3, 0.0, np.where(z < 0.7, 2.0, 1.0))
    celltype = np.repeat(ct_z, nx * ny)
    zc = (np.arange(nz - 1) + 0.5) / (nz - 1)
    th = np.deg2rad(-60.0 + 120.0 * zc)
    fx, fy = np.cos(th), np.sin(th)
    d = np.zeros((nz - 1, 6))  # xx, xy, xz, yy, yz, zz
    d[:, 0] = SLAB_DT_ + (SLAB_DL - SLAB_DT_) * fx * fx
    d[:, 1] = (SLAB_DL - SLAB_DT_) * fx * fy
    d[:, 3] = SLAB_DT_ + (SLAB_DL - SLAB_DT_) * fy * fy
    d[:, 5] = SLAB_DT_
    D = np.repeat(d, (nx - 1) * (ny - 1), axis=0)
    mask = np.zeros(nx * ny * nz, np.uint8)
    mask[: 2 * nx * ny] = 1
    return celltype, D, mask


def slab_main(args, world, rank, local, pg):
    import torch
    cep = importlib.import_module("2ddrugsimulation_b200")
    torch.cuda.set_device(local)
    nx = args.nx if args.nx != 512 else 256
    ny, nz = nx, SLAB_NZ
    n = nx * ny * nz
    celltype, D, mask = slab_fields(nx, ny, nz)
    rng = np.random.default_rng(5150 + rank)
    hill = np.zeros(14)
    hill[0::2] = 10 ** rng.uniform(-1, 2, 7)
    hill[1::2] = rng.uniform(0.6, 1.8, 7)
    cmax = 10 ** rng.uniform(-2, 1)
    concs = [cmax, 3 * cmax]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    res = {}
    fmt = format_arg(cep, args)
    for prec in ("mixed", "fp64"):
        slabs = []
        for c in concs:
            cells = cep.Batch("ord2011", n, prec)
            cells.init(celltype=celltype, conc=np.full(n, c), hill=hill, quirks=False)
            fem = cep.Fem.grid(3, nx, ny, nz, TISSUE_H, TISSUE_DT, D, fmt=cep.FEM_AUTO if fmt is None else fmt)
            fem.set_solver(TISSUE_RTOL)
            fmt = fem.format
            t = cep.Tissue(cells, fem, TISSUE_DT)
            t.set_stimulus(mask, 1000.0, 0.0, 1.0, 1)
            slabs.append(t)
        group = cep.TissueGroup(slabs)
        for _ in range(args.warmup):
            group.run(args.seg)
            flush.zero_()
        torch.cuda.synchronize()
        it0 = sum(t.stats()["cg_iters"] for t in slabs)
        group.set_timing(True)
        barrier(pg)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clk:
            start.record()
            for _ in range(args.steps):
                group.run(args.seg)
                flush.zero_()
            stop.record()
            torch.cuda.synchronize()
        barrier(pg)
        timing = group.timing()
        ms = max_over_ranks(start.elapsed_time(stop), pg)
        st = [t.stats() for t in slabs]
        cg = sum(x["cg_iters"] for x in st) - it0
        res[prec] = dict(value=n * len(slabs) * args.seg * args.steps * world / (ms / 1e3), ms_per_step=ms / args.steps,
                         clocks=clk.summary(), cg_iters_per_solve=cg / (len(slabs) * args.seg * args.steps),
                         not_converged=sum(x["not_converged"] for x in st), width=slabs[0].fem.ell_width,
                         timing=timing)
        group.close()
        for t in slabs:
            t.close()
        del slabs
        torch.cuda.empty_cache()
    if rank != 0:
        return
    mixed, fp64 = res["mixed"], res["fp64"]
    peaks = measured_peaks()
    hbm, src = hbm_peak(peaks)
    roofs = {prec: phase_rooflines("ord2011", prec, 2 * n, args.steps * args.seg, res[prec]["timing"], fmt,
                                   res[prec]["width"], res[prec]["cg_iters_per_solve"], cep.N_STATES["ord2011"],
                                   peaks, hbm, src) for prec in ("mixed", "fp64")}
    rm = roofs["mixed"]
    cpu = None
    if not args.no_cpu:
        from oracle import oracle as O
        cx, cz, steps = 16, 8, 600
        ct_s, D_s, m_s = slab_fields(cx, cx, cz)
        t0 = time.perf_counter()
        O.tissue_run("ord2011", 3, cx, cx, cz, TISSUE_H, D_s, TISSUE_DT, steps, m_s, 1000.0, 0.0, 1.0, 1, conc=concs[0],
                     hill=hill, rtol=TISSUE_RTOL, celltype=ct_s)
        secs = time.perf_counter() - t0
        cpu = {"value": cx * cx * cz * steps / secs, "unit": "node-steps/s", "cores": 1, "kind": "port",
               "sample": f"{cx}x{cx}x{cz} slab, {steps} Godunov steps ({secs:.1f} s)"}
    line = {
        "metric": "ORd 3D slab node-steps/s (Godunov: ionic + Jacobi-PCG, anisotropic), mixed vs FP64",
        "value": mixed["value"], "unit": "node-steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": mixed["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64 (mixed ionic), f64 PCG", "data": "synthetic",
        "config": {"workload": f"3D slab {nx}x{ny}x{nz} trilinear hex nodes, dx 0.025 cm, endo/M/epi ORd layers "
                               f"30/40/30 %, fibre angle -60..+60 deg transmurally, D 0.0013/0.00045 cm^2/ms, "
                               f"endocardial-surface S1 (2 node planes, 1 ms), dt 0.01 ms, Jacobi-PCG rtol 1e-8, 7-channel Hill drug at 2 "
                               f"concentrations (2 slabs stepped as one group); {args.seg} Godunov steps per bench step",
                   "nodes_per_slab": n, "slabs_per_gpu": 2, "sparse_format": ["csr", "ell", "stencil", "classed"][fmt],
                   "l2": "flushed between timed steps (256 MiB write)", "parallelism": f"slab sharding x{world}"},
        "fp64": {"value": fp64["value"], "ms_per_step": fp64["ms_per_step"], "clocks": fp64["clocks"],
                 "cg_iters_per_solve": fp64["cg_iters_per_solve"], "phases": roofs["fp64"]},
        "mixed_over_fp64": mixed["value"] / fp64["value"], "cg_iters_per_solve": mixed["cg_iters_per_solve"],
        "not_converged": mixed["not_converged"] + fp64["not_converged"],
        "roofline": rm["ionic"] if rm["ionic_share"] >= 0.5 else rm["diffusion"], "phases": rm,
        "gpu_launches": args.steps * args.seg * 3, "clocks": mixed["clocks"],
        "cpu_baseline": cpu, "e2e": None,
    }
    return line


def main():
    args = parse()
    model = model_of(args.workload)
    if args.workload == "ord_slab":
        world, rank, local, pg = dist_setup()
        line = slab_main(args, world, rank, local, pg)
        if line is not None:
            print(json.dumps(line))
        if pg is not None:
            pg.destroy_process_group()
        return
    if args.workload == "serve":
        print(json.dumps(serve_main(args)))
        return
    if args.workload == "tt06_sheet":
        world, rank, local, pg = dist_setup()
        if args.impl == "reference":
            if rank == 0:
                cpu = tissue_cpu(args)
                print(json.dumps({"impl": "reference", "metric": "TT2006 monodomain node-steps/s", "value": cpu["value"],
                                  "unit": "node-steps/s", "n_gpus": args.gpus, "steps": args.steps,
                                  "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                                  "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                                  "config": {"workload": "TT2006 sheet (oracle port; the reference tissue solver "
                                                         "needs PETSc, absent)", "sample": cpu["sample"]},
                                  "cpu_baseline": cpu, "e2e": {"value": cpu["value"], "unit": "node-steps/s",
                                                               "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
            return
        line = tissue_main(args, world, rank, local, pg)
        if line is not None:
            print(json.dumps(line))
        if pg is not None:
            pg.destroy_process_group()
        return
    world, rank, local, pg = dist_setup()
    conc, hill = population(model, args.samples, args.concs, seed=1234)
    threads = os.cpu_count() or 1
    if args.impl == "reference":
        if rank != 0:
            return
        per_thread = 400000  # one 2000-ms beat per thread per bench step
        rates = []
        kind = "port"
        for _ in range(args.warmup + args.steps):
            r, kind, _ = cpu_rate(model, conc, hill, threads, per_thread)
            rates.append(r)
        v = statistics.mean(rates[args.warmup:])
        sample = (f"{threads} instances spread evenly over the {len(conc)}-instance population x {per_thread} fixed "
                  f"steps (one 2000-ms beat) per bench step")
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "cell-steps/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": config_of(args, model, len(conc), world) | {"sample": sample},
                "cpu_baseline": {"value": v, "unit": "cell-steps/s", "cores": threads, "kind": kind, "sample": sample},
                "e2e": {"value": v, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return
    peaks = measured_peaks() if rank == 0 else {}
    res, n, launches = run_ours(args, world, rank, local, pg, model)
    if rank != 0:
        if pg is not None:
            pg.destroy_process_group()
        return
    cpu = None
    if not args.no_cpu:
        steps = calibrate_cpu(model, conc, hill, threads, args.cpu_seconds)
        r, kind, secs = cpu_rate(model, conc, hill, threads, steps)
        cpu = {"value": r, "unit": "cell-steps/s", "cores": threads, "kind": kind,
               "sample": f"{threads} instances spread evenly over the population x {steps} fixed steps, one per "
                         f"thread ({secs:.1f} s)"}
    mixed, fp64 = res["mixed"], res["fp64"]
    fl = flops_per_step(model)
    steps_per_bench_step = args.seg * beat_launches(args)  # time steps every instance takes per bench step
    cell_steps_launch = n * steps_per_bench_step  # per bench step (kernel_ms is per bench step)

    def roof(kernel_ms, peak_key, label, per_step=fl, source="bench.py FMA probe on this GPU (2 flop/FMA)"):
        ach = per_step * cell_steps_launch / (kernel_ms * 1e-3) / 1e12
        pk = peaks.get(peak_key)
        tr = TRAFFIC_PER_INSTANCE.get(model)
        return {"bound": label, "achieved": ach, "peak": pk, "unit": "TFLOP/s",
                "frac": (ach / pk) if pk else None, "traffic": (tr * n) if tr else None,
                "flops_per_cell_step": per_step, "peak_source": source}

    sfu = sfu_ops_per_step(model)

    comp = res["compliant"]
    line = {
        "metric": METRIC, "value": comp["value"], "unit": "cell-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": comp["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32+f64 (mixed; FP64 for the drug-depolarised instances, concurrently)", "data": "synthetic",
        "config": config_of(args, model, n, world),
        "compliant": {k: comp[k] for k in ("n_candidates", "candidate_fraction", "refine_above_vm",
                                           "kernel_ms_mixed", "kernel_ms_fp64_candidates", "clocks")} | {
            "us_per_step_fp64_candidates": comp["kernel_ms_fp64_candidates"] * 1e3 / steps_per_bench_step,
            "us_per_step_mixed": comp["kernel_ms_mixed"] * 1e3 / steps_per_bench_step,
            "what": "value = the mixed population (stream 1) with the instances whose diastolic Vm after the "
                    "screening beat stays above refine_above_vm in FP64 (stream 2), one beat of both per step: "
                    "the path whose records meet APD90 <= 0.1 ms against FP64 for every instance"},
        "mixed_plain": {"value": mixed["value"], "ms_per_step": mixed["ms_per_step"], "kernel_ms": mixed["kernel_ms"],
                        "note": "mixed precision for every instance, no FP64 refinement (misses the APD90 bar "
                                "for non-repolarising instances)"},
        "fp64": {"value": fp64["value"], "ms_per_step": fp64["ms_per_step"], "kernel_ms": fp64["kernel_ms"],
                 "us_per_step": fp64["kernel_ms"] * 1e3 / steps_per_bench_step,
                 "roofline": roof(fp64["kernel_ms"], "fp64_tflops", "fp64"), "clocks": fp64["clocks"]},
        "mixed_over_fp64": comp["value"] / fp64["value"],
        "mixed_plain_over_fp64": mixed["value"] / fp64["value"],
        "kernel_ms": mixed["kernel_ms"],
        # The mixed kernel is bound by the special-function unit: every
        # division, exponential and logarithm is one MUFU operation (16 per
        # SM per clock on B200), ~390 per cell-step against ~1,900 issue
        # slots. "flop" here = one such algorithmic operation.
        "roofline": roof(mixed["kernel_ms"], "sfu_tops", "sfu", per_step=sfu,
                         source="bench.py ex2.approx throughput probe on this GPU (1 op/MUFU)"),
        "roofline_fp32_pipe": roof(mixed["kernel_ms"], "fp32_tflops", "fp32"),
        "gpu_launches": launches,
        "clocks": comp["clocks"],
        "cpu_baseline": cpu,
        "e2e": comp.get("e2e"),
        "e2e_mixed_plain": res.get("e2e"),
        "instances_nonfinite": mixed["n_nonfinite"] + fp64["n_nonfinite"] + comp["n_nonfinite"],
        "peaks": {k: v for k, v in peaks.items() if k != "measured_peaks_json"},
    }
    if world == 1 and not args.no_sub and args.workload == "cipa_pop":
        line["sub_results"] = sub_results(args)
    print(json.dumps(line))
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
