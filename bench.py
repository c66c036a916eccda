#!/usr/bin/env python
"""Throughput of the FDMT + normalise + boxcar + cluster search path on B200.

    python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]
                    [--workload config2|config0|config1|config3|config4|config4fwd]
                    [--form both|batched] [--no-e2e] [--no-cpu-baseline] [--dry-run]
                    [--save-schedules FILE | --schedules FILE]

--gpus N without torchrun relaunches this script as N ranks through
torch.distributed.run (127.0.0.1); under torchrun the ranks come from the
environment.

Workload (default ``config2``): the batched multi-beam search — 48 beams of
uneven shapes (nchan from {256, 512, 1024, 4096}, 2^14..2^17 samples, max
delay = nchan, 1200-1600 MHz, 0-3 injected pulses), seeded synthetic N(0,1)
data generated on the device.  A step is one pass of the whole path over all
48 beams: FDMT -> per-row statistics -> fused normalise + boxcar (widths
1..32, S/N > 7) + compaction -> 3-pass clustering (+-16 samples, +-8 rows,
any width) -> delegates copied to the host.  The headline is the batched
form (every beam's FDMT + statistics + boxcar replayed from one CUDA graph,
then one sort and one clustering for all beams), pipelined: run i + 1's
graph is submitted before run i is collected, so run i's sort and
clustering overlap the next run's FDMT (``batched_sync`` times the same
form one run at a time); the plain per-beam form
(the same kernels with host round trips per beam) is timed beside it and
must return identical results.  ``config0`` is the single
512 x 32768 beam of the reference's CPU-runnable case; ``config4fwd`` one
1024 x 65536 beam (used for profiling: its input exceeds L2).  The other
workloads print their own line with the same metric: ``config1`` one raw
32-channel GUPPI chunk through the coherent stage (fused unpack + FFT, chirp,
inverse FFTs, detection) into the FDMT and search; ``config3`` a 4096 x 2^17
plane with FP32 / FP16 / BF16 FDMT planes (error against FP64, recall against
FP32); ``config4`` forward against adjoint FDMT with the gradient checks.

Metric: channel*samples per second over the whole job (all ranks).
``value`` is device-timed with inputs already in HBM (the working set of
each beam, 0.1-11 GB, exceeds the 126 MB L2 between uses, so no flush is
needed); ``e2e`` is the same metric through the public API with each beam's
input copied from pinned host memory every step and the delegates read back.
Under torchrun each rank processes its own 48-beam set (weak scaling, no
collective on the data path); the step time is the max over ranks.

CPU figures (rank 0, one GPU): ``cpu_baseline`` is the reference's own
CFdmtCpu (built from its sources into oracle/_ref) plus the oracle's
row-normalise / boxcar / cluster on a bounded sample of the beams;
``cpu_baseline_variant`` the same with the reference's other CPU FDMT
(FDMTCPU, Pravir plan), labelled as a different FDMT variant.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

METRIC = "chan*samples/s FDMT+boxcar search, batched vs plain, 1 B200; % HBM peak"
UNIT = "chan*samples/s"
SEARCH = dict(widths_mode=0, param=5, thr=7.0, metrics=(16, 8, 1 << 30))


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["config2", "config0", "config4fwd", "config3", "config4",
                                           "config1"], default="config2")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--dry-run", action="store_true",
                    help="rank coordination only (launch, barrier, max over ranks, per-rank beam "
                         "sets) with no GPU work: prints the line's shape with value null")
    ap.add_argument("--form", choices=["both", "batched"], default="both",
                    help="batched: time only the batched form (profiling runs; no plain-form "
                         "numbers, no FDMT roofline)")
    ap.add_argument("--save-schedules", metavar="FILE",
                    help="write the autotuner's FDMT schedule of every beam (JSON)")
    ap.add_argument("--schedules", metavar="FILE",
                    help="use these FDMT schedules (from --save-schedules) instead of autotuning: "
                         "a profiled run then executes the kernels an unprofiled run chose")
    return ap.parse_args(argv)


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def beams_for(workload: str, rank: int):
    """The workload's beams for one rank: every rank gets the same shapes
    (weak scaling: fixed work per GPU) with its own noise (another data seed
    per rank)."""
    import dataclasses

    from cpp_projects_b200 import synth
    if workload == "config0":
        beams = [synth.config0(seed=1)]
    elif workload == "config4fwd":
        beams = [synth.config4(seed=4)]
    elif workload == "config3":
        beams = [synth.config3(seed=3)]
    else:
        beams = synth.config2(seed=2)
    if rank:
        beams = [dataclasses.replace(b, seed=b.seed + 1_000_003 * rank) for b in beams]
    return beams


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while running."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.tmp = None

    def start(self):
        if shutil.which("nvidia-smi") is None:
            return self
        self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = subprocess.Popen(
            ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
             "-i", str(self.gpu), "-lms", "200"], stdout=self.tmp, stderr=subprocess.DEVNULL)
        # let the sampler start up (and print its first line) before the
        # caller times anything: its start-up competes for the host
        t0 = time.time()
        while time.time() - t0 < 3.0 and os.path.getsize(self.tmp.name) == 0:
            time.sleep(0.05)
        return self

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.tmp.flush()
        lines = [ln.split(",") for ln in Path(self.tmp.name).read_text().splitlines() if ln.strip()]
        os.unlink(self.tmp.name)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for f in lines:
            try:
                sm.append(float(f[1])); smax = float(f[2])
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, f[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
def cpu_reference_leg(beams, max_seconds: float = 15.0, min_steps: int = 1):
    """The reference's own CPU FDMT (CFdmtCpu, oracle/_ref, all host threads)
    followed by the oracle's CPU restatement of per-row normalisation, boxcar
    (OpenMP over rows) and clustering, on the given beams (cycled) until
    max_seconds of work.  Returns (chan*samples/s, seconds, sample text, kind)."""
    from oracle import pyoracle
    threads = os.cpu_count() or 1
    ref = pyoracle.ref_lib() is not None
    done, secs, k = 0, 0.0, 0
    names = []
    while (secs < max_seconds and k < 64) or k < min_steps:
        b = beams[k % len(beams)]
        from cpp_projects_b200 import synth
        x = synth.filterbank(b)
        t0 = time.perf_counter()
        if ref:
            dm = pyoracle.ref_fdmt_cpu(b.fmin, b.fmax, x, b.nchan, b.nsamp, b.max_dt, threads=threads)
        else:
            dm = pyoracle.fdmt_f32(b.fmin, b.fmax, x, b.nchan, b.nsamp, b.max_dt)
        z, _, _ = pyoracle.norm_rows(dm)
        c = pyoracle.boxcar_mt(z, SEARCH["thr"], SEARCH["widths_mode"], SEARCH["param"], cap=1 << 27)
        if len(c):
            pyoracle.cluster(c, SEARCH["metrics"])
        secs += time.perf_counter() - t0
        done += b.nchan * b.nsamp
        names.append(f"{b.nchan}x{b.nsamp}")
        k += 1
    kind = "reference" if ref else "port"
    sample = (f"{k} beam(s) [{', '.join(names[:6])}{', ...' if k > 6 else ''}]: "
              f"{'reference CFdmtCpu' if ref else 'oracle FDMT port'} ({threads} threads) + "
              f"oracle row-normalise/boxcar ({threads} threads)/cluster (1 thread)")
    return done / secs, secs, sample, kind, threads


def cpu_pravir_leg(beams, max_seconds: float = 6.0):
    """A second CPU figure, labelled as a different FDMT variant: the
    reference's other CPU FDMT (FDMTCPU, Pravir plan, oracle/_ref, all host
    threads; its output rows are its own delay grid) followed by the same
    row-normalise / boxcar / cluster restatement, on the given beams (cycled)
    until max_seconds of work.  None when oracle/_ref holds no FDMTCPU."""
    from cpp_projects_b200 import synth
    from oracle import pyoracle
    if pyoracle.ref_pravir_lib() is None:
        return None
    threads = os.cpu_count() or 1
    done, secs, k = 0, 0.0, 0
    names = []
    while (secs < max_seconds and k < 64) or k < 1:
        b = beams[k % len(beams)]
        x = synth.filterbank(b)
        t0 = time.perf_counter()
        dm = pyoracle.ref_pravir_cpu(b.fmin, b.fmax, x, b.nchan, b.nsamp, b.max_dt, threads=threads)
        if dm is None:
            return None
        z, _, _ = pyoracle.norm_rows(dm)
        c = pyoracle.boxcar_mt(z, SEARCH["thr"], SEARCH["widths_mode"], SEARCH["param"], cap=1 << 27)
        if len(c):
            pyoracle.cluster(c, SEARCH["metrics"])
        secs += time.perf_counter() - t0
        done += b.nchan * b.nsamp
        names.append(f"{b.nchan}x{b.nsamp}")
        k += 1
    return {"value": done / secs, "unit": UNIT, "cores": threads, "kind": "reference",
            "label": "different FDMT variant (the reference's FDMTCPU, Pravir plan)",
            "sample": (f"{k} beam(s) [{', '.join(names[:6])}{', ...' if k > 6 else ''}]: reference FDMTCPU "
                       f"({threads} threads) + oracle row-normalise/boxcar ({threads} threads)/cluster "
                       f"(1 thread)"),
            "seconds": secs}


def stratified(beams):
    """The workload's beams ordered for bounded samples: the smallest beam of
    every channel count, then the second smallest of every count, ... (every
    channel class appears in the first few beams of a sample)."""
    by = {}
    for b in sorted(beams, key=lambda b: b.nchan * b.nsamp):
        by.setdefault(b.nchan, []).append(b)
    out = []
    for k in range(max(len(v) for v in by.values())):
        out += [v[k] for n, v in sorted(by.items()) if k < len(v)]
    return out


def reference_gpu_leg(sample, warmup: int, nbeams: int = 4):
    """The reference's own GPU search path, built from its sources into
    oracle/_ref/libref_gpu.so: CFdmtGpu::process_image, then (the reference has
    no per-row normalisation: this build's, as a stand-in) its
    gather_candidates_in_dynamicalArray and complete_clusterization with its
    log, on one beam of each channel count (the first `nbeams` of the
    stratified sample), wall clock with device synchronisation.  None when the
    library or a GPU is missing."""
    try:
        import torch
    except ImportError:
        return None
    from oracle import pyoracle
    if not torch.cuda.is_available() or pyoracle.ref_gpu_lib() is None:
        return None
    from cpp_projects_b200 import search
    from cpp_projects_b200.pipeline import device_filterbank
    lib = pyoracle.ref_gpu_lib()
    dev = torch.device("cuda", 0)
    beams = sample[:nbeams]
    thr = torch.tensor([SEARCH["thr"]], device=dev)
    metrics = torch.tensor(list(SEARCH["metrics"]), dtype=torch.int32, device=dev)
    log = str(Path(tempfile.gettempdir()) / "bench_ref_gpu.log").encode()
    secs, units = 0.0, 0
    for rep in range(max(1, warmup) + 1):   # the first pass warms up
        for b in beams:
            x = device_filterbank(b.nchan, b.nsamp, b.fmin, b.fmax, b.seed, b.pulses, dev)
            f = pyoracle.RefFdmtGpu(b.fmin, b.fmax, b.nchan, b.nsamp, b.max_dt)
            out = torch.empty((b.max_dt, b.nsamp), device=dev)
            z = torch.empty_like(out)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            if f.process_image(x.data_ptr(), out.data_ptr()) != 0:
                return None
            search.norm_rows(out, out=z)
            lib.ref_search_dynamic(z.data_ptr(), b.max_dt, b.nsamp, thr.data_ptr(), SEARCH["param"],
                                   metrics.data_ptr(), log, 1e-3, 0.0)
            torch.cuda.synchronize()
            if rep > 0:
                secs += time.perf_counter() - t0
                units += b.nchan * b.nsamp
            del f, out, z, x
    return {"value": units / secs, "unit": UNIT,
            "sample": f"{len(beams)} beam(s) [{', '.join(f'{b.nchan}x{b.nsamp}' for b in beams)}]: the "
                      "reference's CFdmtGpu + gather_candidates_in_dynamicalArray + complete_clusterization "
                      "(built from its sources for sm_100a), per-row normalisation by this build",
            "seconds": secs}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    beams = beams_for(args.workload, 0)
    sample = stratified(beams)
    for _ in range(args.warmup):
        cpu_reference_leg(sample[:1], max_seconds=0.0)
    done, secs_total, texts, kind, threads = 0.0, 0.0, "", "port", 1
    for s in range(args.steps):
        r, secs, texts, kind, threads = cpu_reference_leg(sample[s % 4:], max_seconds=10.0)
        done += r * secs
        secs_total += secs
    value = done / secs_total
    pravir = cpu_pravir_leg(sample, max_seconds=5.0)
    ref_gpu = reference_gpu_leg(sample, args.warmup)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs_total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded N(0,1) + injected pulses, generated on the host)",
            "impl": "reference",
            "config": {"workload": args.workload, "beams": len(beams),
                       "chan_samples_per_rank": int(sum(b.nchan * b.nsamp for b in beams)),
                       "nchan_set": sorted({b.nchan for b in beams}),
                       "search": "pow2 widths 1..32, S/N > 7, clusters +-16 samples/+-8 rows/any width",
                       "timed": "a bounded sample of the workload's beams per step (cpu_baseline.sample), "
                                "rate in channel-samples per second"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": texts},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "cpu_baseline_variant": pravir, "reference_gpu": ref_gpu}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
def run_ours(args):
    import torch

    from cpp_projects_b200.pipeline import (SCHEDULE_FIELDS, BatchedSearch, BeamShape, SearchPipeline,
                                            device_filterbank, tuned_schedule)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if not torch.cuda.is_available():
        print(json.dumps({"metric": METRIC, "error": "no CUDA device"}))
        return 1
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    from cpp_projects_b200.ranks import Ranks
    ranks = Ranks("nccl", dev)
    if args.warmup < 3:
        args.warmup = 3  # the timing rules require >= 3 warm-up steps

    beams = beams_for(args.workload, rank)
    shapes = [BeamShape(b.nchan, b.nsamp, b.fmin, b.fmax, b.max_dt) for b in beams]
    capacity = (1 << 26) if args.workload == "config2" else (1 << 24)
    schedules = None
    if args.schedules:
        schedules = json.loads(Path(args.schedules).read_text())["schedules"]
        if len(schedules) != len(shapes):
            raise SystemExit(f"{args.schedules}: {len(schedules)} schedules for {len(shapes)} beams")
    # both forms use the same FDMT plans: autotuned per shape, or the given schedules
    pipe = SearchPipeline(shapes, widths_mode=SEARCH["widths_mode"], param=SEARCH["param"],
                          thr=SEARCH["thr"], metrics=SEARCH["metrics"], capacity=capacity,
                          device=dev, fuse_depth=-2, schedules=schedules)
    if schedules is None:
        schedules = [tuned_schedule(s) for s in shapes]
    if args.save_schedules and rank == 0:
        Path(args.save_schedules).write_text(json.dumps({"fields": list(SCHEDULE_FIELDS),
                                                         "schedules": schedules}))
    # the batch holds every beam's candidates at once (config2: ~96M)
    batch = BatchedSearch(shapes, widths_mode=SEARCH["widths_mode"], param=SEARCH["param"],
                          thr=SEARCH["thr"], metrics=SEARCH["metrics"], capacity=capacity * 2,
                          use_graph=True, schedules=schedules)
    inputs = [device_filterbank(b.nchan, b.nsamp, b.fmin, b.fmax, b.seed, b.pulses, dev, gain=b.gain)
              for b in beams]
    torch.cuda.synchronize()

    barrier = ranks.barrier
    max_over_ranks = ranks.max

    # ---- device-resident timing: plain per-beam form -------------------------
    plain = args.form == "both"
    clocks = ClockSampler(local).start()
    plain_results, plain_launches, plain_ms, fdmt_ms = None, None, None, None
    if plain:
        for _ in range(args.warmup):
            pipe.run(inputs)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        fdmt_ev = []
        launches0 = pipe.launches
        e0.record()
        for _ in range(args.steps):
            plain_results = pipe.run(inputs, fdmt_timing=fdmt_ev)
        e1.record()
        torch.cuda.synchronize()
        plain_launches = (pipe.launches - launches0) // args.steps
        barrier()
        plain_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
        fdmt_ms = sum(a.elapsed_time(b) for a, b in fdmt_ev) / args.steps
    units = pipe.chan_samples * world

    # ---- device-resident timing: batched form (the headline) -----------------
    for _ in range(args.warmup):
        batch.run(inputs)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    b0.record()
    results = None
    for _ in range(args.steps):
        results = batch.run(inputs)
    b1.record()
    torch.cuda.synchronize()
    barrier()
    sync_ms = max_over_ranks(b0.elapsed_time(b1) / args.steps)
    sync_results = results

    # ---- device-resident timing: pipelined batched form (the headline) -----
    # run i + 1's FDMT + statistics + boxcar (its CUDA graph on the batch's
    # stage-1 stream) is submitted before run i is collected, so run i's sort
    # and clustering overlap it; every run still processes all beams
    for _ in range(args.warmup):
        batch.submit(inputs)
        batch.collect()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record()
    batch.submit(inputs)
    for i in range(args.steps):
        if i + 1 < args.steps:
            batch.submit(inputs)
        results = batch.collect()
    p1.record()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    step_ms = max_over_ranks(p0.elapsed_time(p1) / args.steps)
    value = units / (step_ms / 1e3)
    ncand = sum(r.n_candidates for r in results)
    launches = batch.launches_per_run(ncand)

    def _equal(xs, ys):
        return all(a.n_candidates == b.n_candidates and np.array_equal(a.delegates, b.delegates)
                   and np.array_equal(a.group_sizes, b.group_sizes) for a, b in zip(xs, ys))
    same_sync = _equal(sync_results, results)
    same = plain and _equal(plain_results, results) and same_sync

    peak, peak_kind = measured_peaks()
    fdmt_bytes = pipe.fdmt_alg_bytes()
    sched = pipe.fdmt_sched_bytes()
    sched_bytes = sum(sched)
    # achieved: the bytes this schedule must move (input, each plane that
    # reaches HBM written and read once, output) over the FDMT's event time;
    # traffic: those bytes scaled by the DRAM / schedule-byte ratio measured
    # with ncu on one FDMT of each channel count (profiles/traffic.json)
    achieved = sched_bytes / (fdmt_ms / 1e3) / 1e9 if plain else None
    traffic = None
    tf = ROOT / "profiles" / "traffic.json"
    if tf.exists():
        ratio = json.loads(tf.read_text()).get("fdmt_dram_over_sched", {})
        if all(str(b.nchan) in ratio for b in beams):
            traffic = sum(sb * ratio[str(b.nchan)] for sb, b in zip(sched, beams))
    compulsory = sum(4.0 * b.nsamp * (b.nchan + 3 * b.max_dt) for b in beams)
    # the autotuner's schedules: beams per (head depth or input segment, HBM passes)
    sched_counts = {}
    for p in pipe.plans:
        passes = p.passes()
        first = "head %d" % p.info.fuse_depth if p.info.fuse_depth else (
            "input segment" if passes and passes[0][2] > 0 else "level 0")
        key = f"{first}, {p.info.hbm_passes} merge passes"
        sched_counts[key] = sched_counts.get(key, 0) + 1
    pipe_bytes = fdmt_bytes + pipe.search_alg_bytes()

    # ---- end to end: pinned host inputs, copied every step ------------------
    e2e = None
    if not args.no_e2e:
        host = [torch.empty(x.shape, dtype=x.dtype, pin_memory=True) for x in inputs]
        for h, x in zip(host, inputs):
            h.copy_(x)
        torch.cuda.synchronize()
        h2d = sum(h.numel() * h.element_size() for h in host)
        for _ in range(2):  # eager run, then the capture of copies + compute
            batch.run_host(host, inputs)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record()
        d2h = 0
        for _ in range(args.steps):
            # every beam's input copied from pinned host memory, overlapped
            # with the search of the beams before it
            rs = batch.run_host(host, inputs)
            # the candidate counter, then per beam the delegates and group sizes
            d2h += 4 + sum(r.delegates.nbytes + 4 * len(r.group_sizes) for r in rs)
        f1.record()
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        barrier()
        e2e_ms = max_over_ranks(f0.elapsed_time(f1) / args.steps)
        # the bound: the same host buffers copied to the device and nothing else
        copy_ms = []
        for _ in range(3):
            f0.record()
            for h, x in zip(host, inputs):
                x.copy_(h, non_blocking=True)
            f1.record()
            torch.cuda.synchronize()
            copy_ms.append(f0.elapsed_time(f1))
        copy_ms = max_over_ranks(min(copy_ms[1:]))
        e2e = {"value": units / (e2e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h // args.steps, "ms_per_step": e2e_ms,
               "wall_ms_per_step": 1e3 * wall / args.steps,
               "h2d_gbs": h2d / e2e_ms / 1e6,
               "copy_only": {"ms_per_step": copy_ms, "gbs": h2d / copy_ms / 1e6,
                             "frac": copy_ms / e2e_ms,
                             "what": "the step's host inputs copied to the device alone (pinned, one stream)"}}
        del host

    # ---- CPU baseline (rank 0, N=1 only) -------------------------------------
    cpu = cpu_variant = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        small = stratified(beams)
        rate, secs, sample, kind, threads = cpu_reference_leg(small, max_seconds=12.0)
        cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": kind, "sample": sample,
               "seconds": secs}
        cpu_variant = cpu_pravir_leg(small, max_seconds=5.0)

    ndel = sum(len(r.delegates) for r in results)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded N(0,1) + injected dispersed pulses, generated on device)",
            "config": {"workload": args.workload,
                       "beams": len(beams), "chan_samples_per_rank": pipe.chan_samples,
                       "nchan_set": sorted({b.nchan for b in beams}),
                       "search": "pow2 widths 1..32, S/N > 7, clusters +-16 samples/+-8 rows/any width",
                       "l2": "no flush: each beam's working set (>= 100 MB) exceeds L2 between uses",
                       "form": "batched, pipelined: one CUDA graph for every beam's FDMT + "
                               "statistics + boxcar, one sort and one clustering for all beams; run "
                               "i + 1's graph submitted before run i's sort and clustering (two "
                               "candidate buffers)",
                       "parallelism": f"{world} independent rank(s), beams sharded, no collective"},
            "roofline": {"bound": "hbm",
                         "kernel": "FDMT (fused head or level 0, then fused merge segments)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak if plain else None, "peak_source": peak_kind,
                         "traffic": traffic,
                         "bytes": "achieved = schedule bytes per step / FDMT time; traffic = DRAM bytes "
                                  "per step (ncu ratio per channel count x schedule bytes)",
                         "sched_bytes_per_step": sched_bytes,
                         "level_by_level_bytes_per_step": fdmt_bytes,
                         "level_by_level_gbs": fdmt_bytes / (fdmt_ms / 1e3) / 1e9 if plain else None,
                         "compulsory_io_bytes_per_step": compulsory,
                         "compulsory_io": "input read + FDMT output written + row statistics and "
                                          "boxcar reads of the output",
                         "fdmt_ms_per_step": fdmt_ms, "schedules": sched_counts,
                         "timed_in": "plain per-beam form (events around each beam's FDMT; "
                                     "same autotuned plans as the batched form)"},
            "batched_sync": {"value": units / (sync_ms / 1e3), "ms_per_step": sync_ms,
                             "same_results_as_pipelined": same_sync,
                             "form": "each run's sort and clustering before the next run starts"},
            "plain": {"value": units / (plain_ms / 1e3), "ms_per_step": plain_ms,
                      "gpu_launches": plain_launches,
                      "batched_speedup": plain_ms / step_ms, "same_results_as_batched": same}
                     if plain else None,
            "pipeline_balg": {"bytes_per_step": pipe_bytes,
                              "gbs": pipe_bytes / (step_ms / 1e3) / 1e9,
                              "frac_of_peak": pipe_bytes / (step_ms / 1e3) / 1e9 / peak},
            "e2e": e2e, "cpu_baseline": cpu, "cpu_baseline_variant": cpu_variant,
            "clocks": clk, "gpu_launches": launches,
            "candidates": ncand, "delegates": ndel,
        }
        print(json.dumps(line), flush=True)
    ranks.close()
    return 0


def _cand_keys(cands, n, cols):
    """(row, sample, width) of each candidate as one int64 (device)."""
    import torch
    c = cands[:n].long()
    return (c[:, 1] * cols + c[:, 0]) * 64 + c[:, 2]


def run_config3(args):
    """Reduced-precision FDMT: one 4096 x 2^17 beam (1100-1500 MHz, bandpass
    gain, 20 pulses) through FDMT + row statistics + boxcar (widths 1..64,
    S/N > 7) + clustering with FP32, FP16 and BF16 planes between FDMT levels.
    Reports each form's device time, the 16-bit forms' FDMT difference from
    the FP32 form (on the first 8192 samples; the error against FP64 is
    asserted by the GPU tests), and candidate / delegate / injected-pulse
    recall of the 16-bit forms against FP32."""
    import torch

    from cpp_projects_b200 import search
    from cpp_projects_b200.pipeline import BeamShape, SearchPipeline, device_filterbank

    if not torch.cuda.is_available():
        print(json.dumps({"metric": METRIC, "error": "no CUDA device"}))
        return 1
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    args.warmup = max(args.warmup, 3)
    b = beams_for("config3", 0)[0]
    shape = BeamShape(b.nchan, b.nsamp, b.fmin, b.fmax, b.max_dt)
    x = device_filterbank(b.nchan, b.nsamp, b.fmin, b.fmax, b.seed, b.pulses, dev, gain=b.gain)
    search_cfg = dict(widths_mode=0, param=6, thr=7.0, metrics=(16, 8, 1 << 30))
    peak, peak_kind = measured_peaks()
    tw = 8192
    y32 = None                     # the FP32 form's first tw samples (the loop starts with it)
    forms = {}
    keys = {}
    clocks = ClockSampler(0).start()
    for name, prec in (("f32", 0), ("f16", 1), ("bf16", 2)):
        pipe = SearchPipeline([shape], capacity=1 << 27, device=dev, fuse_depth=-2, precision=prec,
                              **search_cfg)
        for _ in range(args.warmup):
            pipe.run([x])
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev = []
        e0.record()
        for _ in range(args.steps):
            res = pipe.run([x], fdmt_timing=ev)[0]
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        fdmt_ms = sum(a.elapsed_time(c) for a, c in ev) / args.steps
        alg = pipe.fdmt_alg_bytes()
        plane = pipe.plane[: b.max_dt * b.nsamp].view(b.max_dt, b.nsamp)
        y = plane[:, :tw].double().cpu().numpy()
        if y32 is None:
            y32 = y
        err = y - y32
        # the candidates of the last run are still in the pipeline's buffer
        keys[name] = _cand_keys(pipe.cands, res.n_candidates, b.nsamp)
        # an injected pulse is found when a candidate lies at its delay row
        # (+-16) and its arrival at the lowest channel (t0 + span, -64 .. +width+64)
        c = pipe.cands[: res.n_candidates]
        found = 0
        for p in b.pulses:
            t_end = p.t0 + p.span
            ok = (((c[:, 1] - p.span).abs() <= 16) & (c[:, 0] >= t_end - 64)
                  & (c[:, 0] <= t_end + p.width + 64))
            found += bool(ok.any().item())
        forms[name] = {
            "value": b.nchan * b.nsamp / (ms / 1e3), "ms_per_step": ms, "fdmt_ms": fdmt_ms,
            "fdmt_alg_bytes": alg, "fdmt_gbs": alg / (fdmt_ms / 1e3) / 1e9,
            "fdmt_frac": alg / (fdmt_ms / 1e3) / 1e9 / peak, "fuse_depth": pipe.plans[0].info.fuse_depth,
            "diff_vs_f32": {"max_rel_to_maxabs": float(np.abs(err).max() / np.abs(y32).max()),
                            "rms_rel": float(np.sqrt((err ** 2).mean() / (y32 ** 2).mean()))},
            "candidates": res.n_candidates, "delegates": len(res.delegates),
            "injected_found": f"{found}/{len(b.pulses)}",
            "_delegates": res.delegates,
        }
        del pipe
        torch.cuda.empty_cache()
    clk = clocks.stop()
    ref = keys["f32"]
    for name in ("f16", "bf16"):
        k = keys[name]
        hit = torch.isin(ref, k).sum().item()
        extra = (~torch.isin(k, ref)).sum().item()
        d32, d16 = forms["f32"]["_delegates"], forms[name]["_delegates"]
        dhit = sum(bool(((np.abs(d16["mdt"] - r["mdt"]) <= 8) & (np.abs(d16["mt"] - r["mt"]) <= 16)).any())
                   for r in d32)
        forms[name]["recall_vs_f32"] = {
            "candidates": hit / max(1, ref.numel()), "extra_candidates": extra,
            "delegates": dhit / max(1, len(d32))}
    for f in forms.values():
        f.pop("_delegates")
    h = forms["f16"]
    line = {
        "metric": METRIC, "value": h["value"], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": h["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 sums, f16 planes",
        "data": "synthetic (seeded N(0,1) x bandpass gain + 20 dispersed pulses, generated on device)",
        "config": {"workload": "config3", "nchan": b.nchan, "nsamp": b.nsamp, "band_mhz": [b.fmin, b.fmax],
                   "max_dt": b.max_dt, "search": "pow2 widths 1..64, S/N > 7, clusters +-16/+-8/any",
                   "l2": "no flush: 2 GiB input and output exceed L2", "form": "plain per-beam"},
        "roofline": {"bound": "hbm", "kernel": "FDMT, FP16 planes", "achieved": h["fdmt_gbs"],
                     "peak": peak, "unit": "GB/s", "frac": h["fdmt_frac"], "peak_source": peak_kind,
                     "traffic": None},
        "precision": forms, "clocks": clk, "e2e": None, "cpu_baseline": None,
    }
    print(json.dumps(line), flush=True)
    return 0


def _pulse_cells(plane, stats, beam, search):
    """The (row, start, width) cell of each injected pulse: the largest S/N
    at the pulse's width within +-4 rows and +-16 samples of its nominal
    position (row = delay span, start = arrival at the lowest channel)."""
    cells = []
    rows, cols = plane.shape
    for p in beam.pulses:
        d0, t0 = int(round(p.span)), p.t0 + int(round(p.span))
        grid = [(d, t, p.width) for d in range(max(0, d0 - 4), min(rows, d0 + 5))
                for t in range(max(0, t0 - 16), min(cols - p.width, t0 + 17))]
        snr = search.snr_cells(plane, stats, grid).cpu().numpy()
        cells.append(grid[int(np.argmax(snr))])
    return np.array(cells, np.int32)


def run_config4(args):
    """Differentiable FDMT: one 1024 x 65536 beam (8 pulses, 10 % of channels
    with RFI sinusoids of amplitude 5), per-channel weights w (initially 1),
    loss = -sum of boxcar S/N at the 8 pulse cells.  Times the forward FDMT,
    the adjoint FDMT and the whole forward + backward step (device events);
    checks the weight gradient against central finite differences (eps 0.05)
    of the loss on 4 channels (the FP64 gradient check is a GPU test); runs
    30 steps of projected gradient ascent on w in [0, 1] to show the S/N
    gain."""
    import torch

    from cpp_projects_b200 import CFdmtGpu, search, synth
    from cpp_projects_b200.autograd import boxcar_snr, fdmt
    from cpp_projects_b200.pipeline import device_filterbank

    if not torch.cuda.is_available():
        print(json.dumps({"metric": METRIC, "error": "no CUDA device"}))
        return 1
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    args.warmup = max(args.warmup, 3)
    b = synth.config4(seed=4, rfi=True)
    x = device_filterbank(b.nchan, b.nsamp, b.fmin, b.fmax, b.seed, b.pulses, dev, rfi=b.rfi)
    plan = CFdmtGpu(b.fmin, b.fmax, b.nchan, b.nsamp, b.max_dt, fuse_depth=-2)
    y = plan(x)
    cells = _pulse_cells(y, search.row_stats(y), b, search)
    gy = torch.randn_like(y)
    gx = torch.empty_like(x)
    peak, peak_kind = measured_peaks()

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps

    w = torch.ones(b.nchan, device=dev, requires_grad=True)

    def step():
        w.grad = None
        loss = -boxcar_snr(fdmt(w[:, None] * x, plan), cells).sum()
        loss.backward()
        return loss

    clocks = ClockSampler(0).start()
    fwd_ms = timed(lambda: plan.process_image(x, y))
    adj_ms = timed(lambda: plan.adjoint(gy, gx))
    step_ms = timed(step)
    clk = clocks.stop()
    loss = step()
    g_gpu = w.grad.double().cpu().numpy()

    # central differences of the loss on 4 channels, through this build's own
    # forward path (FP32; eps 0.05 keeps the difference well above FP32
    # rounding of a loss of ~1e3); the FP64 gradient check is a GPU test
    eps = 0.05
    rng = np.random.default_rng(0)
    fd = []
    with torch.no_grad():
        for c in rng.choice(b.nchan, 4, replace=False):
            e = torch.zeros(b.nchan, device=dev)
            e[int(c)] = eps
            lp = -boxcar_snr(fdmt((1.0 + e)[:, None] * x, plan), cells).sum().item()
            lm = -boxcar_snr(fdmt((1.0 - e)[:, None] * x, plan), cells).sum().item()
            fd.append({"channel": int(c), "fd": (lp - lm) / (2 * eps), "gpu": float(g_gpu[c])})
    gscale = float(np.abs(g_gpu).max())

    # projected gradient ascent on the weights
    snr0 = float(-loss.item())
    wv = torch.ones(b.nchan, device=dev, requires_grad=True)
    opt = torch.optim.Adam([wv], lr=0.05)
    for _ in range(30):
        opt.zero_grad()
        l = -boxcar_snr(fdmt(wv[:, None] * x, plan), cells).sum()
        l.backward()
        opt.step()
        with torch.no_grad():
            wv.clamp_(0.0, 1.0)
    with torch.no_grad():
        snr1 = float(boxcar_snr(fdmt(wv[:, None] * x, plan), cells).sum().item())
    rfi_ch = np.array([c for c, _, _, _ in b.rfi])
    wf = wv.detach().cpu().numpy()
    clean = np.setdiff1d(np.arange(b.nchan), rfi_ch)

    alg = plan.alg_bytes
    units = b.nchan * b.nsamp
    line = {
        "metric": METRIC, "value": units / (step_ms / 1e3), "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded N(0,1) + 8 dispersed pulses + RFI sinusoids on 10% of channels)",
        "config": {"workload": "config4", "nchan": b.nchan, "nsamp": b.nsamp, "max_dt": b.max_dt,
                   "step": "w*x -> FDMT -> S/N at 8 pulse cells -> backward (adjoint boxcar, adjoint FDMT)",
                   "l2": "no flush: 256 MiB planes exceed L2"},
        "roofline": {"bound": "hbm", "kernel": "adjoint FDMT (level gathers + level-0 adjoint)",
                     "achieved": alg / (adj_ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": alg / (adj_ms / 1e3) / 1e9 / peak, "peak_source": peak_kind, "traffic": None},
        "adjoint": {"forward_fdmt_ms": fwd_ms, "adjoint_fdmt_ms": adj_ms, "ratio": adj_ms / fwd_ms,
                    "forward_fuse_depth": plan.info.fuse_depth},
        "gradient_check": {"loss_gpu": float(loss.item()), "max_abs_grad": gscale,
                           "finite_differences_eps_0.05": fd},
        "weight_optimisation": {"snr_sum_before": snr0, "snr_sum_after_30_adam_steps": snr1,
                                "mean_w_rfi_channels": float(wf[rfi_ch].mean()),
                                "mean_w_clean_channels": float(wf[clean].mean())},
        "clocks": clk, "e2e": None, "cpu_baseline": None,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_config1(args):
    """Full pipeline from raw voltages: one GUPPI-like chunk (32 coarse
    channels x 2 pols x 4 128 768 int8 samples, 1200-1328 MHz, a pulse at
    DM 56.8) through unpack + forward FFT (2^20, one fused four-step transform
    reading the int8 samples) -> FP64 chirp at DM 56.8 ->
    inverse FFTs (1024 fine channels) -> detection + transpose + dedispersion
    shifts -> calc_fdmt_inputs -> FDMT of data and mask (max delay 1024) ->
    fdmt_normalization -> per-row normalisation + boxcar (widths 1..32, S/N
    > 7) + clustering (+-16 samples, +-8 rows, any width).  value: fine
    channel-samples (1024 x 129 024) per second of the device-timed step;
    e2e: the same with every chunk copied from pinned host memory (double
    buffered: the next chunk's copy overlaps this chunk's processing) and the
    delegates read back."""
    import torch

    from cpp_projects_b200 import search, synth
    from cpp_projects_b200.chunk import CChunk_gpu
    from cpp_projects_b200.cluster import complete_clusterization

    if not torch.cuda.is_available():
        print(json.dumps({"metric": METRIC, "error": "no CUDA device"}))
        return 1
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    args.warmup = max(args.warmup, 3)
    vc = synth.config1()
    raw = synth.voltage_chunk(vc, dev)
    ch = CChunk_gpu(vc.fmin, vc.fmax, vc.npol, vc.nchan, vc.len_sft, 0, 0, vc.dm, 0.0, 1, 7.0, 1, vc.nbin,
                    vc.nfft, vc.noverlap, vc.tsamp, max_dt=vc.max_dt, dms=[vc.dm])
    cplx = ch.complex_buffer(dev)
    cands_buf = torch.empty((1 << 24, 4), dtype=torch.int32, device=dev)
    units = ch.rows * ch.msamp
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]

    def step(src):
        ev[0].record()
        ch.unpack_fft(src, cplx)
        ev[1].record()
        planes = ch.process_spectrum(cplx)
        ev[2].record()
        y = planes[0]
        st = search.row_stats(y)
        cands, n = search.boxcar_gather(y, 7.0, 0, 5, stats=st, out=cands_buf)
        cl = complete_clusterization(cands, (16, 8, 1 << 30)) if n else None
        ev[3].record()
        return n, cl

    clocks = ClockSampler(0).start()   # started (and settled) before the warm-up
    for _ in range(args.warmup):
        step(raw)
    torch.cuda.synchronize()
    t = {"unpack+fft": 0.0, "coherent+fdmt": 0.0, "search": 0.0}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        n, cl = step(raw)
        torch.cuda.synchronize()
        t["unpack+fft"] += ev[0].elapsed_time(ev[1])
        t["coherent+fdmt"] += ev[1].elapsed_time(ev[2])
        t["search"] += ev[2].elapsed_time(ev[3])
    e1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    step_ms = sum(t.values()) / args.steps
    dl = cl.delegate_records() if cl is not None else np.zeros(0)
    top = dl[np.argmax(dl["msnr"])] if len(dl) else None
    # e2e: every step's raw chunk copied from pinned host memory (a stream of
    # chunks, as the GUPPI reader delivers them) and its delegates read back.
    # Two device buffers: chunk i+1 crosses PCIe on a copy stream while chunk
    # i is processed; the timed region starts before the first copy.
    host = raw.cpu().pin_memory()
    draw = [torch.empty_like(raw), torch.empty_like(raw)]
    cs = torch.cuda.Stream()
    copied = [torch.cuda.Event(), torch.cuda.Event()]
    freed = [torch.cuda.Event(), torch.cuda.Event()]
    main = torch.cuda.current_stream()

    def copy_in(i):
        b = i % 2
        cs.wait_event(freed[b])
        with torch.cuda.stream(cs):
            draw[b].copy_(host, non_blocking=True)
            copied[b].record(cs)

    def run_stream(nsteps):
        d2h = 0
        go = torch.cuda.Event()
        go.record(main)        # the copy stream starts after the timing event
        cs.wait_event(go)
        copy_in(0)
        for i in range(nsteps):
            if i + 1 < nsteps:
                copy_in(i + 1)
            b = i % 2
            main.wait_event(copied[b])
            n2, cl2 = step(draw[b])
            freed[b].record(main)
            recs = cl2.delegate_records() if cl2 is not None else np.zeros(0)
            d2h += 4 + recs.nbytes
        return d2h

    for b in range(2):
        freed[b].record(main)
    run_stream(2)
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record()
    d2h = run_stream(args.steps)
    f1.record()
    torch.cuda.synchronize()
    e2e_ms = f0.elapsed_time(f1) / args.steps
    peak, peak_kind = measured_peaks()
    line = {
        "metric": METRIC, "value": units / (step_ms / 1e3), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int8 in, FP64 chirp phase, f32",
        "data": "synthetic GUPPI-like int8 voltages (uniform [-8, 7] + a pulse at DM 56.8), generated on device",
        "config": {"workload": "config1", "coarse_channels": vc.nchan, "pols": vc.npol // 2,
                   "samples_per_channel": vc.len_chunk, "band_mhz": [vc.fmin, vc.fmax], "nbin": vc.nbin,
                   "nfft": vc.nfft, "noverlap": vc.noverlap, "fine_channels": ch.rows, "msamp": ch.msamp,
                   "coherent_dms": [vc.dm], "max_dt": vc.max_dt,
                   "search": "pow2 widths 1..32, S/N > 7, clusters +-16/+-8/any",
                   "l2": "no flush: 512 MiB raw chunk and 2 GiB spectra exceed L2"},
        "stages_ms": {k: v / args.steps for k, v in t.items()},
        "roofline": None,
        "e2e": {"value": units / (e2e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": int(host.numel()),
                "d2h_bytes_per_step": d2h // args.steps, "ms_per_step": e2e_ms},
        "candidates": int(n), "delegates": int(len(dl)),
        "brightest": None if top is None else {"mt": int(top["mt"]), "mdt": int(top["mdt"]),
                                               "mwidth": int(top["mwidth"]), "snr": float(top["msnr"])},
        # the chunk's dedispersion shifts align every fine channel to the
        # bottom of the band: t0 (top of band) plus the cross-band delay
        "pulse_expected_mt": int((vc.t0 + 4.148808e3 * vc.dm * (vc.fmin ** -2 - vc.fmax ** -2) / vc.tsamp)
                                 // vc.len_sft),
        "cpu_baseline": None, "clocks": clk,
    }
    print(json.dumps(line), flush=True)
    return 0


def launch_ranks(args, argv) -> int:
    """--gpus N without a launcher: start N ranks of this script (one process
    per GPU) through torch.distributed.run on 127.0.0.1, with a bound on the
    whole job; they print the line (rank 0)."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(ROOT / "bench.py")] + list(argv)
    env = dict(os.environ, OMP_NUM_THREADS=os.environ.get("OMP_NUM_THREADS", "1"))
    try:
        return subprocess.call(cmd, env=env, timeout=3600)
    except subprocess.TimeoutExpired:
        print(json.dumps({"metric": METRIC, "error": f"{args.gpus}-rank job exceeded 3600 s"}), flush=True)
        return 1


def run_dry(args) -> int:
    """The multi-rank plumbing without GPU work: every rank builds its beam
    set, meets the others at the barrier and takes the maximum over ranks of
    a stand-in step time; rank 0 prints the line with each rank's beam seeds."""
    import torch
    from cpp_projects_b200.ranks import Ranks
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    gpu = torch.cuda.is_available()
    ranks = Ranks("nccl" if gpu else "gloo", torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
                  if gpu else None, timeout_s=60)
    beams = beams_for(args.workload, rank)
    ranks.barrier()
    slowest = ranks.max(float(rank + 1))
    seeds = [b.seed for b in beams]
    all_seeds = [seeds]
    if world > 1:
        import torch.distributed as dist
        all_seeds = [None] * world
        dist.all_gather_object(all_seeds, seeds)
    ranks.barrier()
    ranks.close()
    if rank == 0:
        print(json.dumps({"metric": METRIC, "value": None, "unit": UNIT, "n_gpus": world, "steps": 0,
                          "warmup": 0, "dry_run": True, "scaling": "weak",
                          "config": {"workload": args.workload, "beams": len(beams),
                                     "parallelism": f"{world} independent rank(s), beams sharded, no collective"},
                          "slowest_rank_stand_in": slowest, "rank_seeds": all_seeds}), flush=True)
    return 0


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    args = parse_args(argv)
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return launch_ranks(args, argv)
    if args.dry_run:
        return run_dry(args)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "config1":
        return run_config1(args)
    if args.workload == "config3":
        return run_config3(args)
    if args.workload == "config4":
        return run_config4(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
