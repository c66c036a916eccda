"""Time one FDMT variant on the current GPU (CUDA events, inputs resident).

    python -m cpp_projects_b200.fdmt_timing --nchan 1024 --ncols 65536 \
        [--max-dt 1024] [--fmin 1200 --fmax 1600] [--fuse -2] [--tile 0] \
        [--seg-levels 0] [--seg-rows 0] \
        [--precision f32|f16|bf16] [--adjoint] [--reps 10] [--warmup 3] [--profile-one]
        [--print-tuned]

Prints one JSON line: the plan's fused depth and merge passes ([first
level, last level] of each pass after the head), milliseconds per call, the
level-by-level algorithmic bytes of one call and the resulting GB/s, and the
bytes this schedule cannot avoid (every plane that reaches HBM written and
read once).  Used
for the autotuner's choices, for the reduced-precision and adjoint timings,
and as the command under ncu for the per-kernel captures.

For 512, 1024 and 2048 channels the line also carries the figure the
reference's FDMT drivers print, "GFLP/sec": a constant operation count per
test size (MyVSLib_C++/Constants.h:6-9; 1024 channels use the 512 x 1024
count, as fdmt_class_v0/kernel.cu:24,176-199 selects it) divided by the time
per call.
"""
from __future__ import annotations

import argparse
import json

import torch

from .fdmt import CFdmtGpu

PRECISIONS = {"f32": 0, "f16": 1, "bf16": 2}
# giga-operations per call of the reference's FDMT test sizes (Constants.h:6-9)
REFERENCE_GFLOP = {512: 0.00320386, 1024: 0.006518622, 2048: 0.0586616}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--nchan", type=int, default=1024)
    ap.add_argument("--ncols", type=int, default=65536)
    ap.add_argument("--max-dt", type=int, default=0, help="default: nchan")
    ap.add_argument("--fmin", type=float, default=1200.0)
    ap.add_argument("--fmax", type=float, default=1600.0)
    ap.add_argument("--fuse", type=int, default=-2, help="-2 autotune, -1 default head, 0 none, k")
    ap.add_argument("--tile", type=int, default=0)
    ap.add_argument("--seg-levels", type=int, default=0, help="merge levels per fused pass (1: none)")
    ap.add_argument("--seg-rows", type=int, default=0, help="output rows per fused tile (0: auto)")
    ap.add_argument("--seg-threads", type=int, default=0, help="threads per segment CTA (0: auto; 256/512/1024)")
    ap.add_argument("--seg-flags", type=int, default=0, help="1: one input buffer per segment CTA")
    ap.add_argument("--precision", choices=sorted(PRECISIONS), default="f32")
    ap.add_argument("--adjoint", action="store_true")
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--profile-one", action="store_true",
                    help="after the timing, one more call between cudaProfilerStart / Stop (for "
                         "ncu --profile-from-start off: one FDMT's launches, none of the tuning)")
    ap.add_argument("--print-tuned", action="store_true",
                    help="autotune this shape and print the chosen schedule as command-line options "
                         "(--fuse k --tile t --seg-levels s --seg-rows r), then exit")
    a = ap.parse_args(argv)
    max_dt = a.max_dt or a.nchan
    if a.print_tuned:
        from . import _capi
        from .fdmt import autotune_desc
        t, _ = autotune_desc(_capi.FdmtDesc(fmin=a.fmin, fmax=a.fmax, nchan=a.nchan, ncols=a.ncols,
                                            max_dt=max_dt, precision=PRECISIONS[a.precision]))
        print(f"--fuse {t.fuse_depth} --tile {t.head_tile} --seg-levels {t.seg_levels} --seg-rows {t.seg_rows} "
              f"--seg-threads {t.seg_threads} --seg-flags {t.seg_flags}")
        return 0
    dev = torch.device("cuda", 0)
    f = CFdmtGpu(a.fmin, a.fmax, a.nchan, a.ncols, max_dt, fuse_depth=a.fuse, head_tile=a.tile,
                 precision=PRECISIONS[a.precision], seg_levels=a.seg_levels, seg_rows=a.seg_rows,
                 seg_threads=a.seg_threads, seg_flags=a.seg_flags)
    g = torch.Generator(device=dev).manual_seed(1)
    if a.adjoint:
        src = torch.randn((max_dt, a.ncols), device=dev, generator=g)
        dst = torch.empty((a.nchan, a.ncols), device=dev)
        run = lambda: f.adjoint(src, dst)  # noqa: E731
    else:
        src = torch.randn((a.nchan, a.ncols), device=dev, generator=g)
        dst = torch.empty((max_dt, a.ncols), device=dev)
        run = lambda: f.process_image(src, dst)  # noqa: E731
    for _ in range(a.warmup):
        run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.reps):
        run()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / a.reps
    if a.profile_one:
        torch.cuda.profiler.start()
        run()
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
    print(json.dumps({"passes": f.passes(),"nchan": a.nchan, "ncols": a.ncols, "max_dt": max_dt, "precision": a.precision,
                      "adjoint": a.adjoint, "fuse_depth": f.info.fuse_depth,
                      "hbm_passes": f.info.hbm_passes, "seg_levels": f.info.seg_levels, "ms": ms,
                      "seg_threads": a.seg_threads, "seg_flags": a.seg_flags,
                      "sched_bytes": f.info.sched_bytes,
                      "alg_bytes": f.alg_bytes, "alg_gbs": f.alg_bytes / (ms / 1e3) / 1e9,
                      "reference_gflop_per_s": (REFERENCE_GFLOP[a.nchan] / (ms / 1e3)
                                                if a.nchan in REFERENCE_GFLOP else None)}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
