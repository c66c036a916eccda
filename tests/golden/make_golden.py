"""Regenerates the golden fixtures in this folder from the reference checkout.

    python tests/golden/make_golden.py [/path/to/reference]

* ``cluster_golden.json`` — the reference's only committed golden outputs,
  ``clusterization_forpravir/Candidates1.csv`` (dynamic gather, Q=1) and
  ``Candidates2.csv`` (heap gather, W=2), parsed, together with the input
  plane their driver builds (clusterization_forpravir/clusterization_test.cu:
  63-112: a 3x16 plane of 2.0 with 140 at (0,4), 120 at (0,11), 100 at (2,4);
  threshold 4.0).
* ``fdmt_ref_*.npz`` — outputs of the reference's own CFdmtCpu::process_image
  (built from its sources by oracle/Makefile, one thread) on small seeded
  inputs, so the GPU tests can compare against the reference itself on a box
  where the reference checkout does not exist.
"""
from __future__ import annotations

import csv
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

FDMT_CASES = [
    # name, fmin, fmax, nchan, ncols, max_dt, seed, b_ones
    ("c64", 1200.0, 1600.0, 64, 512, 64, 21, False),
    ("c100_odd", 1100.0, 1500.0, 100, 300, 77, 22, False),
    ("c48_ones", 1200.0, 1600.0, 48, 256, 48, 0, True),
]


def fdmt_input(nchan, ncols, seed):
    return np.random.default_rng(seed).standard_normal((nchan, ncols)).astype(np.float32)


def read_csv(path: Path):
    rows = []
    with open(path) as f:
        for r in csv.DictReader(f):
            rows.append([int(r["mt"]), int(r["mdt"]), int(r["mwidth"]), float(r["msnr"])])
    return rows


def main(ref_root: str = "/root/reference") -> None:
    ref = Path(ref_root)
    d = ref / "clusterization_forpravir"
    golden = {
        "source": "clusterization_forpravir/Candidates{1,2}.csv",
        "plane": {"rows": 3, "cols": 16, "base": 2.0,
                  "spikes": [[0, 4, 140.0], [0, 11, 120.0], [2, 4, 100.0]]},
        "thr": 4.0,
        "dynamic_Q": 1,
        "heap_W": 2,
        "metrics": [2, 1, 2],
        "candidates1_dynamic": read_csv(d / "Candidates1.csv"),
        "candidates2_heap": read_csv(d / "Candidates2.csv"),
    }
    (HERE / "cluster_golden.json").write_text(json.dumps(golden, indent=1))

    from oracle import pyoracle
    pyoracle.build()
    if pyoracle.ref_lib() is None:
        raise SystemExit("reference CFdmtCpu not built: run make -C oracle")
    for name, fmin, fmax, nchan, ncols, max_dt, seed, ones in FDMT_CASES:
        x = None if ones else fdmt_input(nchan, ncols, seed)
        out = pyoracle.ref_fdmt_cpu(fmin, fmax, x, nchan, ncols, max_dt, b_ones=ones, threads=1)
        np.savez_compressed(HERE / f"fdmt_ref_{name}.npz", out=out,
                            params=np.array([fmin, fmax, nchan, ncols, max_dt, seed, int(ones)],
                                            np.float64))


if __name__ == "__main__":
    main(*sys.argv[1:])
