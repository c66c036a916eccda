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
* ``file512.npz`` — the reference's own FDMT test input
  (``fdmt_class_v0/file512.bin``: a 512 x 512 float32 filterbank of small
  integers, stored here as int8, which holds it exactly) with the SHA-256 and
  four rows of the reference's outputs on it: CFdmtCpu (1200-1600 MHz, max
  delay 512; the file's own band and delay were in test folders that are
  absent) and a fresh FDMTCPU (Pravir plan; tsamp 1, dt_max 511, dt_step 1,
  dt_min 0, as fdmt_pr_restr/kernel.cu:357-361 builds it from a 512-row
  maximum delay).
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


def main(ref_root: str | None = None) -> None:
    from oracle import pyoracle
    ref = Path(ref_root) if ref_root else pyoracle.reference_dir()
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


FILE512 = dict(fmin=1200.0, fmax=1600.0, nchan=512, ncols=512, max_dt=512, pravir_dt_max=511)
FILE512_ROWS = [0, 1, 255, 511]


def make_file512(ref_root: str | None = None) -> None:
    import hashlib

    from oracle import pyoracle
    ref = Path(ref_root) if ref_root else pyoracle.reference_dir()
    x = np.fromfile(ref / "fdmt_class_v0" / "file512.bin", np.float32)
    q = x.astype(np.int8)
    if not np.array_equal(q.astype(np.float32), x):
        raise SystemExit("file512.bin is not int8-valued")
    c = FILE512
    x = x.reshape(c["nchan"], c["ncols"])
    keith = pyoracle.ref_fdmt_cpu(c["fmin"], c["fmax"], x, c["nchan"], c["ncols"], c["max_dt"], threads=1)
    pravir = pyoracle.ref_pravir_cpu(c["fmin"], c["fmax"], x, c["nchan"], c["ncols"], c["pravir_dt_max"],
                                     1, 0, tsamp=1.0, threads=1)
    if keith is None or pravir is None:
        raise SystemExit("reference FDMTs not built: run make -C oracle")
    np.savez_compressed(
        HERE / "file512.npz", input_i8=q.reshape(c["nchan"], c["ncols"]),
        params=np.array([c["fmin"], c["fmax"], c["nchan"], c["ncols"], c["max_dt"], c["pravir_dt_max"]],
                        np.float64),
        rows=np.array(FILE512_ROWS, np.int32),
        keith_sha256=np.array(hashlib.sha256(keith.tobytes()).hexdigest()),
        keith_rows=keith[FILE512_ROWS],
        pravir_sha256=np.array(hashlib.sha256(pravir.tobytes()).hexdigest()),
        pravir_shape=np.array(pravir.shape, np.int64),
        pravir_rows=pravir[FILE512_ROWS])


if __name__ == "__main__":
    main(*sys.argv[1:])
    make_file512(*sys.argv[1:])
