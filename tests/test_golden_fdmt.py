"""FDMT against outputs of the reference's own CFdmtCpu::process_image,
committed as tests/golden/fdmt_ref_*.npz by tests/golden/make_golden.py (so
the GPU box, which has no reference checkout, still compares against the
reference itself)."""
from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import pyoracle

GOLD = sorted((Path(__file__).parent / "golden").glob("fdmt_ref_*.npz"))


def load(path):
    z = np.load(path)
    fmin, fmax, nchan, ncols, max_dt, seed, ones = z["params"]
    nchan, ncols, max_dt, seed, ones = int(nchan), int(ncols), int(max_dt), int(seed), bool(ones)
    x = None if ones else np.random.default_rng(seed).standard_normal((nchan, ncols)).astype(np.float32)
    return float(fmin), float(fmax), nchan, ncols, max_dt, x, ones, z["out"]


@pytest.mark.parametrize("path", GOLD, ids=[p.stem for p in GOLD])
def test_oracle_reproduces_reference_output(path):
    fmin, fmax, nchan, ncols, max_dt, x, ones, ref = load(path)
    got = pyoracle.fdmt_f32(fmin, fmax, x, nchan, ncols, max_dt, b_ones=ones)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("path", GOLD, ids=[p.stem for p in GOLD])
def test_gpu_reproduces_reference_output(cuda, path):
    from cpp_projects_b200 import CFdmtGpu
    fmin, fmax, nchan, ncols, max_dt, x, ones, ref = load(path)
    f = CFdmtGpu(fmin, fmax, nchan, ncols, max_dt)
    out = torch.empty((max_dt, ncols), device=cuda)
    f.process_image(None if ones else torch.from_numpy(x).to(cuda), out, ones)
    assert np.array_equal(out.cpu().numpy().view(np.uint32), ref.view(np.uint32))


# --- the reference's own FDMT test input (fdmt_class_v0/file512.bin) ----------
FILE512 = Path(__file__).parent / "golden" / "file512.npz"
REF_FILE512 = pyoracle.reference_dir() / "fdmt_class_v0" / "file512.bin"


def load512():
    import hashlib
    z = np.load(FILE512)
    fmin, fmax, nchan, ncols, max_dt, pravir_dt_max = z["params"]
    x = z["input_i8"].astype(np.float32)
    sha = lambda a: hashlib.sha256(np.ascontiguousarray(a, np.float32).tobytes()).hexdigest()  # noqa: E731
    return (float(fmin), float(fmax), int(nchan), int(ncols), int(max_dt), int(pravir_dt_max), x, z, sha)


def test_file512_fixture_is_the_reference_input():
    if not REF_FILE512.exists():
        pytest.skip("reference checkout absent")
    _, _, nchan, ncols, _, _, x, _, _ = load512()
    assert np.array_equal(x, np.fromfile(REF_FILE512, np.float32).reshape(nchan, ncols))


def test_oracle_reproduces_reference_on_file512():
    fmin, fmax, nchan, ncols, max_dt, pdt, x, z, sha = load512()
    keith = pyoracle.fdmt_f32(fmin, fmax, x, nchan, ncols, max_dt)
    assert sha(keith) == str(z["keith_sha256"])
    assert np.array_equal(keith[z["rows"]].view(np.uint32), z["keith_rows"].view(np.uint32))
    pravir = pyoracle.pravir_fdmt(fmin, fmax, x, nchan, ncols, pdt, 1, 0)
    assert pravir.shape == tuple(z["pravir_shape"]) and sha(pravir) == str(z["pravir_sha256"])
    assert np.array_equal(pravir[z["rows"]].view(np.uint32), z["pravir_rows"].view(np.uint32))


@pytest.mark.gpu
def test_gpu_reproduces_reference_on_file512(cuda):
    from cpp_projects_b200 import FDMTGPU, CFdmtGpu
    fmin, fmax, nchan, ncols, max_dt, pdt, x, z, sha = load512()
    d_in = torch.from_numpy(x).to(cuda)
    f = CFdmtGpu(fmin, fmax, nchan, ncols, max_dt)
    out = torch.empty((max_dt, ncols), device=cuda)
    f.process_image(d_in, out, False)
    assert sha(out.cpu().numpy()) == str(z["keith_sha256"])
    p = FDMTGPU(fmin, fmax, nchan, ncols, 1.0, pdt, 1, 0)
    pout = torch.empty((p.out_rows, ncols), device=cuda)
    p.execute(d_in, d_in.numel(), pout, pout.numel())
    assert sha(pout.cpu().numpy()) == str(z["pravir_sha256"])
