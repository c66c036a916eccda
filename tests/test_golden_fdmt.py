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
