"""GPU parity of the Pravir plan kind (FDMTGPU.execute, the reference's
FDMT::execute of MyVSLib_C++/FDMT_PRAVIR/) against the oracle, which is
bit-identical to the reference's own FDMTCPU; and of its adjoint against the
oracle's FP32 adjoint (same summation order)."""
import numpy as np
import pytest
import torch

from cpp_projects_b200 import FDMTGPU
from oracle import pyoracle

pytestmark = pytest.mark.gpu

CASES = [
    (1200.0, 1600.0, 64, 1000, 64, 1, 0),
    (1200.0, 1600.0, 100, 777, 80, 1, 0),
    (1100.0, 1500.0, 48, 600, 50, 2, 4),
    (1200.0, 1600.0, 512, 32768, 512, 1, 0),   # config-0 shape
    (1200.0, 1328.0, 37, 999, 40, 1, 0),
    (1200.0, 1600.0, 3, 64, 5, 1, 0),
]


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("case", CASES)
def test_pravir_bit_exact_vs_oracle(cuda, case):
    fmin, fmax, nch, ns, dtm, st, dmin = case
    x = np.random.default_rng(nch + ns).standard_normal((nch, ns)).astype(np.float32)
    f = FDMTGPU(fmin, fmax, nch, ns, 1e-3, dtm, st, dmin)
    assert f.get_dt_grid_final() == list(range(dmin, dtm + 1, st))[: f.out_rows]
    d_out = torch.full((f.out_rows, ns), float("nan"), device=cuda)
    f.execute(torch.from_numpy(x).to(cuda), x.size, d_out, d_out.numel())
    want = pyoracle.pravir_fdmt(fmin, fmax, x, nch, ns, dtm, st, dmin)
    assert np.array_equal(_bits(d_out.cpu().numpy()), _bits(want))
    if ns <= 4096 and pyoracle.ref_pravir_lib() is not None:
        ref = pyoracle.ref_pravir_cpu(fmin, fmax, x, nch, ns, dtm, st, dmin, threads=4)
        assert np.array_equal(_bits(d_out.cpu().numpy()), _bits(ref))


def test_pravir_size_checks(cuda):
    f = FDMTGPU(1200.0, 1600.0, 64, 1000, 1e-3, 64)
    x = torch.zeros((64, 1000), device=cuda)
    with pytest.raises(ValueError):
        f.execute(x, 64 * 999, torch.zeros((65, 1000), device=cuda), 65 * 1000)
    with pytest.raises(ValueError):
        f.execute(x, 64 * 1000, torch.zeros((64, 1000), device=cuda), 64 * 1000)


@pytest.mark.parametrize("case", CASES[:3] + CASES[4:5])
def test_pravir_adjoint_bit_exact(cuda, case):
    fmin, fmax, nch, ns, dtm, st, dmin = case
    f = FDMTGPU(fmin, fmax, nch, ns, 1e-3, dtm, st, dmin)
    g = np.random.default_rng(7).standard_normal((f.out_rows, ns)).astype(np.float32)
    gx = f.adjoint(torch.from_numpy(g).to(cuda)).cpu().numpy()
    want = pyoracle.pravir_adjoint(fmin, fmax, g, nch, ns, dtm, st, dmin)
    assert np.array_equal(_bits(gx), _bits(want))
