"""GPU parity of the reduced-precision FDMT (FP16 / BF16 planes between
levels, FP32 sums, FP32 output): bit-identical to the oracle's emulation of
the same 16-bit stores (levels from the fused head's depth on), whatever the
fusion depth; the error against the FP64 FDMT is asserted with its bound."""
import numpy as np
import pytest
import torch

from cpp_projects_b200 import CFdmtGpu
from oracle import pyoracle

pytestmark = pytest.mark.gpu

CASES = [
    (1200.0, 1600.0, 64, 1024, 64),
    (1100.0, 1500.0, 512, 4100, 512),
    (1100.0, 1500.0, 100, 2048, 77),     # odd sub-band counts (carried rows)
    (1200.0, 1328.0, 1024, 3001, 1024),  # ragged length, no vector stores at the end
    (1200.0, 1600.0, 300, 4097, 300),
    (1200.0, 1600.0, 256, 1, 256),
]


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("prec", [1, 2])
@pytest.mark.parametrize("fuse", [0, -1, -2])
def test_lowp_bit_exact_vs_emulation(cuda, case, prec, fuse):
    fmin, fmax, nchan, ncols, max_dt = case
    x = np.random.default_rng(21).standard_normal((nchan, ncols)).astype(np.float32)
    f = CFdmtGpu(fmin, fmax, nchan, ncols, max_dt, fuse_depth=fuse, precision=prec)
    d_out = torch.full((max_dt, ncols), float("nan"), device=cuda)
    f.process_image(torch.from_numpy(x).to(cuda), d_out, False)
    want = pyoracle.fdmt_lowp(fmin, fmax, x, nchan, ncols, max_dt, prec, f.info.fuse_depth)
    assert np.array_equal(_bits(d_out.cpu().numpy()), _bits(want))


@pytest.mark.parametrize("prec", [1, 2])
def test_lowp_ones_mode_and_external_workspace(cuda, prec):
    fmin, fmax, nchan, ncols, max_dt = 1200.0, 1600.0, 512, 2048, 512
    f = CFdmtGpu(fmin, fmax, nchan, ncols, max_dt, fuse_depth=0, precision=prec, external_ws=True)
    ws = torch.empty(f.workspace_size(), dtype=torch.uint8, device=cuda)
    d_out = torch.zeros((max_dt, ncols), device=cuda)
    f.process_image_ws(None, d_out, True, ws)
    want = pyoracle.fdmt_lowp(fmin, fmax, None, nchan, ncols, max_dt, prec, 0, b_ones=True)
    assert np.array_equal(d_out.cpu().numpy(), want)
    # two 16-bit ping-pong planes (2 bytes per value, 128-byte row pitch):
    # even levels below the last in one, odd levels in the other
    rows = f.rows_per_level()[:-1]
    pitch = (ncols + 63) // 64 * 64

    def plane(r):
        return (int(r) * pitch * 2 + 255) // 256 * 256
    assert f.workspace_size() == plane(rows[0::2].max()) + plane(rows[1::2].max())


def test_lowp_error_against_fp64_on_device(cuda):
    fmin, fmax, nchan, ncols, max_dt = 1100.0, 1500.0, 1024, 8192, 1024
    rng = np.random.default_rng(4)
    g = np.exp(rng.uniform(np.log(0.5), np.log(2.0), nchan)).astype(np.float32)[:, None]
    x = rng.standard_normal((nchan, ncols)).astype(np.float32) * g
    y64 = pyoracle.fdmt_f64(fmin, fmax, x, nchan, ncols, max_dt)
    d_in = torch.from_numpy(x).to(cuda)
    for prec, bound in ((1, 1.5e-3), (2, 1.2e-2)):  # relative RMS error bound
        f = CFdmtGpu(fmin, fmax, nchan, ncols, max_dt, fuse_depth=-2, precision=prec)
        y = f(d_in).cpu().numpy().astype(np.float64)
        assert np.sqrt(((y - y64) ** 2).mean() / (y64 ** 2).mean()) < bound
