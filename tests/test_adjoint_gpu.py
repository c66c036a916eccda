"""GPU checks of the adjoint FDMT and the boxcar S/N gradient:
* the adjoint is bit-identical to the oracle's FP32 adjoint (same summation
  order), and agrees with the FP64 transpose (dot-product test);
* S/N at cells equals the S/N the boxcar search reports for those cells;
* the gradient of -sum S/N with respect to per-channel weights, through
  torch.autograd with both adjoints, matches the FP64 reference gradient and
  central finite differences (eps 1e-3) of the FP64 loss."""
import numpy as np
import pytest
import torch

from cpp_projects_b200 import CFdmtGpu, search, synth
from cpp_projects_b200.autograd import boxcar_snr, fdmt
from oracle import pyoracle

pytestmark = pytest.mark.gpu

CASES = [
    (1200.0, 1600.0, 64, 1024, 64),
    (1100.0, 1500.0, 100, 2046, 77),     # odd sub-band counts, ncols % 4 == 2
    (1200.0, 1328.0, 1024, 3001, 1024),  # ragged length
    (1200.0, 1600.0, 300, 4097, 300),
    (1200.0, 1600.0, 3, 64, 5),
]


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("case", CASES)
def test_adjoint_bit_exact_vs_oracle(cuda, case):
    fmin, fmax, nchan, ncols, max_dt = case
    g = np.random.default_rng(31).standard_normal((max_dt, ncols)).astype(np.float32)
    f = CFdmtGpu(fmin, fmax, nchan, ncols, max_dt)
    gx = f.adjoint(torch.from_numpy(g).to(cuda)).cpu().numpy()
    want = pyoracle.fdmt_adjoint_f32(fmin, fmax, g, nchan, ncols, max_dt)
    assert np.array_equal(_bits(gx), _bits(want))
    # the workspace form gives the same bits
    fw = CFdmtGpu(fmin, fmax, nchan, ncols, max_dt, external_ws=True)
    ws = torch.empty(fw.adjoint_workspace_size(), dtype=torch.uint8, device=cuda)
    out = torch.full((nchan, ncols), float("nan"), device=cuda)
    fw.adjoint_ws(torch.from_numpy(g).to(cuda), out, ws)
    assert np.array_equal(_bits(out.cpu().numpy()), _bits(want))


def test_adjoint_dot_product_against_forward(cuda):
    fmin, fmax, nchan, ncols, max_dt = 1200.0, 1600.0, 512, 8192, 512
    rng = np.random.default_rng(5)
    x = torch.from_numpy(rng.standard_normal((nchan, ncols)).astype(np.float32)).to(cuda)
    g = torch.from_numpy(rng.standard_normal((max_dt, ncols)).astype(np.float32)).to(cuda)
    f = CFdmtGpu(fmin, fmax, nchan, ncols, max_dt, fuse_depth=-2)
    a = (f(x).double() * g.double()).sum().item()
    b = (x.double() * f.adjoint(g).double()).sum().item()
    assert abs(a - b) <= 1e-5 * abs(a)


def test_snr_cells_equal_search_snr(cuda):
    beam = synth.config0()
    x = torch.from_numpy(synth.filterbank(beam)).to(cuda)
    y = CFdmtGpu(beam.fmin, beam.fmax, beam.nchan, beam.nsamp, beam.max_dt)(x)
    st = search.row_stats(y)
    cands, n = search.boxcar_gather(y, 7.0, 0, 5, stats=st)
    c = search.cands_to_numpy(cands)[:2000]
    cells = np.stack([c["mdt"], c["mt"], 1 << c["mwidth"]], 1)
    snr = search.snr_cells(y, st, cells).cpu().numpy()
    assert np.array_equal(snr.view(np.uint32), c["msnr"].view(np.uint32))


def _problem(nchan=128, ncols=4096, seed=6):
    rng = np.random.default_rng(seed)
    fmin, fmax = 1200.0, 1600.0
    pulses = [synth.Pulse(int(rng.integers(200, ncols - 400)), float(rng.uniform(0.2, 0.8) * (nchan - 1)),
                          int(rng.integers(2, 9)), 1.5) for _ in range(4)]
    beam = synth.Beam(nchan, ncols, fmin, fmax, nchan, seed, pulses)
    x = synth.filterbank(beam)
    rfi = rng.choice(nchan, nchan // 10, replace=False)
    t = np.arange(ncols)
    for c in rfi:
        x[c] += np.float32(5.0) * np.sin(2 * np.pi * rng.uniform(0.01, 0.2) * t + rng.uniform(0, 6.28)).astype(np.float32)
    cells = np.array([[int(round(p.span)), p.t0 + int(round(p.span)), p.width] for p in pulses])
    return beam, x, cells


def _loss64(beam, x, w, cells):
    y = pyoracle.fdmt_f64(beam.fmin, beam.fmax, x * w[:, None], beam.nchan, beam.nsamp, beam.max_dt)
    snr, grads = pyoracle.snr_cells_f64(y, cells)
    return -snr.sum(), y, grads


def test_weight_gradient_vs_fp64_and_finite_differences(cuda):
    beam, x, cells = _problem()
    rng = np.random.default_rng(7)
    w0 = rng.uniform(0.5, 1.0, beam.nchan)
    xd = torch.from_numpy(x).to(cuda)
    w = torch.tensor(w0, dtype=torch.float32, device=cuda, requires_grad=True)
    plan = CFdmtGpu(beam.fmin, beam.fmax, beam.nchan, beam.nsamp, beam.max_dt, fuse_depth=-2)
    loss = -boxcar_snr(fdmt(w[:, None] * xd, plan), cells).sum()
    loss.backward()
    g_gpu = w.grad.double().cpu().numpy()
    # FP64 reference gradient: dL/dy from the FP64 S/N, then the FP64 adjoint
    l64, y64, grads = _loss64(beam, x.astype(np.float64), w0, cells)
    gy = np.zeros_like(y64)
    for k, (d, t, wd) in enumerate(cells):
        gy[d] -= grads[k]
    gx = pyoracle.fdmt_adjoint_f64(beam.fmin, beam.fmax, gy, beam.nchan, beam.nsamp, beam.max_dt)
    g64 = (gx * x.astype(np.float64)).sum(1)
    # bounds about 10x the errors measured on a B200 (loss 8.2e-8 relative,
    # weight gradient 1.8e-7 of its largest entry)
    assert abs(loss.item() - l64) <= 1e-6 * abs(l64)
    assert np.abs(g_gpu - g64).max() <= 2e-6 * np.abs(g64).max()
    # central finite differences of the FP64 loss, eps 1e-3, on a few channels
    for c in rng.choice(beam.nchan, 6, replace=False):
        wp, wm = w0.copy(), w0.copy()
        wp[c] += 1e-3
        wm[c] -= 1e-3
        fd = (_loss64(beam, x.astype(np.float64), wp, cells)[0]
              - _loss64(beam, x.astype(np.float64), wm, cells)[0]) / 2e-3
        # measured: <= 4.7e-7 relative, <= 1.9e-8 of the largest entry
        assert g_gpu[c] == pytest.approx(fd, rel=5e-6, abs=2e-7 * np.abs(g64).max())


def test_input_gradient_vs_fp64(cuda):
    beam, x, cells = _problem(nchan=64, ncols=2048, seed=9)
    xd = torch.from_numpy(x).to(cuda).requires_grad_(True)
    plan = CFdmtGpu(beam.fmin, beam.fmax, beam.nchan, beam.nsamp, beam.max_dt)
    loss = -boxcar_snr(fdmt(xd, plan), cells).sum()
    loss.backward()
    _, y64, grads = _loss64(beam, x.astype(np.float64), np.ones(beam.nchan), cells)
    gy = np.zeros_like(y64)
    for k, (d, t, wd) in enumerate(cells):
        gy[d] -= grads[k]
    gx = pyoracle.fdmt_adjoint_f64(beam.fmin, beam.fmax, gy, beam.nchan, beam.nsamp, beam.max_dt)
    # measured 1.1e-7 of the largest entry
    assert np.abs(xd.grad.double().cpu().numpy() - gx).max() <= 1e-6 * np.abs(gx).max()
