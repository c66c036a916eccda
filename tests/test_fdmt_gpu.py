"""GPU parity of the FDMT (through the C ABI) against the oracle, which is
itself bit-exact against the reference's CFdmtCpu.  Integer row tables plus
round-to-nearest float arithmetic make the GPU result bit-identical."""
import numpy as np
import pytest
import torch

from cpp_projects_b200 import BfsError, CFdmtGpu, synth
from cpp_projects_b200._capi import BFS_ERR_ARG
from oracle import pyoracle

pytestmark = pytest.mark.gpu

CASES = [
    (1200.0, 1600.0, 64, 1024, 64),
    (1200.0, 1600.0, 512, 4096, 512),
    (1100.0, 1500.0, 100, 2048, 77),
    (1200.0, 1600.0, 48, 2000, 48),
    (1200.0, 1328.0, 1024, 3000, 1024),
    (1200.0, 1600.0, 3, 64, 5),
    (1200.0, 1600.0, 2, 33, 3),
    (1200.0, 1600.0, 256, 1, 256),     # a single time sample
    (1200.0, 1600.0, 300, 4097, 300),  # ragged length
]


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("fuse", [0, -1])
def test_fdmt_bit_exact_vs_oracle(cuda, case, fuse):
    fmin, fmax, nchan, ncols, max_dt = case
    x = np.random.default_rng(11).standard_normal((nchan, ncols)).astype(np.float32)
    f = CFdmtGpu(fmin, fmax, nchan, ncols, max_dt, fuse_depth=fuse)
    d_in = torch.from_numpy(x).to(cuda)
    d_out = torch.full((max_dt, ncols), float("nan"), device=cuda)
    f.process_image(d_in, d_out, False)
    got = d_out.cpu().numpy()
    want = pyoracle.fdmt_f32(fmin, fmax, x, nchan, ncols, max_dt)
    assert np.array_equal(_bits(got), _bits(want))


@pytest.mark.parametrize("case", CASES[:5] + CASES[8:])
@pytest.mark.parametrize("fuse,tile", [(-2, 0), (3, 512), (5, 256), (2, 512)])
def test_fdmt_autotuned_and_wide_tiles_bit_exact(cuda, case, fuse, tile):
    fmin, fmax, nchan, ncols, max_dt = case
    x = np.random.default_rng(12).standard_normal((nchan, ncols)).astype(np.float32)
    try:
        f = CFdmtGpu(fmin, fmax, nchan, ncols, max_dt, fuse_depth=fuse, head_tile=tile)
    except BfsError as e:  # an explicit depth deeper than this plan's head allows
        assert fuse > 0 and e.status == BFS_ERR_ARG
        pytest.skip(f"fuse_depth {fuse} not usable for {nchan} channels")
    d_out = torch.full((max_dt, ncols), float("nan"), device=cuda)
    f.process_image(torch.from_numpy(x).to(cuda), d_out, False)
    want = pyoracle.fdmt_f32(fmin, fmax, x, nchan, ncols, max_dt)
    assert np.array_equal(_bits(d_out.cpu().numpy()), _bits(want))


@pytest.mark.parametrize("d", range(2, 9))
def test_level0_constant_division_matches_ieee_divide_for_every_float(cuda, d):
    """The level-0 running means divide by r + 1 with a multiply / fused
    multiply-add split; all 2^32 bit patterns must give __fdiv_rn's bits."""
    import ctypes
    from cpp_projects_b200 import _capi
    bad, first = ctypes.c_uint64(), ctypes.c_uint32()
    _capi.call("bfs_selftest_divide", d, ctypes.byref(bad), ctypes.byref(first), None)
    assert bad.value == 0, f"d={d}: {bad.value} mismatches, first bits {first.value:#010x}"


@pytest.mark.parametrize("shape", [(64, 2048, 64), (64, 2048, 96), (64, 2048, 128)])
@pytest.mark.parametrize("fuse", [0, -1])
def test_fdmt_bit_exact_on_special_values(cuda, shape, fuse):
    """Signed zeros, subnormals, tiny and huge magnitudes reach the level-0
    divisions on both sides of the split-division guard (|x| >= 2^-64)."""
    nchan, ncols, max_dt = shape
    rng = np.random.default_rng(13)
    x = rng.standard_normal((nchan, ncols)).astype(np.float32)
    specials = np.array([0.0, -0.0, 1e-40, -1e-40, 1e-30, -1e-30, 2.0 ** -64, -(2.0 ** -65),
                         1e-20, 1e30, -1e30, 3.0e38 / 256], np.float32)
    idx = rng.integers(0, x.size, size=x.size // 4)
    x.reshape(-1)[idx] = specials[rng.integers(0, specials.size, size=idx.size)]
    x[:, :64] = -0.0  # whole runs of negative zeros: -0 sums stay -0
    f = CFdmtGpu(1200.0, 1600.0, nchan, ncols, max_dt, fuse_depth=fuse)
    d_out = torch.full((max_dt, ncols), float("nan"), device=cuda)
    f.process_image(torch.from_numpy(x).to(cuda), d_out, False)
    want = pyoracle.fdmt_f32(1200.0, 1600.0, x, nchan, ncols, max_dt)
    assert np.array_equal(_bits(d_out.cpu().numpy()), _bits(want))


def test_autotune_returns_a_valid_choice(cuda):
    from cpp_projects_b200 import _capi
    from cpp_projects_b200.fdmt import autotune, autotune_desc
    depth, tile, ms = autotune(1200.0, 1600.0, 1024, 65536, 1024)
    assert depth in (0, 2, 3, 4, 5) and ms > 0
    assert tile in ((0,) if depth == 0 else (256, 512))
    assert autotune(1200.0, 1600.0, 1024, 65536, 1024)[:2] == (depth, tile)  # cached
    d = _capi.FdmtDesc(fmin=1200.0, fmax=1600.0, nchan=1024, ncols=65536, max_dt=1024)
    t, ms2 = autotune_desc(d)
    assert (t.fuse_depth, t.head_tile) == (depth, tile) and ms2 == ms
    assert t.seg_levels in (1, 2, 3, 4) and t.seg_rows in ((0,) if t.seg_levels == 1 else (16, 24, 28, 32))
    # the tuned plan is the one the autotuning plan request builds, and bit-exact
    x = np.random.default_rng(7).standard_normal((1024, 4096)).astype(np.float32)
    f = CFdmtGpu(1200.0, 1600.0, 1024, 4096, 1024, fuse_depth=t.fuse_depth, head_tile=t.head_tile,
                 seg_levels=t.seg_levels, seg_rows=t.seg_rows)
    d_out = torch.empty((1024, 4096), device=cuda)
    f.process_image(torch.from_numpy(x).to(cuda), d_out, False)
    want = pyoracle.fdmt_f32(1200.0, 1600.0, x, 1024, 4096, 1024)
    assert np.array_equal(_bits(d_out.cpu().numpy()), _bits(want))


@pytest.mark.parametrize("fuse", [0, -1])
def test_fdmt_ones_mode(cuda, fuse):
    fmin, fmax, nchan, ncols, max_dt = 1200.0, 1600.0, 512, 2048, 512
    f = CFdmtGpu(fmin, fmax, nchan, ncols, max_dt, fuse_depth=fuse)
    d_out = torch.zeros((max_dt, ncols), device=cuda)
    f.process_image(None, d_out, True)
    want = pyoracle.fdmt_f32(fmin, fmax, None, nchan, ncols, max_dt, b_ones=True)
    assert np.array_equal(d_out.cpu().numpy(), want)


def test_fdmt_config0_full_size_bit_exact_and_fp64_error(cuda):
    beam = synth.config0()
    x = synth.filterbank(beam)
    f = CFdmtGpu(beam.fmin, beam.fmax, beam.nchan, beam.nsamp, beam.max_dt)
    d_out = torch.empty((beam.max_dt, beam.nsamp), device=cuda)
    f.process_image(torch.from_numpy(x).to(cuda), d_out)
    got = d_out.cpu().numpy()
    want = pyoracle.fdmt_f32(beam.fmin, beam.fmax, x, beam.nchan, beam.nsamp, beam.max_dt)
    assert np.array_equal(_bits(got), _bits(want))
    f64 = pyoracle.fdmt_f64(beam.fmin, beam.fmax, x.astype(np.float64), beam.nchan,
                            beam.nsamp, beam.max_dt)
    rel = np.abs(got - f64).max() / np.abs(f64).max()
    print(f"config0 FDMT max error vs FP64, relative to max |out|: {rel:.3e}")
    assert rel < 1e-5


def test_fdmt_deterministic_and_stream_ordered(cuda):
    fmin, fmax, nchan, ncols, max_dt = 1200.0, 1600.0, 1024, 8192, 1024
    x = torch.randn((nchan, ncols), device=cuda, generator=torch.Generator(cuda).manual_seed(3))
    f = CFdmtGpu(fmin, fmax, nchan, ncols, max_dt)
    s = torch.cuda.Stream()
    outs = []
    with torch.cuda.stream(s):
        for _ in range(2):
            o = torch.empty((max_dt, ncols), device=cuda)
            f.process_image(x, o)
            outs.append(o)
    s.synchronize()
    assert torch.equal(outs[0], outs[1])


def test_fdmt_rejects_bad_sizes(cuda):
    f = CFdmtGpu(1200.0, 1600.0, 64, 128, 64)
    with pytest.raises(ValueError):
        f.process_image(torch.zeros(10, device=cuda), torch.zeros((64, 128), device=cuda))


@pytest.mark.parametrize("case", CASES[:5] + CASES[7:])
@pytest.mark.parametrize("kind", ["keith", "pravir"])
def test_row_mask_fdmt_equals_the_transform(cuda, case, kind):
    """The channel-count form of the FDMT of a 0/1 row mask gives exactly the
    level-by-level transform of that plane (and b_ones is its all-1 case)."""
    import ctypes
    from cpp_projects_b200 import FDMTGPU, _capi
    from cpp_projects_b200._tensors import dev_ptr
    fmin, fmax, nchan, ncols, max_dt = case
    if kind == "pravir":
        if ncols <= max_dt:
            pytest.skip("Pravir plans need offsets below ncols")
        f = FDMTGPU(fmin, fmax, nchan, ncols, 1e-3, max_dt)
        rows = f.out_rows
    else:
        f = CFdmtGpu(fmin, fmax, nchan, ncols, max_dt, fuse_depth=0)
        rows = max_dt
    m = (np.random.default_rng(nchan).random(nchan) > 0.2).astype(np.float32)
    plane = torch.from_numpy(np.repeat(m[:, None], ncols, 1)).to(cuda)
    want = torch.empty((rows, ncols), device=cuda)
    _capi.call("bfs_fdmt_execute", f._plan, dev_ptr(plane), dev_ptr(want), 0, None)
    got = torch.full((rows, ncols), float("nan"), device=cuda)
    _capi.call("bfs_fdmt_execute_row_mask", f._plan, dev_ptr(plane), ncols, dev_ptr(got), None)
    assert torch.equal(got, want)
    if kind == "keith":
        ones = torch.full((rows, ncols), float("nan"), device=cuda)
        f.process_image(None, ones, True)
        oracle_ones = pyoracle.fdmt_f32(fmin, fmax, None, nchan, ncols, max_dt, b_ones=True)
        assert np.array_equal(ones.cpu().numpy(), oracle_ones)

