"""CPU checks of the adjoint oracle: the FP64 adjoint is the transpose of the
FP64 FDMT (dot-product test), the FP32 adjoint agrees with it, and the FP64
S/N-at-cells gradient agrees with central finite differences."""
import numpy as np
import pytest

from oracle import pyoracle

CASES = [
    (1200.0, 1600.0, 64, 500, 64),
    (1100.0, 1500.0, 100, 333, 77),   # odd sub-band counts
    (1200.0, 1600.0, 3, 40, 5),
    (1200.0, 1328.0, 256, 257, 256),
]


@pytest.mark.parametrize("case", CASES)
def test_adjoint_is_the_transpose(case):
    fmin, fmax, nchan, ncols, mdt = case
    rng = np.random.default_rng(1)
    x = rng.standard_normal((nchan, ncols))
    g = rng.standard_normal((mdt, ncols))
    y = pyoracle.fdmt_f64(fmin, fmax, x, nchan, ncols, mdt)
    gx = pyoracle.fdmt_adjoint_f64(fmin, fmax, g, nchan, ncols, mdt)
    a, b = (y * g).sum(), (x * gx).sum()
    assert abs(a - b) <= 1e-12 * max(abs(a), 1.0) * 1e3
    gx32 = pyoracle.fdmt_adjoint_f32(fmin, fmax, g.astype(np.float32), nchan, ncols, mdt)
    assert np.abs(gx32 - gx).max() <= 1e-6 * np.abs(gx).max()


def test_snr_gradient_matches_finite_differences():
    rng = np.random.default_rng(2)
    y = rng.standard_normal((4, 300))
    y[1, 100:108] += 3.0
    cells = np.array([[1, 100, 8], [1, 98, 4], [3, 0, 1], [2, 296, 4]])
    snr, grads = pyoracle.snr_cells_f64(y, cells)
    eps = 1e-6
    for k, (d, t, w) in enumerate(cells):
        for u in (0, t, t + w - 1, 150, 299):
            yp, ym = y.copy(), y.copy()
            yp[d, u] += eps
            ym[d, u] -= eps
            fd = (pyoracle.snr_cells_f64(yp, cells[k:k + 1])[0][0]
                  - pyoracle.snr_cells_f64(ym, cells[k:k + 1])[0][0]) / (2 * eps)
            assert grads[k][u] == pytest.approx(fd, rel=1e-5, abs=1e-8)
