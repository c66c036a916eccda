"""Candidate output formats: the report text is byte-identical to the
reference's own COutChunkHeader::writeReport (built from its source) and
parses back like its read_outputlogfile_line; fragments (GPU) follow the
reference's cutQuadraticFragment rule."""
import json

import numpy as np
import pytest
import torch

from cpp_projects_b200 import reports
from oracle import pyoracle

RECORDS = [(1024, 129024, 3, 35001, 2, 310.58838, 56.8, 0, 0),
           (512, 32768, 256, 10250, 4, 7.0001, 0.0, 3, 11),
           (4096, 131072, 4095, 0, 32, 12345.678, -1.25, 99, 0)]


def test_report_bytes_match_the_reference(tmp_path):
    want = tmp_path / "ref.txt"
    if not pyoracle.ref_write_report(want, RECORDS, 1.25e-3):
        pytest.skip("reference report writer not built (oracle/_ref)")
    got = tmp_path / "ours.txt"
    reports.write_report(got, [reports.COutChunkHeader(*r) for r in RECORDS], 1.25e-3)
    assert got.read_bytes() == want.read_bytes()


def test_report_lines_parse_like_the_reference(tmp_path):
    path = tmp_path / "r.txt"
    reports.write_report(path, [reports.COutChunkHeader(*r) for r in RECORDS], 2e-4)
    for i, r in enumerate(RECORDS):
        ours = reports.read_outputlogfile_line(path, i)
        assert ours["numBlock"] == r[7] + 1 and ours["numChunk"] == r[8] + 1
        assert (ours["nrows"], ours["ncols"], ours["sucRow"], ours["sucCol"], ours["width"]) == r[:5]
        ref = pyoracle.ref_read_report_line(path, i)
        if ref is None:
            continue
        assert ref["ok"]
        for k in ("numBlock", "numChunk", "nrows", "ncols", "sucRow", "sucCol", "width"):
            assert ours[k] == ref[k], k
        assert np.float32(ours["snr"]) == np.float32(ref["snr"])
        assert np.float32(ours["cohDisp"]) == np.float32(ref["cohDisp"])
    path.write_text("no keys here\n")
    assert reports.read_outputlogfile_line(path, 0) is None


@pytest.mark.gpu
@pytest.mark.parametrize("shape,target", [((64, 1000), (3, 10)), ((64, 1000), (63, 999)),
                                          ((64, 1000), (0, 960)), ((100, 40), (99, 39)),
                                          ((50, 50), (10, 49)), ((1, 7), (0, 6))])
def test_fragment_follows_the_reference_rule(cuda, tmp_path, shape, target):
    rng = np.random.default_rng(sum(shape))
    plane = rng.standard_normal(shape).astype(np.float32)
    fr = reports.cut_quadratic_fragment(torch.from_numpy(plane).to(cuda), *target, width=4, snr=9.5,
                                        coh_dm=56.8)
    want, rb, cb = pyoracle.cut_quadratic_fragment(plane, *target)
    assert (fr.m_nBeginRow, fr.m_nBeginCol, fr.m_dim) == (rb, cb, want.shape[0])
    assert np.array_equal(fr.m_vctData.reshape(want.shape), want)
    p = fr.save_npy(tmp_path / "frag")
    assert np.array_equal(np.load(p), want)
    meta = json.loads(p.with_suffix(".json").read_text())
    assert meta["dim"] == want.shape[0] and meta["snr"] == 9.5 and meta["coherent_dm"] == 56.8
