"""The C++ drop-in header (include/bfs_dropin.hpp) compiles a reference-style
driver unchanged (CPU) and, on the GPU, gives the same FDMT (both plan kinds)
as the oracle and the expected delegate log for the reference's clustering
test plane."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from cpp_projects_b200 import _capi
from oracle import pyoracle

ROOT = Path(__file__).resolve().parent.parent
CUDA = Path("/usr/local/cuda")


def build_demo(tmp: Path) -> Path:
    exe = tmp / "dropin_demo"
    cmd = ["g++", "-std=c++17", "-O2", str(ROOT / "tests/cpp/dropin_demo.cpp"), "-I", str(ROOT / "include"),
           "-I", str(CUDA / "include"), "-L", str(_capi.LIB_PATH.parent), "-lbfs_b200",
           "-L", str(CUDA / "lib64"), "-lcudart", f"-Wl,-rpath,{_capi.LIB_PATH.parent}",
           f"-Wl,-rpath,{CUDA / 'lib64'}", "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_dropin_header_compiles_a_reference_style_driver(tmp_path):
    assert build_demo(tmp_path).exists()


@pytest.mark.gpu
def test_dropin_driver_runs_and_matches(cuda, tmp_path):
    exe = build_demo(tmp_path)
    x = np.random.default_rng(5).standard_normal((64, 1024)).astype(np.float32)
    x.tofile(tmp_path / "in.bin")
    r = subprocess.run([str(exe), str(tmp_path / "in.bin"), str(tmp_path / "out.bin"),
                        str(tmp_path / "ouput.log"), str(tmp_path / "pravir.bin")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(tmp_path / "out.bin", np.float32).reshape(64, 1024)
    want = pyoracle.fdmt_f32(1200.0, 1600.0, x, 64, 1024, 64)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    pr = np.fromfile(tmp_path / "pravir.bin", np.float32).reshape(-1, 1024)
    pwant = pyoracle.pravir_fdmt(1200.0, 1600.0, x, 64, 1024, 64)
    assert pr.shape == pwant.shape and np.array_equal(pr.view(np.uint32), pwant.view(np.uint32))
    from cpp_projects_b200 import reports
    want_rep = tmp_path / "want.report"
    reports.write_report(want_rep, [reports.COutChunkHeader(3, 16, 0, 4, 1, 140.0, 56.8, 0, 0)], 1.25e-3)
    assert (tmp_path / "ouput.log.report").read_bytes() == want_rep.read_bytes()
    body = [ln.split() for ln in (tmp_path / "ouput.log").read_text().splitlines()[1:]]
    assert body == [["1", "4", "4e-05", "0", "1", "140", "3"],
                    ["2", "4", "4e-05", "2", "1", "100", "3"],
                    ["3", "11", "0.00011", "0", "1", "120", "3"]]
