"""CPU: the search oracle reproduces the reference's golden candidate lists
(clusterization_forpravir/Candidates{1,2}.csv) and its clustering rules; the
boxcar kernel's register-window schedule is checked for every width set."""
import json
import re
from pathlib import Path

import numpy as np
import pytest

from oracle import pyoracle

GOLDEN = json.loads((Path(__file__).parent / "golden" / "cluster_golden.json").read_text())


def golden_plane():
    p = GOLDEN["plane"]
    a = np.full((p["rows"], p["cols"]), p["base"], np.float32)
    for r, c, v in p["spikes"]:
        a[r, c] = v
    return a


def as_rows(c):
    return [(int(r["mt"]), int(r["mdt"]), int(r["mwidth"]), f"{float(r['msnr']):.6g}") for r in c]


def golden_rows(key):
    return [(a, b, c, f"{d:.6g}") for a, b, c, d in GOLDEN[key]]


def test_oracle_dynamic_gather_matches_candidates1_csv():
    got = pyoracle.boxcar(golden_plane(), GOLDEN["thr"], 0, GOLDEN["dynamic_Q"])
    # the reference's order comes from atomicInc: compare as sets
    assert sorted(as_rows(got)) == sorted(golden_rows("candidates1_dynamic"))


def test_oracle_heap_gather_matches_candidates2_csv_in_order():
    got = pyoracle.boxcar(golden_plane(), GOLDEN["thr"], 1, GOLDEN["heap_W"])
    assert as_rows(got) == golden_rows("candidates2_heap")


def test_oracle_clustering_of_golden_heap_candidates():
    c = pyoracle.boxcar(golden_plane(), GOLDEN["thr"], 1, GOLDEN["heap_W"])
    perm, offs, dl = pyoracle.cluster(c, GOLDEN["metrics"])
    assert len(offs) - 1 == 3
    d = c[dl]
    assert [(int(r["mt"]), int(r["mdt"]), int(r["mwidth"]), float(r["msnr"])) for r in d] == \
        [(4, 0, 1, 140.0), (4, 2, 1, 100.0), (11, 0, 1, 120.0)]
    assert list(np.diff(offs)) == [3, 3, 3]


def test_oracle_select_delegates_tree_tie_rule():
    # The reference reduces 64 lanes with `if (arr[t+s] > arr[t])` for s = 32..1.
    # Maximum tied at lanes 5 and 40: lane 40 travels 40 -> 8 -> 0 and meets
    # lane 5's value (5 -> 1) only in the last step, where lane 0 keeps its own:
    # the tree picks position 40, not the lowest lane.
    c = np.zeros(64, pyoracle.CAND_DTYPE)
    c["msnr"] = 1.0
    c["msnr"][5] = 5.0
    c["msnr"][40] = 5.0
    perm = np.arange(64, dtype=np.int32)
    offs = np.array([0, 64], np.int32)
    assert pyoracle.select_delegates(c, perm, offs)[0] == 40
    # more members than lanes: lane 1 scans 1, 65 (first strict max kept)
    c = np.zeros(70, pyoracle.CAND_DTYPE)
    c["msnr"] = 1.0
    c["msnr"][2] = 5.0
    c["msnr"][65] = 5.0
    perm = np.arange(70, dtype=np.int32)
    offs = np.array([0, 70], np.int32)
    assert pyoracle.select_delegates(c, perm, offs)[0] == 2


def test_oracle_boxcar_truncated_windows_and_edges():
    plane = np.array([[1, 2, 3, 4, 5]], np.float32)
    got = pyoracle.boxcar(plane, -1.0, 0, 3)  # widths 1,2,4,8
    widths = {(int(r["mt"]), int(r["mwidth"])) for r in got}
    # w=4 only fits from t=0,1; w=8 never
    assert (0, 2) in widths and (1, 2) in widths and (2, 2) not in widths
    assert not any(w == 3 for _, w in widths)


@pytest.mark.parametrize("wmax", [1, 2, 3, 4, 5, 6, 7, 8, 16, 32, 64, 128])
def test_boxcar_sliding_window_schedule(wmax):
    """k_boxcar_reg's register window: with S starts per thread, step w reads
    window values w-1 .. w+S-2; the first S/4 float4s are loaded up front and
    the vector starting at value w+S-2 at step w.  Every value must be loaded
    before the step that first reads it, and every float4 read of the thread
    with the highest start must stay inside the tile of kRegTile + 4 ceil((W-1)/4)
    values."""
    src = (Path(__file__).resolve().parent.parent / "cpp_projects_b200" / "csrc" / "search.cu").read_text()
    S = int(re.search(r"constexpr int kRegStarts = (\d+);", src).group(1))
    threads = int(re.search(r"constexpr int kRegThreads = (\d+);", src).group(1))
    vec = (S + wmax - 1 + 3) // 4
    span = threads * S + 4 * ((wmax - 1 + 3) // 4)
    loaded = set(range(S))
    for w in range(1, wmax + 1):
        b = w + S - 2
        if b % 4 == 0 and b // 4 >= S // 4 and b // 4 < vec:
            loaded |= set(range(b, b + 4))
        assert set(range(w - 1, w + S - 1)) <= loaded, (w, sorted(loaded))
    last_vec = max([S // 4 - 1] + [(w + S - 2) // 4 for w in range(1, wmax + 1)
                                    if (w + S - 2) % 4 == 0 and (w + S - 2) // 4 < vec])
    top = (threads - 1) * (S // 4) + last_vec       # float4 index of the highest read
    assert 4 * top + 3 < span
