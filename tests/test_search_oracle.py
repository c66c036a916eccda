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
def test_boxcar_pair_window_schedule(wmax):
    """k_boxcar_pair's register window: a lane's S starts read positions
    w-1 .. w+S-2 at width step w, each position a pair {row 0, row 1}, two
    positions per float4.  The first kPre float4s are loaded up front and the
    one starting at position w+S-2+kAhead at step w (kAhead steps early).
    Every position must be loaded before the step that first reads it, and
    the last lane's highest float4 must stay inside the warp's staged tile,
    whose logical float4 f sits at f + f // 4 (one float4 of padding after
    every four)."""
    src = (Path(__file__).resolve().parent.parent / "cpp_projects_b200" / "csrc" / "search.cu").read_text()
    S = int(re.search(r"constexpr int kPairStarts = (\d+);", src).group(1))
    ahead = int(re.search(r"constexpr int kAhead = (\d+);", src).group(1))
    assert "constexpr int kPairWarpTile = 32 * kPairStarts;" in src
    npos = S + wmax - 1
    nvec = (npos + 1) // 2
    npre = min((S + ahead + 1) // 2, nvec)
    loaded = set()
    for v in range(npre):
        loaded |= {2 * v, 2 * v + 1}
    highest = npre - 1
    for w in range(1, wmax + 1):
        pn = w + S - 2 + ahead
        if pn % 2 == 0 and npre <= pn // 2 < nvec:
            loaded |= {pn, pn + 1}
            highest = max(highest, pn // 2)
        assert set(range(w - 1, w + S - 1)) <= loaded, (w, sorted(loaded))
    span = (32 * S + wmax - 1 + 3) // 4 * 4          # staged positions of a warp
    nf4 = span // 2
    f_top = 31 * S // 2 + highest                      # the last lane's highest logical float4
    assert f_top < nf4
    assert f_top + f_top // 4 < nf4 + nf4 // 4         # inside the padded array


@pytest.mark.parametrize("rows,cols", [(4096, 32768), (256, 131072), (1024, 16749), (512, 24485), (3, 5),
                                       (7, 1), (2, 8193), (65535, 3)])
def test_row_stats_partition(rows, cols):
    """k_row_stats' work split (emulated from the constants in its sources):
    the cluster size per row (1..kStatMaxCluster, doubled while the grid is
    under two waves of 8 CTAs per SM and each thread keeps >= 32 samples),
    each CTA's range (a multiple of 4 samples), the scalars before the first
    4-sample piece whose plane index is a multiple of 4, the pieces strided
    over the threads and the tail scalars: every sample of a row is added
    exactly once, and each piece starts on a 16-byte boundary of a 16-byte
    aligned plane.  The assignment depends on the plane index only."""
    root = Path(__file__).resolve().parent.parent / "cpp_projects_b200" / "csrc"
    common = (root / "search_common.cuh").read_text()
    T = int(re.search(r"constexpr int kStatThreads = (\d+);", common).group(1))
    maxc = int(re.search(r"constexpr int kStatMaxCluster = (\d+);", common).group(1))
    src = (root / "search.cu").read_text()
    assert "static_cast<long long>(rows) * split < 16LL * sms" in src
    assert "cols / (2 * split) >= 32 * kStatThreads" in src
    sms = 148
    split = 1
    while split < maxc and rows * split < 16 * sms and cols // (2 * split) >= 32 * T:
        split *= 2
    assert split & (split - 1) == 0 and split <= 8   # a portable cluster size
    for r in sorted({0, 1, 2, 3, rows - 1} & set(range(rows))):
        seen = np.zeros(cols, np.int64)
        per = ((cols + split - 1) // split + 3) & ~3
        for rank in range(split):
            beg = min(cols, rank * per)
            end = min(cols, beg + per)
            phase = (r * cols + beg) & 3
            lead = min(end - beg, (4 - phase) & 3)
            n4 = (end - beg - lead) >> 2
            tail = end - beg - lead - 4 * n4
            assert 0 <= lead < 4 and 0 <= tail < 4 and lead + 4 <= T
            if n4:
                assert (r * cols + beg + lead) % 4 == 0   # 16-byte aligned given an aligned plane
                base = beg + lead + 4 * np.arange(n4)
                for j in range(4):
                    np.add.at(seen, base + j, 1)
            for k in range(T):
                if k < lead:
                    seen[beg + k] += 1
                elif 4 <= k < 4 + tail:
                    seen[beg + lead + 4 * n4 + (k - 4)] += 1
        assert (seen == 1).all(), (r, split)
