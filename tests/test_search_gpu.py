"""GPU parity of normalisation, boxcar gather, clustering, delegates and the
statistical preprocessing against the oracle and the reference's golden CSVs.
Integer outputs (candidate lists, groups, delegates) must be identical; float
outputs bit-identical unless a tolerance is written next to the assert."""
import json
from pathlib import Path

import numpy as np
import pytest
import torch

from cpp_projects_b200 import BfsError, cluster, preproc, search, synth
from cpp_projects_b200._capi import BFS_ERR_OVERFLOW
from oracle import pyoracle

pytestmark = pytest.mark.gpu

GOLDEN = json.loads((Path(__file__).parent / "golden" / "cluster_golden.json").read_text())


def normalise_with(y, stats):
    """(x - mean_r) / std_r in float32, one rounding per operation (the
    oracle's and the product's arithmetic), with given row statistics."""
    r = y.shape[0]
    m, sd = stats[:r, None], stats[r:, None]
    with np.errstate(divide="ignore", invalid="ignore"):
        z = ((y - m).astype(np.float32) / sd).astype(np.float32)
    z[np.broadcast_to(sd == 0, z.shape)] = 0.0
    return z


def golden_plane():
    p = GOLDEN["plane"]
    a = np.full((p["rows"], p["cols"]), p["base"], np.float32)
    for r, c, v in p["spikes"]:
        a[r, c] = v
    return a


def rows_of(c):
    return [(int(r["mt"]), int(r["mdt"]), int(r["mwidth"]), f"{float(r['msnr']):.6g}") for r in c]


def golden_rows(key):
    return [(a, b, c, f"{d:.6g}") for a, b, c, d in GOLDEN[key]]


def same_cands(a, b):
    return (len(a) == len(b) and np.array_equal(a["mt"], b["mt"]) and np.array_equal(a["mdt"], b["mdt"])
            and np.array_equal(a["mwidth"], b["mwidth"])
            and np.array_equal(a["msnr"].view(np.uint32), b["msnr"].view(np.uint32)))


def test_golden_dynamic_and_heap_paths(cuda):
    d = torch.from_numpy(golden_plane()).to(cuda)
    c1, n1 = search.gather_candidates_in_dynamicalArray(d, 3, 16, GOLDEN["thr"], GOLDEN["dynamic_Q"])
    assert sorted(rows_of(search.cands_to_numpy(c1))) == sorted(golden_rows("candidates1_dynamic"))
    thr_dev = torch.tensor([GOLDEN["thr"]], device=cuda)  # threshold bound to device memory
    c2, n2 = search.gather_candidates_in_heap_with_plan(d, 3, 16, thr_dev, GOLDEN["heap_W"])
    assert rows_of(search.cands_to_numpy(c2)) == golden_rows("candidates2_heap")


def test_golden_clusterization_main_log(cuda, tmp_path):
    d = torch.from_numpy(golden_plane()).to(cuda)
    log = tmp_path / "ouput.log"
    cl = cluster.clusterization_main(d, 3, 16, GOLDEN["thr"], GOLDEN["heap_W"], GOLDEN["metrics"],
                                     str(log), 1e-5, 0.0)
    lines = log.read_text().splitlines()
    assert lines[0].split() == ["N", "t,", "bin", "t,", "sec", "dedisp", "width", "SNR", "num"]
    body = [ln.split() for ln in lines[1:]]
    assert body == [["1", "4", "4e-05", "0", "1", "140", "3"],
                    ["2", "4", "4e-05", "2", "1", "100", "3"],
                    ["3", "11", "0.00011", "0", "1", "120", "3"]]
    assert cl.ngroups == 3


PLANES = [(8, 5000), (3, 1024), (1, 37), (17, 2049), (64, 3000)]


@pytest.mark.parametrize("shape", PLANES)
@pytest.mark.parametrize("mode,param", [(0, 5), (0, 0), (0, 6), (0, 7), (0, 8), (1, 4), (1, 33)])
def test_boxcar_matches_oracle(cuda, shape, mode, param):
    rng = np.random.default_rng(hash((shape, mode, param)) % 2**32)
    x = rng.standard_normal(shape).astype(np.float32)
    thr = 2.5
    want = pyoracle.boxcar(x, thr, mode, param)
    got, n = search.boxcar_gather(torch.from_numpy(x).to(cuda), thr, mode, param)
    got = search.cands_to_numpy(got)
    assert n == len(want) and same_cands(got, want)


def test_boxcar_with_fused_row_normalisation(cuda):
    rng = np.random.default_rng(5)
    x = (rng.standard_normal((32, 4100)) * 3 + 1.5).astype(np.float32)
    z, m, s = pyoracle.norm_rows(x)
    d = torch.from_numpy(x).to(cuda)
    zg, st = search.norm_rows(d)
    # FP64 statistics summed in another order: equal after rounding to float
    # except in rare half-way cases; allow 1 ulp on the stats and the plane.
    stg = st.cpu().numpy()
    assert np.abs(stg[:32].view(np.int32) - m.view(np.int32)).max() <= 1
    assert np.abs(stg[32:].view(np.int32) - s.view(np.int32)).max() <= 1
    assert np.abs(zg.cpu().numpy().view(np.int32) - z.view(np.int32)).max() <= 1
    got, n = search.boxcar_gather(d, 3.0, 0, 5, stats=st)
    # the boxcar's fused normalisation against the oracle's, both given the
    # GPU's statistics: identical lists (the statistics themselves are within
    # 1 ulp of the oracle's, asserted above)
    want = pyoracle.boxcar(normalise_with(x, stg), 3.0, 0, 5)
    assert n == len(want) and same_cands(search.cands_to_numpy(got), want)
    # and given the oracle's own statistics, the oracle's own normalised plane
    st_o = torch.from_numpy(np.concatenate([m, s])).to(cuda)
    got_o, n_o = search.boxcar_gather(d, 3.0, 0, 5, stats=st_o)
    want_o = pyoracle.boxcar(z, 3.0, 0, 5)
    assert n_o == len(want_o) and same_cands(search.cands_to_numpy(got_o), want_o)


def test_boxcar_fast_snr_mode_is_within_two_ulp(cuda):
    x = np.random.default_rng(9).standard_normal((16, 8192)).astype(np.float32)
    want = pyoracle.boxcar(x, 2.0, 0, 5)
    got, _ = search.boxcar_gather(torch.from_numpy(x).to(cuda), 2.0, 0, 5, snr_fast=True)
    got = search.cands_to_numpy(got)
    key = lambda c: set(zip(c["mt"].tolist(), c["mdt"].tolist(), c["mwidth"].tolist()))
    diff = key(got) ^ key(want)
    # the fast quotient differs from the IEEE one by <= 2 ulp: only candidates
    # within 2 ulp of the threshold can change side
    assert len(diff) <= 2
    common = np.intersect1d(got[["mt", "mdt", "mwidth"]], want[["mt", "mdt", "mwidth"]])
    assert len(common) >= len(want) - 2


def test_boxcar_capacity_overflow_and_empty(cuda):
    x = torch.randn((4, 4096), device=cuda)
    with pytest.raises(BfsError) as e:
        search.boxcar_gather(x, -100.0, 0, 2, capacity=10)
    assert e.value.status == BFS_ERR_OVERFLOW
    c, n = search.boxcar_gather(x, 1e30, 1, 4)
    assert n == 0 and c.shape[0] == 0


def _random_cands(rng, n, tmax=50, dmax=10, wmax=6):
    c = np.zeros(n, pyoracle.CAND_DTYPE)
    c["mt"] = rng.integers(0, tmax, n)
    c["mdt"] = rng.integers(0, dmax, n)
    c["mwidth"] = rng.integers(0, wmax, n)
    c["msnr"] = rng.integers(0, 8, n).astype(np.float32) * 0.5 + 7.0  # many exact ties
    return c


@pytest.mark.parametrize("n,metrics", [(1, (2, 1, 2)), (9, (2, 1, 2)), (500, (2, 1, 2)),
                                       (5000, (16, 8, 1 << 30)), (20000, (0, 0, 0))])
def test_cluster_matches_oracle(cuda, n, metrics):
    c = _random_cands(np.random.default_rng(n), n)
    perm, offs, dl = pyoracle.cluster(c, metrics)
    cl = cluster.complete_clusterization(search.cands_from_numpy(c, cuda), metrics)
    assert cl.ngroups == len(offs) - 1
    np.testing.assert_array_equal(cl.perm.cpu().numpy(), perm)
    np.testing.assert_array_equal(cl.offsets.cpu().numpy(), offs)
    np.testing.assert_array_equal(cl.delegates.cpu().numpy(), dl)


def test_select_delegates_large_groups_with_ties(cuda):
    rng = np.random.default_rng(4)
    c = _random_cands(rng, 3000)
    perm = rng.permutation(3000).astype(np.int32)
    offs = np.array([0, 1, 70, 500, 2999, 3000], np.int32)
    want = pyoracle.select_delegates(c, perm, offs)
    got = cluster.select_delegates(search.cands_from_numpy(c, cuda),
                                   torch.from_numpy(perm).to(cuda), torch.from_numpy(offs).to(cuda))
    np.testing.assert_array_equal(got.cpu().numpy(), want)


def test_calc_fdmt_inputs_matches_oracle(cuda):
    rng = np.random.default_rng(12)
    x = rng.standard_normal((256, 3000)).astype(np.float32)
    x[17] *= 40.0  # an RFI row that must be zapped
    x[200] += 3.0
    want_x, want_mask, want_stats = pyoracle.calc_fdmt_inputs(x)
    d = torch.from_numpy(x).to(cuda)
    buff = torch.empty(4 + 2 * 256, device=cuda)
    mask = torch.empty_like(d)
    preproc.calc_fdmt_inputs(d, 256, 3000, buff, mask)
    assert want_mask[17].max() == 0.0 and want_mask[16].min() == 1.0
    np.testing.assert_array_equal(mask.cpu().numpy(), want_mask)
    # FP64 reductions in another order; equal up to 1 ulp after rounding
    assert np.abs(buff.cpu().numpy().view(np.int32) - want_stats.view(np.int32)).max() <= 1
    assert np.abs(d.cpu().numpy() - want_x).max() <= 1e-6 * np.abs(want_x).max()


def test_fdmt_normalization_bit_exact(cuda):
    rng = np.random.default_rng(1)
    f = rng.standard_normal(100003).astype(np.float32) * 50
    nrm = rng.uniform(0, 600, 100003).astype(np.float32)
    nrm[:10] = 0.0
    out = torch.empty(100003, device=cuda)
    preproc.fdmt_normalization(torch.from_numpy(f).to(cuda), torch.from_numpy(nrm).to(cuda),
                               100003, out)
    assert np.array_equal(out.cpu().numpy(), pyoracle.fdmt_normalize(f, nrm))


def test_config0_search_chain_finds_the_pulse(cuda):
    from cpp_projects_b200 import CFdmtGpu
    beam = synth.config0()
    x = torch.from_numpy(synth.filterbank(beam)).to(cuda)
    f = CFdmtGpu(beam.fmin, beam.fmax, beam.nchan, beam.nsamp, beam.max_dt)
    dm = f(x)
    st = search.row_stats(dm)
    cands, n = search.boxcar_gather(dm, 7.0, 0, 5, stats=st)
    assert n > 0
    cl = cluster.complete_clusterization(cands, (16, 8, 1 << 30))
    best = cl.delegate_records()
    top = best[np.argmax(best["msnr"])]
    assert abs(int(top["mdt"]) - 256) <= 8 and 10240 <= int(top["mt"]) <= 10270
    # parity of the whole chain with the oracle on the same plane: the FDMT
    # bit for bit, the row statistics within 1 ulp, then (given the same
    # statistics) the full candidate list, the groups and the delegates
    y = dm.cpu().numpy()
    want_y = pyoracle.fdmt_f32(beam.fmin, beam.fmax, synth.filterbank(beam), beam.nchan, beam.nsamp,
                               beam.max_dt)
    assert np.array_equal(y.view(np.uint32), want_y.view(np.uint32))
    stg = st.cpu().numpy()
    _, m, sd = pyoracle.norm_rows(y)
    assert np.abs(stg[:512].view(np.int32) - m.view(np.int32)).max() <= 1
    assert np.abs(stg[512:].view(np.int32) - sd.view(np.int32)).max() <= 1
    want = pyoracle.boxcar(normalise_with(y, stg), 7.0, 0, 5)
    assert n == len(want) and same_cands(search.cands_to_numpy(cands), want)
    perm, offs, dl = pyoracle.cluster(want, (16, 8, 1 << 30))
    assert cl.ngroups == len(offs) - 1
    np.testing.assert_array_equal(cl.perm.cpu().numpy(), perm)
    np.testing.assert_array_equal(cl.offsets.cpu().numpy(), offs)
    np.testing.assert_array_equal(cl.delegates.cpu().numpy(), dl)


@pytest.mark.parametrize("rows,cols", [(4096, 8192), (256, 131072), (1024, 16749), (33, 4099), (5, 3)])
def test_row_stats_do_not_depend_on_the_planes_address(cuda, rows, cols):
    """The row statistics' order of additions follows each row's plane index,
    so a plane 4 bytes past a 16-byte boundary (scalar loads) gives the same
    bits as its 16-byte aligned copy (16-byte loads), and both stay within
    1 ulp of the oracle's FP64 sums."""
    rng = np.random.default_rng(rows + cols)
    x = (rng.standard_normal(rows * cols + 1) * 2.0 + 0.25).astype(np.float32)
    flat = torch.from_numpy(x).to(cuda)
    shifted = flat[1:].view(rows, cols)                # 4 bytes past the allocation's start
    assert shifted.data_ptr() % 16 == 4
    aligned = shifted.clone()
    assert aligned.data_ptr() % 16 == 0
    st_s = search.row_stats(shifted).cpu().numpy()
    st_a = search.row_stats(aligned).cpu().numpy()
    assert np.array_equal(st_s.view(np.int32), st_a.view(np.int32))
    _, m, s = pyoracle.norm_rows(x[1:].reshape(rows, cols))
    assert np.abs(st_a[:rows].view(np.int32) - m.view(np.int32)).max() <= 1
    assert np.abs(st_a[rows:].view(np.int32) - s.view(np.int32)).max() <= 1
