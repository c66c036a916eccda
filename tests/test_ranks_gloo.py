"""The multi-rank path on CPU: two gloo ranks (one process each, as torchrun
starts them) through the same coordination bench.py uses on GPUs — the
timing barrier, the maximum over ranks, one beam set per rank (weak
scaling, no collective on the data path) — and the reference arm, which runs
on rank 0 only."""
import contextlib
import io
import json
import os
import socket
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import bench
    from cpp_projects_b200.ranks import Ranks
    ranks = Ranks("gloo", timeout_s=60)
    ranks.barrier()
    step_ms = 10.0 * (rank + 1)                    # this rank's measured time
    slowest = ranks.max(step_ms)
    beams = bench.beams_for("config2", rank)
    ranks.barrier()
    ranks.close()
    res = {"rank": rank, "world": ranks.world, "slowest": slowest,
           "nbeams": len(beams), "shapes": [[b.nchan, b.nsamp] for b in beams],
           "seeds": [b.seed for b in beams]}
    Path(out_dir, f"rank{rank}.json").write_text(json.dumps(res))


def test_two_gloo_ranks_share_timing_and_shard_beams(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    r = [json.loads((tmp_path / f"rank{i}.json").read_text()) for i in range(world)]
    assert all(x["world"] == world for x in r)
    assert all(x["slowest"] == 10.0 * world for x in r)    # max over ranks, seen by every rank
    assert r[0]["nbeams"] == r[1]["nbeams"] == 48          # weak scaling: a full set per rank
    assert r[0]["shapes"] == r[1]["shapes"]                # the same work on every rank
    assert set(r[0]["seeds"]).isdisjoint(r[1]["seeds"])    # independent data per rank


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    sys.path.insert(0, str(ROOT))
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    args = bench.parse_args(["--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3"])
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        rc = bench.run_reference(args)
    assert rc == 0 and buf.getvalue() == ""


def test_bench_gpus_2_launches_two_ranks():
    """bench.py --gpus 2 without a launcher starts two ranks itself
    (torch.distributed.run on 127.0.0.1; gloo here, no GPU) and prints one
    line with n_gpus = 2 and one 48-beam set per rank."""
    import subprocess
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--gpus", "2", "--dry-run"],
                       capture_output=True, text=True, timeout=300, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["n_gpus"] == 2 and line["dry_run"] and line["slowest_rank_stand_in"] == 2.0
    s0, s1 = line["rank_seeds"]
    assert len(s0) == len(s1) == 48 and set(s0).isdisjoint(s1)


def test_stratified_sample_covers_every_channel_count_first():
    sys.path.insert(0, str(ROOT))
    import bench
    beams = bench.beams_for("config2", 0)
    s = bench.stratified(beams)
    assert sorted(b.seed for b in s) == sorted(b.seed for b in beams)
    assert [b.nchan for b in s[:4]] == [256, 512, 1024, 4096]
    # within a channel count, smallest first
    for n in (256, 512, 1024, 4096):
        sizes = [b.nsamp for b in s if b.nchan == n]
        assert sizes == sorted(sizes)
