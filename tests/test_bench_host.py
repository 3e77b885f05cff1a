"""Host logic of bench.py: the N > 1 replica plumbing on world-size-2 gloo ranks (CPU),
the algorithmic byte counts and the clock-record parser."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

import bench  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    d = bench.init_dist(world, "gloo")
    cpu = torch.device("cpu")
    bench.barrier(d, cpu)
    m = bench.max_over_ranks(10.0 + rank * 5.0, d, cpu)
    # every rank takes the same collective steps; the max is the slowest rank's time
    q.put((rank, m, bench.dist_env()))
    d.destroy_process_group()


def test_replica_timing_max_over_ranks_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, m, env in out:
        assert m == 15.0
        assert env == (world, rank, rank)


def test_single_rank_plumbing_is_identity():
    assert bench.max_over_ranks(3.5, None, None) == 3.5
    bench.barrier(None, None)


def test_step_bytes_match_the_byte_model():
    """3 substeps x (14 state/store passes + 1 control read of v) in FP64 plus
    (16 product passes in y-planes + 24 passes of the z-padded slab) at the product precision."""
    w = bench.workload()
    nxh = w["nx"] // 2
    nspec = nxh * w["nz"] * w["ny"]
    nmid = nxh * (w["nz"] * 3 // 2) * w["ny"]
    for s_nl in (8, 16):
        expect = 3 * (16 * 15 * nspec + s_nl * (16 * nspec + 24 * nmid))
        assert bench.step_bytes(w, s_nl) == expect


def test_clock_parser(tmp_path):
    c = bench.ClockSampler("0")
    c.path = str(tmp_path / "c.csv")
    with open(c.path, "w") as f:
        f.write("0, 1800, 1965, 700.0, 0x0, Not Active, Not Active, Not Active, Not Active\n")
        f.write("0, 1700, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active\n")
        f.write("0, 1750, 1965, 980.0, 0x4, Not Active, Not Active, Not Active, Active\n")
    s = c.summary()
    assert s["sm_mhz"] == 1750.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]


def test_measured_peaks_has_a_number():
    peak, kind = bench.measured_peaks()
    assert peak > 1000 and kind in ("measured", "fallback")


def test_gpus_n_without_launcher_relaunches_n_ranks(monkeypatch):
    """`bench.py --gpus 4` with no WORLD_SIZE in the environment runs itself as 4 ranks under
    torch.distributed.run on 127.0.0.1 (one process per GPU), passing the arguments through."""
    seen = {}

    def fake_call(cmd):
        seen["cmd"] = cmd
        return 0

    monkeypatch.delenv("WORLD_SIZE", raising=False)
    monkeypatch.setattr(bench.subprocess, "call", fake_call)
    assert bench.main(["--gpus", "4", "--steps", "7", "--warmup", "3"]) == 0
    cmd = seen["cmd"]
    assert cmd[1:3] == ["-m", "torch.distributed.run"]
    assert "--nproc-per-node=4" in cmd and "--master-addr=127.0.0.1" in cmd
    assert cmd[-6:] == ["--gpus", "4", "--steps", "7", "--warmup", "3"]
    assert cmd[-7].endswith("bench.py")
