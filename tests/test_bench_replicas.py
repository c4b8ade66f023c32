"""The replica path of bench.py on CPU: world size 2 over gloo.  Every rank reports
its own step and end-to-end times; the job's are the slowest rank's."""
import os
import socket
import sys

import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, REPO)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    # rank 0 is slower on the step, rank 1 on the end-to-end path
    got = bench.max_over_ranks([10.0 + rank * 5.0, 80.0 - rank * 20.0], dist, "cpu")
    out[rank] = got
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo_world_2():
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[0] == [15.0, 80.0] and out[1] == [15.0, 80.0]


def test_max_over_ranks_without_process_group():
    sys.path.insert(0, REPO)
    import bench
    assert bench.max_over_ranks([3, 4.5], None, "cpu") == [3.0, 4.5]


def test_peaks_fall_back_when_file_absent(tmp_path, monkeypatch):
    """Without a peaks file the roofline denominators are the labelled fallback;
    with one, its figures are used as written."""
    sys.path.insert(0, REPO)
    import json
    import bench
    monkeypatch.setattr(bench, "REPO", str(tmp_path))
    got = bench.measured_peaks()
    assert got == bench.FALLBACK_PEAKS and got is not bench.FALLBACK_PEAKS
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 7000.0, "bf16_tflops": 1600.0}))
    assert bench.measured_peaks() == {"hbm_gbs": 7000.0, "bf16_tflops": 1600.0}
    (tmp_path / "MEASURED_PEAKS.json").write_text("{not json")
    assert bench.measured_peaks()["source"] == "fallback"
