"""bench.py's multi-rank path on CPU: two gloo ranks on 127.0.0.1.

N GPUs run independent replicas with no collective in the data path; the only
collectives are the barriers and the max over ranks of each timed region, and
the whole-job value counts every rank's atoms over the slowest rank's time.
Both ranks must get the same numbers."""
import json
import socket
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, outdir):
    import datetime
    import os

    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    sys.path.insert(0, str(ROOT))
    import bench
    ms = bench.max_over_ranks(10.0 + 5.0 * rank, world, torch.device("cpu"))
    value = bench.replicas_value(1000, 20, world, ms)
    dist.barrier()
    dist.destroy_process_group()
    Path(outdir, f"rank{rank}.json").write_text(json.dumps({"ms": ms, "value": value}))


def test_two_ranks_agree_on_the_slowest_time(tmp_path):
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(world)]
    assert res[0] == res[1]
    assert res[0]["ms"] == 15.0
    assert res[0]["value"] == 1000 * 20 * 2 / 0.015
