"""The bench's multi-rank plumbing on CPU: two gloo ranks (world size 2).

`bench.py` runs one replica per GPU ("replicas only": the transforms shard by
lane with no exchange), times each rank on its own device and reports the
maximum over ranks; the reference arm runs on rank 0 alone.  The rank logic is
exercised here with the gloo backend on 127.0.0.1, no GPU.
"""
import io
import json
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(world),
                       "RANK": str(rank), "LOCAL_RANK": str(rank), "AFC_BENCH_BACKEND": "gloo"})
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    import bench
    w, r, _ = bench.dist_init()
    out = {"world": w, "rank": r}
    out["max"] = bench.max_over_ranks(float(rank + 1) * 0.5, w, torch.device("cpu"))
    bench.barrier(w)
    # reference arm: rank 0 prints one line, the other ranks exit 0 without work
    bench.SHAPE = (8, 8, 8)
    args = type("A", (), {"steps": 1, "warmup": 1, "gpus": w})()
    buf = io.StringIO()
    with redirect_stdout(buf):
        rc = bench.run_reference(args)
    out["ref_rc"] = rc
    out["ref_out"] = buf.getvalue()
    bench.barrier(w)
    dist.destroy_process_group()
    q.put(out)


@pytest.mark.timeout(300)
def test_two_gloo_ranks_max_and_reference_arm():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort(key=lambda d: d["rank"])
    assert all(d["world"] == 2 for d in res)
    assert all(d["max"] == 1.0 for d in res)          # max over ranks of 0.5, 1.0
    assert all(d["ref_rc"] == 0 for d in res)
    assert res[1]["ref_out"] == ""                    # only rank 0 runs the reference arm
    line = json.loads(res[0]["ref_out"].strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"
