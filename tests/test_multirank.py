"""The multi-rank path of bench.py on the host: two ranks over gloo (the
backend bench.py takes when no GPU is present) meet at the barrier, agree on
the maximum of their timings, derive different replica scenes from their
ranks, and run the reference arm on rank 0 alone while rank 1 leaves
without work."""
import json
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, port, out_dir):
    import contextlib
    import io
    import sys
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": "2",
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import torch.distributed as dist

    import bench
    world, r, _ = bench.dist_setup()
    assert (world, r) == (2, rank) and dist.get_backend() == "gloo"
    bench.barrier(world)
    ms = bench.max_over_ranks(world, 10.0 + rank)
    spec = bench.scene_spec(rank, 16)
    sys.argv = ["bench.py", "--impl", "reference", "--scale", "16", "--steps", "1",
                "--warmup", "0"]
    args = bench.parse_args()
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        bench.run_reference(args, world, r)
    bench.barrier(world)
    dist.destroy_process_group()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"max_ms": ms, "seed": spec["seed"], "stdout": buf.getvalue()}, f)


def test_two_ranks_over_gloo(tmp_path):
    import torch.multiprocessing as mp
    mp.spawn(_rank_main, args=(_free_port(), str(tmp_path)), nprocs=2, join=True)
    res = [json.load(open(os.path.join(str(tmp_path), f"rank{k}.json"))) for k in (0, 1)]
    assert res[0]["max_ms"] == res[1]["max_ms"] == pytest.approx(11.0)
    assert res[0]["seed"] != res[1]["seed"]
    line = json.loads(res[0]["stdout"].strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert res[1]["stdout"] == ""
