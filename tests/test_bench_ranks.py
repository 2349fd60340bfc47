"""The multi-GPU bench path on CPU: replicas only, no data-path collective;
the job time is the max over ranks (gloo, world size 2, 127.0.0.1)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        w, r, local = bench.dist_setup()
        ms = 10.0 + 5.0 * rank  # the slower rank sets the job time
        job = bench.max_over_ranks(ms, dist, device="cpu")
        out[rank] = (w, r, local, job, bench.replica_value(w, 100, 30.0, job))
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time():
    world, port = 2, _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][:3] == (2, 0, 0) and res[1][:3] == (2, 1, 1)
    for r in range(world):
        assert res[r][3] == pytest.approx(15.0)
        # 2 replicas x 100 steps x 30 s in 15 ms of job time
        assert res[r][4] == pytest.approx(2 * 100 * 30.0 / 86400.0 / 0.015)


def test_output_line_is_strict_json():
    """A forecast that went non-finite reports null: the line stays strict JSON."""
    import json
    import numpy as np
    sys.path.insert(0, ROOT)
    import bench
    line = {"value": 1.5, "accuracy": {"L2": float("nan"), "curve": [1e-8, np.float64("inf"), -np.inf],
                                       "drift": (np.float64(2.0), np.nan)}, "n": 3, "s": "x"}
    out = json.loads(json.dumps(bench.strict_json(line), allow_nan=False))
    assert out == {"value": 1.5, "accuracy": {"L2": None, "curve": [1e-8, None, None], "drift": [2.0, None]},
                   "n": 3, "s": "x"}
