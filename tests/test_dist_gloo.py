"""The multi-rank harness on CPU: two gloo ranks, the max-over-ranks timing and
the per-rank ensembles (replicas, no data-path collective)."""

import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from menodax_b200 import _dist
    from workloads import systems

    r, w, _ = _dist.init(backend="gloo", timeout_s=60)
    cfg = systems.robertson_config(size=8, seed=_dist.shard_seed(42, r))
    _dist.barrier(w)
    out[r] = _dist.max_over_ranks(10.0 * (r + 1), w)
    out[2 + r] = float(cfg["params"][0, 0])
    _dist.finalize(w)


def test_two_gloo_ranks_take_the_max_and_draw_disjoint_ensembles():
    ctx = mp.get_context("spawn")
    out = ctx.Array("d", 4)
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[0] == out[1] == 20.0
    assert out[2] != out[3]
    assert np.isfinite(out[2])
