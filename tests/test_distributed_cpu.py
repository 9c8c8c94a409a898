"""Multi-process plumbing of the N > 1 paths on CPU, world size 2 over gloo
(127.0.0.1): the bench's whole-job reduction of the replicas, the NCCL unique
id shared through a torch.distributed store, and the per-rank configuration
of a decomposed run."""
import datetime
import os
import socket

import pytest
import torch.multiprocessing as mp

from plasmasim_b200 import PicConfig, rank_config


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _combine_worker(rank, port, q):
    import torch.distributed as dist

    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=2, timeout=datetime.timedelta(seconds=60))
    try:
        q.put((rank, bench.combine_over_ranks(10.0 + rank, 100 * (rank + 1), dist, device="cpu")))
    finally:
        dist.destroy_process_group()


def test_bench_combines_replicas_over_gloo():
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_combine_worker, args=(r, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = dict(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
    assert out[0] == out[1] == (11.0, 300.0)  # slowest rank's time, all ranks' pushes


def _uid_worker(rank, port, q):
    import torch.distributed as dist

    from plasmasim_b200.decomp import NcclTransport

    store = dist.TCPStore("127.0.0.1", port, 2, rank == 0, timeout=datetime.timedelta(seconds=60))
    q.put((rank, NcclTransport.share_unique_id(store, rank)))


def test_nccl_unique_id_travels_through_the_store():
    from plasmasim_b200 import build as pbuild

    if not os.path.isfile(pbuild.LIB):
        pytest.skip("library not built")
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_uid_worker, args=(r, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = dict(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
    assert len(out[0]) == 128 and out[0] == out[1] and any(out[0])


def test_rank_config_numbers_ranks_like_main():
    """rank = myrank_y PROCESS_Nx + myrank_x (:205-206); random-stream keys
    (rank) * 10000 + the single-rank keys (:442-443)."""
    cfg = PicConfig(nx=8, ny=8, nz=8, np=4)
    seen = set()
    for r in range(6):
        c = rank_config(cfg, 3, 2, r)
        assert (c.rank_x, c.rank_y) == (r % 3, r // 3)
        assert (c.procs_x, c.procs_y) == (3, 2)
        assert (c.seed_p, c.seed_v) == (10000 * r, 10000 * r + 50)
        seen.add((c.rank_x, c.rank_y))
    assert len(seen) == 6
