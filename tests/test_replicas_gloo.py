"""Multi-process path on CPU: world_size-2 gloo ranks split independent
proofs (replicas, no data-path collective) and reduce only the timing
(max over ranks) and the proof count (sum).  Each rank proves its share with
the oracle here; on GPUs bench.py does the same with liblgpu."""
import os
import pathlib
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "oracle"))
    import hashlib

    import lgref
    import importlib.util

    spec = importlib.util.spec_from_file_location("lg_replicas", ROOT / "ligerito-rust_b200" / "replicas.py")
    rep = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(rep)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seeds = list(range(5))
        mine = rep.shard(seeds, rank, world)
        cfg = lgref.config(1, 8, 4, [6], [2])
        digests = {s: hashlib.sha256(lgref.prove(cfg, lgref.splitmix(s, 1 << 12))).hexdigest() for s in mine}
        t_max = rep.reduce_max(float(rank + 1))
        n_tot = rep.reduce_sum(float(len(mine)))
        out_q.put((rank, mine, digests, t_max, n_tot))
    finally:
        dist.destroy_process_group()


def test_replica_shards_cover_every_proof_once():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert res[0][1] == [0, 2, 4] and res[1][1] == [1, 3]
    assert all(r[3] == 2.0 and r[4] == 5.0 for r in res)
    # the same proof regardless of which rank made it
    sys.path.insert(0, str(ROOT / "oracle"))
    import hashlib

    import lgref

    cfg = lgref.config(1, 8, 4, [6], [2])
    for r in res:
        for s, d in r[2].items():
            assert d == hashlib.sha256(lgref.prove(cfg, lgref.splitmix(s, 1 << 12))).hexdigest()


def test_shard_validation():
    import importlib.util

    spec = importlib.util.spec_from_file_location("lg_replicas", ROOT / "ligerito-rust_b200" / "replicas.py")
    rep = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(rep)
    assert rep.shard([], 0, 1) == []
    assert sorted(rep.shard(range(7), 0, 3) + rep.shard(range(7), 1, 3) + rep.shard(range(7), 2, 3)) == list(range(7))
    with pytest.raises(ValueError):
        rep.shard([1], 2, 2)
