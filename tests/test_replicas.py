"""Replica parallelism on CPU: world_size-2 gloo ranks share a frequency x polarisation sweep."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from giem2g_b200.replicas import instances, shard, shard_instances


def test_shard_partitions_instances():
    for n in range(0, 20):
        for w in range(1, 6):
            got = sorted(i for r in range(w) for i in shard(n, r, w))
            assert got == list(range(n))
    with pytest.raises(ValueError):
        shard(4, 2, 2)


def test_instances_order():
    assert instances([0.1, 1.0], [1, 0]) == [(0, 1), (0, 0), (1, 1), (1, 0)]


def test_polarisations_of_a_frequency_stay_on_one_rank():
    """Sharding is by frequency: EY and EX of one frequency (one tensor build, shared tensor reads in the
    batched solver) land on the same rank for every world size, and every instance on exactly one rank."""
    for nf in range(0, 9):
        freqs = [10.0 ** (k - 3) for k in range(nf)]
        for w in range(1, 6):
            owner = {}
            for r in range(w):
                for key in shard_instances(freqs, [1, 0], r, w):
                    assert key not in owner
                    owner[key] = r
            assert sorted(owner) == sorted(instances(freqs, [1, 0]))
            for fi in range(nf):
                assert owner[(fi, 1)] == owner[(fi, 0)] == fi % w


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    from giem2g_b200.replicas import max_over_ranks, run_sweep
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        freqs = [0.01, 0.1, 1.0]
        res = run_sweep(lambda fi, p: {"rank": rank, "val": freqs[fi] * (p + 1)}, freqs, [1, 0], rank, world)
        t = max_over_ranks(1.0 + rank)
        q.put((rank, res, t))
    finally:
        dist.destroy_process_group()


def test_two_rank_sweep_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = {}
    for _ in range(2):
        r, res, t = q.get(timeout=120)
        out[r] = (res, t)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    res0, t0 = out[0]
    assert out[1][0] is None
    assert t0 == 2.0 and out[1][1] == 2.0
    assert sorted(res0) == sorted(instances([0, 1, 2], [1, 0]))
    for key in instances([0, 1, 2], [1, 0]):
        assert res0[key]["rank"] == key[0] % 2  # whole frequencies per rank
        assert abs(res0[key]["val"] - [0.01, 0.1, 1.0][key[0]] * (key[1] + 1)) < 1e-15
