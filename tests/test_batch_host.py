"""Host-side logic of the batched workload: the seeded instance generator,
the rank partition and the cross-rank reduction of the disorder average
(world_size 2 over gloo on CPU; the per-rank partial sums come from the
FP64 oracle, standing in for each rank's GPU batch)."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from helix_b200 import systems as S


def test_disorder_instances_are_seeded_and_in_range():
    a = S.disorder_instance(123)
    b = S.disorder_instance(123)
    np.testing.assert_array_equal(a.h_diag, b.h_diag)
    np.testing.assert_array_equal(a.meta["J"], b.meta["J"])
    assert (a.meta["h"], a.meta["lam"], a.meta["T"]) == (b.meta["h"], b.meta["lam"], b.meta["T"])
    shapes = set()
    for s in range(200):
        p = S.disorder_instance(s)
        n, L = p.n_spins, p.max_depth - 1
        assert 3 <= n <= 5 and 2 <= L <= 4
        assert 0.5 <= p.meta["h"] <= 1.5 and 0.05 <= p.meta["lam"] <= 0.2 and 0.5 <= p.meta["T"] <= 2.0
        assert len(p.baths) == n and p.modes == 3 * n
        shapes.add((n, L))
    assert len(shapes) == 9


def test_shard_instances_partitions_and_balances():
    problems = S.disorder_batch(512, seed=7)
    sizes = [S.state_bytes(p) for p in problems]
    for world in (1, 2, 3, 8):
        parts = S.shard_instances(sizes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(512))
        loads = [sum(sizes[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(sizes)
        assert parts == S.shard_instances(sizes, world)  # every rank computes the same partition


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, problems, steps, out):
    import torch
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    parts = S.shard_instances([S.state_bytes(p) for p in problems], world)
    partial = np.zeros(steps)
    for i in parts[rank]:
        o = O.Oracle(problems[i])
        r, _ = o.run(steps, trace=True)
        o.close()
        s = np.where(np.arange(problems[i].dim) & 1, 1.0, -1.0)
        partial += np.real(np.einsum("tii->ti", r)) @ s
    t = torch.tensor(np.concatenate([partial, [len(parts[rank])]]), dtype=torch.float64)
    dist.all_reduce(t)
    if rank == 0:
        out.put(t.numpy().copy())
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_disorder_average_equals_single_process():
    problems = [p for p in S.disorder_batch(10, seed=40) if p.hierarchy_size() <= 500][:5]
    steps = 5
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, problems, steps, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    total, count = res[:steps], res[steps]
    assert count == len(problems)
    from oracle import oracle as O
    ref = np.zeros(steps)
    for p in problems:
        o = O.Oracle(p)
        r, _ = o.run(steps, trace=True)
        o.close()
        s = np.where(np.arange(p.dim) & 1, 1.0, -1.0)
        ref += np.real(np.einsum("tii->ti", r)) @ s
    np.testing.assert_allclose(total, ref, rtol=0, atol=1e-12)
