"""Host side of the data-parallel mini-batch split, on CPU with two gloo ranks:
row ranges cover every mini-batch exactly once, the accumulator all-reduce sums
the ranks' shares, and the iteration report combines NaN status and error
means as one process would compute them, and the gradient engine's NaN status
is the same on every rank."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from phaser_b200.distributed import allreduce_sum, combine_report, combine_status, split_rows


def test_split_rows_partitions_every_batch():
    for B in (1, 2, 7, 64, 255, 256):
        for world in (1, 2, 3, 8):
            rows = [split_rows(B, world, r) for r in range(world)]
            assert rows[0][0] == 0 and rows[-1][1] == B
            assert all(a[1] == b[0] for a, b in zip(rows, rows[1:]))
            sizes = [b1 - b0 for b0, b1 in rows]
            assert max(sizes) - min(sizes) <= 1


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, q):
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        # accumulators: each rank contributes its rows' share
        f32 = torch.zeros(10)
        f64 = torch.zeros(4, dtype=torch.float64)
        b0, b1 = split_rows(10, world, rank)
        f32[b0:b1] = torch.arange(b0, b1, dtype=torch.float32) + 1
        f64 += rank + 1
        allreduce_sum((f32, f64))
        # report: rank 0 saw NaN in group 3, rank 1 none; error means over disjoint rows
        rep = torch.tensor([3.0 if rank == 0 else -1.0, 2.0, [1.0, 4.0][rank], [2.0, 6.0][rank]],
                           dtype=torch.float64)
        combine_report(rep)
        empty = torch.tensor([-1.0, 0.0, float('nan'), 0.0], dtype=torch.float64)
        combine_report(empty)
        # gradient-engine status: rank 1 saw group 5 go non-finite, rank 0 nothing -> 5 on both;
        # both fine -> -1
        st = torch.tensor([[-1, 5][rank]], dtype=torch.int32)
        combine_status(st)
        ok = torch.tensor([-1], dtype=torch.int32)
        combine_status(ok)
        q.put((rank, f32.tolist(), f64.tolist(), rep.tolist(), empty.tolist(), int(st[0]), int(ok[0])))
    finally:
        dist.destroy_process_group()


def test_allreduce_and_report_over_two_gloo_ranks():
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, f32, f64, rep, empty, st, ok in out:
        assert st == 5 and ok == -1
        assert f32 == [float(i + 1) for i in range(10)]
        assert f64 == [3.0] * 4
        assert rep[0] == 3.0 and rep[1] == 2.0
        assert rep[3] == 8.0 and rep[2] == pytest.approx((1.0 * 2 + 4.0 * 6) / 8)
        assert empty[0] == -1.0 and empty[3] == 0.0 and empty[2] != empty[2]
