"""bench.py's multi-process path on CPU: two gloo ranks (world size 2), as
`torchrun --nproc-per-node 2 bench.py` runs them one per GPU.  Every rank takes
part in the max-over-ranks reduction of its timed region and the whole-job rate
counts the work of every replica (weak scaling); the reference arm lets rank 0
alone run.  No GPU is used: the reduction helpers take the device as an argument
(CPU tensors with gloo here, CUDA tensors with NCCL in the bench)."""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, out):
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=ws)
    sys.path.insert(0, ROOT)
    import bench
    ms = 10.0 + 5.0 * rank                     # rank 1 is the slow one
    got = bench.max_over_ranks(ms, dist, device='cpu')
    rate = bench.job_rate(1000, 20, ws, got * 1e-3)
    out.put((rank, got, rate))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_timing_is_the_slowest_rank_and_rate_counts_every_replica():
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    ws, port = 2, _free_port()
    ps = [ctx.Process(target=_rank, args=(r, ws, port, q)) for r in range(ws)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=90) for _ in range(ws))
    for p in ps:
        p.join(60)
        assert p.exitcode == 0
    assert [r for r, _, _ in res] == [0, 1]
    assert all(got == 15.0 for _, got, _ in res)             # the max over ranks, on every rank
    assert all(rate == pytest.approx(1000 * 20 * 2 / 15e-3) for _, _, rate in res)


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, None) == 3.5
    assert bench.job_rate(10, 4, 1, 2.0) == 20.0


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    """Under torchrun only rank 0 times the CPU reference; the others exit with no work."""
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv('WORLD_SIZE', '2')
    monkeypatch.setenv('RANK', '1')
    assert bench.reference_arm(None) is None
    assert capsys.readouterr().out == ''
