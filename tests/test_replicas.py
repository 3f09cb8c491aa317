"""Multi-rank host logic of the replica runs (nuc3d_b200.replicas, used by
bench.py under torchrun): world size 2 over gloo on CPU.  Each rank owns an
independent box; the ranks meet only at barriers and at the max over ranks of
the timed region, and only rank 0 reports."""

import multiprocessing as mp
import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank, world, port):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT / "nuc3d-cartisian_b200" / "python"))
    sys.path.insert(0, str(ROOT))


def _worker(rank, world, port, q):
    _env(rank, world, port)
    from nuc3d_b200.replicas import Replicas, rank_info, whole_job_rate
    import bench
    info = rank_info()
    reps = Replicas(info, backend="gloo", timeout_s=60.0)
    reps.barrier()
    t_local = 1.0 + 0.5 * rank           # this rank's device-timed seconds
    t_max = reps.max(t_local)
    rate = whole_job_rate(1000.0, info.world, t_max)
    # the reference arm runs on rank 0 only; the other ranks exit without work
    ref_line = bench.run_reference(None, info.rank, info.world) if info.rank != 0 else "root"
    reps.barrier()
    reps.close()
    q.put((info.rank, info.world, t_max, rate, ref_line))


def _lonely(port, q):
    _env(0, 2, port)
    from nuc3d_b200.replicas import Replicas, rank_info
    try:
        Replicas(rank_info(), backend="gloo", timeout_s=3.0)
        q.put("joined")
    except Exception as e:  # the missing peer ends the wait with an error
        q.put(type(e).__name__)


def _run(target, args_list, timeout=120):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=target, args=a + (q,)) for a in args_list]
    for p in ps:
        p.start()
    out = [q.get(timeout=timeout) for _ in ps]
    for p in ps:
        p.join(timeout=30)
        assert p.exitcode == 0
    return out


def test_two_ranks_max_over_ranks_and_root_only_report():
    port = _free_port()
    out = sorted(_run(_worker, [(r, 2, port) for r in range(2)]))
    assert [o[0] for o in out] == [0, 1]
    for rank, world, t_max, rate, ref in out:
        assert world == 2
        assert t_max == 1.5                      # the slowest rank's time on every rank
        assert rate == pytest.approx(2 * 1000.0 / 1.5)
    assert out[1][4] is None                     # rank 1 does no reference work


def test_missing_peer_ends_with_an_error_not_a_hang():
    port = _free_port()
    (res,) = _run(_lonely, [(port,)], timeout=90)
    assert res != "joined"


def test_single_process_needs_no_group():
    sys.path.insert(0, str(ROOT / "nuc3d-cartisian_b200" / "python"))
    from nuc3d_b200.replicas import Replicas, rank_info, whole_job_rate
    info = rank_info(env={})
    assert (info.rank, info.world, info.local_rank) == (0, 1, 0) and info.is_root
    reps = Replicas(info)
    assert reps.dist is None and reps.max(2.5) == 2.5
    assert whole_job_rate(10.0, 1, 2.0) == 5.0
