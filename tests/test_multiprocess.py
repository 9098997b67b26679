"""CPU, world size 2 over gloo: the multi-GPU bench path is replicas only (no
data-path collective), so what crosses ranks is the timing -- a barrier and
the max over ranks of the timed region -- and the reference arm runs on
rank 0 alone.  Two spawned ranks exercise exactly bench.py's helpers."""
import multiprocessing as mp
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
    sys.path.insert(0, ROOT)
    import bench

    ws, r, local, dist = bench._dist()
    t = bench._max_over_ranks(10.0 + 5.0 * rank, dist, local)
    bench._barrier(dist)
    args = type("Args", (), {"steps": 1, "warmup": 3, "config": "headline"})()
    ref = bench.bench_reference(args, ws, r, local, dist) if r != 0 else "rank 0 not run here"
    dist.destroy_process_group()
    q.put((r, ws, t, ref))


def test_replica_timing_helpers_on_two_gloo_ranks():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_worker, args=(r, port, q)) for r in (0, 1)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=180) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[0] for r in res] == [0, 1]
    assert all(r[1] == 2 for r in res)
    assert all(r[2] == 15.0 for r in res)  # both ranks see the slower rank's time
    assert res[1][3] is None  # the reference arm does no work off rank 0
