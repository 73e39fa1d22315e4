"""bench.py's multi-GPU bookkeeping on CPU: replicas time themselves and the
job's time is the slowest rank's (gloo, two processes); the reference arm
does its work on rank 0 only."""
import importlib.util
import os
import socket

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        bench = _bench()
        t = bench.max_over_ranks(dist, 1.0 + rank, "cpu")
        out.put((rank, t))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_two_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    got = sorted(q.get(timeout=5) for _ in range(2))
    assert got == [(0, 2.0), (1, 2.0)]


def test_max_over_ranks_single_process_is_identity():
    assert _bench().max_over_ranks(None, 0.25, "cpu") == 0.25


def test_reference_arm_works_on_rank_zero_only(monkeypatch, capsys):
    bench = _bench()
    monkeypatch.setenv("RANK", "1")

    class Args:
        steps, warmup, gpus = 10, 3, 2
    assert bench.run_reference(Args()) == 0
    assert capsys.readouterr().out == ""
