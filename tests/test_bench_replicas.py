"""The multi-GPU form of the benchmark is independent replicas: each rank works
alone and only the step time (max over ranks) and the bytes processed (sum)
are reduced. Checked here with two gloo ranks on the CPU."""
import multiprocessing as mp
import os
import socket


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, q) -> None:
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench

        step_ms = [3.5, 4.25][rank]        # replica step times
        text_bytes = [1 << 30, 1 << 30][rank]
        ms = bench.allreduce_max(step_ms, world)
        total = bench.allreduce_sum(float(text_bytes), world)
        bench.barrier(world)
        q.put((rank, ms, total, total / (ms * 1e-3) / 1e9))
    finally:
        dist.destroy_process_group()


def test_two_replicas_reduce_max_time_and_summed_bytes():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, total, gbps in out:
        assert ms == 4.25 and total == float(2 << 30)
        assert abs(gbps - (2 << 30) / 4.25e-3 / 1e9) < 1e-9
