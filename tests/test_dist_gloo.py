"""Multi-process (world size 2, gloo, CPU) tests of the benchmark's multi-GPU host logic.

The path has no exchange step: `bench.py --gpus N` runs N independent replicas (one pi
computation per rank) and reports all ranks' digits over the slowest rank's time. These tests
run that host logic on CPU ranks: each rank computes pi with GMP products through the engine
(no GPU), checks its digits, and the ranks agree on the maximum time.
"""
import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, q):
    import ctypes
    import importlib.util
    import time

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
        bench = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(bench)
        pkg = bench.load_pkg()
        lib = ctypes.CDLL(pkg.LIBPIB200)
        lib.pib_pi.argtypes = [ctypes.c_size_t, ctypes.c_int, ctypes.c_uint, ctypes.c_size_t, ctypes.c_int,
                               ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_double)]
        D = 1000 + 500 * rank                  # replicas may differ in size; timing is per rank
        buf = ctypes.create_string_buffer(D + 2)
        t0 = time.perf_counter()
        assert lib.pib_pi(D, 0, 1, 1, 0, buf, D + 2, None) == 0
        elapsed = time.perf_counter() - t0 + 0.25 * rank   # make the ranks' times differ
        digits = buf.raw[: D + 2].decode()
        ref = open(os.path.join(ROOT, "tests", "golden", "pi_1000.txt")).read()
        ok = digits.startswith(ref) if D >= 1000 else ref.startswith(digits)
        tmax = bench.dist_max(elapsed)
        q.put((rank, ok, elapsed, tmax, bench.replica_throughput(D, 1, world, tmax)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_agree_on_max_time():
    import socket

    with socket.socket() as sk:  # a free port on the loopback interface
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=5) for _ in range(2))
    assert all(r[1] for r in res), "a replica's digits differ from the golden file"
    tmax = max(r[2] for r in res)
    assert all(abs(r[3] - tmax) < 1e-9 for r in res)      # both ranks see the slowest rank's time
    assert abs(res[0][4] - 1000 * 2 / tmax) < 1e-6


def test_dist_max_is_identity_without_process_group():
    import importlib.util

    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    assert bench.dist_max(3.5) == 3.5
    assert bench.replica_throughput(100, 2, 4, 8.0) == 100.0
