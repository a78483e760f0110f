#!/usr/bin/env python
"""Benchmark of the multiply hot path (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--workload mul]

Workload "mul" (default): the standalone multiply at its headline size, one balanced
2^24 x 2^24-limb product per step (seeded splitmix64 operands, top bit set), the size at
which the 50%-of-HBM-roofline target is stated. `value` is the algorithmic GB/s of the
device-resident product (B_mul = 400 * (na + nb) bytes per product, operands already in
HBM); `e2e` is the same metric through the host C ABI call pg_mul (host buffers, copies in
the timed region). Every product moves ~2.5 GB through HBM, far above the 126 MB L2, so no
explicit flush is needed between steps.

--impl reference times the reference's own CPU product, pi::GmpMultiplier::multiply
(compiled unchanged from its sources into oracle/_ref/libpiref.so), on a bounded sample:
one 2^22 x 2^22-limb product per thread on every host core.

Multi-GPU (torchrun): the products are independent, so each rank runs its own replica
("replicas only", no collective on the data path); value = total work / max rank time.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
METRIC = "pi digits/s at 100M (batched vs per-call GPU, bit-exact); mul GB/s vs HBM"


def load_pkg():
    import importlib.util

    spec = importlib.util.spec_from_file_location("pi_compute_b200", os.path.join(ROOT, "pi-compute_b200", "__init__.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules["pi_compute_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    import importlib.util

    spec = importlib.util.spec_from_file_location("pi_oracle", os.path.join(ROOT, "oracle", "oracle.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules["pi_oracle"] = mod
    spec.loader.exec_module(mod)
    return mod


def measured_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def b_mul(na: int, nb: int) -> int:
    """Algorithmic bytes of one product (fixed formula: 16(na+nb) I/O + 3 transforms x 128(na+nb))."""
    return 400 * (na + nb)


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_gmp_sample(n: int = 1 << 22, threads: int = 0, seconds: float = 10.0) -> dict:
    """Reference CPU product throughput: GmpMultiplier::multiply on every core, bounded sample."""
    orc = load_oracle()
    pkg = sys.modules.get("pi_compute_b200") or load_pkg()
    threads = threads or (os.cpu_count() or 1)
    a = pkg.random_operand(n, 11)
    b = pkg.random_operand(n, 12)
    done = [0] * threads
    stop = time.perf_counter() + seconds
    use_ref = orc.ref_available()

    def work(i):
        while True:
            (orc.ref_mul if use_ref else orc.mul_gmp)(a, b)
            done[i] += 1
            if time.perf_counter() >= stop:
                break

    t0 = time.perf_counter()
    ts = [threading.Thread(target=work, args=(i,)) for i in range(threads)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    dt = time.perf_counter() - t0
    total = sum(done)
    return {"value": round(b_mul(n, n) * total / dt / 1e9, 4), "unit": "GB/s", "cores": threads,
            "kind": "reference" if use_ref else "port",
            "sample": f"{total} products of {n}x{n} limbs (pi::GmpMultiplier::multiply -> mpz_mul, "
                      f"one per thread, {threads} threads) in {dt:.1f} s"}


def run_reference(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return
    steps = []
    for _ in range(args.warmup):
        pass  # CPU runs need no warm-up; the sample below is timed as is
    for _ in range(max(1, args.steps)):
        steps.append(cpu_gmp_sample(seconds=max(3.0, 20.0 / max(1, args.steps))))
    v = statistics.median(s["value"] for s in steps)
    cb = dict(steps[0])
    cb["value"] = v
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "GB/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": "multiply, balanced 2^24 x 2^24 limbs (sampled at 2^22 x 2^22 on CPU)",
                       "parallelism": "host threads"},
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_b200(args):
    import torch

    world, rank, local = dist_setup()
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    pkg = load_pkg()
    eng = pkg.Engine(local)
    lib = eng.lib

    n = 1 << args.logn
    na = nb = n
    a_h = pkg.random_operand(na, 1234 + rank)
    b_h = pkg.random_operand(nb, 5678 + rank)
    a_d = torch.from_numpy(a_h.view(np.int64)).to(f"cuda:{local}")
    b_d = torch.from_numpy(b_h.view(np.int64)).to(f"cuda:{local}")
    out_d = torch.empty(na + nb, dtype=torch.int64, device=f"cuda:{local}")
    stream = torch.cuda.ExternalStream(lib.pg_stream(eng.ctx), device=f"cuda:{local}")

    def step():
        st = lib.pg_mul_device(eng.ctx, a_d.data_ptr(), na, b_d.data_ptr(), nb, out_d.data_ptr())
        if st != 0:
            raise pkg.PgError(st, eng.last_error())

    # correctness gate on this box: residues of the product modulo independent primes
    step()
    if lib.pg_sync(eng.ctx) != 0:
        raise pkg.PgError(-1, eng.last_error())
    r = out_d.cpu().numpy().view(np.uint64)
    A, B, R = pkg.limbs_to_int(a_h), pkg.limbs_to_int(b_h), pkg.limbs_to_int(r)
    for q in (2**61 - 1, 1000000007, 998244353):
        assert (A % q) * (B % q) % q == R % q, "product check failed"
    del A, B, R, r

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    l0 = lib.pg_launch_count(eng.ctx)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    ev[0].record(stream)
    for i in range(args.steps):
        step()
        ev[i + 1].record(stream)
    torch.cuda.synchronize()
    launches = lib.pg_launch_count(eng.ctx) - l0
    per = [ev[i].elapsed_time(ev[i + 1]) for i in range(args.steps)]
    total_ms = ev[0].elapsed_time(ev[-1])
    if lib.pg_sync(eng.ctx) != 0:
        raise pkg.PgError(-1, eng.last_error())
    clk = clocks.stop()

    # end-to-end through the host C ABI (pinned staging, H2D, product, D2H inside the timed region)
    out_h = np.zeros(na + nb, dtype=np.uint64)
    for _ in range(max(1, args.warmup // 2)):
        eng.mul_limbs(a_h, b_h)
    torch.cuda.synchronize()
    e2e_steps = max(2, min(args.steps, 5))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        out_h = eng.mul_limbs(a_h, b_h)
    e2e_s = (time.perf_counter() - t0) / e2e_steps

    t_ms = torch.tensor([total_ms], device=f"cuda:{local}")
    if world > 1:
        torch.distributed.all_reduce(t_ms, op=torch.distributed.ReduceOp.MAX)
    total_ms = float(t_ms.item())
    ms_per_step = total_ms / args.steps
    bal = b_mul(na, nb)
    value = bal * args.steps * world / (total_ms / 1e3) / 1e9
    peaks = measured_peaks()
    achieved = bal / (statistics.mean(per) / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        traffic = json.load(open(tpath)).get(f"mul_{args.logn}")

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32 mod p (NTT), u64 limbs", "data": "synthetic",
            "config": {"workload": f"multiply, balanced 2^{args.logn} x 2^{args.logn} limbs "
                                   f"(3-prime NTT, 32-bit coefficients, L = 2^{pkg_logL(na, nb)})",
                       "na": na, "nb": nb, "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (~2.5 GB of HBM traffic per product)"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": round(achieved / peaks["hbm_gbs"], 4), "traffic": traffic,
                         "peak_source": peaks["source"],
                         "what": "one whole product (all its kernels) against B_mul = 400*(na+nb) bytes"},
            "e2e": {"value": round(bal / e2e_s / 1e9, 3), "unit": "GB/s", "h2d_bytes_per_step": 8 * (na + nb),
                    "d2h_bytes_per_step": 8 * (na + nb), "ms_per_step": round(e2e_s * 1e3, 3),
                    "path": "pg_mul (host C ABI)"},
            "gpu_launches": int(launches),
            "clocks": clk,
        }
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_gmp_sample(seconds=args.cpu_seconds)
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def pkg_logL(na, nb):
    conv = 2 * (na + nb) - 1
    return max(6, (conv - 1).bit_length())


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="mul", choices=["mul"])
    ap.add_argument("--logn", type=int, default=24)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
