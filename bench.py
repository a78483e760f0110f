#!/usr/bin/env python
"""Benchmark: pi digits/s at 100M digits on one B200, plus the multiply's HBM roofline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--digits D]

Step (workload "pi", the default): one complete computation of pi to D = 100,000,000 digits
through the engine's C entry point pib_pi in level-batched mode: device-resident binary
splitting of 7,051,375 terms, integer Newton reciprocal and sqrt(10005) with the final exact
correction, divide-and-conquer decimal conversion (large products on the B200), the digit
string in host memory. The digits of the first step are checked against the reference
program's sha256 (tests/golden/pi_golden.json). `value` = D / wall seconds per step (the
pipeline is host-orchestrated around device work, so the clock is the host clock with the
device synchronised on both sides); `e2e` = the same through the command-line program
(process start, CUDA context, output file), end to end like the reference's pi_compute.

`roofline` is measured live in the same run on the hot path's unit, one balanced
2^24 x 2^24-limb product (operands in HBM, CUDA events on the library's stream), against the
fixed algorithmic bytes B_mul = 400 * (na + nb) and the measured HBM copy bandwidth.

`cpu_baseline` = the reference's own program (oracle/_ref/pi_compute_ref, compiled unchanged
from its sources) on every host core, bounded sample: pi to 10M digits. `--impl reference`
runs that program at the full D digits once (about a minute on 16 cores) and reports digits/s.

Multi-GPU (torchrun): each rank computes pi independently (replicas only: the computation runs on
one GPU and the path has no exchange step); value = total digits / max rank time.
"""
from __future__ import annotations

import argparse
import ctypes
import hashlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
METRIC = "pi digits/s at 100M (batched vs per-call GPU, bit-exact); mul GB/s vs HBM"
PIB_MODE_PER_CALL = 1
PIB_MODE_BATCHED = 2
PI_COMPUTE_REF = os.path.join(ROOT, "oracle", "_ref", "pi_compute_ref")


def load_pkg():
    import importlib.util

    spec = importlib.util.spec_from_file_location("pi_compute_b200", os.path.join(ROOT, "pi-compute_b200", "__init__.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules["pi_compute_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    """oracle/oracle.py (the cpu_baseline leg times the reference's own GmpMultiplier through it)."""
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


def golden_sha(digits: int):
    g = json.load(open(os.path.join(ROOT, "tests", "golden", "pi_golden.json")))
    e = g.get(str(digits))
    return e["sha256"] if e else None


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
        sm, busy, smax, reasons = [], [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                v = float(f[1])
                sm.append(v)
                smax = float(f[2])
                if float(f[3]) > 250:  # under load
                    busy.append(v)
            except ValueError:
                continue
            for n, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        med = statistics.median(busy or sm) if sm else None
        return {"sm_mhz": med, "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm),
                "samples_under_load": len(busy)}


def dist_max(x: float, device=None) -> float:
    """Maximum of x over all ranks (identity without an initialised process group)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(units_per_rank: float, steps: int, world: int, max_seconds: float) -> float:
    """Whole-job throughput of independent replicas: all ranks' units over the slowest rank's time."""
    return units_per_rank * steps * world / max_seconds


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_reference_program(digits: int, threads: int) -> tuple[float, str]:
    """Wall seconds of the reference's pi_compute (unchanged sources) and the sha256 of its output."""
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "pi.txt")
        t0 = time.perf_counter()
        subprocess.run([PI_COMPUTE_REF, "--digits", str(digits), "--threads", str(threads), "--output", out],
                       check=True, stdout=subprocess.DEVNULL, cwd=td)
        dt = time.perf_counter() - t0
        sha = hashlib.sha256(open(out, "rb").read()).hexdigest()
    return dt, sha


def cpu_baseline(digits: int = 10_000_000) -> dict:
    threads = os.cpu_count() or 1
    if not os.path.exists(PI_COMPUTE_REF):
        return {"value": None, "unit": "digits/s", "cores": threads, "kind": "reference",
                "sample": "reference program not built"}
    dt, sha = run_reference_program(digits, threads)
    return {"value": round(digits / dt, 1), "unit": "digits/s", "cores": threads, "kind": "reference",
            "sample": f"reference pi_compute (GmpMultiplier, mpf finish) to {digits:,} digits with --threads "
                      f"{threads}: {dt:.2f} s; sha256 {sha[:16]}"}


def run_reference(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    dt, sha = run_reference_program(args.digits, threads)
    v = args.digits / dt
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 1), "unit": "digits/s", "n_gpus": args.gpus,
            "steps": 1, "warmup": 0, "ms_per_step": round(dt * 1e3, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64 limbs (GMP)", "data": "none (pi)",
            "config": {"workload": f"pi to {args.digits:,} digits (Chudnovsky, binary splitting + mpf finish)",
                       "parallelism": f"{threads} host threads"},
            "cpu_baseline": {"value": round(v, 1), "unit": "digits/s", "cores": threads, "kind": "reference",
                             "sample": f"one full {args.digits:,}-digit run of the reference program "
                                       f"({dt:.1f} s, sha256 {sha[:16]})"},
            "e2e": {"value": round(v, 1), "unit": "digits/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def product_roofline(pkg, eng, torch, local, logn=24, steps=5) -> dict:
    """Live roofline of the hot path's unit: balanced 2^logn x 2^logn product, operands in HBM."""
    lib = eng.lib
    n = 1 << logn
    a_h = pkg.random_operand(n, 1234)
    b_h = pkg.random_operand(n, 5678)
    a_d = torch.from_numpy(a_h.view(np.int64)).to(f"cuda:{local}")
    b_d = torch.from_numpy(b_h.view(np.int64)).to(f"cuda:{local}")
    out_d = torch.empty(2 * n, dtype=torch.int64, device=f"cuda:{local}")
    stream = torch.cuda.ExternalStream(lib.pg_stream(eng.ctx), device=f"cuda:{local}")

    def step():
        st = lib.pg_mul_device(eng.ctx, a_d.data_ptr(), n, b_d.data_ptr(), n, out_d.data_ptr())
        if st != 0:
            raise pkg.PgError(st, eng.last_error())

    step()
    if lib.pg_sync(eng.ctx) != 0:
        raise pkg.PgError(-1, eng.last_error())
    r = out_d.cpu().numpy().view(np.uint64)
    A, B, R = pkg.limbs_to_int(a_h), pkg.limbs_to_int(b_h), pkg.limbs_to_int(r)
    for q in (2**61 - 1, 1000000007, 998244353):
        assert (A % q) * (B % q) % q == R % q, "product check failed"
    for _ in range(3):
        step()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    torch.cuda.synchronize()
    l0 = lib.pg_launch_count(eng.ctx)
    ev[0].record(stream)
    for i in range(steps):
        step()
        ev[i + 1].record(stream)
    torch.cuda.synchronize()
    launches = lib.pg_launch_count(eng.ctx) - l0
    per = [ev[i].elapsed_time(ev[i + 1]) for i in range(steps)]
    bal = 400 * 2 * n
    achieved = bal / (statistics.mean(per) / 1e3) / 1e9
    peaks = measured_peaks()
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        traffic = json.load(open(tpath)).get(f"mul_{logn}")
    return {"bound": "hbm", "achieved": round(achieved, 2), "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": round(achieved / peaks["hbm_gbs"], 4), "traffic": traffic, "peak_source": peaks["source"],
            "what": f"one balanced 2^{logn} x 2^{logn}-limb product (all its kernels, {launches // steps} launches) "
                    f"against B_mul = 400*(na+nb) bytes; {statistics.mean(per):.3f} ms per product",
            "ms_per_product": round(statistics.mean(per), 4), "launches": int(launches)}


def run_b200(args):
    import torch

    world, rank, local = dist_setup()
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    pkg = load_pkg()
    lib = ctypes.CDLL(pkg.LIBPIB200)
    lib.pib_pi.argtypes = [ctypes.c_size_t, ctypes.c_int, ctypes.c_uint, ctypes.c_size_t, ctypes.c_int,
                           ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_double)]
    lib.pib_pi.restype = ctypes.c_int
    lib.pib_last_error.restype = ctypes.c_char_p
    D = args.digits
    threads = os.cpu_count() or 1
    # batched: the device pipeline (pg_pi); per-call: the reference's BinarySplitting and mpf finish
    # with every product of at least --threshold limbs sent to the B200 one call at a time
    mode = PIB_MODE_PER_CALL if args.mode == "per-call" else PIB_MODE_BATCHED
    # the digits land in page-locked host memory (allocated once, outside the timed region), so that
    # the 100 MB device-to-host copy of every step runs at the link's speed
    pinned = torch.empty(D + 2, dtype=torch.uint8, pin_memory=True)
    buf = ctypes.cast(ctypes.c_void_p(pinned.data_ptr()), ctypes.c_char_p)

    def digits_bytes() -> bytes:
        return ctypes.string_at(pinned.data_ptr(), D + 2)
    stats = (ctypes.c_double * 8)()

    def step():
        st = lib.pib_pi(D, mode, threads, args.threshold, local, buf, D + 2, stats)
        if st != 0:
            raise RuntimeError(lib.pib_last_error().decode())
        return list(stats)

    # correctness gate: the first computation must equal the reference's digits
    step()
    want = golden_sha(D)
    got = hashlib.sha256(digits_bytes()).hexdigest()
    if want is not None and got != want:
        raise RuntimeError(f"digits differ from the reference run: sha256 {got} != {want}")
    # the clock sampler (an nvidia-smi process) starts during the warm-up, so that its start-up
    # does not compete with the timed steps' host work; it keeps sampling through the timed region
    clocks = ClockSampler(local)
    clocks.start()
    for _ in range(max(0, args.warmup - 1)):
        step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    per, phases, launches = [], [], 0
    t_all = time.perf_counter()
    for _ in range(args.steps):
        t0 = time.perf_counter()
        s = step()
        torch.cuda.synchronize()
        per.append(time.perf_counter() - t0)
        phases.append(s[:4])
        launches += int(s[4])
    total = time.perf_counter() - t_all
    clk = clocks.stop()
    total = dist_max(total, device=f"cuda:{local}")
    value = replica_throughput(D, args.steps, world, total)

    eng = pkg.Engine(local)
    roof = product_roofline(pkg, eng, torch, local, logn=args.logn)
    eng.close()

    # The metric's other half: the same digits with the per-call drop-in (the reference's
    # BinarySplitting and mpf finish, every product of >= --threshold limbs sent to the B200 one
    # pi::Multiplier call at a time), once, after the timed batched steps; every rank runs it so the
    # ranks stay in step.
    per_call = None
    if mode == PIB_MODE_BATCHED and not args.no_per_call:
        t0 = time.perf_counter()
        st = lib.pib_pi(D, PIB_MODE_PER_CALL, threads, args.threshold, local, buf, D + 2, stats)
        dt = time.perf_counter() - t0
        if st != 0:
            raise RuntimeError(lib.pib_last_error().decode())
        pc = list(stats)
        pc_sha = hashlib.sha256(digits_bytes()).hexdigest()
        bs_batched = float(np.mean([p[0] for p in phases]))
        per_call = {"seconds": round(dt, 3), "value": round(D / dt, 1), "unit": "digits/s",
                    "threshold_limbs": args.threshold, "host_threads": threads,
                    "phases_s": {"binary_splitting": round(pc[0], 3), "final_formula": round(pc[1], 3),
                                 "decimal_conversion": round(pc[2], 3)},
                    "gpu_products": int(pc[5]), "gmp_products": int(pc[6]), "gpu_launches": int(pc[4]),
                    "digits_sha256": pc_sha, "matches_reference": (pc_sha == want) if want else None,
                    "batched_over_per_call": round(dt / (total / args.steps), 2),
                    "batched_over_per_call_bs": round(pc[0] / bs_batched, 2) if bs_batched > 0 else None,
                    "how": "pib_pi(PIB_MODE_PER_CALL): the reference's BinarySplitting and mpf finish over "
                           "pi::B200Multiplier, one run after the timed batched steps, host wall clock"}

    if rank == 0:
        # end to end through the command-line program, like the reference's pi_compute
        e2e = None
        if not args.no_e2e:
            # five fresh processes (CUDA start-up dominates and varies from run to run): the median
            runs, sha, parts = [], None, []
            env = {k: v for k, v in os.environ.items() if k != "PI_B200_TRACE"}  # the untraced path
            with tempfile.TemporaryDirectory() as td:
                out = os.path.join(td, "pi.txt")
                for _ in range(5):
                    w0 = time.time_ns()
                    t0 = time.perf_counter()
                    flags = ["--batched"] if mode == PIB_MODE_BATCHED else ["--gpu", "--gpu-threshold", str(args.threshold)]
                    cp = subprocess.run([pkg.PI_B200_BIN, *flags, "--digits", str(D), "--threads", str(threads),
                                         "--device", str(local), "--output", out, "--verbose"], check=True, env=env,
                                        stdout=subprocess.PIPE, text=True)
                    wall = time.perf_counter() - t0
                    w1 = time.time_ns()
                    runs.append(wall)
                    got_sha = hashlib.sha256(open(out, "rb").read()).hexdigest()
                    sha = got_sha if sha in (None, got_sha) else "differs between runs"
                    # "Process: main X ms, device context Y ms, compute Z ms, file W ms" (--verbose)
                    ms, clock = None, None
                    for line in cp.stdout.splitlines():
                        if line.strip().startswith("Process:"):
                            ms = [float(t.split()[-2]) for t in line.split(":", 1)[1].split(",")]
                        elif line.strip().startswith("Clock:"):
                            clock = [int(t.split()[-2]) for t in line.split(":", 1)[1].split(",")]
                    if ms and len(ms) == 4:
                        # start-up: launch to main (+ argument parsing); exit: the exit stamp to the return of
                        # subprocess.run (driver tear-down of the context); wall clocks of one host
                        start = (clock[0] - w0) / 1e9 + ms[0] / 1e3 if clock else None
                        end = (w1 - clock[1]) / 1e9 if clock else None
                        parts.append([wall - sum(ms) / 1e3 + ms[0] / 1e3] + [m / 1e3 for m in ms[1:]]
                                     + ([start, end] if clock else [float("nan"), float("nan")]))
            e2e_s = float(np.median(runs))
            breakdown = None
            if parts:
                med = np.median(np.array(parts), axis=0)
                breakdown = {"process_start_and_exit": round(float(med[0]), 3),
                             "of_which_start": round(float(med[4]), 3) if np.isfinite(med[4]) else None,
                             "of_which_exit": round(float(med[5]), 3) if np.isfinite(med[5]) else None,
                             "device_context_and_tables": round(float(med[1]), 3),
                             "compute": round(float(med[2]), 3), "file_write": round(float(med[3]), 3),
                             "how": "median over the runs of the CLI's own timing (--verbose); process start and "
                                    "exit = wall clock minus the timed parts"}
            e2e = {"value": round(D / e2e_s, 1), "unit": "digits/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": D + 2, "seconds": round(e2e_s, 3),
                   "runs_s": [round(x, 3) for x in runs],
                   "path": ("pi_b200 --batched" if mode == PIB_MODE_BATCHED else "pi_b200 --gpu")
                           + " (process start, CUDA context, output file)",
                   "sha256_matches_reference": (sha == want) if want else None, "breakdown_s": breakdown}
        ph = np.mean(np.array(phases), axis=0)
        line = {
            "metric": METRIC, "value": round(value, 1), "unit": "digits/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1e3 * total / args.steps, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32 mod p (NTT), u64 limbs", "data": "none (pi)",
            "config": {"workload": (f"pi to {D:,} digits: level-batched device binary splitting + Newton final "
                                    f"formula + scaled-remainder-tree digit conversion on B200 products")
                       if mode == PIB_MODE_BATCHED else
                                   (f"pi to {D:,} digits: the reference's splitting and mpf finish, every product of "
                                    f">= {args.threshold} limbs on the B200 one call at a time (per-call drop-in)"),
                       "mode": args.mode,
                       "digits": D, "terms": None, "parallelism": f"replicas x{world}",
                       "l2": "every product of the top tree levels moves GBs through HBM (far above the 126 MB L2)",
                       "phases_s": {"binary_splitting": round(ph[0], 3), "final_formula": round(ph[1], 3),
                                    "decimal_conversion": round(ph[2], 3)},
                       "step_s": [round(x, 4) for x in per],
                       "step_phases_s": [[round(v, 4) for v in s3[:3]] for s3 in phases],
                       "digits_sha256": got, "matches_reference": (got == want) if want else None},
            "roofline": roof,
            "per_call": per_call,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk,
        }
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline()
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def run_mul(args):
    """Workload "mul": only the product's live roofline (for profiling the hot path's unit)."""
    import torch

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    pkg = load_pkg()
    eng = pkg.Engine(local)
    roof = product_roofline(pkg, eng, torch, local, logn=args.logn, steps=max(1, args.steps))
    eng.close()
    if rank == 0:
        n = 1 << args.logn
        ms = roof["ms_per_product"]
        print(json.dumps({"metric": "mul GB/s vs HBM (B_mul = 400*(na+nb))", "value": roof["achieved"],
                          "unit": "GB/s", "n_gpus": 1, "steps": args.steps, "warmup": 3, "ms_per_step": ms,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                          "dtype": "u32 mod p (NTT), u64 limbs", "data": "synthetic",
                          "config": {"workload": f"multiply, balanced 2^{args.logn} x 2^{args.logn} limbs", "na": n,
                                     "nb": n}, "roofline": roof, "gpu_launches": roof["launches"]}), flush=True)


def run_sweep(args):
    """Workload "sweep": the standalone multiply sweep. Seeded operands (splitmix64, a seed per size
    and shape) of n = 2^j and 3*2^(j-1) limbs, j = 10..24; balanced a*b, 1:4, 1:16 and squares;
    every product's first run checked (word for word against mpz_mul's sha256 where tests/golden
    holds the case, 2^24 included; modulo three primes otherwise), then `--trials` timed runs
    (CUDA events on the context's stream, operands in HBM). Reports median ms, GB/s of
    B_mul = 400 (na + nb) / B_sqr = 536 n and the fraction of measured HBM bandwidth; GMP's mpz_mul
    (the reference's GmpMultiplier, one core) beside it up to 2^20 limbs."""
    import torch

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    pkg = load_pkg()
    eng = pkg.Engine(local)
    lib = eng.lib
    dev = f"cuda:{local}"
    stream = torch.cuda.ExternalStream(lib.pg_stream(eng.ctx), device=dev)
    peaks = measured_peaks()
    sizes = []
    for j in range(10, 25):
        sizes.append(1 << j)
        if j < 24:
            sizes.append(3 << (j - 1))
    rows = []
    # products with a committed mpz_mul hash (tests/golden) use that case's seeds and are compared
    # word for word; the others are checked modulo three primes
    golden = {}
    for fn in ("products.json", "products_top.json"):
        for c in json.load(open(os.path.join(ROOT, "tests", "golden", fn))):
            golden[(c["na"], c["nb"])] = c
    launches0 = lib.pg_launch_count(eng.ctx)
    for n in sizes:
        for shape, nb in (("balanced", n), ("1:4", n // 4), ("1:16", n // 16), ("square", 0)):
            g = golden.get((n, nb))
            seed = g["seed"] if g else n * 8 + len(rows) % 4
            a_h = pkg.random_operand(n, seed)
            b_h = pkg.random_operand(nb, seed + 7) if nb else a_h
            a_d = torch.from_numpy(a_h.view(np.int64)).to(dev)
            b_d = torch.from_numpy(b_h.view(np.int64)).to(dev) if nb else a_d
            m = n + (nb if nb else n)
            out_d = torch.empty(m, dtype=torch.int64, device=dev)

            def step():
                if nb:
                    st = lib.pg_mul_device(eng.ctx, a_d.data_ptr(), n, b_d.data_ptr(), nb, out_d.data_ptr())
                else:
                    st = lib.pg_sqr_device(eng.ctx, a_d.data_ptr(), n, out_d.data_ptr())
                if st != 0:
                    raise pkg.PgError(st, eng.last_error())

            step()
            if lib.pg_sync(eng.ctx) != 0:
                raise pkg.PgError(-1, eng.last_error())
            r_h = out_d.cpu().numpy().view(np.uint64)
            if g:
                r_t = r_h[: int(np.max(np.nonzero(r_h)[0])) + 1] if r_h.any() else r_h[:0]
                ok = len(r_t) == g["len"] and hashlib.sha256(r_t.astype("<u8").tobytes()).hexdigest() == g["sha256"]
                checked = "sha256 = mpz_mul's (tests/golden)"
            else:
                A, B, R = pkg.limbs_to_int(a_h), pkg.limbs_to_int(b_h), pkg.limbs_to_int(r_h)
                ok = all((A % q) * (B % q) % q == R % q for q in (2**61 - 1, 1000000007, 998244353))
                checked = "mod 2^61-1, 1e9+7, 998244353"
            if not ok:
                raise RuntimeError(f"product check failed at n={n} shape={shape}")
            step()
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.trials + 1)]
            torch.cuda.synchronize()
            ev[0].record(stream)
            for i in range(args.trials):
                step()
                ev[i + 1].record(stream)
            torch.cuda.synchronize()
            ms = statistics.median(ev[i].elapsed_time(ev[i + 1]) for i in range(args.trials))
            balg = 400 * (n + nb) if nb else 536 * n
            gbs = balg / (ms / 1e3) / 1e9
            rows.append({"na": n, "nb": nb if nb else n, "shape": shape, "ms": round(ms, 4), "gbs": round(gbs, 1),
                         "frac": round(gbs / peaks["hbm_gbs"], 4), "checked": checked})
            del a_d, b_d, out_d
    launches = lib.pg_launch_count(eng.ctx) - launches0
    eng.close()
    # GMP mpz_mul on one host core, the reference's GmpMultiplier::multiply (oracle/_ref)
    cpu = []
    oracle = None
    try:
        oracle = load_oracle()
    except Exception:
        pass
    if oracle is not None and oracle.ref_available():
        for n in (1 << 10, 1 << 14, 1 << 18, 1 << 20):
            a_h, b_h = pkg.random_operand(n, 7), pkg.random_operand(n, 8)
            reps = max(1, (1 << 20) // n)
            t0 = time.perf_counter()
            for _ in range(reps):
                oracle.ref_mul(a_h, b_h)
            cpu.append({"na": n, "nb": n, "ms": round((time.perf_counter() - t0) * 1e3 / reps, 3)})
    if rank == 0:
        head = next(r for r in rows if r["na"] == 1 << 24 and r["shape"] == "balanced")
        print(json.dumps({"metric": "mul GB/s vs HBM (B_mul = 400*(na+nb))", "value": head["gbs"], "unit": "GB/s",
                          "n_gpus": 1, "steps": args.trials, "warmup": 1, "ms_per_step": head["ms"],
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                          "dtype": "u32 mod p (NTT), u64 limbs", "data": "synthetic (splitmix64)",
                          "config": {"workload": "multiply sweep: 2^10..2^24 limbs and 3*2^(j-1), balanced, 1:4, "
                                                 "1:16, square", "trials": args.trials,
                                     "l2": "timed back to back; operands above 2^21 limbs exceed the 126 MB L2"},
                          "sweep": rows, "gpu_launches": int(launches),
                          "cpu_baseline": {"kind": "reference", "cores": 1,
                                           "sample": "GmpMultiplier::multiply (mpz_mul) on balanced operands",
                                           "rows": cpu}}), flush=True)


def run_batch_workload(args):
    """Workload "batch": a synthetic batch of products with sizes drawn log-uniform in
    [2^6, 2^18] limbs from one seed, run as one pg_mul_batch call and, for comparison, as the
    same products issued one pg_mul_device call at a time (the per-call drop-in's pattern).
    Metric: sum of B_mul = 400*(na+nb) bytes over the batch / batch time."""
    import torch

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    pkg = load_pkg()
    eng = pkg.Engine(local)
    lib = eng.lib
    dev = f"cuda:{local}"
    rng = np.random.default_rng(3)
    nj = args.batch_jobs
    na = np.maximum(1, (2.0 ** rng.uniform(6, 18, nj)).astype(np.int64))
    nb = np.maximum(1, (2.0 ** rng.uniform(6, 18, nj)).astype(np.int64))
    pad = lambda x: (x + 1) // 2 * 2  # keep every operand 16-byte aligned
    oa = np.concatenate([[0], np.cumsum(pad(na))])
    ob = np.concatenate([[0], np.cumsum(pad(nb))])
    oo = np.concatenate([[0], np.cumsum(pad(na + nb))])
    g = torch.Generator(device=dev).manual_seed(5)
    A = torch.randint(-2**63, 2**63 - 1, (int(oa[-1]),), dtype=torch.int64, device=dev, generator=g)
    B = torch.randint(-2**63, 2**63 - 1, (int(ob[-1]),), dtype=torch.int64, device=dev, generator=g)
    O1 = torch.zeros(int(oo[-1]), dtype=torch.int64, device=dev)
    O2 = torch.zeros_like(O1)
    a0, b0, o1, o2 = A.data_ptr(), B.data_ptr(), O1.data_ptr(), O2.data_ptr()
    jobs = (pkg.PgJob * nj)()
    for i in range(nj):
        jobs[i] = pkg.PgJob(a0 + 8 * int(oa[i]), int(na[i]), b0 + 8 * int(ob[i]), int(nb[i]), None, 0, None, 0, 0,
                            o1 + 8 * int(oo[i]), int(na[i] + nb[i]))
    stream = torch.cuda.ExternalStream(lib.pg_stream(eng.ctx), device=dev)

    def batch():
        st = lib.pg_mul_batch(eng.ctx, jobs, nj)
        if st != 0:
            raise pkg.PgError(st, eng.last_error())

    def per_call():
        for i in range(nj):
            st = lib.pg_mul_device(eng.ctx, a0 + 8 * int(oa[i]), int(na[i]), b0 + 8 * int(ob[i]), int(nb[i]),
                                   o2 + 8 * int(oo[i]))
            if st != 0:
                raise pkg.PgError(st, eng.last_error())
        if lib.pg_sync(eng.ctx) != 0:
            raise pkg.PgError(-1, eng.last_error())

    def timed(fn, steps):
        for _ in range(max(3, args.warmup)):
            fn()
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
        l0 = lib.pg_launch_count(eng.ctx)
        ev[0].record(stream)
        for i in range(steps):
            fn()
            ev[i + 1].record(stream)
        torch.cuda.synchronize()
        return statistics.median([ev[i].elapsed_time(ev[i + 1]) for i in range(steps)]), \
            (lib.pg_launch_count(eng.ctx) - l0) // steps

    ms_b, launches_b = timed(batch, args.steps)
    ms_p, launches_p = timed(per_call, args.steps)
    same = bool(torch.equal(O1, O2))
    eng.close()
    bytes_alg = 400.0 * float(np.sum(na + nb))
    gbs = bytes_alg / (ms_b / 1e3) / 1e9
    peaks = measured_peaks()
    if rank == 0:
        print(json.dumps({
            "metric": "batched products: sum B_mul / batch time", "value": round(gbs, 2), "unit": "GB/s",
            "n_gpus": 1, "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": round(ms_b, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32 mod p (NTT), u64 limbs",
            "data": "synthetic",
            "config": {"workload": f"{nj} products, na and nb log-uniform in [2^6, 2^18] limbs (seed 3)",
                       "sum_limbs": int(np.sum(na + nb))},
            "per_call": {"ms": round(ms_p, 4), "launches": int(launches_p),
                         "value": round(bytes_alg / (ms_p / 1e3) / 1e9, 2)},
            "speedup_vs_per_call": round(ms_p / ms_b, 3), "results_identical": same,
            "roofline": {"bound": "hbm", "achieved": round(gbs, 2), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": round(gbs / peaks["hbm_gbs"], 4), "traffic": None, "peak_source": peaks["source"]},
            "gpu_launches": int(launches_b)}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--digits", type=int, default=100_000_000)
    ap.add_argument("--threshold", type=int, default=1024)
    ap.add_argument("--logn", type=int, default=24)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-per-call", action="store_true",
                    help="pi workload: skip the one per-call drop-in run after the timed batched steps")
    ap.add_argument("--workload", default="pi", choices=["pi", "mul", "batch", "sweep"])
    ap.add_argument("--mode", default="batched", choices=["batched", "per-call"],
                    help="pi workload: device pipeline (default) or the per-call drop-in multiplier")
    ap.add_argument("--trials", type=int, default=5, help="timed runs per size and shape (sweep)")
    ap.add_argument("--batch-jobs", type=int, default=4096)
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "mul":
        run_mul(args)
    elif args.workload == "batch":
        run_batch_workload(args)
    elif args.workload == "sweep":
        run_sweep(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
