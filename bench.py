#!/usr/bin/env python
"""Frequency solves per second on the 2160-element dynamic sweep.

One step = one frequency solve of the hot path: GHMATECD (complex Stokes
H/G assembly with the boundary-condition column swap and the right-hand
side) + LINSOLVE (LU with partial pivoting and solve), for the next
frequency of a 128-point sweep (omega log-uniform in [0.1, 10], seed 3) on
the 48x45 planar mesh with +-10% node jitter (seed 0): 2160 elements,
NPG = 4, n = 6480 complex unknowns.  The per-mesh static work (GHMATECE)
is done once before timing.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torchrun: one independent replica per GPU (the sweep is
sharded by frequency, no collective on the data path), timed on the device
with CUDA events, max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
import __graft_entry__  # noqa: E402

__graft_entry__.load_package()
from bem_mececcs_b200 import meshgen  # noqa: E402

METRIC = "freq-solves/sec @2160 elem: mixed+batched vs plain FP64 GPU at <=1e-8 rel err"
UNIT = "freq-solves/s"
WORKLOAD = ("2160-element planar mesh (48x45 quads over [-5,5]^2, +-10% interior node jitter, "
            "seed 0), NPG=4, mu=1, nu=0.25, rho=1, damping 0.01, unit traction patch r<1; "
            "128-frequency sweep omega log-uniform [0.1,10] (seed 3); n=6480 complex unknowns")


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


# ---------------------------------------------------------------------------
# Clock sampling during the timed region (nvidia-smi, 200 ms).
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, bus_id: str | None):
        self.proc = None
        self.path = None
        self.bus_id = bus_id

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                   "-lms", "200"]
            if self.bus_id:
                cmd += ["-i", self.bus_id]
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(cmd, stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as fh:
            for line in fh:
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    smax.append(float(f[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, f[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


# ---------------------------------------------------------------------------
# CPU baseline: the oracle's restatement of the reference CPU path.
# ---------------------------------------------------------------------------
def cpu_freq_solve_seconds(s, d, zh_sys, zfi_sys, fr, *, budget_s=8.0):
    """Time of one frequency solve on the host: GHMATECD (OpenMP over element
    columns, timed on a bounded sample of columns and scaled), ZGEMV and
    ZGESV (OpenBLAS, all threads) on the full system.  Returns
    (seconds, sample description, threads)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from scipy.linalg import lapack
    p = oracle.OracleProblem(s, d)
    p.ghmatece()
    nbe = s.nbe
    zh = np.zeros(p.nn * p.nn, dtype=np.complex128)
    zg = np.zeros(p.nn * p.nn, dtype=np.complex128)
    t0 = time.perf_counter()
    p.ghmatecd_cols(fr, 0, 32, zh, zg)
    t_probe = time.perf_counter() - t0
    cols = int(min(nbe - 32, max(32, budget_s / max(t_probe / 32, 1e-9))))
    t0 = time.perf_counter()
    p.ghmatecd_cols(fr, 32, 32 + cols, zh, zg)
    t_asm = (time.perf_counter() - t0) * nbe / cols
    del zh, zg
    a = np.array(zh_sys.reshape(p.nn, p.nn, order="F"), order="F", copy=True)
    b = zfi_sys.copy()
    t0 = time.perf_counter()
    _ = a @ b  # ZGEMV-sized matrix-vector product
    _, _, x, info = lapack.zgesv(a, b, overwrite_a=True, overwrite_b=True)
    t_lu = time.perf_counter() - t0
    if info != 0:
        raise RuntimeError(f"CPU ZGESV info={info}")
    try:
        from threadpoolctl import threadpool_info
        threads = max(i.get("num_threads", 1) for i in threadpool_info()) or os.cpu_count()
    except Exception:
        threads = os.cpu_count()
    sample = (f"GHMATECD on {cols} of {nbe} element columns (scaled x{nbe / cols:.1f}, "
              f"{t_asm:.2f} s est.), full ZGEMV+ZGESV n={p.nn} ({t_lu:.2f} s)")
    return t_asm + t_lu, sample, int(threads)


# ---------------------------------------------------------------------------
def run_ours(args):
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=torch.device(f"cuda:{local}"))
    from bem_mececcs_b200 import capi
    from bem_mececcs_b200.solver import BemSolver

    s, d = meshgen.config_mesh("c2_2160")
    freqs = meshgen.sweep_frequencies(128, seed=3)
    mine = freqs[rank::world]
    sol = BemSolver(s, device=local)
    sol.ghmatece(compute_gest=True)
    sol.set_bc(d.kode, d.bc.astype(np.complex128), d.dam, d.rho)
    ctx = sol.ctx
    stream = torch.cuda.Stream(device=local)
    ctx.set_stream(stream.cuda_stream)

    def step(i):
        sol.ghmatecd(float(mine[i % len(mine)]))
        ctx.check(ctx.L.bem_linsolve_async(ctx.h), "bem_linsolve_async")

    for i in range(args.warmup):
        step(i)
    ctx.sync()

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    props = torch.cuda.get_device_properties(local)
    bus = None
    try:
        bus = f"{props.pci_domain_id:08X}:{props.pci_bus_id:02X}:{props.pci_device_id:02X}.0"
    except Exception:
        pass
    sampler = ClockSampler(bus)

    # --- device-resident throughput (value) ---
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    ctx.prof_reset()
    ctx.prof(True)
    l0 = ctx.launches
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(args.steps):
        step(args.warmup + i)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = ctx.launches - l0
    prof = ctx.prof_read()
    ctx.prof(False)
    clocks = sampler.stop()
    ctx.sync()
    ms_max = max_over_ranks(ms)
    barrier()

    # --- end to end through the C-ABI with host buffers (e2e) ---
    nn = sol.nn
    zdfi_pin = torch.empty(nn * 16, dtype=torch.uint8, pin_memory=True).numpy().view(np.complex128)
    kode_pin = torch.empty(nn * 4, dtype=torch.uint8, pin_memory=True).numpy().view(np.int32)
    zfi_pin = torch.empty(nn * 16, dtype=torch.uint8, pin_memory=True).numpy().view(np.complex128)
    zdfi_pin[:] = d.bc
    kode_pin[:] = d.kode
    zge, zcs, zcp = sol.material
    zge2, zcs2, zcp2 = (capi.f64([z.real, z.imag]) for z in (zge, zcs, zcp))
    c = capi.f64(sol.c)
    L, h = ctx.L, ctx.h

    def e2e_step(i):
        ctx.check(L.bem_dyn_upload(h, capi.ptr(zdfi_pin), capi.ptr(kode_pin)), "bem_dyn_upload")
        ctx.check(L.bem_ghmatecd(h, capi.ptr(zge2), capi.ptr(zcs2), capi.ptr(zcp2), capi.ptr(c),
                                 float(mine[i % len(mine)]), capi.BEM_FAST_SINGULAR), "bem_ghmatecd")
        ctx.check(L.bem_linsolve(h, capi.ptr(zfi_pin)), "bem_linsolve")

    e2e_step(0)
    barrier()
    torch.cuda.synchronize()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for i in range(args.steps):
        e2e_step(i)
    f1.record(stream)
    f1.synchronize()
    e2e_ms = max_over_ranks(f0.elapsed_time(f1))
    if not np.all(np.isfinite(zfi_pin)):
        raise RuntimeError("non-finite solution")

    peak = ctx.fp64_peak_tflops()
    value = world * args.steps / (ms_max * 1e-3)
    e2e_value = world * args.steps / (e2e_ms * 1e-3)
    g = prof["gemm"]
    achieved = g["work"] / (g["ms"] * 1e-3) / 1e12 if g["ms"] > 0 else None
    line = {
        "metric": METRIC,
        "value": round(value, 3),
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_max / args.steps, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "form": "plain FP64 (complex128 assembly and LU)",
                   "n": nn, "parallelism": f"replicas x{world} (frequency-sharded)",
                   "l2": "inputs larger than L2: the 6480x6481 complex128 system is 672 MB"},
        "roofline": {"bound": "tensor", "kernel": "k_gemm_update (LU trailing update, FP64 DMMA)",
                     "achieved": round(achieved, 3) if achieved else None, "peak": round(peak, 3),
                     "unit": "TFLOP/s", "frac": round(achieved / peak, 4) if achieved else None,
                     "traffic": None,
                     "peak_source": "FP64 mma.sync m8n8k4 loop measured in this run "
                                    "(MEASURED_PEAKS.json has no FP64 figure)",
                     "kernel_share": {k: round(v["ms"] / ms, 4) for k, v in prof.items()}},
        "kernels": prof,
        "e2e": {"value": round(e2e_value, 3), "unit": UNIT,
                "h2d_bytes_per_step": int(nn * 16 + nn * 4), "d2h_bytes_per_step": int(nn * 16)},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sol.ghmatecd(float(mine[0]))
        zh_sys, zfi_sys = sol.get_system()
        secs, sample, threads = cpu_freq_solve_seconds(s, d, zh_sys, zfi_sys, float(mine[0]))
        line["cpu_baseline"] = {"value": round(1.0 / secs, 5), "unit": UNIT, "cores": threads,
                                "kind": "port", "sample": sample}
    ctx.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_reference(args):
    """The reference's CPU path (the oracle's restatement of GHMATECD + the
    OpenBLAS ZGESV it links) on the host cores, on our arm's workload."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    s, d = meshgen.config_mesh("c2_2160")
    freqs = meshgen.sweep_frequencies(128, seed=3)
    p = oracle.OracleProblem(s, d)
    p.ghmatece()
    steps = max(1, min(args.steps, 3))
    warm = min(args.warmup, 1)
    times, sample, threads = [], "", 1
    for i in range(warm + steps):
        fr = float(freqs[i % len(freqs)])
        zh, zfi, _, _ = p.system(fr) if i == 0 else (zh, zfi, None, None)
        secs, sample, threads = cpu_freq_solve_seconds(s, d, zh, zfi, fr)
        if i >= warm:
            times.append(secs)
    value = len(times) / sum(times)
    line = {"metric": METRIC, "value": round(value, 5), "unit": UNIT, "n_gpus": world,
            "steps": len(times), "warmup": warm, "ms_per_step": round(1e3 * sum(times) / len(times), 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "form": "reference CPU path (oracle restatement)",
                       "n": 3 * s.nbe, "parallelism": "host threads"},
            "cpu_baseline": {"value": round(value, 5), "unit": UNIT, "cores": threads,
                             "kind": "port", "sample": sample},
            "e2e": {"value": round(value, 5), "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    a = parse_args()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)
