#!/usr/bin/env python
"""Frequency solves per second on the 2160-element dynamic sweep.

A frequency solve is the hot path for one omega: GHMATECD (complex Stokes
H/G assembly with the boundary-condition column swap and the right-hand
side) + LINSOLVE (LU with partial pivoting and solve).  Frequencies come
from a 128-point sweep (omega log-uniform in [0.1, 10], seed 3) on the
48x45 boundary grid with +-10% node jitter (seed 0) closed by enclosing
elements: 2160 boundary elements, NPG = 4, n = 6480 complex unknowns.  The
per-mesh static work (GHMATECE) is done once before timing.

Headline (`value`): the mixed+batched form, one step = one lockstep batch of
`bem_sweep_batch_limit` frequency solves, 7 on this mesh (FP64 assembly,
FP32 LU on TF32 tensor cores, FP64 iterative refinement), checked against
the plain FP64 path at 1e-8.  The plain FP64 GPU path (one frequency at a
time) is measured in the same run.

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
WORKLOAD = ("2160 boundary elements (48x45 quads over [-5,5]^2 at z=0, +-10% interior node jitter, "
            "seed 0) closed by 2904 enclosing elements (bottom at z=-2.5, 4-layer walls), NPG=4, "
            "mu=1, nu=0.25, rho=1, damping 0.01, unit traction patch r<1; 128-frequency sweep "
            "omega log-uniform [0.1,10] (seed 3); n=6480 complex unknowns")


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40,
                    help="timed lockstep steps (40: about 2 s, so the clock sampler sees the timed region)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch", type=int, default=0,
                    help="frequencies per lockstep batch (0: the library's limit for this mesh, "
                         "bem_sweep_batch_limit)")
    ap.add_argument("--refine", type=int, default=2,
                    help="FP64 refinement steps of the mixed form (2: max error 2.6e-13 against the plain FP64 "
                         "path over the 128 frequencies, the target being 1e-8)")
    ap.add_argument("--lanes", type=int, default=2,
                    help="contexts of the same mesh, each on its own stream, that take the headline's lockstep "
                         "batches in turn, so that one lane's latency-bound panels overlap the other's updates")
    ap.add_argument("--serve-count", type=int, default=2000,
                    help="requests of the serving stream replayed in the mixed form (0 skips the "
                         "stream; the 128-request served sweep always runs)")
    ap.add_argument("--serve-plain-count", type=int, default=120,
                    help="requests of the same stream (its first ones) replayed in the plain FP64 form, "
                         "whose service rate is far below the arrival rate")
    ap.add_argument("--no-precision", action="store_true",
                    help="skip the precision block (per-result errors against the FP64 oracle)")
    ap.add_argument("--no-serve", action="store_true", help="skip the served measurements")
    ap.add_argument("--small-count", type=int, default=512,
                    help="small meshes (24..600 elements) of the batching measurement (0 skips it)")
    ap.add_argument("--autotune", metavar="CACHE", default=None,
                    help="tune the headline sweep's switches and lockstep batch on this GPU, store the "
                         "result in the JSON file CACHE and print it (no bench line)")
    ap.add_argument("--profile-case", action="store_true",
                    help="run only warmup+steps headline sweep batches and print a launch count "
                         "(a small, short command to run under ncu); no bench line")
    ap.add_argument("--profile-plain", action="store_true",
                    help="run only warmup+steps plain FP64 solves (bem_ghmatecd + bem_linsolve) of the "
                         "headline mesh and print a launch count (for ncu); no bench line")
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def frequency_shard(freqs, rank, world):
    """This replica's frequencies: every world-th one from its rank on.  The
    shares are disjoint, cover the sweep and differ in length by at most one;
    no rank needs another's data."""
    return freqs[rank::world]


def max_over_ranks(x, world, device):
    """The slowest rank's time (ms): the job ends when its last replica does.
    One all-reduce, taken by every rank at the same point."""
    if world == 1:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def job_rate(world, units_per_rank, ms):
    """Whole-job throughput: the units all replicas processed over the slowest
    replica's time."""
    return world * units_per_rank / (ms * 1e-3)


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
_TIMING_LIB: list = []


def _timing_build(oracle):
    """The oracle compiled with the reference's CPU flags on this host, once
    per process: (library path or None, what was timed)."""
    if not _TIMING_LIB:
        path, why = oracle.timing_lib(tempfile.mkdtemp(prefix="bem_cpu_"))
        flags = " ".join(oracle.REFERENCE_CFLAGS)
        _TIMING_LIB.append((path, f"oracle port built with the reference's flags ({flags})" if path else
                            f"oracle port, parity build -O2 (the {flags} build failed: {why})"))
    return _TIMING_LIB[0]


def cpu_freq_solve_seconds(s, d, zh_sys, zfi_sys, fr, *, budget_s=8.0):
    """Time of one frequency solve on the host: GHMATECD (OpenMP over element
    columns, timed on a bounded sample of columns and scaled), ZGEMV and
    ZGESV (OpenBLAS, all threads) on the full system.  GHMATECD runs the
    oracle compiled the way the reference compiles its CPU path.  Returns
    (seconds, sample description, threads)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from scipy.linalg import lapack
    lib_path, built = _timing_build(oracle)
    p = oracle.OracleProblem(s, d, lib_path=lib_path)
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
              f"{t_asm:.2f} s est.; {built}), full ZGEMV+ZGESV n={p.nn} ({t_lu:.2f} s, OpenBLAS)")
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
    mine = frequency_shard(freqs, rank, world)
    sol = BemSolver(s, device=local)
    limit = sol.sweep_batch_limit("mixed")
    B, R = (min(args.batch, limit) if args.batch > 0 else limit), args.refine
    t0 = time.perf_counter()
    sol.ghmatece(compute_gest=True)  # returns once HESTdiag and GESTdiag are on the host
    static_ms = (time.perf_counter() - t0) * 1e3
    sol.set_bc(d.kode, d.bc.astype(np.complex128), d.dam, d.rho)
    ctx = sol.ctx
    stream = torch.cuda.Stream(device=local)
    ctx.set_stream(stream.cuda_stream)
    nn = sol.nn
    zge, zcs, zcp = sol.material
    zge2, zcs2, zcp2 = (capi.f64([z.real, z.imag]) for z in (zge, zcs, zcp))
    c = capi.f64(sol.c)
    L, h = ctx.L, ctx.h
    # lanes: more contexts of the same mesh on their own streams; step i runs on lane i % NL
    lanes = [(ctx, stream)]
    extra = []
    for _ in range(max(1, args.lanes) - 1):
        s2 = BemSolver(s, device=local)
        s2.ghmatece(compute_gest=True)
        s2.set_bc(d.kode, d.bc.astype(np.complex128), d.dam, d.rho)
        st2 = torch.cuda.Stream(device=local)
        s2.ctx.set_stream(st2.cuda_stream)
        extra.append(s2)
        lanes.append((s2.ctx, st2))
    NL = len(lanes)

    def batch_freqs(i):
        return capi.f64([mine[(i * B + j) % len(mine)] for j in range(B)])

    def sweep_step(i, x_out=None, lane=None):
        fr = batch_freqs(i)
        lc = lanes[i % NL if lane is None else lane][0]
        lc.check(L.bem_sweep(lc.h, capi.ptr(zge2), capi.ptr(zcs2), capi.ptr(zcp2), capi.ptr(c),
                             capi.ptr(fr), B, capi.BEM_FORM_MIXED, B, R, capi.ptr(x_out), None),
                 "bem_sweep")

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def timed(fn, steps, prof=False):
        barrier()
        torch.cuda.synchronize()
        if prof:
            ctx.prof_reset()
            ctx.prof(True)
        l0 = ctx.launches
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(steps):
            fn(i)
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        out = {"ms": ms, "launches": ctx.launches - l0}
        if prof:
            out["prof"] = ctx.prof_read()
            ctx.prof(False)
        ctx.sync()
        return out

    def timed_lanes(fn, steps):
        """timed() over every lane: all lanes start after one event on lane
        0's stream; the time is the latest lane's end."""
        barrier()
        torch.cuda.synchronize()
        l0 = sum(lc.launches for lc, _ in lanes)
        e0 = torch.cuda.Event(enable_timing=True)
        e0.record(lanes[0][1])
        for _, st in lanes[1:]:
            st.wait_event(e0)
        for i in range(steps):
            fn(i)
        ends = []
        for _, st in lanes:
            e1 = torch.cuda.Event(enable_timing=True)
            e1.record(st)
            ends.append(e1)
        torch.cuda.synchronize()
        ms = max(e0.elapsed_time(e1) for e1 in ends)
        for lc, _ in lanes:
            lc.sync()
        return {"ms": ms, "launches": sum(lc.launches for lc, _ in lanes) - l0}

    if args.autotune:
        from bem_mececcs_b200 import autotune
        best = autotune.tune_sweep(sol, mine, form="mixed", refine=R, steps=3, cache_path=args.autotune)
        print(json.dumps({"autotune": "2160-element sweep", "n": nn, **best}), flush=True)
        ctx.close()
        return

    if args.profile_case:
        for i in range(args.warmup + args.steps):
            sweep_step(i)
        ctx.sync()
        print(json.dumps({"profile_case": "mixed sweep", "batch": B, "batches": args.warmup + args.steps,
                          "launches": ctx.launches}), flush=True)
        ctx.close()
        return
    if args.profile_plain:
        for i in range(args.warmup + args.steps):
            sol.ghmatecd(mine[i % len(mine)])
            sol.linsolve()
        ctx.sync()
        print(json.dumps({"profile_case": "plain FP64 solve", "solves": args.warmup + args.steps,
                          "launches": ctx.launches}), flush=True)
        ctx.close()
        return

    # --- accuracy of the mixed form against the plain FP64 path, every
    #     frequency of this rank's share of the sweep (untimed) ---
    xm, corr = sol.sweep(mine, form="mixed", batch=B, refine=R)
    xp, _ = sol.sweep(mine, form="plain", batch=sol.sweep_batch_limit("plain"))
    errs = [float(np.linalg.norm(xm[i] - xp[i]) / np.linalg.norm(xp[i])) for i in range(len(mine))]
    max_err = max(errs)
    del xm, xp

    props = torch.cuda.get_device_properties(local)
    bus = None
    try:
        bus = f"{props.pci_domain_id:08X}:{props.pci_bus_id:02X}:{props.pci_device_id:02X}.0"
    except Exception:
        pass

    # --- headline: mixed + batched sweep, device-resident (value) ---
    for i in range(max(args.warmup, NL)):
        sweep_step(i)
    for lc, _ in lanes:
        lc.sync()
    sampler = ClockSampler(bus)
    sampler.start()
    time.sleep(0.3)
    t_mix = timed_lanes(lambda i: sweep_step(args.warmup + i), args.steps)
    clocks = sampler.stop()
    ms_mix = max_over_ranks(t_mix["ms"], world, f"cuda:{local}")
    # per-kernel-class times, launches and algorithmic bytes: a separate
    # profiled pass (CUDA events around every launch; no graph replay)
    # (lane 0 alone: the classes of one lane's step, without the other lane's overlap)
    t_prof = timed(lambda i: sweep_step(args.warmup + args.steps + i, lane=0), max(3, args.steps // 2), prof=True)

    # --- the plain FP64 GPU path, one frequency at a time (the comparison) ---
    def plain_step(i):
        sol.ghmatecd(float(mine[i % len(mine)]))
        ctx.check(L.bem_linsolve_async(h), "bem_linsolve_async")

    kp = max(3, args.steps // 2)
    for i in range(2):
        plain_step(i)
    ctx.sync()
    t_plain = timed(plain_step, kp, prof=True)
    ms_plain = max_over_ranks(t_plain["ms"], world, f"cuda:{local}")

    # --- end to end through the C-ABI with host buffers (e2e) ---
    # every step uploads its boundary conditions from pinned host memory and
    # reads its solutions back into pinned host memory; each lane's host
    # thread keeps two steps in flight (bem_sweep_async into one of two
    # output buffers, then it waits for the previous step's solutions)
    import threading
    pins = []
    for _ in lanes:
        zp = torch.empty(nn * 16, dtype=torch.uint8, pin_memory=True).numpy().view(np.complex128)
        kp_ = torch.empty(nn * 4, dtype=torch.uint8, pin_memory=True).numpy().view(np.int32)
        xps = [torch.empty(B * nn * 16, dtype=torch.uint8, pin_memory=True).numpy().view(np.complex128)
               for _ in range(2)]
        zp[:] = d.bc
        kp_[:] = d.kode
        pins.append((zp, kp_, xps))

    def e2e_step(i, lane):
        """Enqueues step i on the lane; returns an event after its read-back."""
        lc, st = lanes[lane]
        zp, kp_, xps = pins[lane]
        lc.check(L.bem_dyn_upload(lc.h, capi.ptr(zp), capi.ptr(kp_)), "bem_dyn_upload")
        fr = batch_freqs(i)
        lc.check(L.bem_sweep_async(lc.h, capi.ptr(zge2), capi.ptr(zcs2), capi.ptr(zcp2), capi.ptr(c),
                                   capi.ptr(fr), B, capi.BEM_FORM_MIXED, B, R, capi.ptr(xps[(i // NL) % 2])),
                 "bem_sweep_async")
        ev = torch.cuda.Event()
        ev.record(st)
        return ev

    for li in range(NL):
        e2e_step(li, li).synchronize()
        lanes[li][0].sync()
    errors = []

    def e2e_lane(li):
        try:
            prev = None
            for i in range(li, args.steps, NL):
                ev = e2e_step(i, li)
                if prev is not None:
                    prev.synchronize()  # the previous step's solutions are on the host
                prev = ev
            if prev is not None:
                prev.synchronize()
            lanes[li][0].sync()  # the status of the lane's calls
        except Exception as e:  # reported after the join
            errors.append(e)

    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ths = [threading.Thread(target=e2e_lane, args=(li,)) for li in range(NL)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3, world, f"cuda:{local}")
    if errors:
        raise errors[0]
    if not all(np.all(np.isfinite(x)) for p in pins for x in p[2]):
        raise RuntimeError("non-finite solution")

    # --- the plain FP64 form batched as the mixed one is (bem_sweep PLAIN) ---
    Bp = sol.sweep_batch_limit("plain")

    def plain_sweep_step(i):
        fr = capi.f64([mine[(i * Bp + j) % len(mine)] for j in range(Bp)])
        ctx.check(L.bem_sweep(h, capi.ptr(zge2), capi.ptr(zcs2), capi.ptr(zcp2), capi.ptr(c),
                              capi.ptr(fr), Bp, capi.BEM_FORM_PLAIN, Bp, 0, None, None), "bem_sweep")

    plain_sweep_step(0)
    ctx.sync()
    kpb = max(2, args.steps // 4)
    t_plain_b = timed(lambda i: plain_sweep_step(1 + i), kpb)
    ms_plain_b = max_over_ranks(t_plain_b["ms"], world, f"cuda:{local}")

    mpeaks = ctx.peaks()
    value = job_rate(world, args.steps * B, ms_mix)
    value_plain = job_rate(world, kp, ms_plain)
    value_plain_b = job_rate(world, kpb * Bp, ms_plain_b)
    e2e_value = job_rate(world, args.steps * B, e2e_ms)
    pm = t_prof["prof"]
    pp = t_plain["prof"]
    shares = {k: round(v["ms"] / t_prof["ms"], 4) for k, v in pm.items()}
    # Roofline of the headline form's dominant class among those bound by HBM
    # or the tensor cores.  The panel (latency: barriers per column) and the
    # assembly (the FP64 pipe) have no HBM or tensor roof to be measured
    # against; `dominant_by_time` names the largest class of all.
    peaks = _peaks()
    top_all = max(pm, key=lambda k: pm[k]["ms"])
    roofed = [k for k in pm if k not in ("panel", "assembly") and pm[k]["ms"] > 0] or [top_all]
    top = max(roofed, key=lambda k: pm[k]["ms"])
    roof = _roofline(top, pm[top], peaks, mpeaks)
    roof["dominant_by_time"] = {"class": top_all, "share": round(pm[top_all]["ms"] / t_prof["ms"], 4),
                                "this_class_share": round(pm[top]["ms"] / t_prof["ms"], 4),
                                "note": NOTES.get(top_all, "")}
    roof_all = {k: _roofline(k, v, peaks, mpeaks) for k, v in pm.items() if v["ms"] > 0}
    g64 = pp["gemm"]
    plain_gemm = g64["work"] / (g64["ms"] * 1e-3) / 1e12 if g64["ms"] > 0 else None
    line = {
        "metric": METRIC,
        "value": round(value, 3),
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_mix / args.steps, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64 assembly + f32/tf32 LU + f64 refinement",
        "data": "synthetic",
        "config": {"workload": WORKLOAD,
                   "form": f"mixed+batched: {B} frequencies per step in lockstep on {NL} lanes (contexts of the "
                           f"mesh on their own streams, taking the steps in turn), FP64 assembly, "
                           f"FP32 LU with TF32 tensor-core updates, {R} FP64 refinement steps",
                   "step": f"one batch of {B} frequency solves",
                   "n": nn, "parallelism": f"replicas x{world} (frequency-sharded)",
                   "l2": "inputs larger than L2: each 6480x6481 complex128 system is 672 MB"},
        "gpu_launches": int(t_mix["launches"]),
        "clocks": clocks,
        "e2e": {"value": round(e2e_value, 3), "unit": UNIT,
                "h2d_bytes_per_step": int(nn * 16 + nn * 4), "d2h_bytes_per_step": int(B * nn * 16),
                "how": f"bem_dyn_upload + bem_sweep_async per step from pinned host memory, {NL} lanes of one "
                       "host thread each, two steps in flight per lane (waits on the previous step's read-back)"},
        "roofline": roof,
        "rooflines_all": {k: {kk: v[kk] for kk in ("achieved", "frac", "ms") if kk in v} |
                          ({"tensor_frac": v["tensor"]["frac"]} if "tensor" in v else {}) |
                          ({"fp64_frac": v["fp64"]["frac"]} if "fp64" in v else {})
                          for k, v in roof_all.items()},
        "peaks_measured_tflops": mpeaks,
        "kernel_share": shares,
        "kernels": pm,
        "kernels_steps": max(3, args.steps // 2),
        "cuda_graphs": os.environ.get("BEM_GRAPHS", "1") != "0",
        "static_per_mesh": {"ghmatece_ms": round(static_ms, 3),
                            "kelvin_evals": s.nbe * (s.n - 1) * s.npg ** 2 + 4 * s.nbe * s.npg ** 2,
                            "note": "GHMATECE once per mesh (HESTdiag + GESTdiag on the device), host wall "
                                    "clock of the first call, set-up included; outside the timed sweep"},
        "accuracy": {"max_rel_err_vs_plain_fp64": max_err, "median_rel_err_vs_plain_fp64": float(np.median(errs)),
                     "frequencies_checked": len(errs), "refinement_steps": R, "tolerance": 1e-8,
                     "last_correction": float(max(corr))},
        "plain_fp64": {"value": round(value_plain, 3), "unit": UNIT,
                       "form": "one frequency at a time: bem_ghmatecd + bem_linsolve (the reference's order); "
                               "FP64 LU with panel pairs, trailing update by cuBLAS ZGEMM",
                       "ms_per_solve": round(ms_plain / kp, 3), "steps": kp,
                       "gemm_tflops": round(plain_gemm, 3) if plain_gemm else None,
                       "kernel_share": {k: round(v["ms"] / t_plain["ms"], 4) for k, v in pp.items()}},
        "plain_fp64_batched": {"value": round(value_plain_b, 3), "unit": UNIT,
                               "form": f"bem_sweep PLAIN, {Bp} frequencies per step in lockstep, FP64 LU "
                                       "(panel pairs, trailing update by strided-batched cuBLAS ZGEMM)",
                               "ms_per_step": round(ms_plain_b / kpb, 3), "steps": kpb},
        "speedup_vs_plain_fp64": round(value / value_plain, 3),
        "speedup_vs_plain_fp64_batched": round(value / value_plain_b, 3),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sol.ghmatecd(float(mine[0]))
        zh_sys, zfi_sys = sol.get_system()
        secs, sample, threads = cpu_freq_solve_seconds(s, d, zh_sys, zfi_sys, float(mine[0]))
        del zh_sys, zfi_sys
        line["cpu_baseline"] = {"value": round(1.0 / secs, 5), "unit": UNIT, "cores": threads,
                                "kind": "port", "sample": sample}
    ctx.close()
    for s2 in extra:
        s2.close()
    if rank == 0 and not args.no_precision:
        line["precision"] = run_precision(args, local)
    if not args.no_serve:
        line["served"] = run_served(args, s, d, mine, local)
    if args.small_count > 0:
        line["batched_small_meshes"] = run_small_batch(args, local)
    line["summary"] = _summary(line)
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def _summary(line):
    """The figures a reader needs first, compact and last on the line (a log
    that keeps only the end of the output still holds them)."""
    out = {"mixed_batched": line["value"], "e2e": line["e2e"]["value"],
           "plain_fp64": line["plain_fp64"]["value"],
           "plain_fp64_batched": line["plain_fp64_batched"]["value"],
           "speedup_vs_plain_fp64": line["speedup_vs_plain_fp64"],
           "speedup_vs_plain_fp64_batched": line["speedup_vs_plain_fp64_batched"],
           "plain_gemm_tflops": line["plain_fp64"]["gemm_tflops"],
           "max_rel_err_mixed_vs_plain": float(f"{line['accuracy']['max_rel_err_vs_plain_fp64']:.3g}"),
           "roofline": {"class": line["roofline"].get("class"), "frac": line["roofline"]["frac"],
                        "traffic_per_launch": line["roofline"]["traffic"]}}
    if "cpu_baseline" in line:
        out["cpu_baseline"] = line["cpu_baseline"]["value"]
    pr = line.get("precision")
    if pr:
        out["rel_err_vs_oracle_2160"] = {k: {f: float(f"{max(v[f].values()):.3g}") for f in ("mixed", "plain")}
                                         for k, v in pr["c3_2160_vs_oracle"].items()}
        out["rel_err_mixed_vs_plain_8640"] = {k: float(f"{v:.3g}") for k, v in pr["c3_8640_vs_plain_gpu"].items()}
    sv = line.get("served")
    if sv:
        out["served_sweep_2160"] = {"mixed": sv["sweep_2160"]["mixed"]["solves_per_s"],
                                    "plain": sv["sweep_2160"]["plain"]["solves_per_s"],
                                    "speedup": sv["sweep_2160"]["speedup_mixed_vs_plain"]}
        if "stream" in sv:
            out["served_stream"] = {f: {k: sv["stream"][f][k] for k in
                                        ("requests", "completed", "solves_per_s", "p50_ms", "p99_ms")}
                                    for f in ("mixed", "plain") if f in sv["stream"]}
    sb = line.get("batched_small_meshes")
    if sb:
        out["small_meshes"] = {"batch_mixed": sb["batch_mixed"]["solves_per_s"],
                               "batch_plain": sb["batch_plain"]["solves_per_s"],
                               "one_by_one_plain": sb["one_by_one_plain"]["solves_per_s"]}
    return out


PRECISION_OMEGAS = (0.5, 2.0, 8.0)


def run_precision(args, device):
    """The precision form's per-result errors.  2160 elements (the jittered
    mesh of seed 1) at omega 0.5, 2, 8: the mixed and the plain GPU solutions
    against the FP64 oracle's (raw solution, boundary displacements and
    tractions after the un-swap).  8640 elements (seed 2, n = 25920): the
    mixed form against the plain FP64 GPU path, which the oracle pins
    wherever both run (the oracle would need tens of GB and minutes per
    omega at this size)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from bem_mececcs_b200.solver import BemSolver, unswap_host

    def rel(a, b):
        return float(np.linalg.norm(np.ravel(a - b)) / np.linalg.norm(np.ravel(b)))

    out = {"note": "relative 2-norm errors per result; mixed target <= 1e-8, plain parity <= 1e-10"}
    s3, d3 = meshgen.config_mesh("c3_2160")
    with BemSolver(s3, device=device) as sol:
        sol.ghmatece()
        sol.set_bc(d3.kode, d3.bc.astype(np.complex128), d3.dam, d3.rho)
        xm, corr = sol.sweep(d3.freqs, form="mixed", batch=len(d3.freqs), refine=args.refine)
        xp, _ = sol.sweep(d3.freqs, form="plain", batch=len(d3.freqs))
        zge = sol.material[0]
    p = oracle.OracleProblem(s3, d3)
    p.ghmatece()
    res = {}
    for i, fr in enumerate(d3.freqs):
        odisp, otrac, ox = p.solve(float(fr), use_openblas=True)
        r = {}
        for form, x in (("mixed", xm[i]), ("plain", xp[i])):
            disp, trac = unswap_host(x, d3.kode, d3.bc, zge)
            r[form] = {"x": rel(x, ox), "disp": rel(disp, odisp), "trac": rel(trac, otrac)}
        r["last_correction"] = float(corr[i])
        res[f"{fr:g}"] = r
    out["c3_2160_vs_oracle"] = res
    s4, d4 = meshgen.config_mesh("c3_8640")
    with BemSolver(s4, device=device) as sol:
        sol.ghmatece()
        sol.set_bc(d4.kode, d4.bc.astype(np.complex128), d4.dam, d4.rho)
        xm, corr = sol.sweep(d4.freqs, form="mixed", batch=1, refine=args.refine)
        xp, _ = sol.sweep(d4.freqs, form="plain", batch=1)
    out["c3_8640_vs_plain_gpu"] = {f"{fr:g}": rel(xm[i], xp[i]) for i, fr in enumerate(d4.freqs)}
    out["c3_8640_last_correction"] = {f"{fr:g}": float(corr[i]) for i, fr in enumerate(d4.freqs)}
    return out


def run_small_batch(args, device):
    """The batching form's small meshes: --small-count meshes of 24..600
    elements (rectangular jittered grids, seeded), random Poisson ratio in
    [0.15, 0.35] and damping in [0.005, 0.05], omega uniform in [0.1, 10].
    bem_batch_solve (padded lockstep classes) in both forms against the same
    problems solved one after another through bem_ghmatecd + bem_linsolve
    (each problem on its own context and stream).  Per-mesh static work
    (upload, GHMATECE) is done before the clocks; each form runs once
    untimed, then the median of three timed passes is reported."""
    import torch
    from bem_mececcs_b200 import capi, serve
    from bem_mececcs_b200.solver import BemSolver, batch_solve
    rng = np.random.Generator(np.random.PCG64(5))
    probs = []
    for _ in range(args.small_count):
        nx, ny = serve.grid_for(int(rng.integers(24, 601)))
        nu = float(rng.uniform(0.15, 0.35))
        dam = float(rng.uniform(0.005, 0.05))
        m = meshgen.enclosed_grid(nx, ny, jitter=0.10, seed=int(rng.integers(1 << 30)), rnu=nu,
                                  depth=2.5, layers=4)
        dd = meshgen.traction_patch(m, dam=dam)
        sol = BemSolver(m, device=device)
        sol.ghmatece()
        sol.set_bc(dd.kode, dd.bc, dam, 1.0)
        probs.append((sol, float(rng.uniform(0.1, 10.0))))
    nns = [p[0].nn for p in probs]
    driver = capi.Context(device)
    out = {"problems": len(probs), "n_range": [min(nns), max(nns)],
           "flops_lu_total": float(sum(8.0 / 3.0 * n ** 3 for n in nns))}
    def timed(fn, reps=3):
        # one untimed pass sizes every buffer (each context's system, the
        # driver's class buffers and staging) and caches the lockstep
        # capacities; then the median of `reps` passes
        res = fn()
        walls = []
        for _ in range(reps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            res = fn()
            walls.append(time.perf_counter() - t0)
        return float(np.median(walls)), res

    for form in ("mixed", "plain"):
        dt, (_, corr) = timed(lambda: batch_solve(driver, probs, form=form))
        out[f"batch_{form}"] = {"solves_per_s": round(len(probs) / dt, 2), "wall_s": round(dt, 3),
                                "max_last_correction": float(np.max(corr))}

    def one_by_one():
        for sol, fr in probs:
            sol.ghmatecd(fr)
            sol.ctx.check(sol.ctx.L.bem_linsolve_async(sol.ctx.h), "bem_linsolve_async")
        for sol, _ in probs:
            sol.ctx.sync()

    dt, _ = timed(one_by_one)
    out["one_by_one_plain"] = {"solves_per_s": round(len(probs) / dt, 2), "wall_s": round(dt, 3)}
    out["speedup_batch_mixed_vs_one_by_one_plain"] = round(
        out["batch_mixed"]["solves_per_s"] / out["one_by_one_plain"]["solves_per_s"], 2)
    driver.close()
    for sol, _ in probs:
        sol.ctx.close()
    return out


def _served_summary(st, wall_s):
    return {"solves_per_s": round(st["solves_per_s"], 3), "p50_ms": round(st["p50_ms"], 2),
            "p99_ms": round(st["p99_ms"], 2), "completed": int(st["completed"]),
            "rhs_only": int(st["rhs_only"]), "evictions": int(st["evictions"]),
            "max_busy": int(st["max_busy"]), "peak_gb": round(st["peak_bytes"] / 1e9, 2),
            "wall_s": round(wall_s, 2)}


def run_served(args, s, d, mine, device):
    """The serving form (bem_server_*, one request per (mesh, omega, BCs)):
    (1) this rank's share of the 128-frequency sweep on the 2160 mesh,
    submitted as one burst of requests; (2) the seeded serving stream
    (Poisson arrivals at 50/s, 240..12000 elements, 30% right-hand-side-only),
    replayed in real time: its first --serve-count requests (all 2000 by
    default) in the mixed form, its first --serve-plain-count in the plain
    FP64 form.  HBM budget 160 GB.  Latency = submit to result on the host."""
    from bem_mececcs_b200 import serve
    mat = (s.ge, s.rnu, d.dam, d.rho)
    bc = d.bc.astype(np.complex128)
    out = {"budget_gb": 160.0}
    sweep = {}
    for form in ("mixed", "plain"):
        srv = serve.Server(device=device, budget_bytes=160e9, form=form, refine=args.refine)
        mid = srv.add_mesh(s)
        srv.wait(srv.submit(mid, mat, 0.05, bc, d.kode))  # warm-up (an omega not in the sweep)
        srv.reset_stats()
        t0 = time.perf_counter()
        ids = [srv.submit(mid, mat, float(f), bc, d.kode) for f in mine]
        for i in ids:
            srv.wait(i)
        sweep[form] = _served_summary(srv.stats(), time.perf_counter() - t0)
        srv.close()
    sweep["speedup_mixed_vs_plain"] = round(sweep["mixed"]["solves_per_s"] /
                                            max(sweep["plain"]["solves_per_s"], 1e-9), 3)
    out["sweep_2160"] = sweep
    if args.serve_count > 0:
        reqs = serve.serving_workload(count=max(args.serve_count, args.serve_plain_count))
        meshes, prepared = {}, []
        for r in reqs:
            if r.key not in meshes:
                meshes[r.key] = serve.request_mesh(r)
            prepared.append((r, *serve.request_bc(meshes[r.key], r)))
        stream = {"stream_length": len(reqs), "arrival_rate_per_s": 50.0,
                  "elements": [int(min(r.grid[0] * r.grid[1] for r in reqs)),
                               int(max(r.grid[0] * r.grid[1] for r in reqs))]}
        for form, count in (("mixed", args.serve_count), ("plain", args.serve_plain_count)):
            if count <= 0:
                continue
            srv = serve.Server(device=device, budget_bytes=160e9, form=form, refine=args.refine)
            last = max(r.key for r, _, _ in prepared[:count])
            ids_mesh = {k: srv.add_mesh(m) for k, m in meshes.items() if k <= last}
            wm = serve.request_mesh(serve.Request(0.0, (12, 10), 1, 0.0, mat, (0, 0, 1)))
            w = srv.add_mesh(wm)
            srv.wait(srv.submit(w, mat, 1.0, *serve.request_bc(wm, serve.Request(
                0.0, (12, 10), 1, 0.0, mat, (0.0, 0.0, 1.0)))))
            srv.reset_stats()
            t0 = time.perf_counter()
            ids = []
            for r, rbc, rk in prepared[:count]:
                dt = r.t - (time.perf_counter() - t0)
                if dt > 0:
                    time.sleep(dt)
                ids.append(srv.submit(ids_mesh[r.key], r.material, r.fr, rbc, rk))
            for i in ids:
                srv.wait(i, timeout=1800.0)
            stream[form] = _served_summary(srv.stats(), time.perf_counter() - t0) | {"requests": count}
            srv.close()
        out["stream"] = stream
    return out


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return json.load(fh)
    except Exception:
        return {}


# Flops of one Stokes evaluation with its Gauss-weighted accumulation into H
# and G, and of one element's geometry at one Gauss point, counted once on the
# reference's arithmetic (SOLFUND, NONSINGD) by an operation-counting
# restatement of the oracle that a test keeps equal to these figures.  Two
# complex exponentials (2 exp + 2 sincos calls) per evaluation come on top.
STOKES_FLOPS_PER_EVAL = 613
GEOMETRY_FLOPS_PER_GAUSS_POINT = 98

KERNELS = {
    "assembly": "k_dyn_diag + k_dyn_offdiag + k_rhs_reduce (FP64 Stokes assembly, BC swap, RHS)",
    "panel": "k_panel_push (LU panel, one 16-CTA cluster per problem; pivot candidates pushed by remote "
             "stores before one cluster barrier per column)",
    "laswp_trsm": "k_l11_inv + k_laswp_tc (row interchanges + U12 = L11^-1 A12 on TF32 tensor cores, FP32)",
    "gemm": "k_pack_l21 + k_gemm_tc2 (FP32 LU trailing update by CTA pairs, tcgen05 kind::tf32 cta_group::2, "
            "M = 256, one N = 256 MMA per K step, K = 256 per four-panel group, TMA reduce-add)",
    "solves": "k_tri_inv + k_trsv_f32 (cooperative forward + back substitution with inverted diagonal blocks)",
    "residual": "k_resid_partial + k_resid_final (FP64 refinement residual)",
}
NOTES = {
    "panel": "latency bound: a CTA barrier and a cluster barrier (remote-store mailboxes) per column",
    "solves": "latency bound: one split group barrier per 64-row step, the next step's rows loading meanwhile",
    "laswp_trsm": "latency bound: per 64-column tile a gather, two tensor-core products and the stores",
    "assembly": "FP64-pipe bound (two complex exponentials per Gauss point); bytes are the systems written",
}


# DRAM bytes (read + write) per algorithmic byte of the trailing update, from
# one ncu capture of a K = 256 k_gemm_tc2 launch on 2 problems of n = 6480
# (1.054 GB against 1.044 GB of C read and written once).  The launch's
# traffic is C (the operands stay in L2), so it grows in proportion to the
# algorithmic bytes and scales to any launch by them.
GEMM_DRAM_PER_ALGO_BYTE = 1.054 / 1.044


def _roofline(name, k, peaks, mpeaks):
    """Roofline of one kernel class over the timed region: achieved
    algorithmic bytes (bem_prof_bytes) per second against the measured HBM
    copy bandwidth; the trailing update also against the tcgen05 TF32 peak.
    traffic: DRAM bytes per launch (average over the class's launches), where
    an ncu capture gives the ratio to the algorithmic bytes."""
    secs = k["ms"] * 1e-3
    hbm = peaks.get("hbm_gbs", 6650.0)
    gbs = k.get("bytes", 0.0) / secs / 1e9 if secs > 0 else 0.0
    out = {"bound": "hbm", "class": name, "kernel": KERNELS.get(name, name), "achieved": round(gbs, 1),
           "peak": hbm, "unit": "GB/s", "frac": round(gbs / hbm, 4), "traffic": None,
           "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)",
           "ms": round(k["ms"], 3), "launches": k["launches"]}
    if name in NOTES:
        out["note"] = NOTES[name]
    if name == "gemm":
        tf = k["work"] / secs / 1e12
        peak = mpeaks["tf32_umma_n128"]
        per_launch = k.get("bytes", 0.0) / max(1, k["launches"])
        out["traffic"] = round(GEMM_DRAM_PER_ALGO_BYTE * per_launch)
        out["algorithmic_bytes_per_launch"] = round(per_launch)
        out["traffic_note"] = ("bytes per launch: dram read+write / algorithmic C bytes = "
                               f"{GEMM_DRAM_PER_ALGO_BYTE:.3f} from ncu on one K = 256 launch of 2 problems "
                               "(profiles/k_gemm_tc2_k256_2160.md), times this run's algorithmic bytes per launch")
        out["tensor"] = {"achieved_tflops": round(tf, 2), "peak_tflops": round(peak, 1),
                         "frac": round(tf / peak, 4),
                         "peak_source": "measured: tcgen05 kind::tf32 M=128 N=128 issue-rate "
                                        "microbenchmark (bem_measure_peaks)"}
    if name == "assembly" and secs > 0:
        evals = k["work"] / secs
        out["stokes_evals_per_s"] = round(evals, 1)
        tf = evals * STOKES_FLOPS_PER_EVAL / 1e12
        fp64 = mpeaks.get("fp64_fma") if isinstance(mpeaks, dict) else None
        out["fp64"] = {"achieved_tflops": round(tf, 2), "flops_per_eval": STOKES_FLOPS_PER_EVAL,
                       "transcendentals_per_eval": "2 exp + 2 sincos, not in the flops",
                       "peak_tflops": fp64, "frac": round(tf / fp64, 4) if fp64 else None,
                       "peak_source": "measured: FP64 FMA issue-rate microbenchmark (bem_measure_peaks)"}
    return out


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
