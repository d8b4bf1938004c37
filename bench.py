#!/usr/bin/env python
"""Benchmark of the B200 force-evaluation hot path (one JSON line on rank 0).

Headline workload: Lennard-Jones FCC 40³ (256,000 atoms, a=5.26 Å, σ_disp
0.1 Å, ε=0.0104 eV, σ=3.4 Å, c=8.5 Å, periodic), plain FP64 E+F+virial.  A
step is one evaluate! call: the full cell-list rebuild plus the pair kernel
and the reductions, on synthetic seeded input.

  value  atoms/s with positions resident in HBM (pfw_set_geometry_device +
         pfw_evaluate_device per step), per-step CUDA events on the
         library's launch stream; L2 flushed between steps outside the events
  e2e    the same through the reference-facing C ABI with HOST buffers
         (pinned X in, E/F/W out, copies inside the timed region)

--impl reference times the reference's CPU algorithm (restated in oracle/,
the reference being a Julia package that cannot run on this machine) with
all host threads on the same workload.  Under torchrun each GPU evaluates
its own replica (weak scaling; the single-box path is replicas only).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "potentialframework.jl_b200"))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "atoms/s E+F+virial, plain vs mixed/batched/surrogate at stated force RMSE"
FALLBACK_HBM = 6650.0


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-forms", action="store_true")
    return p.parse_args()


def env_rank():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def workload():
    from pfw_b200 import workloads as WL
    s = WL.lj_fcc(seed=2, nc=40)
    return s, dict(workload="lj_fcc40_256000", atoms=len(s), potential="lennard_jones",
                   epsilon=WL.LJ_EPS, sigma=WL.LJ_SIGMA, cutoff=WL.LJ_CUTOFF, lattice_a=5.26,
                   displacement_sigma=0.1, box=list(np.diag(s.H)), periodic=True)


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return d.get("hbm_gbs", FALLBACK_HBM), "measured"
    return FALLBACK_HBM, "fallback"


def profile_traffic(name):
    """Per-launch DRAM bytes of a kernel, from a committed ncu summary line
    `traffic_bytes_per_launch = N` in profiles/<name>.md (None if absent)."""
    path = os.path.join(ROOT, "profiles", name + ".md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.strip().startswith("traffic_bytes_per_launch"):
            try:
                return float(line.split("=")[1].split()[0])
            except Exception:
                return None
    return None


class Clocks:
    """nvidia-smi sampler for the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.f = tempfile.NamedTemporaryFile("w+", delete=False, suffix=".csv")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(device), f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = []
        for line in open(self.f.name):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 7:
                try:
                    rows.append((float(parts[0]), float(parts[1]), parts[3:7]))
                except ValueError:
                    pass
        os.unlink(self.f.name)
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for _, _, r in rows for k in range(4) if r[k].lower() == "active"})
        return dict(sm_mhz=statistics.median(r[0] for r in rows), sm_max_mhz=max(r[1] for r in rows),
                    samples=len(rows), reasons=reasons)


def cpu_baseline(s, seconds=12.0, max_reps=20):
    """Restated reference CPU algorithm (oracle/, phase-coloured threads) on the
    full workload, repeated for about `seconds`."""
    from oracle import oracle as O
    from pfw_b200 import workloads as WL
    nthreads = os.cpu_count() or 1
    times = []
    t0 = time.perf_counter()
    while len(times) < max_reps and (time.perf_counter() - t0) < seconds:
        t = time.perf_counter()
        O.pair_evaluate(s.X, s.H, s.pbc, s.species, "lj", (WL.LJ_EPS, WL.LJ_SIGMA), WL.LJ_CUTOFF,
                        nthreads=nthreads)
        times.append(time.perf_counter() - t)
    med = statistics.median(times)
    return dict(value=len(s) / med, unit="atoms/s", cores=nthreads, kind="port",
                sample=f"full {len(s)}-atom LJ box, {len(times)} evaluate! calls (median), "
                       f"restated reference CPU algorithm (oracle/), {nthreads} threads")


def run_reference(args):
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    s, cfg = workload()
    from oracle import oracle as O
    from pfw_b200 import workloads as WL
    nthreads = os.cpu_count() or 1
    call = lambda: O.pair_evaluate(s.X, s.H, s.pbc, s.species, "lj", (WL.LJ_EPS, WL.LJ_SIGMA), WL.LJ_CUTOFF,
                                   nthreads=nthreads)
    for _ in range(args.warmup):
        call()
    t = time.perf_counter()
    for _ in range(args.steps):
        call()
    dt = (time.perf_counter() - t) / max(args.steps, 1)
    v = len(s) / dt
    cfg = dict(cfg, parallelism="cpu threads", note="reference is Julia (not installable here); "
               "its CPU algorithm restated in oracle/ is timed")
    line = dict(impl="reference", metric=METRIC, value=v, unit="atoms/s", n_gpus=args.gpus, steps=args.steps,
                warmup=args.warmup, ms_per_step=dt * 1e3, higher_is_better=True, scaling="weak", vs_baseline=None,
                dtype="f64", data="synthetic", config=cfg,
                cpu_baseline=dict(value=v, unit="atoms/s", cores=nthreads, kind="port",
                                  sample=f"full {len(s)}-atom LJ box per step"),
                e2e=dict(value=v, unit="atoms/s", h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line), flush=True)
    return 0


def run_b200(args):
    import ctypes

    import torch

    from pfw_b200 import lib
    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    s, cfg = workload()
    n = len(s)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    h = lib.Handle(lib.FP64, device=local)
    h.check(h.L.pfw_set_stream(h.ws, ctypes.c_void_p(stream.cuda_stream)))
    h.lj(cfg["epsilon"], cfg["sigma"], cfg["cutoff"])
    X_dev = torch.from_numpy(s.X).to(dev)
    sp_dev = torch.from_numpy(s.species).to(dev)
    E_dev = torch.zeros(1, dtype=torch.float64, device=dev)
    F_dev = torch.zeros((n, 3), dtype=torch.float64, device=dev)
    W_dev = torch.zeros(9, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def step():
        h.set_geometry_device(n, ctypes.c_void_p(X_dev.data_ptr()), s.H, s.pbc, ctypes.c_void_p(sp_dev.data_ptr()))
        h.evaluate_device(lib.MODEL_PAIR, 7, ctypes.c_void_p(E_dev.data_ptr()), ctypes.c_void_p(F_dev.data_ptr()),
                          ctypes.c_void_p(W_dev.data_ptr()))

    for _ in range(max(args.warmup, 3)):
        step()
    h.check(h.L.pfw_set_diagnostics(h.ws, 1))
    ms_buf = np.zeros(4)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    stage = []
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    l0 = h.launches
    for k in range(args.steps):
        flush.zero_()  # L2 flush (256 MB write), outside the step's events
        starts[k].record(stream)
        step()
        ends[k].record(stream)
        h.L.pfw_stage_times(h.ws, ms_buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 4)
        stage.append(ms_buf.copy())
    torch.cuda.synchronize()
    launches = h.launches - l0
    clk = clocks.stop()
    h.check(h.L.pfw_set_diagnostics(h.ws, 0))
    step_ms = [a.elapsed_time(b) for a, b in zip(starts, ends)]
    ms = sum(step_ms) / len(step_ms)
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    value = world * n / (ms * 1e-3)
    stage = np.array(stage)
    kern_ms = float(stage[:, 1].mean())
    geom_ms = float(stage[:, 0].mean())

    # e2e through the host C ABI: pinned X in, E/F/W out, copies timed
    Xh = torch.from_numpy(s.X).pin_memory()
    sph = torch.from_numpy(s.species).pin_memory()
    Fh = torch.zeros((n, 3), dtype=torch.float64).pin_memory()
    Eh = np.zeros(1)
    Wh = np.zeros(9)
    Hf = np.asarray(s.H).ravel(order="F").copy()
    pb = np.array([1, 1, 1], np.uint8)
    dp = ctypes.POINTER(ctypes.c_double)

    def e2e_step():
        h.check(h.L.pfw_set_geometry(h.ws, n, ctypes.cast(Xh.data_ptr(), dp), Hf.ctypes.data_as(dp),
                                     pb.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
                                     ctypes.cast(sph.data_ptr(), ctypes.POINTER(ctypes.c_int32))))
        h.check(h.L.pfw_evaluate(h.ws, lib.MODEL_PAIR, 7, Eh.ctypes.data_as(dp), ctypes.cast(Fh.data_ptr(), dp),
                                 Wh.ctypes.data_as(dp)))

    for _ in range(3):
        e2e_step()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - t0) / args.steps
    if dist:
        t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    npairs = h.pair_count()
    E_ref = float(Eh[0])

    line = None
    if rank == 0:
        peak, peak_kind = measured_peaks()
        alg_bytes = 49.0 * n  # X 24 B + species 1 B read, F 24 B written per atom
        achieved = alg_bytes / (kern_ms * 1e-3) / 1e9
        fp64_peak = h.probe_fp64()
        alg_flops = npairs * 65.0  # 62 flop + 1 sqrt + 2 div per in-cutoff unordered pair
        traffic = profile_traffic("pair_lj_fp64")
        line = dict(
            metric=METRIC, value=value, unit="atoms/s", n_gpus=world, steps=args.steps, warmup=args.warmup,
            ms_per_step=ms, higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f64",
            data="synthetic (seeded FCC lattice, Gaussian displacements)",
            config=dict(cfg, parallelism=f"replicas x{world}" if world > 1 else "single GPU",
                        l2="256 MB flush between steps, outside the per-step events",
                        unordered_pairs=npairs, energy_eV=E_ref),
            roofline=dict(bound="hbm", kernel="k_pair64<LJ>", achieved=achieved, peak=peak, unit="GB/s",
                          frac=achieved / peak, peak_source=peak_kind, traffic=traffic,
                          kernel_ms=kern_ms, geometry_ms=geom_ms, algorithmic_bytes_per_launch=alg_bytes,
                          fp64_pipe=dict(achieved_tflops=alg_flops / (kern_ms * 1e-3) / 1e12, peak_tflops=fp64_peak,
                                         frac=alg_flops / (kern_ms * 1e-3) / 1e12 / fp64_peak,
                                         peak_source="measured DFMA probe (pfw_probe_fp64_peak)",
                                         algorithmic_flops_per_launch=alg_flops)),
            e2e=dict(value=world * n / e2e_s, unit="atoms/s", ms_per_step=e2e_s * 1e3, h2d_bytes_per_step=28 * n,
                     d2h_bytes_per_step=24 * n + 8 + 72, api="pfw_set_geometry + pfw_evaluate (host buffers)"),
            gpu_launches=launches, clocks=clk)
        if not args.no_forms:
            line["forms"] = forms(s, dev)
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(s)
    h.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if line:
        print(json.dumps(line), flush=True)
    return 0


def forms(s, dev):
    """Mixed-precision form on the same workload: atoms/s and force error vs FP64."""
    import torch

    from pfw_b200 import lib
    out = {}
    h64 = lib.Handle(lib.FP64, device=dev.index)
    h64.set_geometry(s.X, s.H, s.pbc, s.species)
    h64.lj(0.0104, 3.4, 8.5)
    E64, F64, W64 = h64.evaluate(lib.MODEL_PAIR, 7)
    h32 = lib.Handle(lib.MIXED, device=dev.index)
    h32.set_geometry(s.X, s.H, s.pbc, s.species)
    h32.lj(0.0104, 3.4, 8.5)
    E32, F32, W32 = h32.evaluate(lib.MODEL_PAIR, 7)
    import ctypes
    X_dev = torch.from_numpy(s.X).to(dev)
    sp_dev = torch.from_numpy(s.species).to(dev)
    bufs = [torch.zeros(k, dtype=torch.float64, device=dev) for k in (1, 3 * len(s), 9)]
    stream = torch.cuda.current_stream(dev)
    h32.check(h32.L.pfw_set_stream(h32.ws, ctypes.c_void_p(stream.cuda_stream)))

    def step():
        h32.set_geometry_device(len(s), ctypes.c_void_p(X_dev.data_ptr()), s.H, s.pbc,
                                ctypes.c_void_p(sp_dev.data_ptr()))
        h32.evaluate_device(lib.MODEL_PAIR, 7, *[ctypes.c_void_p(b.data_ptr()) for b in bufs])

    for _ in range(3):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(10):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / 10
    out["mixed_lj"] = dict(value=len(s) / (ms * 1e-3), unit="atoms/s", ms_per_step=ms,
                           force_rmse=float(np.sqrt(np.mean((F32 - F64) ** 2))),
                           force_max_err=float(np.abs(F32 - F64).max()), energy_err=abs(E32 - E64),
                           virial_max_err=float(np.abs(W32 - W64).max()),
                           note="FP32 pair arithmetic, FP64 wrap/shift, Kahan FP64 E/W; errors vs plain FP64")
    h32.close()
    h64.close()
    return out


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
