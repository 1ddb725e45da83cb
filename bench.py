"""Benchmark: plain FP64 GPU Fock builds on (H2O)16 / RHF 6-31G* (6D, 304 functions).

A "step" is one complete two-electron Fock build G(D) = J[D] - K[D]/2 from a
resident density: every Schwarz-surviving ERI (threshold 1e-12) recomputed
(direct SCF) and digested into J and K, with the reference-parity Boys mode.

  value      Fock builds/s with D resident in HBM (dss_build_jk_device),
             per-step CUDA events on the library's stream, L2 flushed (a 512 MiB
             write) between steps, outside the timed events.
  e2e        Fock builds/s through the reference-facing C ABI call
             dss_build_jk: packed-U D from pinned host memory in, packed-U J and
             K back to pinned host memory, copies inside the timed region.
  roofline   the dominant ERI class kernel: algorithmic FP64 flops per launch
             (per-class constants from csrc/gen_eri.py) over its event-timed
             duration, against the FP64 FMA throughput measured by
             dss_probe_fp64_peak in the same run.
  cpu_baseline / --impl reference
             the unmodified reference (oracle/_ref/libdssref.so) on the host
             cores: a bounded sample of its ERI phase (the canonical quartet rows
             it computes in assignExactRepulsionTensor) over the same basis,
             one process per core, scaled to one full Fock build (ERI phase
             only, the digest over the stored tensor is not counted, which
             favours the reference).

N > 1 GPUs (torchrun): independent replicas, one molecule per GPU, no
collective on the data path ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Fock builds/s"
WORKLOAD = "(H2O)16 RHF/6-31G* 6D (304 bf), plain FP64 J+K build, Schwarz 1e-12"


def _workload():
    from dollarstorescf_b200 import basis, geometry, shells

    mol = geometry.water_cluster(3, 3, 2, 16, seed=2024)
    sh = shells.build_shells(mol, basis.builtin_basis("6-31G*"), pure=False)
    return mol, sh


def _dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ---------------------------------------------------------------- reference arm
def _ref_worker(args):
    seconds_budget, seed = args
    sys.path.insert(0, ROOT)
    from oracle import refpy

    _, sh = _workload()
    refpy.setup(sh, build_tensor=False)
    n, secs, _ = refpy.time_eri_random(seconds_budget, seed)
    return n, secs


def reference_rate(budget_s: float = 12.0, cores: int = 0):
    """Reference ERI-phase throughput on the host cores, one process per core
    (the reference's global state rules out threads).  Returns
    (builds/s, quartets/s, cores, sample description)."""
    import multiprocessing as mp

    from oracle import refpy

    if not refpy.available():
        return None
    _, sh = _workload()
    n = sh.nbf()
    npair = n * (n + 1) // 2
    total_quartets = npair * (npair + 1) // 2
    cores = cores or os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        res = pool.map(_ref_worker, [(budget_s, 1000003 * (k + 1)) for k in range(cores)])
    done = sum(r[0] for r in res)
    rate = sum(r[0] / r[1] for r in res if r[1] > 0)  # quartets/s over all processes
    builds = rate / total_quartets
    sample = (f"{done} uniformly drawn canonical function quartets (of {total_quartets}) of the reference's "
              f"ERI phase (electronRepulsionIntegral), {cores} processes x {budget_s:.0f}s; scaled to one "
              f"full Fock build, ERI phase only")
    return builds, rate, cores, sample


def run_reference(args):
    ws, rank, _ = _dist_env()
    if rank != 0:
        return
    from oracle import refpy

    if not refpy.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libdssref.so not built"}))
        return
    t_all = time.perf_counter()
    vals = []
    meta = None
    for step in range(args.warmup + args.steps):
        r = reference_rate(budget_s=6.0)
        if step >= args.warmup:
            vals.append(r[0])
            meta = r
    v = statistics.mean(vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "builds/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / v, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded water cluster)",
        "config": {"workload": WORKLOAD + " -- reference CPU ERI phase", "l2": "n/a (CPU)"},
        "cpu_baseline": {"value": v, "unit": "builds/s", "cores": meta[2], "kind": "reference",
                         "sample": meta[3]},
        "e2e": {"value": v, "unit": "builds/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "eri_quartets_per_s": meta[1], "wall_s": time.perf_counter() - t_all,
    }
    print(json.dumps(line))


# ---------------------------------------------------------------- GPU arm
class ClockSampler:
    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out" if os.path.isdir(os.path.join(ROOT, "gpurun_out")) else "_build",
                                 f"clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) < 7:
                    continue
                try:
                    sm.append(float(p[0]))
                    mx.append(float(p[1]))
                except ValueError:
                    continue
                for nm, v in zip(names, p[3:7]):
                    if v.lower() == "active":
                        reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def _class_flops():
    sys.path.insert(0, os.path.join(ROOT, "dollarstorescf_b200", "csrc"))
    import gen_eri

    return gen_eri.flop_table(2)


def algorithmic_flops(fb, pure: bool):
    """Per class: algorithmic FP64 flops of one build, from the screened
    quartet counts.  Per primitive quartet: Boys 2(L+1)+20 plus the VRR terms
    (2 flops each) that build [e0|f0]^(m), la<=|e|<=la+lb, lc<=|f|<=lc+ld; per
    contracted quartet: the HRR terms (2 flops each) plus the digest, 12 flops
    per Cartesian integral (6 FMAs: 2 for J, 4 for K)."""
    from dollarstorescf_b200 import _lib

    L = _lib.load()
    ft = _class_flops()
    out = []
    for i in range(L.dss_num_classes()):
        l4, sq, pq, wt = fb.class_info(i)
        name = "%d%d%d%d" % tuple(l4)
        f = ft[name]
        ncart = 1
        for l in l4:
            ncart *= (l + 1) * (l + 2) // 2
        flops = pq * (2 * (f["L"] + 1) + 20 + f["vrr_alg"]) + sq * (f["hrr"] + 12 * ncart)
        out.append({"class": name, "shell_quartets": sq, "prim_quartets": pq, "warp_tasks": wt, "flops": flops})
    return out


def run_gpu(args):
    import numpy as np
    import torch

    ws, rank, local = _dist_env()
    if ws > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    device = local if ws > 1 else 0
    torch.cuda.set_device(device)

    from dollarstorescf_b200 import shells
    from dollarstorescf_b200.engine import BOYS_REF, FockBuilder

    mol, sh = _workload()
    fb = FockBuilder(device=device, schwarz_threshold=1e-12, boys_mode=BOYS_REF)
    stream = torch.cuda.ExternalStream(fb.stream_ptr(), device=device)
    n = fb.set_basis(sh)
    # A realistic density: a seeded, idempotent-looking symmetric matrix with a core-like diagonal.
    rng = np.random.default_rng(7)
    A = rng.standard_normal((n, n)) * 0.02
    Dm = A + A.T + np.diag(np.full(n, 0.3))
    Dd = torch.tensor(Dm, dtype=torch.float64, device=f"cuda:{device}")
    Jd = torch.empty_like(Dd)
    Kd = torch.empty_like(Dd)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{device}")

    def one_build():
        fb.jk_device(Dd.data_ptr(), Jd.data_ptr(), Kd.data_ptr())

    # Per-class kernel choice (untimed): thread-per-quartet vs warp-cooperative.
    from dollarstorescf_b200 import autotune

    variants = autotune.tune(fb, Dd.data_ptr(), Jd.data_ptr(), Kd.data_ptr())

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            flush.fill_(1.0)
            one_build()
        stream.synchronize()
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize()
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        t0 = time.perf_counter()
        with ClockSampler(device) as clk:
            for k in range(args.steps):
                flush.fill_(float(k))
                starts[k].record(stream)
                one_build()
                ends[k].record(stream)
            stream.synchronize()
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    tot_ms = sum(step_ms)
    if ws > 1:
        t = torch.tensor([tot_ms], dtype=torch.float64, device=f"cuda:{device}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        tot_ms = float(t.item())
    value = ws * args.steps / (tot_ms * 1e-3)

    # --- e2e through the reference-facing C ABI, pinned host buffers.
    npk = n * (n + 1) // 2
    Dp = torch.tensor(shells.pack(Dm), dtype=torch.float64).pin_memory()
    Jp = torch.empty(npk, dtype=torch.float64).pin_memory()
    Kp = torch.empty(npk, dtype=torch.float64).pin_memory()
    for _ in range(2):
        fb.jk_host_ptrs(Dp.data_ptr(), Jp.data_ptr(), Kp.data_ptr())
    if ws > 1:
        dist.barrier()
    e2e_s = []
    for k in range(args.steps):
        flush.fill_(float(k))
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        fb.jk_host_ptrs(Dp.data_ptr(), Jp.data_ptr(), Kp.data_ptr())
        e2e_s.append(time.perf_counter() - t1)
    e2e_tot = sum(e2e_s)
    if ws > 1:
        t = torch.tensor([e2e_tot], dtype=torch.float64, device=f"cuda:{device}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_tot = float(t.item())
    e2e_value = ws * args.steps / e2e_tot

    # --- per-class profile, roofline of the dominant class kernel.
    per_class_ms = fb.profile_build(Dd.data_ptr(), Jd.data_ptr(), Kd.data_ptr())
    per_class_ms2 = fb.profile_build(Dd.data_ptr(), Jd.data_ptr(), Kd.data_ptr())
    per_class_ms = [min(a, b) if a > 0 and b > 0 else max(a, b) for a, b in zip(per_class_ms, per_class_ms2)]
    fl = algorithmic_flops(fb, sh.pure)
    peak = fb.fp64_peak_tflops()
    dom = max(range(len(fl)), key=lambda i: per_class_ms[i])
    dom_t = per_class_ms[dom] * 1e-3
    achieved = fl[dom]["flops"] / dom_t / 1e12 if dom_t > 0 else 0.0
    total_flops = sum(c["flops"] for c in fl)
    sq, pq, wt = fb.work_stats()
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.isfile(tpath):
        with open(tpath) as f:
            traffic = json.load(f).get("eri_jk_kernel_%s" % fl[dom]["class"])
    kern = fb.kernels_per_build()

    line = {
        "metric": METRIC, "value": value, "unit": "builds/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": tot_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded (H2O)16 cluster, 3x3x2 lattice 3.0 A, rotation + 0.2 A jitter)",
        "config": {"workload": WORKLOAD, "nbf": n, "shells": sh.nshell, "boys": "reference series",
                   "warp_cooperative_classes": sorted(k for k, v in variants.items() if v == 1),
                   "l2": "flushed between steps (512 MiB write)", "parallelism": f"replicas x{ws}"},
        "e2e": {"value": e2e_value, "unit": "builds/s", "h2d_bytes_per_step": npk * 8,
                "d2h_bytes_per_step": 2 * npk * 8},
        "gpu_launches": kern * args.steps,
        "roofline": {"bound": "fp64", "kernel": "eri_jk_kernel<%s>" % fl[dom]["class"], "achieved": achieved,
                     "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak if peak else None,
                     "peak_source": "measured in this run (dss_probe_fp64_peak DFMA loop)",
                     "traffic": traffic},
        "build_tflops": total_flops / (tot_ms / args.steps * 1e-3) / 1e12,
        "eri_shell_quartets_per_s": sq * value / ws, "eri_prim_quartets_per_s": pq * value / ws,
        "work": {"shell_quartets": sq, "prim_quartets": pq, "warp_tasks": wt},
        "per_class_ms": {c["class"]: round(t, 4) for c, t in zip(fl, per_class_ms) if t > 0},
        "clocks": clk.summary(), "wall_s": wall,
    }
    if rank == 0 and not args.no_cpu_baseline:
        r = reference_rate(budget_s=8.0)
        if r is not None:
            line["cpu_baseline"] = {"value": r[0], "unit": "builds/s", "cores": r[2], "kind": "reference",
                                    "sample": r[3]}
    if rank == 0:
        print(json.dumps(line))
    fb.close()
    if ws > 1:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="dss", choices=["dss", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
