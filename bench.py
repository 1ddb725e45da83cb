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
import tempfile
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


def _radical(mol):
    """The molecule without its last hydrogen (an alkyl radical from an alkane)."""
    from dollarstorescf_b200.basis import Molecule

    k = max(i for i, z in enumerate(mol.Z) if z == 1)
    return Molecule([z for i, z in enumerate(mol.Z) if i != k], [p for i, p in enumerate(mol.xyz) if i != k])


def measure_rows(device: int, cpu_baseline: bool):
    """The rows next to the Fock build: device one-electron integrals and device
    UHF, each beside the reference's own CPU code on the same input (one host
    core, the reference is single-threaded).

      one_electron  (H2O)32 6-31G* 6D (608 functions, 96 nuclei): dss_one_electron
                    (S, T, V to host) vs the reference's basis set-up without the
                    ERI tensor (S, T, V and the Loewdin X).
      uhf           CH2 triplet 6-31G* and the n-butyl radical 6-31G (doublet):
                    dss_uhf_solve from the core guess, conv 1e-10, vs the
                    reference's unrestricted solveMOs (ERI tensor + SCF).
      gradient      water dimer 6-31G*: dss_gradient (analytic four-centre term,
                    difference quotients of the one-electron integrals) vs the
                    time of the reference's gradient routine on the same
                    converged state; the four-centre term alone on the dimer
                    and on the (H2O)16 6D bench basis.
    """
    import time as _t

    import numpy as np

    from dollarstorescf_b200 import basis as B
    from dollarstorescf_b200 import geometry, shells
    from dollarstorescf_b200.engine import BOYS_REF, FockBuilder

    out = {}
    w32 = geometry.water_cluster(4, 4, 2, 32, seed=2024)
    sh32 = shells.build_shells(w32, B.builtin_basis("6-31G*"), pure=False)
    with FockBuilder(device=device, schwarz_threshold=1e-12, boys_mode=BOYS_REF) as fb:
        fb.set_basis(sh32)
        fb.one_electron(sh32)
        ts = []
        for _ in range(11):
            t0 = _t.perf_counter()
            fb.one_electron(sh32)
            ts.append(_t.perf_counter() - t0)
    ts.sort()
    # Host-side jitter (pageable copies of 3 x 1.5 MB) spreads single calls; the
    # median of 11 is the reported figure, the fastest call beside it.
    oe = {"workload": "(H2O)32 6-31G* 6D S, T, V (608 functions, 96 nuclei)", "gpu_ms": ts[5] * 1e3,
          "gpu_ms_min": ts[0] * 1e3, "per_s": 1.0 / ts[5]}
    if cpu_baseline:
        from oracle import refpy

        if refpy.available():
            t0 = _t.perf_counter()
            refpy.setup(sh32, build_tensor=False)
            dt = _t.perf_counter() - t0
            oe["cpu_baseline"] = {"seconds": dt, "per_s": 1.0 / dt, "cores": 1, "kind": "reference",
                                  "sample": "the reference's basis set-up without the ERI tensor (S, T, V, X)"}
            oe["gpu_over_cpu"] = dt / ts[5]
    out["one_electron"] = oe

    A = B.molecule_from_angstrom
    cases = [("ch2_631gs_triplet", A(["C", "H", "H"], [[0, 0, 0], [0.9918, 0.4226, 0], [-0.9918, 0.4226, 0]]),
              "6-31G*", 3),
             ("c4h9_631g_doublet", _radical(geometry.alkane(4, 0)), "6-31G", 2)]
    uhf = {}
    for name, mol, bas, mult in cases:
        sh = shells.build_shells(mol, B.builtin_basis(bas), pure=True)
        ne = sh.n_electrons()
        na, nb = (ne + mult) // 2, (ne + 1 - mult) // 2
        r = {"nbf": sh.nbf(), "n_alpha": na, "n_beta": nb}
        with FockBuilder(device=device, schwarz_threshold=1e-12, boys_mode=BOYS_REF) as fb:
            fb.set_basis(sh)
            t0 = _t.perf_counter()
            S, T, V, en = fb.one_electron(sh)
            E, Da, Db, it, rc = fb.uhf(T + V, S, na, nb, en, conv=1e-10, max_iter=1000, raise_on_noconv=False)
            dt = _t.perf_counter() - t0
        r["gpu"] = {"solves_per_s": 1.0 / dt, "iterations": it, "energy": E, "status": rc}
        if cpu_baseline:
            from oracle import refpy

            if refpy.available():
                t0 = _t.perf_counter()
                refpy.setup(sh, charge=0, multiplicity=mult)
                Er, _, itr, _ = refpy.scf(1e-10)
                dtr = _t.perf_counter() - t0
                r["cpu_baseline"] = {"solves_per_s": 1.0 / dtr, "iterations": itr, "energy": Er, "cores": 1,
                                     "kind": "reference", "sample": "one full unrestricted solve (ERI tensor + SCF)"}
                r["abs_dE_vs_reference"] = abs(E - Er)
                r["gpu_over_cpu"] = dtr / dt
        uhf[name] = r
    out["uhf"] = uhf

    # Nuclear gradient of a converged water dimer 6-31G* (dss_gradient: the
    # analytic four-centre term plus central differences of the device
    # one-electron integrals), beside the reference's gradient routine on the
    # same converged state (its values differ from the derivative of its own
    # energy, so only the time compares); the four-centre term alone
    # (dss_eri_gradient) on the dimer and on the (H2O)16 6-31G* 6D bench basis.
    dimer = geometry.water_dimer(0)
    shd = shells.build_shells(dimer, B.builtin_basis("6-31G*"), pure=True)
    gr = {"workload": "(H2O)2 RHF/6-31G* (36 functions, 6 nuclei)"}

    def best_of(f, k=3):
        f()
        ts = []
        for _ in range(k):
            t0 = _t.perf_counter()
            r = f()
            ts.append(_t.perf_counter() - t0)
        return min(ts), r

    with FockBuilder(device=device, schwarz_threshold=1e-12, boys_mode=BOYS_REF) as fb:
        fb.set_basis(shd)
        S, T, V, en = fb.one_electron(shd)
        E, Dc, it, rc = fb.scf(T + V, S, shd.n_electrons() // 2, en, conv=1e-10)
        gr["gpu_s"], g = best_of(lambda: fb.gradient(shd))
        gr["max_abs_net_force"] = float(np.abs(g.sum(axis=0)).max())
        gr["eri_gradient_s"], _ = best_of(lambda: fb.eri_gradient(shd, 2.0 * Dc))
    sh16 = shells.build_shells(geometry.water_cluster(3, 3, 2, 16, seed=2024), B.builtin_basis("6-31G*"), pure=False)
    with FockBuilder(device=device, schwarz_threshold=1e-12, boys_mode=BOYS_REF) as fb:
        fb.set_basis(sh16)
        n16 = sh16.nbf()
        A16 = np.random.default_rng(0).standard_normal((n16, n16)) * 0.05
        D16 = shells.pack(A16 + A16.T)
        t16, _ = best_of(lambda: fb.eri_gradient(sh16, D16))
        gr["eri_gradient_h2o16_6d"] = {"seconds": t16, "nbf": n16, "natom": sh16.natom,
                                       "note": "four-centre term alone, Schwarz 1e-12, a fixed symmetric density"}
    if cpu_baseline:
        from oracle import refpy

        if refpy.available():
            refpy.setup(shd)
            refpy.scf(1e-10)
            t0 = _t.perf_counter()
            refpy.gradient(shd.natom)
            gr["cpu_baseline"] = {"seconds": _t.perf_counter() - t0, "cores": 1, "kind": "reference",
                                  "sample": "scf::getEnergyGradient on the same converged state"}
    out["gradient"] = gr
    return out


# ---------------------------------------------------------------- reference arm
def _ref_init():
    """Pool initializer: the reference's basis set-up, once per process."""
    sys.path.insert(0, ROOT)
    from oracle import refpy

    _, sh = _workload()
    refpy.setup(sh, build_tensor=False)


def _ref_worker(args):
    seconds_budget, seed = args
    from oracle import refpy

    n, secs, _ = refpy.time_eri_random(seconds_budget, seed)
    return n, secs


def reference_rate(budget_s: float = 12.0, cores: int = 0, pool=None):
    """Reference ERI-phase throughput on the host cores, one process per core
    (the reference's global state rules out threads).  pool: a process pool
    made by reference_pool (reused across samples), else one is made here.
    Returns (builds/s, quartets/s, cores, sample description)."""
    from oracle import refpy

    if not refpy.available():
        return None
    _, sh = _workload()
    n = sh.nbf()
    npair = n * (n + 1) // 2
    total_quartets = npair * (npair + 1) // 2
    cores = cores or os.cpu_count() or 1
    own = pool is None
    if own:
        pool = reference_pool(cores)
    try:
        res = pool.map(_ref_worker, [(budget_s, 1000003 * (k + 1) + int(1e6 * time.perf_counter()) % 1000003)
                                     for k in range(cores)])
    finally:
        if own:
            pool.close()
            pool.join()
    done = sum(r[0] for r in res)
    rate = sum(r[0] / r[1] for r in res if r[1] > 0)  # quartets/s over all processes
    builds = rate / total_quartets
    sample = (f"{done} uniformly drawn canonical function quartets (of {total_quartets}) of the reference's "
              f"ERI phase (electronRepulsionIntegral), {cores} processes x {budget_s:.0f}s; scaled to one "
              f"full Fock build, ERI phase only")
    return builds, rate, cores, sample


def reference_pool(cores: int = 0):
    """One spawned process per host core, each with the reference's basis set up."""
    import multiprocessing as mp

    cores = cores or os.cpu_count() or 1
    return mp.get_context("spawn").Pool(cores, initializer=_ref_init)


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
    # One pool for every step (its processes set the basis up once); each step
    # samples 2 s on every core, so the default 3 + 50 steps take about two minutes.
    pool = reference_pool()
    try:
        for step in range(args.warmup + args.steps):
            r = reference_rate(budget_s=2.0, pool=pool)
            if step >= args.warmup:
                vals.append(r[0])
                meta = r
    finally:
        pool.close()
        pool.join()
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
        "estimate": "sampled extrapolation: each step times uniformly drawn canonical function quartets of the "
                    "reference's ERI phase on every host core and scales the rate to the full quartet count of "
                    "one build; not a timed full build (the digest over the stored tensor is left out, which "
                    "favours the reference)",
    }
    print(json.dumps(line))


# ---------------------------------------------------------------- replicas
def max_over_ranks(x: float, device: str) -> float:
    """The largest of every rank's x (an all-reduce MAX on the process group):
    the job's time is the slowest replica's."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(world_size: int, steps: int, seconds: float) -> float:
    """Whole-job builds/s of world_size independent replicas that each ran
    `steps` builds, timed by the slowest one (weak scaling)."""
    return world_size * steps / seconds


# ---------------------------------------------------------------- GPU arm
class ClockSampler:
    def __init__(self, device: int):
        self.device = device
        self.proc = None
        # DSS_CLOCKS_DIR keeps the raw nvidia-smi samples where the caller wants them.
        self.path = os.path.join(os.environ.get("DSS_CLOCKS_DIR") or tempfile.gettempdir(),
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

    # Per-class kernel shape (untimed): thread per quartet in three register
    # tiers or warp-cooperative, the fastest by per-launch events.
    from dollarstorescf_b200 import autotune

    variants = autotune.tune(fb, Dd.data_ptr(), Jd.data_ptr(), Kd.data_ptr(), cache_path=args.tune_cache)
    # Refined on whole builds, where the classes run concurrently (cached like the rest).
    refine = autotune.tune_whole(fb, Dd.data_ptr(), Jd.data_ptr(), Kd.data_ptr(), variants,
                                 cache_path=args.tune_cache)
    # Launch shape of the whole build: one launch per class or persistent grouped launches.
    launch_shape = autotune.tune_launch(fb, Dd.data_ptr(), Jd.data_ptr(), Kd.data_ptr(), cache_path=args.tune_cache)

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
        tot_ms = max_over_ranks(tot_ms, f"cuda:{device}")
    value = replica_rate(ws, args.steps, tot_ms * 1e-3)

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
        e2e_tot = max_over_ranks(e2e_tot, f"cuda:{device}")
    e2e_value = replica_rate(ws, args.steps, e2e_tot)

    # --- mixed-precision incremental builds (G of a density change dD: FP32
    # quartets below Schwarz.|dD| 1e-7, skipped below 1e-12), same timing rules.
    mixed_builds = {}
    for scale in (1e-3, 1e-5):
        dD = torch.tensor(Dm * scale, dtype=torch.float64, device=f"cuda:{device}")
        with torch.cuda.stream(stream):
            for _ in range(args.warmup):
                flush.fill_(1.0)
                fb.jk_mixed_device(dD.data_ptr(), Jd.data_ptr(), Kd.data_ptr())
            stream.synchronize()
            ms_ = []
            for k in range(args.steps):
                flush.fill_(float(k))
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                fb.jk_mixed_device(dD.data_ptr(), Jd.data_ptr(), Kd.data_ptr())
                e1.record(stream)
                e1.synchronize()
                ms_.append(e0.elapsed_time(e1))
        tms = sum(ms_)
        if ws > 1:
            tms = max_over_ranks(tms, f"cuda:{device}")
        mixed_builds[f"dD_scale_{scale:g}"] = {"builds_per_s": replica_rate(ws, args.steps, tms * 1e-3),
                                                "ms_per_build": tms / args.steps}

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
    build_tflops = total_flops / (tot_ms / args.steps * 1e-3) / 1e12
    sq, pq, wt = fb.work_stats()
    traffic = None  # DRAM bytes per launch of the dominant kernel, from the committed ncu capture
    build_traffic = None  # DRAM bytes of one whole build (sum of its launches' captures)
    tpath = os.path.join(ROOT, "profiles", "traffic.txt")
    if os.path.isfile(tpath):
        with open(tpath) as f:
            for ln in f:
                p = ln.split()
                if len(p) == 2 and not ln.startswith("#") and \
                        p[0] == "eri_jk_kernel<%s>/%s" % (fl[dom]["class"], variants.get(fl[dom]["class"], 0)):
                    traffic = int(p[1])
                if len(p) == 2 and not ln.startswith("#") and p[0] == "build":
                    build_traffic = int(p[1])
    kern = fb.kernels_per_build()
    hbm_peak = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            hbm_peak = float(json.load(f)["hbm_gbs"])
    except (OSError, ValueError, KeyError):
        pass

    line = {
        "metric": METRIC, "value": value, "unit": "builds/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": tot_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded (H2O)16 cluster, 3x3x2 lattice 3.0 A, rotation + 0.2 A jitter)",
        "config": {"workload": WORKLOAD, "nbf": n, "shells": sh.nshell, "boys": "reference series",
                   "warp_cooperative_classes": sorted(k for k, v in variants.items() if v == 1),
                   # Autotuned kernel shape per class: 0 thread per quartet, 2/3 the
                   # same with fewer resident blocks (more registers), 1 warp per quartet.
                   "tuned_shapes": variants,
                   "tuned_whole_build": refine,
                   "tuned_launch": launch_shape,
                   "l2": "flushed between steps (512 MiB write)", "parallelism": f"replicas x{ws}"},
        "e2e": {"value": e2e_value, "unit": "builds/s", "h2d_bytes_per_step": npk * 8,
                "d2h_bytes_per_step": 2 * npk * 8},
        "gpu_launches": kern * args.steps,
        # The build's 21 class kernels run concurrently on eight streams (the tuner's
        # shapes are chosen for that), so the roofline is the whole build's: its
        # algorithmic FLOP over its event-timed duration against the DFMA peak.
        # The dominant class launch, timed alone, is reported beside it.
        "roofline": {"bound": "fp64", "kernel": "Fock build: every class kernel (eri_jk_kernel / eri_coop_kernel), "
                                                "concurrent on eight side streams",
                     "achieved": build_tflops, "peak": peak, "unit": "TFLOP/s",
                     "frac": build_tflops / peak if peak else None,
                     "peak_source": "measured in this run (dss_probe_fp64_peak DFMA loop)",
                     "traffic": build_traffic,
                     "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum summed over the 21 class launches "
                                       "of one build, each captured from a flushed L2 (an upper bound), from the "
                                       "committed ncu capture of this workload (profiles/traffic.txt, "
                                       "build_dram_h2o16_631gs.md), not measured in this run",
                     "dominant_kernel_alone": {
                         "kernel": "eri_jk_kernel<%s>" % fl[dom]["class"], "shape": variants.get(fl[dom]["class"]),
                         "achieved": achieved, "frac": achieved / peak if peak else None,
                         "timing": "one launch alone on the stream (dss_profile_build), CUDA events",
                         "traffic": traffic,
                         "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum of this kernel from the "
                                           "committed ncu capture of this workload (profiles/traffic.txt), not "
                                           "measured in this run"}},
        "build_tflops": build_tflops,
        # The digest's compulsory traffic (read D, write J and K) against the measured HBM copy rate.
        "digest": {"bytes_per_build": 3 * n * n * 8,
                   "achieved_GBps": 3 * n * n * 8 / (tot_ms / args.steps * 1e-3) / 1e9,
                   "peak_GBps": hbm_peak, "peak_source": "MEASURED_PEAKS.json hbm_gbs" if hbm_peak else None},
        # Fock builds/s of the mixed-precision incremental form on the same basis:
        # the G of a density change dD = scale x the bench density (screened by
        # Schwarz.|dD|, FP32 below 1e-7, accurate Boys function).
        "mixed_incremental_builds": mixed_builds,
        "eri_shell_quartets_per_s": sq * value / ws, "eri_prim_quartets_per_s": pq * value / ws,
        "work": {"shell_quartets": sq, "prim_quartets": pq, "warp_tasks": wt},
        "per_class_ms": {c["class"]: round(t, 4) for c, t in zip(fl, per_class_ms) if t > 0},
        # Screened shell quartets, primitive quartets and warp tasks of each class.
        "per_class_work": {c["class"]: [c["shell_quartets"], c["prim_quartets"], c["warp_tasks"]]
                           for c in fl if c["shell_quartets"]},
        # Algorithmic TFLOP/s of each class launch (its work / its event-timed duration).
        "per_class_tflops": {c["class"]: round(c["flops"] / (t * 1e-3) / 1e12, 3)
                             for c, t in zip(fl, per_class_ms) if t > 0},
        "clocks": clk.summary(), "wall_s": wall,
    }
    if rank == 0 and not args.no_cpu_baseline:
        r = reference_rate(budget_s=8.0)
        if r is not None:
            line["cpu_baseline"] = {"value": r[0], "unit": "builds/s", "cores": r[2], "kind": "reference",
                                    "sample": r[3]}
    fb.close()
    if rank == 0 and not args.no_forms:
        line["forms"] = measure_forms(device, args.forms_molecules, args.forms_requests)
        line["forms"].update(measure_rows(device, cpu_baseline=not args.no_cpu_baseline))
    if rank == 0:
        print(json.dumps(line))
    if ws > 1:
        dist.destroy_process_group()


def measure_forms(device: int, n_alkanes: int, n_requests: int):
    """SCF solves/s of the plain FP64 GPU form against the mixed-precision,
    batched and served forms, wall-clock timed around each call (each returns
    only after its results are on the host), with per-molecule |dE| of every
    mixed result against the FP64 result of the same molecule.  Every form
    solves the same molecules with the same convergence threshold and iteration
    cap, and its set-up per molecule (shell pairs and Schwarz factors, device
    one-electron integrals) is inside its timed region; solves/s counts the
    molecules that converged.

      scf_h2o32   (H2O)32 6-31G* 6D (608 functions): dss_scf_solve plain
                  (reference Boys, full FP64 build every iteration) vs the
                  incremental mixed-precision form (FP32 below 1e-7).
      alkanes     n_alkanes seeded CnH2n+2 (n ~ U{1..10}) 6-31G, conv 1e-10,
                  64-iteration cap.  plain_sequential: one reused context,
                  dss_set_basis + dss_one_electron + dss_scf_solve per molecule;
                  batched_fp64 / batched_mixed: one dss_batch for all of them.
      serve       n_requests at a Poisson 200 req/s (60% alkanes STO-3G /
                  6-31G*, 40% water-dimer 6-31G* displacements warm-started from
                  the parent density), continuous batching in the FP64 and the
                  mixed form; plain_sequential: the same requests one after
                  another through one reused context; the mixed form again with
                  an arena that holds only part of the stream (admission by
                  memory binds), and half as many requests at 25 req/s.
    """
    import time as _t

    import numpy as np

    from dollarstorescf_b200 import basis as B
    from dollarstorescf_b200 import geometry, serve, shells
    from dollarstorescf_b200.batch import Batch
    from dollarstorescf_b200.engine import BOYS_REF, FockBuilder

    def solve_plain(shs, guesses=None, max_iter=64):
        ok, iters = 0, 0
        with FockBuilder(device=device, schwarz_threshold=1e-12, boys_mode=BOYS_REF) as fb:
            t0 = _t.perf_counter()
            for i, s in enumerate(shs):
                fb.set_basis(s)
                S, T, V, en = fb.one_electron(s)
                g = guesses[i] if guesses is not None else None
                E, D, it, rc = fb.scf(T + V, S, s.n_electrons() // 2, en, conv=1e-10, max_iter=max_iter, guess=g,
                                      raise_on_noconv=False)
                ok += rc == 0
                iters += it
            dt = _t.perf_counter() - t0
        return {"solves_per_s": ok / dt, "molecules": len(shs), "converged": ok, "iterations": iters, "wall_s": dt}

    out = {}
    w32 = geometry.water_cluster(4, 4, 2, 32, seed=2024)
    sh32 = shells.build_shells(w32, B.builtin_basis("6-31G*"), pure=False)
    with FockBuilder(device=device, schwarz_threshold=1e-12, boys_mode=BOYS_REF) as fb:
        fb.set_basis(sh32)
        S, T, V, en = fb.one_electron(sh32)
        ne = sh32.n_electrons() // 2
        res = {"nbf": sh32.nbf()}
        for mode in ("plain", "mixed"):
            t0 = _t.perf_counter()
            E, D, it, rc = fb.scf(T + V, S, ne, en, conv=1e-10, mixed=(mode == "mixed"), fp32_threshold=1e-7)
            dt = _t.perf_counter() - t0
            res[mode] = {"solves_per_s": 1.0 / dt, "iterations": it, "energy": E, "status": rc}
        res["mixed"]["abs_dE_vs_fp64"] = abs(res["mixed"]["energy"] - res["plain"]["energy"])
        res["mixed_over_plain"] = res["mixed"]["solves_per_s"] / res["plain"]["solves_per_s"]
        out["scf_h2o32"] = res

    rng = np.random.default_rng(4)
    alk = [shells.build_shells(geometry.alkane(int(rng.integers(1, 11)), i), B.builtin_basis("6-31G"), pure=True)
           for i in range(n_alkanes)]
    ares = {"molecules": n_alkanes, "conv": 1e-10, "max_iter": 64,
            "note": "solves/s counts converged molecules; some C10 molecules do not converge from the core guess "
                    "(the reference's own loop oscillates or creeps on them too)",
            "plain_sequential": solve_plain(alk)}
    energies = {}
    from dollarstorescf_b200.autotune import tune_batch, tune_batch_launch, tune_batch_whole

    for name, mixed in (("batched_fp64", False), ("batched_mixed", True)):
        with Batch(device=device, schwarz_threshold=1e-12, boys_mode=BOYS_REF) as b:
            # Per-class kernel choice, made once before the timed solve on the
            # first 16 molecules (they cover every class); then the launch shape
            # (per class or persistent groups) on the whole composition.
            hs0 = [b.add(s) for s in alk[:16]]
            ch = tune_batch(b)
            ares.setdefault("tuned_whole_accumulation", tune_batch_whole(b, ch))
            ares.setdefault("tuned_variants", ch)
            hs0 += [b.add(s) for s in alk[16:]]
            ares.setdefault("tuned_launch", tune_batch_launch(b))
            for h in hs0:
                b.remove(h)
            t0 = _t.perf_counter()
            hs = [b.add(s) for s in alk]
            b.solve(conv=1e-10, max_iter=64, mixed=mixed)
            dt = _t.perf_counter() - t0
            r = [b.result(h) for h in hs]
        energies[name] = [(x[0], x[3]) for x in r]
        ok = int(sum(1 for x in r if x[3] == 0))
        ares[name] = {"solves_per_s": ok / dt, "molecules": len(alk), "converged": ok, "wall_s": dt}
    both = [(a[0], m[0]) for a, m in zip(energies["batched_fp64"], energies["batched_mixed"]) if a[1] == 0 and m[1] == 0]
    ares["batched_mixed"]["max_abs_dE_vs_fp64"] = max(abs(a - m) for a, m in both) if both else None
    base = ares["plain_sequential"]["solves_per_s"]
    ares["batched_fp64_over_plain"] = ares["batched_fp64"]["solves_per_s"] / base
    ares["batched_mixed_over_plain"] = ares["batched_mixed"]["solves_per_s"] / base
    ares["batched_mixed_over_batched_fp64"] = (ares["batched_mixed"]["solves_per_s"] /
                                               ares["batched_fp64"]["solves_per_s"])
    out["alkanes_631g"] = ares

    dimer = geometry.water_dimer(3)
    E0, D0 = serve.solve_parent(dimer)
    reqs = serve.make_request_stream(count=n_requests, rate=200.0, seed=11, parent_density=D0, dimer=dimer)
    sres = {"requests": n_requests, "rate_req_per_s": 200.0,
            "plain_sequential": solve_plain([r.shells for r in reqs], [r.guess for r in reqs], max_iter=64)}
    served = {}
    for name, mixed in (("served_fp64", False), ("served_mixed", True)):
        # Three SCF iterations per batch step (one graph replay each) between
        # admissions and retirements: fewer host round trips and pair-list rebuilds.
        sv = serve.serve(reqs, conv=1e-10, boys_mode=BOYS_REF, mixed=mixed, max_iter=64, iterations_per_step=3)
        served[name] = {r.rid: (r.energy, r.status) for r in sv["results"]}
        sres[name] = {k: v for k, v in sv.items() if k != "results"}
    pairs = [(served["served_fp64"][k][0], v[0]) for k, v in served["served_mixed"].items()
             if v[1] == 0 and served["served_fp64"].get(k, (0, 1))[1] == 0]
    sres["served_mixed"]["max_abs_dE_vs_fp64"] = max(abs(a - m) for a, m in pairs) if pairs else None
    base = sres["plain_sequential"]["solves_per_s"]
    sres["served_fp64_over_plain"] = sres["served_fp64"]["solves_per_s"] / base
    sres["served_mixed_over_plain"] = sres["served_mixed"]["solves_per_s"] / base
    # Admission by memory: an arena with room for a quarter of the stream's
    # regions (each request's region bytes summed), so requests wait for
    # finished molecules to free their regions.
    with Batch(device=device, schwarz_threshold=1e-12, boys_mode=BOYS_REF) as probe:
        need = sum(probe.info(n_for_region=r.shells.nbf())[2] for r in reqs)
    arena = max(need // 4, 1)
    sv = serve.serve(reqs, conv=1e-10, boys_mode=BOYS_REF, mixed=True, max_iter=64, arena_bytes=arena,
                     iterations_per_step=3)
    sres["served_mixed_memory_bound"] = dict({k: v for k, v in sv.items() if k != "results"}, arena_bytes=arena)
    # At 200 req/s the queue grows for the whole stream, so p50/p99 above are
    # mostly queueing time (queue_p50 / service_p50 split them).  The same request
    # mix at a rate the mixed form sustains shows the service latency itself.
    low_rate = 25.0
    low = serve.make_request_stream(count=max(1, n_requests // 2), rate=low_rate, seed=11, parent_density=D0,
                                    dimer=dimer)
    sv = serve.serve(low, conv=1e-10, boys_mode=BOYS_REF, mixed=True, max_iter=64)
    sres["served_mixed_at_sustainable_rate"] = dict({k: v for k, v in sv.items() if k != "results"},
                                                     rate_req_per_s=low_rate, requests=len(low))
    out["serve"] = sres
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="dss", choices=["dss", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the SCF / batch / serving measurements")
    ap.add_argument("--forms-molecules", type=int, default=256, help="alkanes in the batched-form measurement")
    ap.add_argument("--forms-requests", type=int, default=200, help="requests in the serving measurement")
    ap.add_argument("--tune-cache", default=None,
                    help="JSON file of autotuner choices: reused when present, written when not (a profiler run "
                         "then repeats the plain run's choices instead of re-timing them under serialisation)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
