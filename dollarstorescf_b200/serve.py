"""Serving loop: continuous batching of SCF requests on one GPU.

Requests (single points, or finite-difference displacements of a parent
geometry warm-started from the parent's density, as the reference's frequency
driver does, chem/scf/Frequency.cpp:121-133) arrive over time.  The loop admits
every request that has arrived into the running batch while the batch arena has
room (admission by device memory), runs SCF iterations of all admitted
molecules together (dss_batch_step: one captured graph per iteration), and
retires molecules as they finish, so new requests join while others are on the
GPU.  Per request it records the latency from arrival to result, split into
the queue time (arrival to admission) and the service time (admission to
result); solves/s counts converged results only.
"""
from __future__ import annotations

import heapq
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from . import basis as basis_mod
from . import geometry
from .batch import Batch
from .engine import BOYS_FAST, BOYS_REF, FockBuilder
from .shells import ShellArrays, build_shells


@dataclass
class Request:
    rid: int
    arrival: float  # seconds after the start of the stream
    shells: ShellArrays
    kind: str
    guess: Optional[np.ndarray] = None  # packed-U alpha density of the parent


@dataclass
class Result:
    rid: int
    kind: str
    energy: float
    iterations: int
    status: int
    arrival: float
    admitted: float
    finished: float

    @property
    def latency(self) -> float:
        return self.finished - self.arrival

    @property
    def queue(self) -> float:
        """Arrival to admission: time spent waiting for a slot (arena memory)."""
        return self.admitted - self.arrival

    @property
    def service(self) -> float:
        """Admission to result: time on the GPU, shared with the other molecules."""
        return self.finished - self.admitted


def poisson_arrivals(rate: float, count: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, count))


def make_request_stream(count: int = 200, rate: float = 200.0, seed: int = 7, parent_density=None,
                        dimer=None) -> List[Request]:
    """The serving workload: 60% alkane single points (CnH2n+2, n ~ U{1..10},
    STO-3G or 6-31G*), 40% +-0.005 bohr displacements of a water dimer
    (6-31G*) along its 18 Cartesian coordinates, warm-started from the parent
    density.  Everything is generated from the seed."""
    rng = np.random.default_rng(seed)
    times = poisson_arrivals(rate, count, seed + 1)
    dimer = dimer if dimer is not None else geometry.water_dimer(seed)
    disps = geometry.displacements(dimer, 0.005)
    b631 = basis_mod.builtin_basis("6-31G*")
    sto = basis_mod.builtin_basis("STO-3G")
    out = []
    for i, t in enumerate(times):
        if rng.random() < 0.6:
            n = int(rng.integers(1, 11))
            bas = sto if rng.random() < 0.5 else b631
            mol = geometry.alkane(n, int(rng.integers(0, 1 << 30)))
            out.append(Request(i, float(t), build_shells(mol, bas, pure=True), f"alkane C{n} {bas.name}"))
        else:
            k = int(rng.integers(0, len(disps)))
            out.append(Request(i, float(t), build_shells(disps[k], b631, pure=True), "dimer displacement",
                               guess=parent_density))
    return out


def solve_parent(dimer, boys_mode: int = BOYS_REF, conv: float = 1e-10):
    """The undisplaced water dimer, whose density warm-starts the displacements."""
    sh = build_shells(dimer, basis_mod.builtin_basis("6-31G*"), pure=True)
    with FockBuilder(schwarz_threshold=1e-12, boys_mode=boys_mode) as fb:
        fb.set_basis(sh)
        S, T, V, en = fb.one_electron(sh)
        E, D, it, rc = fb.scf(T + V, S, sh.n_electrons() // 2, en, conv=conv)
    return E, D


def serve(requests: List[Request], conv: float = 1e-10, max_iter: int = 128, boys_mode: int = BOYS_REF,
          arena_bytes: int = 0, iterations_per_step: int = 1, realtime: bool = True,
          batch: Optional[Batch] = None, mixed: bool = False, **mixed_opts) -> Dict:
    """Runs the request stream; returns per-request results and summary stats.
    realtime=True replays arrivals against the wall clock; False admits each
    request as soon as it is reached in arrival order (a closed loop).
    mixed=True iterates every molecule in the mixed-precision incremental form
    (mixed_opts: its skip_threshold, rebuild_every, final_switch)."""
    own = batch is None
    b = batch if batch is not None else Batch(schwarz_threshold=1e-12, boys_mode=boys_mode, arena_bytes=arena_bytes)
    pending = sorted(requests, key=lambda r: r.arrival)
    qi = 0
    inflight: Dict[int, tuple] = {}
    results: List[Result] = []
    waiting: List[Request] = []
    t0 = time.perf_counter()
    peak_inflight = 0
    admissions_deferred = 0
    # Host wall time of admissions and of steps, the latter split by whether the
    # batch's composition changed since the previous step (which rebuilds its
    # work lists before iterating).
    t_admit = 0.0
    step_changed: List[float] = []
    step_same: List[float] = []
    changed = True
    try:
        while qi < len(pending) or waiting or inflight:
            now = time.perf_counter() - t0
            while qi < len(pending) and (pending[qi].arrival <= now or not realtime):
                waiting.append(pending[qi])
                qi += 1
                if not realtime:
                    break
            # Admission: every waiting request that fits in the arena.
            still = []
            for r in waiting:
                try:
                    ta = time.perf_counter()
                    h = b.add(r.shells, guess=r.guess)
                    t_admit += time.perf_counter() - ta
                    changed = True
                    inflight[h] = (r, time.perf_counter() - t0)
                except Exception as e:  # arena full: wait for a slot to free up
                    if getattr(e, "code", None) == -2:
                        admissions_deferred += 1
                        still.append(r)
                    else:
                        raise
            waiting = still
            peak_inflight = max(peak_inflight, len(inflight))
            if not inflight:
                if qi < len(pending) and realtime:
                    time.sleep(max(0.0, pending[qi].arrival - (time.perf_counter() - t0)))
                continue
            ts = time.perf_counter()
            b.step(iterations_per_step, conv=conv, max_iter=max_iter, mixed=mixed, **mixed_opts)
            (step_changed if changed else step_same).append(time.perf_counter() - ts)
            changed = False
            for h in b.finished_handles():
                if h not in inflight:
                    continue
                E, _, it, st = b.result(h)
                r, adm = inflight.pop(h)
                b.remove(h)
                changed = True
                results.append(Result(r.rid, r.kind, E, it, st, r.arrival, adm, time.perf_counter() - t0))
    finally:
        if own:
            b.close()
    wall = time.perf_counter() - t0
    return _summary(results, wall, peak_inflight, admissions_deferred, t_admit, step_changed, step_same)


def _summary(results: List[Result], wall: float, peak_inflight: int, admissions_deferred: int, t_admit: float,
             step_changed: List[float], step_same: List[float]) -> Dict:
    def pct(vals, q):
        return float(np.percentile(np.array(vals), q) * 1e3) if len(vals) else None

    lat = [r.latency for r in results]
    que = [r.queue for r in results]
    svc = [r.service for r in results]
    ok = sum(1 for r in results if r.status == 0)
    return {
        "results": results,
        "solves": len(results),
        "converged": ok,
        "wall_s": wall,
        "solves_per_s": ok / wall if wall > 0 else 0.0,
        "p50_ms": pct(lat, 50),
        "p99_ms": pct(lat, 99),
        "queue_p50_ms": pct(que, 50),
        "queue_p99_ms": pct(que, 99),
        "service_p50_ms": pct(svc, 50),
        "service_p99_ms": pct(svc, 99),
        "peak_inflight": peak_inflight,
        "admissions_deferred": admissions_deferred,
        "admission_s": t_admit,
        "steps_after_change": len(step_changed),
        "step_after_change_ms": float(np.mean(step_changed) * 1e3) if step_changed else None,
        "steps_unchanged": len(step_same),
        "step_unchanged_ms": float(np.mean(step_same) * 1e3) if step_same else None,
    }


def serve_pipelined(requests: List[Request], pipelines: int = 2, conv: float = 1e-10, max_iter: int = 128,
                    boys_mode: int = BOYS_REF, arena_bytes: int = 0, mixed: bool = False, **mixed_opts) -> Dict:
    """The serving loop over `pipelines` batches, each with its own context and
    stream, stepped by its own host thread (the library calls release the
    interpreter lock).  One batch's eigensolver, DIIS and host-side rebuild
    overlap another batch's ERI launches on the GPU.  Each arrived request goes
    to the batch with the least work in flight (sum of n^2 over its molecules);
    each batch admits by its own arena (arena_bytes per batch) and retires its
    finished molecules after every step, as serve() does."""
    import threading

    batches = [Batch(schwarz_threshold=1e-12, boys_mode=boys_mode, arena_bytes=arena_bytes)
               for _ in range(pipelines)]
    pending = sorted(requests, key=lambda r: r.arrival)
    lock = threading.Lock()
    state = {"qi": 0, "peak": 0, "deferred": 0, "t_admit": 0.0}
    queues: List[List[Request]] = [[] for _ in range(pipelines)]
    load = [0] * pipelines
    inflight_count = [0] * pipelines
    results: List[Result] = []
    step_changed: List[float] = []
    step_same: List[float] = []
    errors: List[BaseException] = []
    t0 = time.perf_counter()

    def dispatch(now: float) -> None:
        # caller holds the lock
        while state["qi"] < len(pending) and pending[state["qi"]].arrival <= now:
            r = pending[state["qi"]]
            state["qi"] += 1
            k = min(range(pipelines), key=lambda j: load[j])
            queues[k].append(r)
            load[k] += r.shells.nbf() ** 2

    def worker(k: int) -> None:
        b = batches[k]
        inflight: Dict[int, tuple] = {}
        changed = True
        try:
            while True:
                with lock:
                    now = time.perf_counter() - t0
                    dispatch(now)
                    mine, queues[k] = queues[k], []
                    finished_all = state["qi"] >= len(pending)
                    next_arrival = pending[state["qi"]].arrival if state["qi"] < len(pending) else None
                still = []
                for r in mine:
                    try:
                        ta = time.perf_counter()
                        h = b.add(r.shells, guess=r.guess)
                        dt = time.perf_counter() - ta
                        inflight[h] = (r, time.perf_counter() - t0)
                        changed = True
                        with lock:
                            state["t_admit"] += dt
                    except Exception as e:  # arena full: retry after a step frees regions
                        if getattr(e, "code", None) == -2:
                            still.append(r)
                        else:
                            raise
                if still:
                    with lock:
                        state["deferred"] += len(still)
                        queues[k] = still + queues[k]
                with lock:
                    inflight_count[k] = len(inflight)
                    state["peak"] = max(state["peak"], sum(inflight_count))
                if not inflight:
                    with lock:
                        empty = not queues[k]
                    if finished_all and empty:
                        return
                    if next_arrival is not None:
                        time.sleep(max(0.0, min(0.005, next_arrival - (time.perf_counter() - t0))))
                    continue
                ts = time.perf_counter()
                b.step(1, conv=conv, max_iter=max_iter, mixed=mixed, **mixed_opts)
                dt = time.perf_counter() - ts
                out = []
                freed = 0
                for h in b.finished_handles():
                    if h not in inflight:
                        continue
                    E, _, it, st = b.result(h)
                    r, adm = inflight.pop(h)
                    b.remove(h)
                    freed += r.shells.nbf() ** 2
                    out.append(Result(r.rid, r.kind, E, it, st, r.arrival, adm, time.perf_counter() - t0))
                with lock:
                    (step_changed if changed else step_same).append(dt)
                    results.extend(out)
                    load[k] -= freed
                changed = bool(out)
        except BaseException as e:  # surfaced to the caller after the join
            with lock:
                errors.append(e)

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(pipelines)]
    try:
        for t in threads:
            t.start()
        for t in threads:
            t.join()
    finally:
        for b in batches:
            b.close()
    if errors:
        raise errors[0]
    wall = time.perf_counter() - t0
    out = _summary(results, wall, state["peak"], state["deferred"], state["t_admit"], step_changed, step_same)
    out["pipelines"] = pipelines
    return out
