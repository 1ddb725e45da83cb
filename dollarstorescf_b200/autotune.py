"""Per-class kernel shape autotuner.

For every shell-quartet class with work in the current basis, times each kernel
shape the library offers for it and keeps the fastest:

  0  one thread per shell quartet, the default register budget (resident
     blocks of 128 threads per SM: 8 / 6 / 4 / 1 for total angular momentum
     L = 0 / 1..2 / 3..4 / >= 5);
  2  the same with one fewer resident block (more registers per thread, fewer
     spills, lower occupancy), L <= 4;
  3  with about half the resident blocks, L <= 4;
  1  one warp per shell quartet with shared-memory programs (the heavy classes
     compiled with it);
  4  one thread per shell quartet in persistent blocks of 8 warps that first
     stage the class's reference-mode Boys records (35 KB per order) in shared
     memory, L <= 2;
  5, 6, 7  shapes 0, 2, 3 on a one-wave grid (the blocks every SM holds at
     once, the warps striding over the tasks): slower alone, but they leave
     SMs to the classes launched beside them in a build.

With the per-class shapes fixed, the launch shape of the whole build is chosen
the same way: one launch per class, or persistent grouped launches (the
thread-per-quartet classes of L <= 2 and of L = 3..4 each in one kernel whose
warps pull warp tasks of every class of the group from a device queue), by
timing whole builds (dss_time_build / dss_batch_time_build).

Timing is per launch with CUDA events (dss_profile_build / dss_batch_profile
run the classes one after another on one stream), best of `repeats`; the
choice is then refined on whole builds (refine_whole), where the classes run
concurrently as they do in production.  The best
shape depends on the class and on its quartet count, so the choice is redone
per basis and can be cached by (class, pure, boys mode, quartet-count bucket).
"""
from __future__ import annotations

import json
import math
import os
from typing import Dict, Optional

from .engine import FockBuilder

# Kernel shapes tried per class (see the module docstring).
VARIANTS = (0, 2, 3, 1, 4, 5, 6, 7, 8)


def tune(fb: FockBuilder, D_ptr: int, J_ptr: int, K_ptr: int, repeats: int = 2,
         cache_path: Optional[str] = None, key_extra: str = "") -> Dict[str, int]:
    """Chooses a variant per class; returns {class name: variant}."""
    cache = {}
    if cache_path and os.path.isfile(cache_path):
        with open(cache_path) as f:
            cache = json.load(f)
    nc = fb.num_classes()
    infos = [fb.class_info(i) for i in range(nc)]
    names = ["%d%d%d%d" % tuple(info[0]) for info in infos]
    keys = [f"{names[i]}|{key_extra}|q{int(math.log2(max(1, infos[i][1])))}" for i in range(nc)]
    todo = [i for i in range(nc) if infos[i][1] > 0 and keys[i] not in cache]
    timings = {}
    for variant in VARIANTS if todo else ():
        ok = []
        for i in todo:
            try:
                fb.set_class_variant(i, variant)
                ok.append(i)
            except Exception:
                pass
        best = [math.inf] * nc
        for _ in range(repeats):
            ms = fb.profile_build(D_ptr, J_ptr, K_ptr)
            for i in ok:
                best[i] = min(best[i], ms[i])
        for i in ok:
            timings.setdefault(i, {})[variant] = best[i]
    choice = {}
    for i in range(nc):
        if infos[i][1] == 0:
            continue
        if keys[i] in cache:
            v = int(cache[keys[i]])
        else:
            t = timings.get(i, {0: 0.0})
            v = min(t, key=t.get)
            cache[keys[i]] = v
        fb.set_class_variant(i, v)
        choice[names[i]] = v
    if cache_path:
        with open(cache_path, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
    return choice


def _median_of(f, k: int) -> float:
    f()
    ts = sorted(f() for _ in range(k))
    return ts[k // 2]


def refine_whole(time_build, set_variant, classes, choice: Dict[str, int], repeats: int = 5,
                 passes: int = 1) -> Dict[str, object]:
    """Coordinate descent of the per-class shapes on the time of whole builds.

    The per-class timings run the classes one after another, but a build runs
    them concurrently on side streams, where a shape that wins alone can lose:
    the warp-cooperative kernels, for one, hold large shared-memory blocks that
    crowd out the light classes running beside them.  Starting from the per-class
    choice, every class (longest first) tries each of its shapes with the others
    fixed and keeps the one whose whole build is fastest (median of `repeats`).
    classes: [(index, name, [shapes])]."""
    best = _median_of(time_build, repeats)
    start = best
    for _ in range(passes):
        improved = False
        for i, name, shapes in classes:
            cur = choice[name]
            for v in shapes:
                if v == cur:
                    continue
                try:
                    set_variant(i, v)
                except Exception:
                    continue
                t = _median_of(time_build, repeats)
                if t < best * 0.995:
                    best, cur, improved = t, v, True
            set_variant(i, cur)
            choice[name] = cur
        if not improved:
            break
    return {"ms_whole_build_per_class_choice": start, "ms_whole_build": best}


def tune_whole(fb: FockBuilder, D_ptr: int, J_ptr: int, K_ptr: int, choice: Dict[str, int],
               repeats: int = 5, cache_path: Optional[str] = None) -> Dict[str, object]:
    """refine_whole for a single-molecule context (dss_time_build); updates
    choice.  With cache_path, a refined choice stored for the same work size is
    applied instead of re-timed."""
    nc = fb.num_classes()
    infos = [fb.class_info(i) for i in range(nc)]
    names = ["%d%d%d%d" % tuple(info[0]) for info in infos]
    cache = {}
    if cache_path and os.path.isfile(cache_path):
        with open(cache_path) as f:
            cache = json.load(f)
    sq, _, _ = fb.work_stats()
    key = f"whole|q{int(math.log2(max(1, sq)))}"
    if key in cache:
        for i in range(nc):
            if names[i] in cache[key]["choice"]:
                fb.set_class_variant(i, int(cache[key]["choice"][names[i]]))
                choice[names[i]] = int(cache[key]["choice"][names[i]])
        # The chosen shapes' launch times, which order the class launches of later builds.
        fb.profile_build(D_ptr, J_ptr, K_ptr)
        return dict(cache[key]["result"], cached=True)
    per = fb.profile_build(D_ptr, J_ptr, K_ptr)
    order = sorted((i for i in range(nc) if infos[i][1] > 0 and names[i] in choice), key=lambda i: -per[i])
    classes = [(i, names[i], VARIANTS) for i in order]
    out = refine_whole(lambda: fb.time_build(D_ptr, J_ptr, K_ptr), fb.set_class_variant, classes, choice, repeats)
    if cache_path:
        cache[key] = {"choice": dict(choice), "result": out}
        with open(cache_path, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
    return out


def tune_batch_whole(batch, choice: Dict[str, int], repeats: int = 3) -> Dict[str, object]:
    """refine_whole for a dss_batch (dss_batch_time_build); updates choice."""
    import ctypes

    nc = batch._L.dss_num_classes()
    ctx = batch._L.dss_batch_context(batch._h)
    per = batch.profile()
    names = {}
    for i in range(nc):
        l4 = (ctypes.c_int * 4)()
        a, b, c = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        batch._L.dss_class_info(ctx, i, l4, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
        names[i] = "%d%d%d%d" % tuple(l4)
    order = sorted((i for i in range(nc) if names[i] in choice and per[i] > 0), key=lambda i: -per[i])
    classes = [(i, names[i], VARIANTS) for i in order]
    return refine_whole(batch.time_build, batch.set_class_variant, classes, choice, repeats)


def tune_launch(fb: FockBuilder, D_ptr: int, J_ptr: int, K_ptr: int, repeats: int = 3,
                cache_path: Optional[str] = None, key_extra: str = "") -> Dict[str, object]:
    """Per-class launches or persistent grouped launches for the whole build,
    whichever times faster (best of `repeats` whole builds each).  With
    cache_path, a choice stored for the same key (the work's size bucket) is
    reused instead of timed."""
    cache = {}
    if cache_path and os.path.isfile(cache_path):
        with open(cache_path) as f:
            cache = json.load(f)
    sq, _, _ = fb.work_stats()
    key = f"launch|{key_extra}|q{int(math.log2(max(1, sq)))}"
    if key in cache:
        fb.set_persistent(bool(cache[key]["persistent"]))
        return dict(cache[key], cached=True)
    t = {}
    for on in (False, True):
        fb.set_persistent(on)
        fb.time_build(D_ptr, J_ptr, K_ptr)
        t[on] = min(fb.time_build(D_ptr, J_ptr, K_ptr) for _ in range(repeats))
    best = min(t, key=t.get)
    fb.set_persistent(best)
    out = {"persistent": best, "ms_per_class_launches": t[False], "ms_persistent": t[True]}
    if cache_path:
        cache[key] = out
        with open(cache_path, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
    return out


def tune_batch_launch(batch, repeats: int = 3) -> Dict[str, object]:
    """tune_launch for a dss_batch (FP64 accumulation over all live molecules).
    Profiles the current composition first: its class launch times order the
    class launches of later builds."""
    batch.profile()
    t = {}
    for on in (False, True):
        batch.set_persistent(on)
        batch.time_build()
        t[on] = min(batch.time_build() for _ in range(repeats))
    best = min(t, key=t.get)
    batch.set_persistent(best)
    return {"persistent": best, "ms_per_class_launches": t[False], "ms_persistent": t[True]}


def tune_batch(batch, repeats: int = 2) -> Dict[str, int]:
    """The same per-class choice for a dss_batch: times every shape of every
    class with work over all live molecules (dss_batch_profile) and keeps the
    fastest.  Returns {class name: variant}."""
    nc = batch._L.dss_num_classes()
    timings: Dict[int, Dict[int, float]] = {}
    for variant in VARIANTS:
        ok = []
        for i in range(nc):
            try:
                batch.set_class_variant(i, variant)
                ok.append(i)
            except Exception:
                pass
        best = [math.inf] * nc
        for _ in range(repeats):
            ms = batch.profile()
            for i in ok:
                best[i] = min(best[i], ms[i])
        for i in ok:
            if best[i] > 0:
                timings.setdefault(i, {})[variant] = best[i]
    choice = {}
    ctx = batch._L.dss_batch_context(batch._h)
    import ctypes

    for i, t in timings.items():
        v = min(t, key=t.get)
        batch.set_class_variant(i, v)
        l4 = (ctypes.c_int * 4)()
        a, b, c = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        batch._L.dss_class_info(ctx, i, l4, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
        choice["%d%d%d%d" % tuple(l4)] = v
    return choice
