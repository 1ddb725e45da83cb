"""Builds libdss.so (the C-ABI engine) in-tree for sm_100a.

Steps: generate the per-class ERI code (csrc/gen_eri.py) and the Boys tables
(csrc/gen_boys_tab.py) into _build/gen/, write one translation unit per
shell-quartet class plus a dispatch unit, compile them in parallel with nvcc
(-gencode arch=compute_100a,code=sm_100a -lineinfo -O3), and link
dollarstorescf_b200/libdss.so with the CUDA runtime linked statically.  The
large Boys cell table is defined once (boys_cell_data.cu) and reaches the
kernels as a pointer; whole-program compilation keeps the kernels free of
call-ABI spills that relocatable device code adds.

Usage: python -m dollarstorescf_b200.build [--lmax 2] [--jobs N]
"""
from __future__ import annotations

import argparse
import hashlib
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
ROOT = os.path.dirname(PKG)
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(ROOT, "_build")
GEN = os.path.join(BUILD, "gen")
LIB = os.path.join(PKG, "libdss.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
          "-Xptxas", "-warn-spills", "-I" + CSRC, "-I" + GEN, "-I" + INCLUDE]


def _classes(lmax: int):
    sys.path.insert(0, CSRC)
    import gen_coop  # noqa: E402
    import gen_eri  # noqa: E402

    return gen_eri.quartet_classes(lmax), gen_eri.pair_classes(lmax), gen_coop.coop_classes(lmax)


def _write_if_changed(path: str, text: str) -> None:
    if os.path.isfile(path):
        with open(path) as f:
            if f.read() == text:
                return
    with open(path, "w") as f:
        f.write(text)


def _class_tu(c, coop: bool) -> str:
    """One translation unit per class: its kernels and host launchers.
    Variants: Boys mode (0 reference, 1 accurate) x 5D/6D, the mixed-precision
    screened form with the accurate Boys function, and the unrestricted
    (two-density) form with the reference Boys function."""
    la, lb, lc, ld = c
    name = f"{la}{lb}{lc}{ld}"
    lines = [f'#include "{"coop_kernels.cuh" if coop else "eri_kernels.cuh"}"', "#include <atomic>", ""]
    combos = [(0, 1, 0), (0, 0, 0), (1, 1, 0), (1, 0, 0), (1, 1, 1), (1, 0, 1)]
    lines.append(f"void dss_launch_eri_jk_{name}(int boys, int pure, int mixed, int uhf, int tier, "
                 f"const EriArgs& a, cudaStream_t s) {{")
    tiers = la + lb + lc + ld <= 4  # dss_has_tiers
    lines.append("  // tier 4..6: tiers 0..2 on a one-wave grid (the resident blocks of every SM; the")
    lines.append("  // warps stride over the tasks), which leaves room for the classes launched beside it.")
    lines.append("  // tier 7: tier 0 on one block per SM of a third of the SMs, so that the local memory")
    lines.append("  // of a class with large per-thread arrays stays within L2 (the rest of the SMs run")
    lines.append("  // the classes beside it).")
    lines.append("  const bool third = tier == 7;")
    lines.append("  if (third) tier = 0;")
    lines.append("  const bool cap = tier >= 4;")
    lines.append("  if (cap) tier -= 4;")
    lines.append("  const int threads = 128;")
    lines.append("  unsigned blocks = (unsigned)(((long long)a.ntasks * 32 + threads - 1) / threads);")
    lines.append("  if (!blocks) return;")
    lines.append(f"  if (cap) {{ const unsigned c = (unsigned)(dss_sm_count() * dss_min_blocks_tier({la + lb + lc + ld}, "
                 f"tier)); if (blocks > c) blocks = c; }}")
    lines.append("  if (third) { const unsigned c = (unsigned)(dss_sm_count() / 3 > 0 ? dss_sm_count() / 3 : 1); "
                 "if (blocks > c) blocks = c; }")
    lines.append("  const dim3 grid(blocks, a.split > 1 ? (unsigned)a.split : 1u);")
    for boys, pure, mixed in combos:
        pb = "true" if pure else "false"
        mb = "true" if mixed else "false"
        if tiers and boys == 0 and not mixed:
            # The plain form: register tier or shared-memory shape chosen per class
            # by the autotuner (tier 3 = class variant 4; split launches keep tier 0).
            if la + lb + lc + ld <= 2:  # dss_has_smem_variant
                lines.append(f"  if (!uhf && boys == 0 && pure == {pure} && mixed == 0 && tier == 3 && a.split <= 1) "
                             f"return dss_launch_eri_smem<{la}, {lb}, {lc}, {ld}, {pb}>(a, s);")
            for t in (2, 1):
                lines.append(f"  if (!uhf && boys == 0 && pure == {pure} && mixed == 0 && tier == {t}) "
                             f"return eri_jk_kernel<{la}, {lb}, {lc}, {ld}, 0, {pb}, false, false, {t}>"
                             f"<<<grid, threads, 0, s>>>(a);")
        lines.append(f"  if (!uhf && boys == {boys} && pure == {pure} && mixed == {mixed}) "
                     f"eri_jk_kernel<{la}, {lb}, {lc}, {ld}, {boys}, {pb}, {mb}><<<grid, threads, 0, s>>>(a);")
    # The unrestricted variant: FP64 with the reference-mode Boys function.
    for pure in (1, 0):
        pb = "true" if pure else "false"
        lines.append(f"  if (uhf && pure == {pure}) "
                     f"eri_jk_kernel<{la}, {lb}, {lc}, {ld}, 0, {pb}, false, true><<<grid, threads, 0, s>>>(a);")
    lines.append("}")
    # Loads (under lazy module loading) the FP64 kernel a plain build of this
    # class launches, so that the first build allocates no code memory.
    lines.append(f"void dss_preload_eri_jk_{name}(int boys, int pure, int variant) {{")
    lines.append("  cudaFuncAttributes fa;")
    for boys in (0, 1):
        for pure in (1, 0):
            pb = "true" if pure else "false"
            if coop:
                lines.append(f"  if (variant == 1 && boys == {boys} && pure == {pure}) "
                             f"{{ cudaFuncGetAttributes(&fa, eri_coop_kernel<{la}, {lb}, {lc}, {ld}, {boys}, {pb}, false>); "
                             f"return; }}")
            if tiers and boys == 0:
                if la + lb + lc + ld <= 2:
                    lines.append(f"  if (variant == 4 && boys == 0 && pure == {pure}) {{ "
                                 f"cudaFuncGetAttributes(&fa, eri_jk_smem_kernel<{la}, {lb}, {lc}, {ld}, {pb}>); "
                                 f"return; }}")
                for t in (2, 1):
                    lines.append(f"  if (variant == {t + 1} && boys == 0 && pure == {pure}) {{ "
                                 f"cudaFuncGetAttributes(&fa, eri_jk_kernel<{la}, {lb}, {lc}, {ld}, 0, {pb}, false, "
                                 f"false, {t}>); return; }}")
            lines.append(f"  if (boys == {boys} && pure == {pure}) "
                         f"cudaFuncGetAttributes(&fa, eri_jk_kernel<{la}, {lb}, {lc}, {ld}, {boys}, {pb}, false>);")
    lines.append("}")
    if (la, lb) == (lc, ld):
        lines.append(f"void dss_launch_schwarz_{la}{lb}(int boys, int pure, const SchwarzArgs& a, cudaStream_t s) {{")
        lines.append("  const int threads = 128;")
        lines.append("  const unsigned blocks = (unsigned)(((long long)a.npair * 32 + threads - 1) / threads);")
        lines.append("  if (!blocks) return;")
        for boys in (0, 1):
            for pure in (1, 0):
                pb = "true" if pure else "false"
                lines.append(f"  if (boys == {boys} && pure == {pure}) "
                             f"schwarz_kernel<{la}, {lb}, {boys}, {pb}><<<blocks, threads, 0, s>>>(a);")
        lines.append("}")
    if coop:
        lines.append(f"void dss_launch_eri_coop_{name}(int boys, int pure, int mixed, const EriArgs& a, "
                     f"cudaStream_t s) {{")
        lines.append("  const unsigned blocks = (unsigned)(((long long)a.ntasks * DSS_COOP_SPLIT + DSS_COOP_WARPS - 1) / "
                     "DSS_COOP_WARPS);")
        lines.append("  if (!blocks) return;")
        for boys, pure, mixed in combos:
            pb = "true" if pure else "false"
            mb = "true" if mixed else "false"
            k = f"eri_coop_kernel<{la}, {lb}, {lc}, {ld}, {boys}, {pb}, {mb}>"
            sm = f"coop_smem_per_warp<{la}, {lb}, {lc}, {ld}, {pb}>() * sizeof(double) * DSS_COOP_WARPS"
            lines.append(f"  if (boys == {boys} && pure == {pure} && mixed == {mixed}) {{")
            lines.append(f"    // per device (the attribute is per context); contexts on several host")
            lines.append(f"    // threads may race here, and setting the attribute twice is harmless")
            lines.append(f"    static std::atomic<bool> attr[64] = {{}};")
            lines.append(f"    int dev = 0;")
            lines.append(f"    cudaGetDevice(&dev);")
            lines.append(f"    const size_t smem = {sm};")
            lines.append(f"    if (dev < 0 || dev >= 64 || !attr[dev].load()) {{ cudaFuncSetAttribute({k}, "
                         f"cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); "
                         f"if (dev >= 0 && dev < 64) attr[dev].store(true); }}")
            lines.append(f"    {k}<<<blocks, 32 * DSS_COOP_WARPS, smem, s>>>(a);")
            lines.append("  }")
        lines.append("}")
    return "\n".join(lines) + "\n"


# Persistent grouped launches: classes of one register budget share a kernel
# (total angular momentum L <= 2 and 3 <= L <= 4); heavier classes keep their
# own launches.  (boys, mixed) combinations: the plain FP64 form and the
# mixed-precision form.
PERSIST_GROUPS = {0: (0, 2, 6), 1: (3, 4, 4)}  # group: (L min, L max, resident blocks)
PERSIST_COMBOS = ((0, 0), (1, 1))


def persist_classes(classes, g):
    lo, hi, _ = PERSIST_GROUPS[g]
    return [c for c in classes if lo <= sum(c) <= hi]


def _persist_tu(classes, g, boys, mixed, pure) -> str:
    """One persistent kernel (group g, one Boys mode / form / function type)
    and its launcher."""
    grp = persist_classes(classes, g)
    minb = PERSIST_GROUPS[g][2]
    pb = "true" if pure else "false"
    mb = "true" if mixed else "false"
    k = f"eri_persist_g{g}_b{boys}_m{mixed}_p{pure}"
    lines = ['#include "eri_kernels.cuh"', "#include <atomic>", ""]
    lines.append(f"__global__ void __launch_bounds__(128, {minb}) {k}(PersistArgs p) {{")
    lines.append("  const int lane = threadIdx.x & 31;")
    lines.append("  const int total = p.start[p.ncls];")
    lines.append("  for (;;) {")
    lines.append("    int base = 0;")
    lines.append("    if (lane == 0) base = atomicAdd(p.head, DSS_PERSIST_CHUNK);")
    lines.append("    base = __shfl_sync(0xffffffffu, base, 0);")
    lines.append("    if (base >= total) return;")
    lines.append("    const int end = min(base + DSS_PERSIST_CHUNK, total);")
    lines.append("    for (int item = base; item < end; ++item) {")
    lines.append("      int c = 0;")
    lines.append("      while (item >= p.start[c + 1]) ++c;")
    lines.append("      const int task = item - p.start[c];")
    lines.append("      switch (p.slot[c]) {")
    for i, (la, lb, lc, ld) in enumerate(grp):
        lines.append(f"        case {i}: eri_jk_task<{la}, {lb}, {lc}, {ld}, {boys}, {pb}, {mb}, false>"
                     f"(p.a, p.tasks[c], task, lane, 0); break;")
    lines.append("        default: break;")
    lines.append("      }")
    lines.append("    }")
    lines.append("  }")
    lines.append("}")
    lines.append(f"void dss_launch_{k}(const PersistArgs& p, cudaStream_t s) {{")
    lines.append("  static std::atomic<int> grid_dev[64] = {};")
    lines.append("  int dev = 0;")
    lines.append("  cudaGetDevice(&dev);")
    lines.append("  int g = (dev >= 0 && dev < 64) ? grid_dev[dev].load() : 0;")
    lines.append("  if (!g) {")
    lines.append("    int per = 0, nsm = 0;")
    lines.append(f"    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, {k}, 128, 0);")
    lines.append("    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);")
    lines.append("    g = (per > 0 ? per : 1) * (nsm > 0 ? nsm : 1);")
    lines.append("    if (dev >= 0 && dev < 64) grid_dev[dev].store(g);")
    lines.append("  }")
    lines.append("  const long long warps = ((long long)p.start[p.ncls] + DSS_PERSIST_CHUNK - 1) / DSS_PERSIST_CHUNK;")
    lines.append("  const long long need = (warps + 3) / 4;")
    lines.append("  const unsigned blocks = (unsigned)(need < g ? need : g);")
    lines.append("  if (!blocks) return;")
    lines.append(f"  {k}<<<blocks, 128, 0, s>>>(p);")
    lines.append("}")
    lines.append(f"void dss_preload_{k}() {{")
    lines.append("  cudaFuncAttributes fa;")
    lines.append(f"  cudaFuncGetAttributes(&fa, {k});")
    lines.append("}")
    return "\n".join(lines) + "\n"


def _persist_dispatch(classes) -> str:
    lines = []
    for g in PERSIST_GROUPS:
        for boys, mixed in PERSIST_COMBOS:
            for pure in (1, 0):
                lines.append(f"void dss_launch_eri_persist_g{g}_b{boys}_m{mixed}_p{pure}(const PersistArgs& p, "
                             f"cudaStream_t s);")
                lines.append(f"void dss_preload_eri_persist_g{g}_b{boys}_m{mixed}_p{pure}();")
    lines.append("void dss_preload_persist() {")
    for g in PERSIST_GROUPS:
        for boys, mixed in PERSIST_COMBOS:
            for pure in (1, 0):
                lines.append(f"  dss_preload_eri_persist_g{g}_b{boys}_m{mixed}_p{pure}();")
    lines.append("}")
    lines.append("int dss_persist_group(int la, int lb, int lc, int ld) {")
    for g in PERSIST_GROUPS:
        for i, (la, lb, lc, ld) in enumerate(persist_classes(classes, g)):
            lines.append(f"  if (la == {la} && lb == {lb} && lc == {lc} && ld == {ld}) return {g * 100 + i};")
    lines.append("  return -1;")
    lines.append("}")
    lines.append("bool dss_launch_persist(int group, int boys, int pure, int mixed, const PersistArgs& p, "
                 "cudaStream_t s) {")
    for g in PERSIST_GROUPS:
        for boys, mixed in PERSIST_COMBOS:
            for pure in (1, 0):
                lines.append(f"  if (group == {g} && boys == {boys} && mixed == {mixed} && pure == {pure}) "
                             f"{{ dss_launch_eri_persist_g{g}_b{boys}_m{mixed}_p{pure}(p, s); return true; }}")
    lines.append("  return false;")
    lines.append("}")
    return "\n".join(lines) + "\n"


def _dispatch_tu(classes, pcls, coop) -> str:
    lines = ['#include "eri_kernels.cuh"', ""]
    for (la, lb, lc, ld) in coop:
        lines.append(f"void dss_launch_eri_coop_{la}{lb}{lc}{ld}(int boys, int pure, int mixed, const EriArgs& a, "
                     f"cudaStream_t s);")
    lines.append("bool dss_has_coop(int la, int lb, int lc, int ld) {")
    for (la, lb, lc, ld) in coop:
        lines.append(f"  if (la == {la} && lb == {lb} && lc == {lc} && ld == {ld}) return true;")
    lines.append("  return false;")
    lines.append("}")
    lines.append("void dss_launch_eri_variant(int la, int lb, int lc, int ld, int boys, int pure, int mixed, int uhf, "
                 "int variant, const EriArgs& a, cudaStream_t s) {")
    for (la, lb, lc, ld) in coop:
        lines.append(f"  if (!uhf && variant == 1 && la == {la} && lb == {lb} && lc == {lc} && ld == {ld}) "
                     f"return dss_launch_eri_coop_{la}{lb}{lc}{ld}(boys, pure, mixed, a, s);")
    lines.append("  dss_launch_eri_jk(la, lb, lc, ld, boys, pure, mixed, uhf, variant >= 2 ? variant - 1 : 0, a, s);")
    lines.append("}")
    for (la, lb, lc, ld) in classes:
        lines.append(f"void dss_preload_eri_jk_{la}{lb}{lc}{ld}(int boys, int pure, int variant);")
    lines.append("void dss_preload_eri_variant(int la, int lb, int lc, int ld, int boys, int pure, int variant) {")
    lines.append("  if (variant == 5 || variant == 8) variant = 0;  // capped grids: same kernels")
    lines.append("  else if (variant >= 6) variant -= 3;")
    for (la, lb, lc, ld) in classes:
        lines.append(f"  if (la == {la} && lb == {lb} && lc == {lc} && ld == {ld}) "
                     f"return dss_preload_eri_jk_{la}{lb}{lc}{ld}(boys, pure, variant);")
    lines.append("}")
    for (la, lb) in pcls:
        lines.append(f"void dss_launch_schwarz_{la}{lb}(int boys, int pure, const SchwarzArgs& a, cudaStream_t s);")
    lines.append("void dss_launch_schwarz(int la, int lb, int boys, int pure, const SchwarzArgs& a, cudaStream_t s) {")
    for (la, lb) in pcls:
        lines.append(f"  if (la == {la} && lb == {lb}) return dss_launch_schwarz_{la}{lb}(boys, pure, a, s);")
    lines.append("}")
    lines.append(_persist_dispatch(classes))
    lines.append("void dss_launch_eri_jk(int la, int lb, int lc, int ld, int boys, int pure, int mixed, int uhf, "
                 "int tier, const EriArgs& a, cudaStream_t s) {")
    for (la, lb, lc, ld) in classes:
        lines.append(f"  if (la == {la} && lb == {lb} && lc == {lc} && ld == {ld}) "
                     f"return dss_launch_eri_jk_{la}{lb}{lc}{ld}(boys, pure, mixed, uhf, tier, a, s);")
    lines.append("}")
    return "\n".join(lines) + "\n"


def _stamp(paths, extra: str) -> str:
    h = hashlib.sha1(extra.encode())
    for p in paths:
        with open(p, "rb") as f:
            h.update(f.read())
    return h.hexdigest()


def build(lmax: int = 2, jobs: int = 0, verbose: bool = False) -> str:
    os.makedirs(GEN, exist_ok=True)
    obj_dir = os.path.join(BUILD, "obj")
    os.makedirs(obj_dir, exist_ok=True)
    eri_gen = os.path.join(GEN, "eri_gen.cuh")
    boys_tab = os.path.join(GEN, "boys_tab.cuh")
    boys_data = os.path.join(GEN, "boys_cell_data.cu")
    gen_stamp = os.path.join(GEN, "stamp")
    want = _stamp([os.path.join(CSRC, "gen_eri.py"), os.path.join(CSRC, "gen_boys_tab.py"),
                   os.path.join(CSRC, "gen_coop.py"), os.path.join(CSRC, "gen_grad.py")], str(lmax))
    have = open(gen_stamp).read() if os.path.isfile(gen_stamp) else ""
    sph_tab = os.path.join(GEN, "sph_tab.h")
    coop_gen = os.path.join(GEN, "coop_gen.cuh")
    grad_gen = os.path.join(GEN, "grad_gen.cuh")
    if have != want or not all(os.path.isfile(x) for x in (eri_gen, boys_tab, boys_data, sph_tab, coop_gen, grad_gen)):
        subprocess.check_call([sys.executable, os.path.join(CSRC, "gen_eri.py"), eri_gen, str(lmax)])
        subprocess.check_call([sys.executable, os.path.join(CSRC, "gen_boys_tab.py"), boys_tab, boys_data])
        subprocess.check_call([sys.executable, os.path.join(CSRC, "gen_coop.py"), coop_gen, str(lmax)])
        subprocess.check_call([sys.executable, os.path.join(CSRC, "gen_grad.py"), grad_gen, str(lmax)])
        with open(gen_stamp, "w") as f:
            f.write(want)
    classes, pcls, coop = _classes(lmax)
    units = []
    for c in classes:
        p = os.path.join(GEN, "eri_class_%d%d%d%d.cu" % c)
        _write_if_changed(p, _class_tu(c, c in coop))
        units.append(p)
    persist_units = set()
    for g in PERSIST_GROUPS:
        for boys, mixed in PERSIST_COMBOS:
            for pure in (1, 0):
                name = f"eri_persist_g{g}_b{boys}_m{mixed}_p{pure}.cu"
                p = os.path.join(GEN, name)
                _write_if_changed(p, _persist_tu(classes, g, boys, mixed, pure))
                units.append(p)
                persist_units.add(name)
    p = os.path.join(GEN, "eri_dispatch.cu")
    _write_if_changed(p, _dispatch_tu(classes, pcls, coop))
    units.append(p)
    units.append(boys_data)
    for name in sorted(os.listdir(CSRC)):
        if name.endswith(".cu"):
            units.append(os.path.join(CSRC, name))
    headers = [os.path.join(CSRC, n) for n in sorted(os.listdir(CSRC)) if n.endswith((".cuh", ".h"))]
    headers += [eri_gen, boys_tab, sph_tab, coop_gen, grad_gen, os.path.join(INCLUDE, "dss.h")]
    all_stamp = _stamp(headers, " ".join(CFLAGS + ARCH))
    # The generated class units only see the kernel headers.
    kernel_headers = [os.path.join(CSRC, n) for n in ("eri_kernels.cuh", "common.cuh", "boys.cuh")]
    kernel_stamp = _stamp(kernel_headers + [eri_gen, boys_tab], " ".join(CFLAGS + ARCH))
    coop_stamp = _stamp(kernel_headers + [eri_gen, boys_tab, coop_gen, os.path.join(CSRC, "coop_kernels.cuh")],
                        " ".join(CFLAGS + ARCH))
    coop_units = {"eri_class_%d%d%d%d.cu" % c for c in coop}

    def compile_one(src: str) -> str:
        obj = os.path.join(obj_dir, os.path.basename(src) + ".o")
        stamp = obj + ".stamp"
        base = os.path.basename(src)
        if base in coop_units:
            hdr = coop_stamp
        elif base.startswith("eri_class_") or base in persist_units:
            hdr = kernel_stamp
        else:
            hdr = all_stamp
        key = hdr + _stamp([src], "")
        if os.path.isfile(obj) and os.path.isfile(stamp) and open(stamp).read() == key:
            return obj
        cmd = [NVCC] + ARCH + CFLAGS + ["-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr[-6000:]}")
        if verbose and r.stderr.strip():
            print(r.stderr)
        with open(stamp, "w") as f:
            f.write(key)
        return obj

    jobs = jobs or max(1, os.cpu_count() or 1)
    with ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(compile_one, units))
    # Link beside the library and rename, so that a reader never sees a partly written file.
    tmp = LIB + ".tmp"
    cmd = [NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-cudart", "static", "-lpthread"]
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--lmax", type=int, default=2)
    ap.add_argument("--jobs", type=int, default=0)
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.lmax, a.jobs, a.verbose))


if __name__ == "__main__":
    main()
