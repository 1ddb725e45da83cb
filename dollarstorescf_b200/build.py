"""Builds libdss.so (the C-ABI engine) in-tree for sm_100a.

Steps: generate the per-class ERI code (csrc/gen_eri.py) and the Boys table
(csrc/gen_boys_tab.py) into _build/gen/, write one translation unit per
shell-quartet class plus a dispatch unit, compile them in parallel with nvcc
(-gencode arch=compute_100a,code=sm_100a -lineinfo -O3), and link
dollarstorescf_b200/libdss.so with the CUDA runtime linked statically.

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
    import gen_eri  # noqa: E402

    return gen_eri.quartet_classes(lmax), gen_eri.pair_classes(lmax)


def _write_if_changed(path: str, text: str) -> None:
    if os.path.isfile(path):
        with open(path) as f:
            if f.read() == text:
                return
    with open(path, "w") as f:
        f.write(text)


def _class_tu(c) -> str:
    la, lb, lc, ld = c
    name = f"{la}{lb}{lc}{ld}"
    lines = [f'#include "eri_kernels.cuh"', ""]
    lines.append(f"void dss_launch_eri_jk_{name}(int boys, int pure, const EriArgs& a, cudaStream_t s) {{")
    lines.append("  const int threads = 128;")
    lines.append("  const unsigned blocks = (unsigned)(((long long)a.ntasks * 32 + threads - 1) / threads);")
    lines.append("  if (!blocks) return;")
    for boys in (0, 1):
        for pure in (1, 0):
            pb = "true" if pure else "false"
            lines.append(f"  if (boys == {boys} && pure == {pure}) "
                         f"eri_jk_kernel<{la}, {lb}, {lc}, {ld}, {boys}, {pb}><<<blocks, threads, 0, s>>>(a);")
    lines.append("}")
    if (la, lb) == (lc, ld):
        lines.append(f"void dss_launch_schwarz_{la}{lb}(int boys, int pure, const SchwarzArgs& a, cudaStream_t s) {{")
        lines.append("  const int threads = 128;")
        lines.append("  const unsigned blocks = (unsigned)((a.npair + threads - 1) / threads);")
        lines.append("  if (!blocks) return;")
        for boys in (0, 1):
            for pure in (1, 0):
                pb = "true" if pure else "false"
                lines.append(f"  if (boys == {boys} && pure == {pure}) "
                             f"schwarz_kernel<{la}, {lb}, {boys}, {pb}><<<blocks, threads, 0, s>>>(a);")
        lines.append("}")
    return "\n".join(lines) + "\n"


def _dispatch_tu(classes, pcls) -> str:
    lines = ['#include "eri_kernels.cuh"', ""]
    for (la, lb) in pcls:
        lines.append(f"void dss_launch_schwarz_{la}{lb}(int boys, int pure, const SchwarzArgs& a, cudaStream_t s);")
    lines.append("void dss_launch_schwarz(int la, int lb, int boys, int pure, const SchwarzArgs& a, cudaStream_t s) {")
    for (la, lb) in pcls:
        lines.append(f"  if (la == {la} && lb == {lb}) return dss_launch_schwarz_{la}{lb}(boys, pure, a, s);")
    lines.append("}")
    lines.append("void dss_launch_eri_jk(int la, int lb, int lc, int ld, int boys, int pure, const EriArgs& a, "
                 "cudaStream_t s) {")
    for (la, lb, lc, ld) in classes:
        lines.append(f"  if (la == {la} && lb == {lb} && lc == {lc} && ld == {ld}) "
                     f"return dss_launch_eri_jk_{la}{lb}{lc}{ld}(boys, pure, a, s);")
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
    gen_stamp = os.path.join(GEN, "stamp")
    want = _stamp([os.path.join(CSRC, "gen_eri.py"), os.path.join(CSRC, "gen_boys_tab.py")], str(lmax))
    have = open(gen_stamp).read() if os.path.isfile(gen_stamp) else ""
    sph_tab = os.path.join(GEN, "sph_tab.h")
    if have != want or not all(os.path.isfile(x) for x in (eri_gen, boys_tab, sph_tab)):
        subprocess.check_call([sys.executable, os.path.join(CSRC, "gen_eri.py"), eri_gen, str(lmax)])
        subprocess.check_call([sys.executable, os.path.join(CSRC, "gen_boys_tab.py"), boys_tab])
        with open(gen_stamp, "w") as f:
            f.write(want)
    classes, pcls = _classes(lmax)
    units = []
    for c in classes:
        p = os.path.join(GEN, "eri_class_%d%d%d%d.cu" % c)
        _write_if_changed(p, _class_tu(c))
        units.append(p)
    p = os.path.join(GEN, "eri_dispatch.cu")
    _write_if_changed(p, _dispatch_tu(classes, pcls))
    units.append(p)
    for name in sorted(os.listdir(CSRC)):
        if name.endswith(".cu"):
            units.append(os.path.join(CSRC, name))
    headers = [os.path.join(CSRC, n) for n in sorted(os.listdir(CSRC)) if n.endswith((".cuh", ".h"))]
    headers += [eri_gen, boys_tab, sph_tab, os.path.join(INCLUDE, "dss.h")]
    all_stamp = _stamp(headers, " ".join(CFLAGS + ARCH))
    # The generated class units only see the kernel headers.
    kernel_headers = [os.path.join(CSRC, n) for n in ("eri_kernels.cuh", "common.cuh", "boys.cuh")]
    kernel_stamp = _stamp(kernel_headers + [eri_gen, boys_tab], " ".join(CFLAGS + ARCH))

    def compile_one(src: str) -> str:
        obj = os.path.join(obj_dir, os.path.basename(src) + ".o")
        stamp = obj + ".stamp"
        hdr = kernel_stamp if os.path.basename(src).startswith("eri_class_") else all_stamp
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
    cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-cudart", "static", "-lpthread"]
    subprocess.check_call(cmd)
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
