"""Build libvoxfea.so in-tree for sm_100a (nvcc cross-compiles; no GPU needed).

    python -m voxelsim_fea_b200.build [--force] [--verbose-ptxas]

Each ``csrc/*.cu`` is compiled to an object under ``_build/`` (in parallel,
skipped when newer than its sources), then linked into
``voxelsim_fea_b200/libvoxfea.so`` with the CUDA runtime linked statically.
"""

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(REPO, "_build")
LIB = os.path.join(HERE, "libvoxfea.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr",
          "-I", os.path.join(REPO, "include")]


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libvoxfea")


def _deps():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        [os.path.join(REPO, "include", "voxfea.h")]


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build(force=False, verbose_ptxas=False, quiet=True):
    os.makedirs(BUILD, exist_ok=True)
    cu = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    deps = _deps()
    cc = nvcc()
    jobs = []
    objs = []
    for src in cu:
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + deps):
            cmd = [cc, *ARCH, *CFLAGS, "-c", src, "-o", obj]
            if verbose_ptxas:
                cmd += ["-Xptxas", "-v"]
            jobs.append((src, cmd))

    def run(job):
        src, cmd = job
        p = subprocess.run(cmd, capture_output=True, text=True)
        return src, p

    failed = []
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
            for src, p in ex.map(run, jobs):
                if p.returncode != 0:
                    failed.append((src, p.stderr))
                elif verbose_ptxas or not quiet:
                    sys.stderr.write(p.stderr)
    if failed:
        msg = "\n".join(f"--- {s}\n{e}" for s, e in failed)
        raise RuntimeError(f"nvcc failed:\n{msg}")
    if force or jobs or _stale(LIB, objs):
        cmd = [cc, *ARCH, "-shared", "-o", LIB, *objs, "-cudart", "static", "-lpthread", "-ldl", "-lrt"]
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError(f"link failed:\n{p.stderr}")
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose_ptxas=a.verbose_ptxas, quiet=False))


if __name__ == "__main__":
    main()
