"""Builds the CUDA backend's shared library (_build/libowec.so) from csrc/ with nvcc for sm_100a.

Objects are rebuilt only when a source or header is newer than them. The CUDA runtime is linked
statically, so the library needs only the driver on the machine that loads it.
"""
import concurrent.futures
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(OUT, "libowec.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include"),
         "--expt-relaxed-constexpr"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    raise RuntimeError("nvcc not found")


def _newest_header():
    hs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    return max(os.path.getmtime(h) for h in hs)


def build(verbose=True, ptxas_info=False):
    os.makedirs(OUT, exist_ok=True)
    nvcc = _nvcc()
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdr = _newest_header()
    jobs = []
    objs = []
    for src in sources:
        obj = os.path.join(OUT, os.path.basename(src).replace(".cu", ".o"))
        objs.append(obj)
        if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr):
            continue
        cmd = [nvcc] + ARCH + FLAGS + (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", src, "-o", obj]
        jobs.append(cmd)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    failed = []
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, len(jobs))) as ex:
        for cmd, r in ex.map(run, jobs):
            if verbose:
                print("nvcc", os.path.basename(cmd[-3]), "->", "ok" if r.returncode == 0 else "FAILED", flush=True)
            if r.returncode != 0:
                failed.append((cmd, r.stdout + r.stderr))
            elif ptxas_info:
                sys.stdout.write(r.stderr)
    if failed:
        msg = "\n".join(" ".join(c) + "\n" + out for c, out in failed)
        raise RuntimeError("CUDA compilation failed:\n" + msg)
    if jobs or not os.path.exists(LIB):
        # linked under another name and renamed over the library in one step, so that a process
        # loading it (or a copy of the tree) never sees a partly written file
        tmp = LIB + ".partial"
        cmd = [nvcc] + ARCH + ["-shared", "-cudart", "static", "-o", tmp] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(ptxas_info="--ptxas" in sys.argv)
    print(LIB)
