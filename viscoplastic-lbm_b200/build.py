"""Build libvlbm.so in-tree for sm_100a.

Every .cu / .cpp file under csrc/ is compiled by nvcc with
`-gencode arch=compute_100a,code=sm_100a`, in parallel, into _build/, and linked
into viscoplastic-lbm_b200/libvlbm.so (static CUDA runtime).  Objects are
rebuilt when their source or any csrc/ header is newer.  The drop-in host
program driver/vlbm_run.cpp is then linked against it into
viscoplastic-lbm_b200/vlbm_run.

Usage: python viscoplastic-lbm_b200/build.py [-j N] [--force]
"""
import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libvlbm.so")
DRIVER = os.path.join(HERE, "vlbm_run")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-Wall", "-I", INCLUDE, "-I", CSRC] + ARCH


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def newest_header():
    hdrs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))
    return max((os.path.getmtime(h) for h in hdrs), default=0.0)


def compile_one(src, force, verbose_ptxas):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if not force and os.path.exists(obj):
        t = os.path.getmtime(obj)
        if t >= os.path.getmtime(src) and t >= newest_header():
            return obj, "", False
    cmd = [nvcc()] + NVCC_FLAGS + ["-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd.insert(1, "-x")
        cmd.insert(2, "cu")
    if verbose_ptxas and src.endswith(".cu"):
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr, True


def build(jobs=None, force=False, verbose_ptxas=False, quiet=False):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sources()
    jobs = jobs or max(1, min(len(srcs), os.cpu_count() or 4))
    objs, logs, changed = [], [], False
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        futs = {ex.submit(compile_one, s, force, verbose_ptxas): s for s in srcs}
        for fu in cf.as_completed(futs):
            obj, log, did = fu.result()
            objs.append(obj)
            changed |= did
            if log:
                logs.append(log)
    if changed or not os.path.exists(LIB):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + sorted(objs) + ["-lcudart_static", "-ldl", "-lrt",
                                                                        "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    drv_src = os.path.join(HERE, "driver", "vlbm_run.cpp")
    if os.path.exists(drv_src) and (not os.path.exists(DRIVER) or os.path.getmtime(DRIVER) < max(
            os.path.getmtime(LIB), os.path.getmtime(drv_src), newest_header())):
        # the drop-in host program, linked against the library next to it
        cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-I", INCLUDE, drv_src, "-o", DRIVER, "-L", HERE, "-lvlbm",
               "-Wl,-rpath,$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"driver build failed:\n{r.stdout}\n{r.stderr}")
    if not quiet:
        print(f"built {LIB} from {len(objs)} objects")
    return LIB, "\n".join(logs)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print -Xptxas -v output")
    a = ap.parse_args()
    _, log = build(a.j, a.force, a.ptxas)
    if a.ptxas:
        print(log)


if __name__ == "__main__":
    sys.exit(main())
