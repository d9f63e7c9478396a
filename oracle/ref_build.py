"""Build the reference's own CUDA program, once per case of ref_cases.py (test infrastructure).

The reference is one CUDA program configured at compile time (var.h, NNF/nnf.h,
IBM/ibmVar.h, IBM/ibmBoundaryCondition.h) and built by compile.sh from every
source of src/CUDA (compile.sh:17-24).  This recipe compiles those sources
where they lie in the reference tree, unmodified, for sm_100a:

* configuration: each of the four configuration headers starts with an include
  guard (`__VAR_H`, `__NNF_H`, `__IBM_VAR_H`, `__IBM_BC_H`).  The recipe writes
  configured copies of them into a scratch folder (text substitutions on the
  reference's own header, each of which must match exactly once) and passes
  them with `-include`, so the guard is set before any source includes the
  original and the original's body is skipped;
* builder: compile.sh compiles the builder file placed in src/CUDA
  (closedBoxBounceBack.cu); here the chosen file of boundaryConditionsBuilders/
  is compiled in its place, or the single-face harness builder of this folder;
* BGK: the collision snippet collisionSchemes/collisionForceNoReg.txt is pasted
  over the regularized collision of lbm.cu (the procedure of doc/updating.md:28-32)
  inside a scratch translation unit, with T_OMEGA, TT_OMEGA and a 7-argument
  gpu_force_term that the snippet uses and the reference does not define;
* simCheckpoint.cu calls std::mkdir(std::string, mode_t) (simCheckpoint.cu:38),
  which no standard header declares: a forced-include shim supplies it;
* particles: createParticles (IBM/ibmParticlesCreation.cpp) is replaced by
  ref_particles.cpp of this folder, which places the case's spheres.

Flags as compile.sh: -rdc=true -O3 --restrict, -lcudadevrt -lcurand, with
`-gencode arch=compute_100a,code=sm_100a`.  Objects are compiled in parallel.
Every case is built twice: with the reference's default dfloat = float
(SINGLE_PRECISION, var.h:18) and with dfloat = double (DOUBLE_PRECISION), the
latter to compare the FP64 oracle with the reference's own FP64 arithmetic.
Outputs go to oracle/_ref/<case>/ (git-ignored): the programs `refsim` and
`refsim_f64` and their stamps; scratch folders are removed after a successful
build.

Usage: python oracle/ref_build.py [--reference DIR] [--case NAME ...] [--force] [-j N]
The reference folder defaults to $VLBM_REFERENCE_ROOT, else /root/reference.
"""
import argparse
import concurrent.futures as cf
import glob
import hashlib
import json
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
sys.path.insert(0, HERE)
import ref_cases  # noqa: E402

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-rdc=true", "-O3", "--restrict", "-w"] + ARCH


def nvcc():
    p = "/usr/local/cuda/bin/nvcc"
    return p if os.path.exists(p) else "nvcc"


def _fmt(v):
    return repr(float(v))


def subst(text, pattern, repl, what):
    """Replace the single line matching `pattern` (multiline regex)."""
    new, n = re.subn(pattern, repl, text, flags=re.M)
    if n != 1:
        raise RuntimeError(f"reference header changed: pattern for {what} matched {n} times")
    return new


def gen_var_h(src, c, case, precision="f32"):
    t = src
    if precision == "f64":
        t = subst(t, r"^#define SINGLE_PRECISION\b.*$", "#define DOUBLE_PRECISION", "precision")
    t = subst(t, r"^#define D3Q19\b.*$", f"#define D3Q{c['q']}", "velocity set")
    t = subst(t, r"^#define IBM\s*$", "#define IBM" if c.get("spheres") else "/* IBM off */", "IBM")
    t = subst(t, r"^// #define POWERLAW\s*$", "#define POWERLAW" if c["rheo"] == "powerlaw" else "", "POWERLAW")
    t = subst(t, r"^// #define BINGHAM\s*$", "#define BINGHAM" if c["rheo"] == "bingham" else "", "BINGHAM")
    t = subst(t, r'^#define ID_SIM\s+".*".*$', f'#define ID_SIM "{case}"', "ID_SIM")
    t = subst(t, r'^#define PATH_FILES\s+".*".*$', '#define PATH_FILES "out"', "PATH_FILES")
    t = subst(t, r"^constexpr int N_STEPS = .*$", f"constexpr int N_STEPS = {int(c['steps'])};", "N_STEPS")
    t = subst(t, r"^constexpr int NX = .*$", f"constexpr int NX = {c['nx']};", "NX")
    t = subst(t, r"^constexpr int NY = .*$", f"constexpr int NY = {c['ny']};", "NY")
    t = subst(t, r"^constexpr int NZ = .*$", f"constexpr int NZ = {c['nz']}/N_GPUS;", "NZ")
    t = subst(t, r"^constexpr dfloat U_MAX = .*$", f"constexpr dfloat U_MAX = {_fmt(c['u_max'])};", "U_MAX")
    t = subst(t, r"^constexpr dfloat TAU = .*$", f"constexpr dfloat TAU = {_fmt(c['tau'])};", "TAU")
    for ax in ("X", "Y", "Z"):
        t = subst(t, rf"^constexpr dfloat F{ax} = .*$",
                  f"constexpr dfloat F{ax} = {_fmt(c['f' + ax.lower()])};", "F" + ax)
    if "rho_bc" in c:
        vals = ", ".join(_fmt(v) for v in c["rho_bc"])
        t = subst(t, r"^__device__ const dfloat RHO_BC\[8\] = .*$", f"__device__ const dfloat RHO_BC[8] = {{ {vals} }};",
                  "RHO_BC")
    # every scheme the cases use; interpolated bounce-back needs the duct macros and stays off
    for name in ("FREE_SLIP", "PRES_ZOU_HE", "VEL_ZOU_HE", "VEL_BOUNCE_BACK"):
        t = subst(t, rf"^#define COMP_{name} false.*$", f"#define COMP_{name} true", "COMP_" + name)
    return t


def gen_nnf_h(src, c):
    t = src
    if c["rheo"] == "powerlaw":
        t = subst(t, r"^constexpr dfloat N_INDEX = .*$", f"constexpr dfloat N_INDEX = {_fmt(c['n_index'])};",
                  "N_INDEX")
        t = subst(t, r"^constexpr dfloat K_CONSISTENCY = .*$",
                  f"constexpr dfloat K_CONSISTENCY = {_fmt(c['k'])};", "K_CONSISTENCY")
    if c["rheo"] == "bingham":
        t = subst(t, r"^constexpr dfloat ETA_P = .*$", f"constexpr dfloat ETA_P = {_fmt(c['eta_p'])};", "ETA_P")
        t = subst(t, r"^constexpr dfloat S_Y = .*$", f"constexpr dfloat S_Y = {_fmt(c['s_y'])};", "S_Y")
    return t


def gen_ibm_var_h(src, c):
    t = src
    ibm = c.get("ibm", {})
    sph = c.get("spheres") or [(20.0, 0, 0, 0)]
    t = subst(t, r"^#define NUM_PARTICLES .*$", f"#define NUM_PARTICLES {len(sph)}", "NUM_PARTICLES")
    t = subst(t, r"^#define IBM_MAX_ITERATION .*$", f"#define IBM_MAX_ITERATION {ibm.get('iterations', 1)}",
              "IBM_MAX_ITERATION")
    t = subst(t, r"^#define PARTICLE_DIAMETER .*$", f"#define PARTICLE_DIAMETER ({_fmt(sph[0][0])})",
              "PARTICLE_DIAMETER")
    t = subst(t, r"^#define IBM_PARTICLES_SAVE .*$", "#define IBM_PARTICLES_SAVE (0)", "IBM_PARTICLES_SAVE")
    t = subst(t, r"^#define IBM_DATA_REPORT .*$", "#define IBM_DATA_REPORT (0)", "IBM_DATA_REPORT")
    t = subst(t, r"^constexpr dfloat PARTICLE_DENSITY = .*$",
              f"constexpr dfloat PARTICLE_DENSITY = {_fmt(ibm.get('density', 2.0))};", "PARTICLE_DENSITY")
    for ax in ("X", "Y", "Z"):
        t = subst(t, rf"^constexpr dfloat G{ax} = .*$",
                  f"constexpr dfloat G{ax} = {_fmt(ibm.get('g' + ax.lower(), 0.0))};", "G" + ax)
    return t


def gen_ibm_bc_h(src, c):
    t = src
    walls = c.get("ibm", {}).get("walls", (0, 1, 0))
    for ax, wall in zip(("X", "Y", "Z"), walls):
        want_wall, want_per = ("", "//") if wall else ("//", "")
        t = subst(t, rf"^\s*(//)?\s*#define IBM_BC_{ax}_WALL\s*$", f"{want_wall}#define IBM_BC_{ax}_WALL",
                  f"IBM_BC_{ax}_WALL")
        t = subst(t, rf"^\s*(//)?\s*#define IBM_BC_{ax}_PERIODIC\s*$", f"{want_per}#define IBM_BC_{ax}_PERIODIC",
                  f"IBM_BC_{ax}_PERIODIC")
    return t


MKDIR_SHIM = """#pragma once
#include <string>
#include <sys/stat.h>
#include <sys/types.h>
namespace std { inline int mkdir(const std::string& p, mode_t m) { return ::mkdir(p.c_str(), m); } }
"""

BGK_OPEN = """    { /* BGK collision (collisionSchemes/collisionForceNoReg.txt) in place of the regularized one */
#define T_OMEGA (1 - OMEGA)
#define TT_OMEGA (1 - 0.5*OMEGA)
#define gpu_force_term(wi, a, b, c, fx, fy, fz) ((wi) * ((fx)*(a) + (fy)*(b) + (fz)*(c)))
"""
BGK_CLOSE = """
#undef gpu_force_term
    }
"""


def gen_bgk_lbm(ref_cuda):
    lines = open(os.path.join(ref_cuda, "lbm.cu")).read().split("\n")
    a = [i for i, l in enumerate(lines) if "// Calculate regularization terms" in l]
    b = [i for i, l in enumerate(lines) if "// Save post collision populations of boundary conditions nodes" in l]
    if len(a) != 1 or len(b) != 1 or not a[0] < b[0]:
        raise RuntimeError("lbm.cu changed: collision paste markers not found once")
    snippet = open(os.path.join(ref_cuda, "collisionSchemes", "collisionForceNoReg.txt")).read()
    return "\n".join(lines[:a[0]]) + "\n" + BGK_OPEN + snippet + BGK_CLOSE + "\n".join(lines[b[0]:])


def source_list(ref_cuda, c, scratch, precision="f32"):
    """compile.sh:17-24 file list, with the builder, lbm.cu and particle creation
    swapped as configured.  The FP64 build leaves out AuxFunctions/ (density
    correction, var.h:37, off): its reduction kernels take float* whatever
    dfloat is, so they compile only with dfloat = float, and nothing else
    calls them."""
    pats = ["IBM/*.cu", "IBM/*.cpp", "IBM/structs/*.cpp", "IBM/structs/*.cu", "IBM/collision/*.cu",
            "AuxFunctions/*.cu", "*.cu", "*.cpp", "boundaryConditionsSchemes/*.cu"]
    if precision == "f64":
        pats.remove("AuxFunctions/*.cu")
    srcs = []
    for p in pats:
        srcs += sorted(glob.glob(os.path.join(ref_cuda, p)))
    srcs = [s for s in srcs if os.path.basename(s) != "closedBoxBounceBack.cu"]
    b = c["builder"]
    if b.startswith("harness:"):
        srcs.append(os.path.join(HERE, "ref_harness_builder.cu"))
    else:
        srcs.append(os.path.join(ref_cuda, "boundaryConditionsBuilders", b + ".cu"))
    if c["op"] == "bgk":
        srcs = [s for s in srcs if os.path.relpath(s, ref_cuda) != "lbm.cu"]
        p = os.path.join(scratch, "lbm_bgk.cu")
        with open(p, "w") as f:
            f.write(gen_bgk_lbm(ref_cuda))
        srcs.append(p)
    if c.get("spheres"):
        srcs = [s for s in srcs if os.path.relpath(s, ref_cuda) != os.path.join("IBM", "ibmParticlesCreation.cpp")]
        srcs.append(os.path.join(HERE, "ref_particles.cpp"))
    return srcs


def case_stamp(case, ref_cuda, precision):
    c = {k: v for k, v in ref_cases.CASES[case].items() if k not in ("oracle", "lib_builder")}
    c["precision"] = precision
    h = hashlib.sha256(json.dumps(c, sort_keys=True, default=str).encode())
    for f in (__file__, os.path.join(HERE, "ref_harness_builder.cu"), os.path.join(HERE, "ref_particles.cpp")):
        if os.path.exists(f):
            h.update(open(f, "rb").read())
    h.update(ref_cuda.encode())
    return h.hexdigest()


def harness_defines(c):
    b = c["builder"]
    if not b.startswith("harness:"):
        return []
    _, face, scheme = b.split(":")
    return [f"-DHARNESS_FACE={face}", f"-DHARNESS_SCHEME={scheme}"]


def gen_spheres_h(c):
    """ref_spheres.h for ref_particles.cpp: the case's spheres as one list
    (a header, since nvcc splits -D values at commas)."""
    flat = ", ".join(f"{float(d)!r}, {float(x)!r}, {float(y)!r}, {float(z)!r}" for d, x, y, z in c["spheres"])
    return f"#pragma once\n#define REF_SPHERES {flat}\n"


def build_case(case, ref_root, force=False, jobs=None, log=print, precision="f32"):
    """Build the case with dfloat = float (var.h's SINGLE_PRECISION, the
    reference's default: oracle/_ref/<case>/refsim) or double
    (DOUBLE_PRECISION: refsim_f64)."""
    c = ref_cases.CASES[case]
    ref_cuda = os.path.join(ref_root, "src", "CUDA")
    outdir = os.path.join(OUT, case)
    suffix = "" if precision == "f32" else "_" + precision
    exe = os.path.join(outdir, "refsim" + suffix)
    stamp_file = os.path.join(outdir, "stamp" + suffix)
    stamp = case_stamp(case, ref_cuda, precision)
    if not force and os.path.exists(exe) and os.path.exists(stamp_file) and open(stamp_file).read() == stamp:
        return exe
    scratch = os.path.join(outdir, "scratch" + suffix)
    if os.path.isdir(scratch):
        shutil.rmtree(scratch)
    gen = os.path.join(scratch, "gen")
    os.makedirs(os.path.join(gen, "NNF"))
    os.makedirs(os.path.join(gen, "IBM"))
    objdir = os.path.join(scratch, "obj")
    os.makedirs(objdir)
    rd = lambda p: open(os.path.join(ref_cuda, p)).read()  # noqa: E731
    files = {
        "var.h": gen_var_h(rd("var.h"), c, case, precision),
        os.path.join("NNF", "nnf.h"): gen_nnf_h(rd(os.path.join("NNF", "nnf.h")), c),
        os.path.join("IBM", "ibmBoundaryCondition.h"): gen_ibm_bc_h(rd(os.path.join("IBM", "ibmBoundaryCondition.h")),
                                                                    c),
        os.path.join("IBM", "ibmVar.h"): gen_ibm_var_h(rd(os.path.join("IBM", "ibmVar.h")), c),
        "mkdir_shim.h": MKDIR_SHIM,
    }
    if c.get("spheres"):
        files["ref_spheres.h"] = gen_spheres_h(c)
    for name, text in files.items():
        with open(os.path.join(gen, name), "w") as f:
            f.write(text)
    pre = []
    for name in ("mkdir_shim.h", "var.h", os.path.join("NNF", "nnf.h"), os.path.join("IBM", "ibmBoundaryCondition.h"),
                 os.path.join("IBM", "ibmVar.h")):
        pre += ["-include", os.path.join(gen, name)]
    incs = ["-I", gen, "-I", ref_cuda, "-I", os.path.join(ref_cuda, "IBM")]
    defs = harness_defines(c)
    srcs = source_list(ref_cuda, c, scratch, precision)

    def one(src):
        obj = os.path.join(objdir, hashlib.md5(src.encode()).hexdigest()[:10] + "_" + os.path.basename(src) + ".o")
        cmd = [nvcc()] + FLAGS + pre + incs + defs + ["-dc", src, "-o", obj]
        if src.endswith(".cpp"):
            cmd[1:1] = ["-x", "cu"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr[-4000:]}")
        return obj

    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        objs = list(ex.map(one, srcs))
    cmd = [nvcc()] + FLAGS + objs + ["-lcudadevrt", "-lcurand", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed for {case}:\n{r.stderr[-4000:]}")
    with open(stamp_file, "w") as f:
        f.write(stamp)
    shutil.rmtree(scratch)
    log(f"built {exe}")
    return exe


def default_reference():
    return os.environ.get("VLBM_REFERENCE_ROOT", "/root/reference")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=default_reference())
    ap.add_argument("--case", action="append")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    a = ap.parse_args()
    if not os.path.isdir(os.path.join(a.reference, "src", "CUDA")):
        print(f"reference sources not found under {a.reference}; nothing built")
        return 0
    cases = a.case or list(ref_cases.CASES)
    failed = []
    for case in cases:
        for precision in ("f32", "f64"):
            try:
                build_case(case, a.reference, a.force, a.j, precision=precision)
            except Exception as e:  # keep building the other cases
                print(f"{case} ({precision}): {e}", file=sys.stderr)
                failed.append(case)
    return 1 if failed else 0


if __name__ == "__main__":
    sys.exit(main())
