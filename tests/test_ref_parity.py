"""Parity with the reference's own CUDA build, run on the same GPU.

oracle/ref_build.py compiles the reference program once per case of
oracle/ref_cases.py (its compile-time configuration, builder and collision)
into oracle/_ref/<case>/, twice: `refsim` with the reference's default
dfloat = float and `refsim_f64` with dfloat = double.  Each test runs both,
reads the macroscopic files their final save writes (lbmReport.cpp:133-172,
raw dfloat [NZ][NY][NX] as src/Post Processing/fileTreat.py:146-168 reads
them), runs the same case through libvlbm (FP32) and through the FP64 oracle,
and compares velocity fields (relative L2 of (ux, uy, uz)) and densities (max
abs):

* reference FP64 vs FP64 oracle: pins the oracle's restatement to the
  reference program itself, to FP64 round-off;
* libvlbm vs reference FP64: the library's own FP32 error;
* reference FP32 vs reference FP64: the reference's own FP32 error;
* libvlbm vs reference FP32: the drop-in claim, which can be no tighter than
  the reference's own FP32 error.

The final save is labelled N_STEPS and holds the macroscopics the last
iteration computed before colliding (main.cu:296, lbm.cu:247-261), i.e. the
state after N_STEPS - 1 steps; libvlbm and the oracle are compared after
N_STEPS - 1 steps.  The reference stores full FP32 populations (values ~w_i);
a slow flow's per-step increments are then a few ulps and their rounding
biases its velocity (0.2 % in the BGK Poiseuille case, 1.4 % in the closed
box at u ~ 1e-4).  The library stores deviations f_i - w_i rho0 and stays
within LIB_VS_REF64 of the reference's FP64 build.
"""
import os
import subprocess

import numpy as np
import pytest

import ref_cases

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(REPO, "oracle", "_ref")

# velocity relative L2 bounds per comparison
REF64_VS_ORACLE = 1e-9    # both FP64, different summation orders
# Power-Law: the reference evaluates gammaDot = (1 - omega/2)|S| / ((1/omega - 1/2)/3)
# (nnf.h:41-44), whose difference 1/omega - 1/2 cancels as omega nears 2; the
# oracle evaluates the equal 3 omega |S|.  FP64 round-off amplified by that
# cancellation over thousands of steps: measured 3e-8 (n = 0.5), 3e-14 (n = 1.5).
REF64_VS_ORACLE_POWERLAW = 1e-7
# the library's FP32 error: relative L2 <= 1e-4, or an RMS velocity error of at
# most 2e-7 (FP32 resolution of the populations) in flows slower than ~2e-3
LIB_VS_REF64 = 1e-4
LIB_VS_REF64_RMS = 2e-7
RHO_LIB_REF64 = 1e-5      # density max abs, library vs reference FP64
# libvlbm vs reference FP32: within the reference's own FP32 error (reference
# FP32 vs FP64) plus the library's, with a margin
LIB_VS_REF32_FACTOR = 1.5
LIB_VS_REF32_FLOOR = 2e-4
# Bingham / Power-Law omega, library vs reference FP64: mean and 99th
# percentile of |d omega| / max omega.  Bingham's omega_p max(0, 1 - tau0/|S|)
# turns FP32 noise of |S| near the yield surface and the channel centre
# (|S| -> 0) into large omega differences on a few nodes; the velocity there is
# unaffected.
OMEGA_MEAN = 5e-3
OMEGA_P99 = 1e-1


def _label(step):
    """Step field of getVarFilename (lbmReport.cpp:55-83): six digits, seven for step 0."""
    return "0" * 7 if step == 0 else f"{step:06d}"


def run_reference(case, workdir, precision="f32"):
    suffix = "" if precision == "f32" else "_f64"
    exe = os.path.join(REF, case, "refsim" + suffix)
    if not os.path.exists(exe):
        pytest.skip(f"reference build for {case} missing (python oracle/ref_build.py)")
    wd = os.path.join(workdir, precision)
    os.makedirs(wd, exist_ok=True)
    r = subprocess.run([exe], cwd=wd, capture_output=True, text=True, timeout=600, stdin=subprocess.DEVNULL)
    assert r.returncode == 0, f"reference program failed ({r.returncode}):\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}"
    mlups = [ln.strip() for ln in r.stdout.splitlines() if "MLUPS" in ln]
    if mlups:
        print(f"REFRUN {case} {precision} {mlups[-1]}")
    c = ref_cases.CASES[case]
    out = {"dir": os.path.join(wd, "out", case)}
    names = ["rho", "ux", "uy", "uz"] + (["omega"] if c["rheo"] else [])
    for v in names:
        p = os.path.join(wd, "out", case, f"{case}_{v}{_label(c['steps'])}.bin")
        a = np.fromfile(p, dtype=np.float32 if precision == "f32" else np.float64)
        assert a.size == c["nx"] * c["ny"] * c["nz"], (p, a.size)
        out[v] = a.reshape(c["nz"], c["ny"], c["nx"])
    return out


def run_library(vlbm, case, storage=0):
    c = ref_cases.CASES[case]
    cfg = vlbm.Config.default(device=0, storage=storage, **ref_cases.lib_config_kwargs(case))
    m = ref_cases.node_map(case, vlbm.build_node_map)
    sim = vlbm.Simulation(cfg, node_map=m)
    sim.step(c["steps"] - 1)
    sim.sync()
    out = sim.macroscopics()
    sim.close()
    return out


def run_oracle(oracle, case):
    """FP64 oracle on the case's oracle lattice, broadcast to the full lattice."""
    c = ref_cases.CASES[case]
    nx, ny, nz = c["oracle"]
    kw = ref_cases.lib_config_kwargs(case)
    kw.update(nx=nx, ny=ny, nz=nz)
    m = ref_cases.node_map(case, lambda b, *s: oracle.reference_builder_map(oracle.BUILDER_NAMES[b], *s), nx, ny, nz)
    o = oracle.Oracle(oracle.Config.default(**kw), m)
    o.step(c["steps"] - 1)
    m = o.macroscopics()
    o.close()
    full = (c["nz"], c["ny"], c["nx"])
    return {k: np.broadcast_to(v, full) for k, v in m.items()}


def u_rel(a, b):
    du = np.sqrt(sum(np.sum((a[k].astype(np.float64) - b[k]) ** 2) for k in ("ux", "uy", "uz")))
    nb = np.sqrt(sum(np.sum(np.asarray(b[k], dtype=np.float64) ** 2) for k in ("ux", "uy", "uz")))
    return float(du / nb)


def u_rms_err(a, b):
    du = sum(np.sum((a[k].astype(np.float64) - b[k]) ** 2) for k in ("ux", "uy", "uz"))
    return float(np.sqrt(du / a["ux"].size))


def rho_max(a, b):
    return float(np.abs(a["rho"].astype(np.float64) - b["rho"]).max())


@pytest.mark.gpu
@pytest.mark.parametrize("case", ref_cases.fluid_cases())
def test_matches_reference_build(vlbm, oracle, case, tmp_path):
    ref32 = run_reference(case, str(tmp_path), "f32")
    ref64 = run_reference(case, str(tmp_path), "f64")
    lib = run_library(vlbm, case)
    oracle.set_threads(os.cpu_count() or 1)
    fp64 = run_oracle(oracle, case)
    res = dict(ref64_fp64=u_rel(ref64, fp64), lib_ref64=u_rel(lib, ref64), ref32_ref64=u_rel(ref32, ref64),
               lib_ref32=u_rel(lib, ref32), lib_ref64_rms=u_rms_err(lib, ref64),
               rho_lib_ref64=rho_max(lib, ref64), rho_ref32_ref64=rho_max(ref32, ref64),
               u_max=float(max(np.abs(ref64[k]).max() for k in ("ux", "uy", "uz"))))
    if "omega" in ref64:
        scale = float(np.abs(ref64["omega"]).max())
        d = np.abs(lib["omega"].astype(np.float64) - ref64["omega"]) / scale
        res.update(omega_mean=float(d.mean()), omega_p99=float(np.percentile(d, 99)))
    print(f"REFPARITY {case} " + " ".join(f"{k}={v:.3e}" for k, v in res.items()))
    for name, f in (("ref32", ref32), ("ref64", ref64), ("lib", lib)):
        for k in ("rho", "ux", "uy", "uz"):
            assert np.all(np.isfinite(f[k])), f"{name} {k} not finite"
    assert res["u_max"] > 1e-4
    tol = REF64_VS_ORACLE_POWERLAW if ref_cases.CASES[case]["rheo"] == "powerlaw" else REF64_VS_ORACLE
    assert res["ref64_fp64"] <= tol, res
    assert res["lib_ref64"] <= LIB_VS_REF64 or res["lib_ref64_rms"] <= LIB_VS_REF64_RMS, res
    assert res["rho_lib_ref64"] <= RHO_LIB_REF64, res
    assert res["lib_ref32"] <= LIB_VS_REF32_FACTOR * res["ref32_ref64"] + LIB_VS_REF32_FLOOR, res
    if "omega_mean" in res:
        assert res["omega_mean"] <= OMEGA_MEAN, res
        assert res["omega_p99"] <= OMEGA_P99, res


# ------------------------------------------------------------------ spheres ---
# Sphere cases: the reference program writes its particle state with
# saveParticlesInfo (IBM/ibmReport.cpp:26-102) after the final step, in
# std::scientific with 7 significant digits; the library writes the same files
# through vlbm_write_particles_csv.  Bounds (lattice units):
#   reference FP64 vs FP64 oracle: fluid velocity relative L2 <= 1e-8; particle
#     position within the CSV resolution (|dx| <= 2e-5), velocity and rotation
#     within 1e-5 of their largest magnitude, Lagrangian nodes |dx| <= 2e-5;
#   library (FP32 fluid, FP64 particles) vs reference FP64: the bounds of the
#     oracle comparison in tests/test_gpu_ibm.py: fluid relative L2 <= 5e-3,
#     position |dx| <= 2e-5 + 1e-3 |x - x0|, velocity and rotation
#     <= 2e-3 of their largest magnitude;
#   library vs reference FP32: within 1.5x the reference's own FP32 error plus
#     the library-vs-FP64 bound.
IBM_REF64_VS_ORACLE_U = 1e-8
IBM_CSV_POS = 2e-5
IBM_REF64_VS_ORACLE_V = 1e-5
IBM_LIB_U = 5e-3
IBM_LIB_V = 2e-3


def _pfile(d, case, var, step):
    return os.path.join(d, f"{case}_{var}{_label(step)}.csv")


def read_pcenters(path):
    """pCenters CSV -> header line and {pos, vel, w, f, M} arrays [n][3]."""
    with open(path) as f:
        header = f.readline().strip()
    a = np.atleast_1d(np.genfromtxt(path, delimiter=",", names=True))
    out = {"header": header}
    for key in ("pos", "vel", "w", "f", "M"):
        out[key] = np.stack([a[f"{key}_{ax}"] for ax in "xyz"], axis=1)
    out["radius"] = a["radius"]
    return out


def read_pnodes(path):
    with open(path) as f:
        header = f.readline().strip()
    a = np.atleast_1d(np.genfromtxt(path, delimiter=",", names=True))
    return header, np.stack([a["pos_x"], a["pos_y"], a["pos_z"]]), a["particle_index"]


def run_library_spheres(vlbm, case, outdir):
    c = ref_cases.CASES[case]
    cfg = vlbm.Config.default(device=0, **ref_cases.lib_config_kwargs(case))
    m = ref_cases.node_map(case, vlbm.build_node_map)
    sim = vlbm.Simulation(cfg, node_map=m)
    sim.add_spheres(vlbm.IbmConfig.default(**ref_cases.ibm_config_kwargs(case)),
                    [vlbm.Sphere(**s) for s in ref_cases.sphere_kwargs(case)])
    sim.step(c["steps"])
    sim.sync()
    out = sim.macroscopics()
    sim.write_particles_csv(outdir, case, c["steps"], save_nodes=True)
    out["dir"] = os.path.join(outdir, case)
    sim.close()
    return out


def run_oracle_spheres(vlbm, oracle, case):
    c = ref_cases.CASES[case]
    cfg = oracle.Config.default(**ref_cases.lib_config_kwargs(case))
    m = ref_cases.node_map(case, lambda b, *s: oracle.reference_builder_map(oracle.BUILDER_NAMES[b], *s))
    sp = [vlbm.Sphere(**s) for s in ref_cases.sphere_kwargs(case)]
    o = oracle.OracleIbm(cfg, m, vlbm.IbmConfig.default(**ref_cases.ibm_config_kwargs(case)), sp)
    o.step(c["steps"])
    out = o.macroscopics()
    out["particles"] = o.particles()
    out["nodes"] = o.nodes()
    o.close()
    return out


def _pdiff(a, b, key):
    return float(np.abs(np.asarray(a[key], dtype=np.float64) - b[key]).max())


@pytest.mark.gpu
@pytest.mark.parametrize("case", ref_cases.sphere_cases())
def test_sphere_case_matches_reference_build(vlbm, oracle, case, tmp_path):
    c = ref_cases.CASES[case]
    steps = c["steps"]
    ref32 = run_reference(case, str(tmp_path), "f32")
    ref64 = run_reference(case, str(tmp_path), "f64")
    lib = run_library_spheres(vlbm, case, str(tmp_path / "lib"))
    oracle.set_threads(os.cpu_count() or 1)
    fp64 = run_oracle_spheres(vlbm, oracle, case)
    p32 = read_pcenters(_pfile(ref32["dir"], case, "pCenters", steps))
    p64 = read_pcenters(_pfile(ref64["dir"], case, "pCenters", steps))
    plib = read_pcenters(_pfile(lib["dir"], case, "pCenters", steps))
    po = fp64["particles"]
    x0 = np.array([[x, y, z] for _, x, y, z in c["spheres"]])
    h64, n64, idx64 = read_pnodes(_pfile(ref64["dir"], case, "pNodes", steps))
    hlib, nlib, idxlib = read_pnodes(_pfile(lib["dir"], case, "pNodes", steps))
    vmax = float(np.abs(p64["vel"]).max())
    wmax = max(float(np.abs(p64["w"]).max()), 1e-12)
    res = dict(
        ref64_fp64=u_rel(ref64, fp64), lib_ref64=u_rel(lib, ref64), ref32_ref64=u_rel(ref32, ref64),
        lib_ref32=u_rel(lib, ref32), rho_lib_ref64=rho_max(lib, ref64),
        pos_ref64_fp64=_pdiff(p64, po, "pos"), vel_ref64_fp64=_pdiff(p64, po, "vel") / vmax,
        w_ref64_fp64=_pdiff(p64, po, "w") / wmax,
        nodes_ref64_fp64=float(np.abs(n64 - fp64["nodes"]).max()),
        nodes_lib_ref64=float(np.abs(nlib - n64).max()),
        pos_lib_ref64=_pdiff(plib, p64, "pos"), vel_lib_ref64=_pdiff(plib, p64, "vel") / vmax,
        w_lib_ref64=_pdiff(plib, p64, "w") / wmax,
        vel_ref32_ref64=_pdiff(p32, p64, "vel") / vmax, vel_lib_ref32=_pdiff(plib, p32, "vel") / vmax,
        disp=float(np.abs(p64["pos"] - x0).max()), v_max=vmax)
    print(f"REFPARITY {case} " + " ".join(f"{k}={v:.3e}" for k, v in res.items()))
    # the library's files are the reference's files: same columns, same rows
    assert plib["header"] == p64["header"]
    assert hlib == h64 and np.array_equal(idxlib, idx64)
    assert np.array_equal(plib["radius"], p64["radius"])
    for name, f in (("ref32", ref32), ("ref64", ref64), ("lib", lib)):
        for k in ("rho", "ux", "uy", "uz"):
            assert np.all(np.isfinite(f[k])), f"{name} {k} not finite"
    assert res["v_max"] > 1e-5 and res["disp"] > 1e-2, res   # the spheres did move
    assert res["ref64_fp64"] <= IBM_REF64_VS_ORACLE_U, res
    assert res["pos_ref64_fp64"] <= IBM_CSV_POS, res
    assert res["vel_ref64_fp64"] <= IBM_REF64_VS_ORACLE_V and res["w_ref64_fp64"] <= IBM_REF64_VS_ORACLE_V, res
    assert res["nodes_ref64_fp64"] <= IBM_CSV_POS, res
    assert res["lib_ref64"] <= IBM_LIB_U, res
    assert res["rho_lib_ref64"] <= RHO_LIB_REF64, res
    dx = np.abs(plib["pos"] - p64["pos"])
    assert np.all(dx <= IBM_CSV_POS + 1e-3 * np.abs(p64["pos"] - x0)), (res, dx)
    assert res["nodes_lib_ref64"] <= IBM_CSV_POS + 1e-3 * res["disp"] * 2, res
    assert res["vel_lib_ref64"] <= IBM_LIB_V and res["w_lib_ref64"] <= IBM_LIB_V, res
    assert res["lib_ref32"] <= LIB_VS_REF32_FACTOR * res["ref32_ref64"] + IBM_LIB_U, res
    assert res["vel_lib_ref32"] <= LIB_VS_REF32_FACTOR * res["vel_ref32_ref64"] + IBM_LIB_V, res
