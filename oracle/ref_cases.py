"""Cases run by the reference's own CUDA build (test infrastructure).

Each entry configures one build of the reference program (its compile-time
configuration in var.h, NNF/nnf.h, IBM/ibmVar.h, the boundary-condition builder
it compiles, the collision it pastes) and the same simulation for libvlbm, so the
tests can run both on the same GPU and compare what they write.

Keys:
  q            velocity set (var.h:19, `#define D3Q19` / `D3Q27`)
  op           "reg" (lbm.cu:263-461, the compiled default) or "bgk"
               (collisionSchemes/collisionForceNoReg.txt pasted over those lines,
               doc/updating.md:28-32)
  rheo         None, "bingham" or "powerlaw" (var.h:26-27)
  builder      reference builder file: boundaryConditionsBuilders/<name>.cu, or
               "harness:<face>:<scheme>" for the single-face builder written here
               (oracle/ref_harness_builder.cu)
  lib_builder  the libvlbm builder id that makes the same node map, or None when
               the map comes from oracle.harness_map
  nx, ny, nz   lattice (var.h:95-100)
  tau          TAU (var.h:104); Bingham: 3*eta_p + 0.5
  fx, fy, fz   FX..FZ (var.h:109-111)
  u_max        U_MAX (var.h:102); UX_BC..RHO_BC (var.h:114-117) follow from it
  eta_p, s_y   ETA_P, S_Y (nnf.h:20-21)
  n_index, k   N_INDEX, K_CONSISTENCY (nnf.h:11-12); GAMMA_0 stays 0
  steps        N_STEPS (var.h:62); the program's final save is labelled N_STEPS
               and holds the macroscopics its last iteration computed before
               colliding, i.e. the state after N_STEPS - 1 steps (main.cu:296,
               lbm.cu:247-261, main.cu:524-527)
  spheres      IBM cases: list of (diameter, cx, cy, cz); ibm: ibmVar.h values
  oracle       lattice the FP64 oracle runs: the case's own, or 1 along each axis the
               flow does not vary on (periodic axes of x/z-invariant channels), the
               fields then broadcast to the full lattice
"""

VAR_BC = {  # var.h:114-117 as functions of U_MAX and RHO_0 = 1
    "ux_bc": lambda u: [0, u, 0, 0, 0, 0, 0, 0],
    "uy_bc": lambda u: [0, u / 2, -u / 2, 0, 0, 0, 0, 0],
    "uz_bc": lambda u: [0, u, -u, 0, 0, 0, 0, 0],
    "rho_bc": lambda u: [1, 1, 1, 1, 1, 1, 1, 1],
}


def powerlaw_k(n, u=0.05, length=64, re=400.0):
    """Consistency for Re = U^(2-n) L^n / K (the lid-cavity Reynolds number)."""
    return u ** (2.0 - n) * length ** n / re


CASES = {
    # BGK Poiseuille channel, 64x32x32, tau 0.9, gx 1e-6, 10,000 steps.
    "poiseuille_bgk_q19": dict(
        q=19, op="bgk", rheo=None, builder="parallelPlatesBounceBack_Y", lib_builder=1, nx=64, ny=32, nz=32,
        tau=0.9, fx=1e-6, fy=0.0, fz=0.0, u_max=0.1, steps=10000, oracle=(1, 32, 1)),
    # Regularized Bingham plane channel, 256x128x64, tau_p 0.8, gx 5e-6, both ends of the yield-stress range.
    "bingham_channel_sy1e-6": dict(
        q=19, op="reg", rheo="bingham", builder="parallelPlatesBounceBack_Y", lib_builder=1, nx=256, ny=128, nz=64,
        tau=0.8, eta_p=0.1, s_y=1e-6, fx=5e-6, fy=0.0, fz=0.0, u_max=0.1, steps=2000, oracle=(1, 128, 1)),
    "bingham_channel_sy1e-4": dict(
        q=19, op="reg", rheo="bingham", builder="parallelPlatesBounceBack_Y", lib_builder=1, nx=256, ny=128, nz=64,
        tau=0.8, eta_p=0.1, s_y=1e-4, fx=5e-6, fy=0.0, fz=0.0, u_max=0.1, steps=2000, oracle=(1, 128, 1)),
    # Regularized Power-Law lid-driven cavity (walls x, y; moving lid y=NY-1; z periodic) on a 64-node
    # cavity: Re 10 for the shear-thinning fluid, Re 100 for the shear-thickening one.  At higher Re the
    # shear-thinning viscosity near the lid corners takes tau towards 1/2: at Re 100 the reference's own
    # FP64 and FP32 builds already differ by 1e-2 after 3000 steps (round-off amplified by the flow), and
    # at Re 400 the FP32 step diverges.
    "powerlaw_lid_q19_n0.5": dict(
        q=19, op="reg", rheo="powerlaw", builder="lidDrivenBounceBack", lib_builder=2, nx=64, ny=64, nz=16,
        tau=0.6, n_index=0.5, k=powerlaw_k(0.5, re=10.0), fx=0.0, fy=0.0, fz=0.0, u_max=0.05, steps=3000,
        oracle=(64, 64, 1)),
    "powerlaw_lid_q19_n1.5": dict(
        q=19, op="reg", rheo="powerlaw", builder="lidDrivenBounceBack", lib_builder=2, nx=64, ny=64, nz=16,
        tau=0.6, n_index=1.5, k=powerlaw_k(1.5, re=100.0), fx=0.0, fy=0.0, fz=0.0, u_max=0.05, steps=3000,
        oracle=(64, 64, 1)),
    # D3Q27 Bingham in a closed box: bounce-back on faces, edges and corners of both velocity sets.
    "closed_box_q27_bingham": dict(
        q=27, op="reg", rheo="bingham", builder="closedBoxBounceBack", lib_builder=3, nx=32, ny=24, nz=20,
        tau=0.8, eta_p=0.1, s_y=2e-6, fx=2e-5, fy=-1e-5, fz=1e-5, u_max=0.1, steps=1500, oracle=(32, 24, 20)),
    # D3Q27 Newtonian plates, bounce-back at y=0 and free slip at y=NY-1.
    "free_slip_q27": dict(
        q=27, op="reg", rheo=None, builder="parallelPlatesBounceBackFreeSlip", lib_builder=7, nx=16, ny=32, nz=8,
        tau=0.7, fx=1e-6, fy=0.0, fz=0.0, u_max=0.1, steps=4000, oracle=(1, 32, 1)),
    # D3Q19 Couette flow between velocity Zou-He plates (uz = +U_MAX at y=NY-1, -U_MAX at y=0).
    "couette_zouhe_q19": dict(
        q=19, op="reg", rheo=None, builder="couetteZouHe", lib_builder=8, nx=8, ny=32, nz=8,
        tau=0.8, fx=0.0, fy=0.0, fz=0.0, u_max=0.02, steps=3000, oracle=(1, 32, 1)),
}

# Zou-He faces of the single-face harness builder (oracle/ref_harness_builder.cu):
# velocity Zou-He on the west, east, front and back faces (no reference builder
# file puts one there; the north and south faces are couetteZouHe.cu above) and
# pressure Zou-He on west, south and back with RHO_BC[1] = 1.002.  Velocity
# faces drive a flow at U_MAX through a lattice that is periodic along the
# face normal; a few hundred steps pin the arithmetic of each face.  The east
# face follows D3Q19_VelZouHe.cu:99-122, which adds its corrections to the
# unknown (incoming) populations instead of rebuilding them from the known
# ones; momentum then builds up step after step and the flow diverges, so that
# case runs 20 steps: it pins the arithmetic, not a flow.
for _face in ("WEST", "EAST", "FRONT", "BACK"):
    CASES[f"vel_zouhe_{_face.lower()}_q19"] = dict(
        q=19, op="reg", rheo=None, builder=f"harness:{_face}:BC_SCHEME_VEL_ZOUHE", lib_builder=None,
        nx=12, ny=10, nz=12, tau=0.8, fx=0.0, fy=0.0, fz=0.0, u_max=0.02, steps=20 if _face == "EAST" else 300,
        oracle=(12, 10, 12))
for _face in ("WEST", "SOUTH", "BACK"):
    CASES[f"pres_zouhe_{_face.lower()}_q19"] = dict(
        q=19, op="reg", rheo=None, builder=f"harness:{_face}:BC_SCHEME_PRES_ZOUHE", lib_builder=None,
        nx=12, ny=10, nz=12, tau=0.8, fx=0.0, fy=0.0, fz=0.0, u_max=0.1, rho_bc=[1.0, 1.002, 1, 1, 1, 1, 1, 1],
        steps=300, oracle=(12, 10, 12))

# Spheres settling in a closed box (IBM, IBM_BC walls on every axis), at most
# three spheres kept apart from each other and from the walls: no contact
# forms, so the reference's contact slots are never filled, and the collision
# kernel launches exactly N(N+1)/2 threads (ibmVar.h:167-175), all inside the
# particle array.  With spheres the final save is made after the last IBM
# step: the program's files labelled N_STEPS hold the state after N_STEPS steps
# (main.cu:293-296, 369-393, 524-535; IBM/ibm.cu:545-648).
IBM_CLOSED = dict(iterations=3, density=2.0, gx=0.0, gy=0.0, gz=-5e-5, walls=(1, 1, 1))
CASES["ibm_settling_closed_box_q19"] = dict(
    q=19, op="reg", rheo=None, builder="closedBoxBounceBack", lib_builder=3, nx=32, ny=32, nz=48,
    tau=0.8, fx=0.0, fy=0.0, fz=0.0, u_max=0.1, steps=301, oracle=(32, 32, 48),
    spheres=[(10.0, 15.5, 16.0, 31.0), (10.0, 16.3, 15.4, 15.0)], ibm=IBM_CLOSED)
CASES["ibm_bingham_closed_box_q19"] = dict(
    q=19, op="reg", rheo="bingham", builder="closedBoxBounceBack", lib_builder=3, nx=32, ny=32, nz=48,
    tau=0.8, eta_p=0.1, s_y=1e-6, fx=0.0, fy=0.0, fz=0.0, u_max=0.1, steps=301, oracle=(32, 32, 48),
    spheres=[(8.0, 10.0, 10.0, 24.0), (8.0, 21.5, 12.0, 30.0), (8.0, 16.0, 22.0, 18.0)], ibm=IBM_CLOSED)


def fluid_cases():
    return [k for k, c in CASES.items() if not c.get("spheres")]


def sphere_cases():
    return [k for k, c in CASES.items() if c.get("spheres")]


def ibm_config_kwargs(case):
    """vlbm.IbmConfig.default keyword arguments (ibmVar.h / ibmBoundaryCondition.h
    values the reference build of the case is configured with)."""
    ib = CASES[case]["ibm"]
    wx, wy, wz = ib["walls"]
    return dict(max_iterations=ib["iterations"], gx=ib["gx"], gy=ib["gy"], gz=ib["gz"],
                wall_x=wx, wall_y=wy, wall_z=wz)


def sphere_kwargs(case):
    """vlbm.Sphere keyword arguments: makeSpherePolar's diameter and centre, at
    rest, movable, PARTICLE_DENSITY (oracle/ref_particles.cpp)."""
    c = CASES[case]
    return [dict(diameter=d, cx=x, cy=y, cz=z, density=c["ibm"]["density"], movable=1)
            for d, x, y, z in c["spheres"]]


def lib_config_kwargs(case):
    """vlbm.Config.default keyword arguments for a case."""
    c = CASES[case]
    kw = dict(nx=c["nx"], ny=c["ny"], nz=c["nz"], vel_set=c["q"], tau=c["tau"], fx=c["fx"], fy=c["fy"],
              fz=c["fz"], rho0=1.0)
    kw["collision"] = 1 if c["op"] == "bgk" else 0
    if c["rheo"] == "bingham":
        kw.update(rheology=1, eta_p=c["eta_p"], yield_stress=c["s_y"])
    elif c["rheo"] == "powerlaw":
        kw.update(rheology=2, n_index=c["n_index"], k_consistency=c["k"], gamma0=0.0)
    else:
        kw["rheology"] = 0
    for key, fn in VAR_BC.items():
        kw[key] = fn(c["u_max"])
    if "rho_bc" in c:
        kw["rho_bc"] = list(c["rho_bc"])
    return kw


def node_map(case, builder_map, nx=None, ny=None, nz=None):
    """The case's node map on (nx, ny, nz) (default: its lattice).  `builder_map(id,
    nx, ny, nz)` makes the named builders' maps; harness cases use oracle.harness_map."""
    import oracle
    c = CASES[case]
    nx, ny, nz = nx or c["nx"], ny or c["ny"], nz or c["nz"]
    if c["lib_builder"] is None:
        _, face, scheme = c["builder"].split(":")
        return oracle.harness_map(face, scheme, nx, ny, nz)
    return builder_map(c["lib_builder"], nx, ny, nz)
