"""ctypes binding of the FP64 oracle (oracle/oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py, always as the checker, never as the product.

Also holds a literal restatement of the reference builders' if-chains
(src/CUDA/boundaryConditionsBuilders/*.cu) used to check libvlbm's builders.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")


def build():
    """Compile liboracle.so with the committed Makefile (g++, OpenMP)."""
    r = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    return LIB_PATH


def _load():
    srcs = [os.path.join(HERE, f) for f in os.listdir(HERE) if f.endswith(".cpp")]
    if not os.path.exists(LIB_PATH) or any(os.path.getmtime(s) > os.path.getmtime(LIB_PATH) for s in srcs):
        build()
    lib = C.CDLL(LIB_PATH)
    P = C.c_void_p
    D = C.POINTER(C.c_double)
    lib.oracle_create.restype = P
    lib.oracle_create.argtypes = [P, C.POINTER(C.c_uint32)]
    lib.oracle_destroy.argtypes = [P]
    lib.oracle_set_threads.argtypes = [C.c_int]
    lib.oracle_step.argtypes = [P, C.c_int]
    lib.oracle_macro.argtypes = [P, D, D, D, D, D]
    lib.oracle_get_pops.argtypes = [P, D]
    lib.oracle_set_pops.argtypes = [P, D]
    lib.oracle_set_omega.argtypes = [P, D]
    lib.oracle_step_count.restype = C.c_longlong
    lib.oracle_step_count.argtypes = [P]
    lib.oracle_bb_role.argtypes = [C.c_int, C.c_int, C.c_int]
    lib.oracle_bb_role.restype = C.c_int
    lib.oracle_free_slip_source.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int)]
    lib.oracle_free_slip_source.restype = C.c_int
    lib.oracle_lattice.argtypes = [C.c_int, C.POINTER(C.c_int)]
    lib.oracle_weight.argtypes = [C.c_int, C.c_int]
    lib.oracle_weight.restype = C.c_double
    if hasattr(lib, "oracle_ibm_create"):
        _bind_ibm(lib)
    return lib


def _bind_ibm(lib):
    P = C.c_void_p
    D = C.POINTER(C.c_double)
    lib.oracle_ibm_create.restype = P
    lib.oracle_ibm_create.argtypes = [P, C.POINTER(C.c_uint32), P, P, C.c_int]
    lib.oracle_ibm_fluid.restype = P
    lib.oracle_ibm_fluid.argtypes = [P]
    lib.oracle_ibm_step.argtypes = [P, C.c_int]
    lib.oracle_ibm_macro.argtypes = [P, D, D, D, D]
    lib.oracle_ibm_particles.argtypes = [P, D, C.c_int]
    lib.oracle_ibm_particles.restype = C.c_int
    lib.oracle_ibm_nodes.argtypes = [P, D, C.c_int]
    lib.oracle_ibm_nodes.restype = C.c_int
    lib.oracle_ibm_destroy.argtypes = [P]
    lib.oracle_sphere_mesh.argtypes = [C.c_double, C.c_double, D, D, C.c_int]
    lib.oracle_sphere_mesh.restype = C.c_int


_lib = _load()


def lib():
    return _lib


def set_threads(n):
    _lib.oracle_set_threads(int(n))


def bb_role(q, direction, i):
    return _lib.oracle_bb_role(q, direction, i)


def velocities(q):
    """The oracle's population ordering, [(cx, cy, cz)] for i < q."""
    out = []
    for i in range(q):
        c = (C.c_int * 3)()
        _lib.oracle_lattice(i, c)
        out.append((c[0], c[1], c[2]))
    return out


def weight(q, i):
    return _lib.oracle_weight(q, i)


def free_slip_source(q, direction, i):
    off = (C.c_int * 3)()
    j = _lib.oracle_free_slip_source(q, direction, i, off)
    return j, [off[0], off[1], off[2]]


class Config(C.Structure):
    """The oracle's configuration: the field layout of vlbm_config (include/vlbm.h),
    which oracle.cpp reads, filled here without loading libvlbm so that CPU
    baselines built on the oracle alone map no product library."""
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("vel_set", C.c_int32), ("collision", C.c_int32), ("rheology", C.c_int32),
        ("storage", C.c_int32), ("device", C.c_int32),
        ("tau", C.c_double), ("rho0", C.c_double),
        ("fx", C.c_double), ("fy", C.c_double), ("fz", C.c_double),
        ("eta_p", C.c_double), ("yield_stress", C.c_double),
        ("n_index", C.c_double), ("k_consistency", C.c_double), ("gamma0", C.c_double),
        ("ux_bc", C.c_double * 8), ("uy_bc", C.c_double * 8),
        ("uz_bc", C.c_double * 8), ("rho_bc", C.c_double * 8),
        ("storage_scale", C.c_double),
        ("layout", C.c_int32),
        ("slab_z_offset", C.c_int32), ("slab_nz_total", C.c_int32),
        ("reserved", C.c_int32 * 5),
        ("duct_outer_radius", C.c_double), ("duct_inner_radius", C.c_double),
        ("duct_outer_velocity", C.c_double), ("duct_outer_rotation", C.c_double),
        ("duct_inner_velocity", C.c_double), ("duct_inner_rotation", C.c_double),
    ]

    @classmethod
    def default(cls, **kw):
        """Reference defaults (var.h:95-117, nnf.h:11-21), then the given fields."""
        c = cls()
        c.nx, c.ny, c.nz = 128, 128, 384
        c.vel_set, c.tau, c.rho0 = 19, 0.6, 1.0
        c.eta_p, c.yield_stress, c.n_index = 0.3, 1e-4, 0.5
        c.k_consistency = c.rho0 * (c.tau - 0.5) / 3.0
        u = 0.1
        for i, (a, b, d) in enumerate(zip([0, u, 0, 0, 0, 0, 0, 0], [0, u / 2, -u / 2, 0, 0, 0, 0, 0],
                                          [0, u, -u, 0, 0, 0, 0, 0])):
            c.ux_bc[i], c.uy_bc[i], c.uz_bc[i], c.rho_bc[i] = a, b, d, 1.0
        for k, v in kw.items():
            if k in ("ux_bc", "uy_bc", "uz_bc", "rho_bc"):
                arr = getattr(c, k)
                for i, val in enumerate(v):
                    arr[i] = val
            else:
                setattr(c, k, v)
        return c


def plates_y_map(nx, ny, nz):
    """Node map of parallelPlatesBounceBack_Y.cu (bounce-back SOUTH at y=0, NORTH
    at y=NY-1), vectorised; equal to reference_builder_map("plates_y", ...)."""
    m = np.full((nz, ny, nx), USED, dtype=np.uint32)
    m[:, 0, :] = _w(BB, S_)
    m[:, ny - 1, :] = _w(BB, N_)
    return m.ravel()


class Oracle:
    """One lattice advanced by the FP64 restatement (reference push/AB scheme)."""

    def __init__(self, cfg, node_map):
        self.cfg = cfg
        self.q = cfg.vel_set
        self.shape = (cfg.nz, cfg.ny, cfg.nx)
        self.n = cfg.nx * cfg.ny * cfg.nz
        m = np.ascontiguousarray(node_map, dtype=np.uint32).ravel()
        assert m.size == self.n
        self._h = _lib.oracle_create(C.byref(cfg), m.ctypes.data_as(C.POINTER(C.c_uint32)))

    def close(self):
        if self._h:
            _lib.oracle_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n=1):
        _lib.oracle_step(self._h, int(n))

    def macroscopics(self):
        out = [np.empty(self.n) for _ in range(5)]
        ptr = [a.ctypes.data_as(C.POINTER(C.c_double)) for a in out]
        _lib.oracle_macro(self._h, *ptr)
        return {k: v.reshape(self.shape) for k, v in zip(("rho", "ux", "uy", "uz", "omega"), out)}

    def populations(self):
        out = np.empty(self.q * self.n)
        _lib.oracle_get_pops(self._h, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out.reshape((self.q,) + self.shape)

    def set_populations(self, pops):
        a = np.ascontiguousarray(pops, dtype=np.float64).ravel()
        _lib.oracle_set_pops(self._h, a.ctypes.data_as(C.POINTER(C.c_double)))


class OracleIbm:
    """Fluid step + immersed-boundary step for spheres, FP64 (reference loop order)."""

    def __init__(self, cfg, node_map, ibm_cfg, spheres):
        self.cfg = cfg
        self.shape = (cfg.nz, cfg.ny, cfg.nx)
        self.n = cfg.nx * cfg.ny * cfg.nz
        m = np.ascontiguousarray(node_map, dtype=np.uint32).ravel()
        arr = (type(spheres[0]) * len(spheres))(*spheres)
        self._keep = arr
        self.np = len(spheres)
        self._h = _lib.oracle_ibm_create(C.byref(cfg), m.ctypes.data_as(C.POINTER(C.c_uint32)),
                                         C.byref(ibm_cfg), C.cast(arr, C.c_void_p), len(spheres))

    def close(self):
        if self._h:
            _lib.oracle_ibm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n=1):
        _lib.oracle_ibm_step(self._h, int(n))

    def macroscopics(self):
        out = [np.empty(self.n) for _ in range(4)]
        _lib.oracle_ibm_macro(self._h, *[a.ctypes.data_as(C.POINTER(C.c_double)) for a in out])
        return {k: v.reshape(self.shape) for k, v in zip(("rho", "ux", "uy", "uz"), out)}

    def particles(self):
        out = np.empty(24 * self.np)
        _lib.oracle_ibm_particles(self._h, out.ctypes.data_as(C.POINTER(C.c_double)), self.np)
        out = out.reshape(self.np, 24)
        return {"pos": out[:, 0:3], "vel": out[:, 3:6], "w": out[:, 6:9], "f": out[:, 9:12],
                "M": out[:, 12:15], "w_avg": out[:, 15:18], "I": out[:, 18:24]}

    def nodes(self):
        n = _lib.oracle_ibm_nodes(self._h, None, 0)
        out = np.empty(3 * n)
        _lib.oracle_ibm_nodes(self._h, out.ctypes.data_as(C.POINTER(C.c_double)), n)
        return out.reshape(3, n)

    def populations(self):
        fl = _lib.oracle_ibm_fluid(self._h)
        q = self.cfg.vel_set
        out = np.empty(q * self.n)
        _lib.oracle_get_pops(fl, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out.reshape((q,) + self.shape)


def sphere_mesh(diameter, mesh_scale=1.0):
    """makeSpherePolar node positions relative to the centre [3][n] and areas [n]."""
    n = _lib.oracle_sphere_mesh(diameter, mesh_scale, None, None, 0)
    xyz = np.empty(3 * n)
    S = np.empty(n)
    _lib.oracle_sphere_mesh(diameter, mesh_scale, xyz.ctypes.data_as(C.POINTER(C.c_double)),
                            S.ctypes.data_as(C.POINTER(C.c_double)), n)
    return xyz.reshape(3, n), S


def treat_data(rho, ux, uy, uz, prev=None, resid_max=1e-5):
    """Report-step data treatment of treatData.cpp:25-89 and stopSim
    treatData.cpp:451-460, in FP64: residual = sum |u - u_old| / sum |u|
    (1 when sum |u| = 0; u_old zero when `prev` is None), avgRho = mean rho,
    avgUzPlanXZ[y] = mean over x, z of uz for the [z][y][x] fields given (the
    mean of this report alone: the reference's array is never cleared between
    reports, macrProc.h:39-40), stop = residual < RESID_MAX or avgRho < 0."""
    u = np.stack([np.asarray(a, dtype=np.float64) for a in (ux, uy, uz)])
    old = np.zeros_like(u) if prev is None else np.stack([np.asarray(a, dtype=np.float64) for a in prev])
    num = np.sqrt(((u - old) ** 2).sum(axis=0)).sum()
    den = np.sqrt((u ** 2).sum(axis=0)).sum()
    residual = num / den if den != 0 else 1.0
    avg_rho = float(np.asarray(rho, dtype=np.float64).mean())
    avg_uz = u[2].mean(axis=(0, 2))
    return {"residual": float(residual), "avg_rho": avg_rho, "avg_uz_plane_xz": avg_uz,
            "stop": bool(residual < resid_max or avg_rho < 0)}


# --------------------------------------------------------------------------
# Literal restatement of the reference builders (node-map words).
# Bit layout src/CUDA/structs/nodeTypeMap.h:15-133.
USED = 1 << 21
SCHEME_OFF, DIR_OFF, UX_OFF, UY_OFF, UZ_OFF = 18, 13, 9, 6, 3
BB, VELBB, VELZH, FREESLIP = 5, 2, 1, 4
(N_, S_, W_, E_, F_, B_, NW, NE, NF, NB, SW, SE, SF, SB, WF, WB, EF, EB,
 NWF, NWB, NEF, NEB, SWF, SWB, SEF, SEB) = range(26)


def _w(scheme, d, ux=0, uz=0):
    return USED | (scheme << SCHEME_OFF) | (d << DIR_OFF) | (ux << UX_OFF) | (uz << UZ_OFF)


def reference_builder_map(name, nx, ny, nz, outer_radius=None, inner_radius=None):
    """Node map as the named reference builder writes it ([nz][ny][nx] uint32).
    The duct builders take OUTER_RADIUS / INNER_RADIUS (default: var.h)."""
    out = np.full((nz, ny, nx), USED, dtype=np.uint32)
    for z in range(nz):
        for y in range(ny):
            for x in range(nx):
                out[z, y, x] = _builder_word(name, x, y, z, nx, ny, nz, outer_radius, inner_radius)
    return out.ravel()


def _builder_word(name, x, y, z, NX, NY, NZ, outer_radius=None, inner_radius=None):
    w = USED
    if name == "periodic":
        return w
    if name == "plates_y":  # parallelPlatesBounceBack_Y.cu
        if y == 0:
            return _w(BB, S_)
        if y == NY - 1:
            return _w(BB, N_)
        return w
    if name == "plates_y_free_slip":  # parallelPlatesBounceBackFreeSlip.cu
        if y == 0:
            return _w(BB, S_)
        if y == NY - 1:
            return _w(FREESLIP, N_)
        return w
    if name == "plates_y_zouhe":  # couetteZouHe.cu
        if y == 0:
            return _w(VELZH, S_, uz=2)
        if y == NY - 1:
            return _w(VELZH, N_, uz=1)
        return w
    if name in ("lid_driven", "square_duct"):  # lidDrivenBounceBack.cu / squareDuctBounceBack.cu
        lid = name == "lid_driven"
        top = (lambda: _w(VELBB, N_, ux=1)) if lid else (lambda: _w(BB, N_))
        if y == 0 and x == 0:
            return _w(BB, SW)
        if y == 0 and x == NX - 1:
            return _w(BB, SE)
        if y == NY - 1 and x == 0:
            return _w(BB, NW)
        if y == NY - 1 and x == NX - 1:
            return _w(BB, NE)
        if y == 0:
            return _w(BB, S_)
        if y == NY - 1:
            return top()
        if x == 0:
            return _w(BB, W_)
        if x == NX - 1:
            return _w(BB, E_)
        return w
    if name in ("closed_box", "lid_cavity_closed"):  # closedBoxBounceBack.cu:56-208
        chain = [
            (y == 0 and x == 0 and z == 0, SWB), (y == 0 and x == 0 and z == NZ - 1, SWF),
            (y == 0 and x == NX - 1 and z == 0, SEB), (y == 0 and x == NX - 1 and z == NZ - 1, SEF),
            (y == NY - 1 and x == 0 and z == 0, NWB), (y == NY - 1 and x == 0 and z == NZ - 1, NWF),
            (y == NY - 1 and x == NX - 1 and z == 0, NEB), (y == NY - 1 and x == NX - 1 and z == NZ - 1, NEF),
            (y == 0 and x == 0, SW), (y == 0 and x == NX - 1, SE), (y == NY - 1 and x == 0, NW),
            (y == NY - 1 and x == NX - 1, NE), (y == 0 and z == 0, SB), (y == 0 and z == NZ - 1, SF),
            (y == NY - 1 and z == 0, NB), (y == NY - 1 and z == NZ - 1, NF), (x == 0 and z == 0, WB),
            (x == 0 and z == NZ - 1, WF), (x == NX - 1 and z == 0, EB), (x == NX - 1 and z == NZ - 1, EF),
            (y == 0, S_), (y == NY - 1, N_), (x == 0, W_), (x == NX - 1, E_), (z == 0, B_), (z == NZ - 1, F_)]
        for cond, d in chain:
            if cond:
                if name == "lid_cavity_closed" and d == N_:
                    return _w(VELBB, N_, ux=1)
                return _w(BB, d)
        return w
    if name == "duct_yz":  # walls on y and z faces, periodic x
        chain = [(y == 0 and z == 0, SB), (y == 0 and z == NZ - 1, SF), (y == NY - 1 and z == 0, NB),
                 (y == NY - 1 and z == NZ - 1, NF), (y == 0, S_), (y == NY - 1, N_), (z == 0, B_),
                 (z == NZ - 1, F_)]
        for cond, d in chain:
            if cond:
                return _w(BB, d)
        return w
    if name in ("circular_duct", "annular_duct"):
        return _duct_word(name == "annular_duct", x, y, NX, NY, outer_radius, inner_radius)
    raise KeyError(name)


FACE_CODES = {"NORTH": N_, "SOUTH": S_, "WEST": W_, "EAST": E_, "FRONT": F_, "BACK": B_}
SCHEME_CODES = {"BC_SCHEME_VEL_ZOUHE": VELZH, "BC_SCHEME_PRES_ZOUHE": 3}


def harness_map(face, scheme, nx, ny, nz):
    """Node map of oracle/ref_harness_builder.cu: `scheme` on `face` with value
    index 1 (UX_BC on west/east, UZ_BC on front/back, UY_BC on north/south,
    RHO_BC for pressure), bounce-back walls on the faces normal to y (normal to
    z when the face is north or south) taking the shared edges, the other axes
    periodic.  [nz][ny][nx] uint32 in the reference's bit layout."""
    d, s = FACE_CODES[face], SCHEME_CODES[scheme]
    m = np.full((nz, ny, nx), USED, dtype=np.uint32)
    if s == 3:
        val = 1
    elif d in (W_, E_):
        val = 1 << UX_OFF
    elif d in (F_, B_):
        val = 1 << UZ_OFF
    else:
        val = 1 << UY_OFF
    sel = {N_: (slice(None), ny - 1, slice(None)), S_: (slice(None), 0, slice(None)),
           W_: (slice(None), slice(None), 0), E_: (slice(None), slice(None), nx - 1),
           F_: (nz - 1, slice(None), slice(None)), B_: (0, slice(None), slice(None))}[d]
    m[sel] = USED | (s << SCHEME_OFF) | (d << DIR_OFF) | val
    if d in (N_, S_):
        m[0, :, :] = _w(BB, B_)
        m[nz - 1, :, :] = _w(BB, F_)
    else:
        m[:, 0, :] = _w(BB, S_)
        m[:, ny - 1, :] = _w(BB, N_)
    return m.ravel()


INTERP, IS_SAVE = 6, 1 << 22
_DIRS8 = [(1, 0), (0, 1), (-1, 0), (0, -1), (1, 1), (-1, 1), (-1, -1), (1, -1)]


def _dist2f(x1, y1, x2, y2):
    """distPoints2D (globalFunctions.h:159-162) with dfloat = float."""
    f = np.float32
    dx, dy = f(x1) - f(x2), f(y1) - f(y2)
    return np.sqrt(f(dx * dx) + f(dy * dy), dtype=np.float32)


def _duct_word(annular, x, y, NX, NY, outer_radius=None, inner_radius=None):
    """circularDuctInterpBounceBack.cu:35-123 / annularDuctInterpBounceBack.cu:35-140
    (OUTER_RADIUS = NY/2 - 1.5, INNER_RADIUS = OUTER_RADIUS/4, DUCT_CENTER_X/Y,
    var.h:142-162), in float as the builders compute it."""
    f = np.float32
    Rd = outer_radius if outer_radius else NY / 2.0 - 1.5
    R = f(Rd)
    r = f(inner_radius if inner_radius else Rd / 4.0)
    xc, yc = f((NX - 1) / 2.0 + 0.5), f((NY - 1) / 2.0 + 0.5)
    xn, yn = f(x) + f(0.5), f(y) + f(0.5)
    dist = _dist2f(xn, yn, xc, yc)
    s2 = np.sqrt(f(2.0), dtype=np.float32)
    w = USED | ((F_ << DIR_OFF) if annular else 0)
    interp = lambda inside: (w & ~((7 << SCHEME_OFF) | (31 << DIR_OFF))) | (INTERP << SCHEME_OFF) | \
        ((S_ if inside else N_) << DIR_OFF)
    if not annular:
        if dist > R:
            return w & ~USED
        if dist > f(R - s2):
            w = interp(False)
        elif dist > f(R - f(2 * s2)):
            w |= IS_SAVE
        else:
            return w
    else:
        if dist > R or dist < r:
            w &= ~USED
        elif dist > f(R - s2):
            w = interp(False)
        elif dist > f(R - f(2 * s2)):
            w |= IS_SAVE
        elif dist < f(r + s2):
            w = interp(True)
        elif dist < f(r + f(2 * s2)):
            w |= IS_SAVE
    for i, (dx, dy) in enumerate(_DIRS8):
        xa, ya = f(xn - f(dx)), f(yn - f(dy))
        unknown = True
        if xa < NX and xa > 0 and ya < NY and ya > 0:
            da = _dist2f(xa, ya, xc, yc)
            unknown = bool(da > R or (annular and da < r))
        if unknown:
            w |= (1 << i) << 23
    return w


BUILDER_NAMES = {0: "periodic", 1: "plates_y", 2: "lid_driven", 3: "closed_box", 4: "square_duct",
                 5: "duct_yz", 6: "lid_cavity_closed", 7: "plates_y_free_slip", 8: "plates_y_zouhe",
                 9: "circular_duct", 10: "annular_duct"}
