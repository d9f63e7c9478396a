"""Python binding of libvlbm (include/vlbm.h) over ctypes.

This module mirrors the reference's simulation interface for Python callers:
the YAML keys of pyvisc (pyvisc/schemes.py:49-74), the compile-time constants
of src/CUDA/var.h and NNF/nnf.h become fields of `Config`; the reference's
main loop (src/CUDA/main.cu:270-507) becomes `Simulation.step()`.

The CUDA library is mandatory: importing this module loads the in-tree
libvlbm.so and raises if it is missing.  There is no CPU fallback.
"""
import ctypes as C
import os
import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libvlbm.so")

if not os.path.exists(_LIB_PATH):
    raise ImportError(
        "libvlbm.so not found next to vlbm.py; build it with "
        "`python viscoplastic-lbm_b200/build.py` (nvcc, sm_100a)")
_lib = C.CDLL(_LIB_PATH)

# ----------------------------------------------------------------- enums --
OK, ERR_INVALID, ERR_CUDA, ERR_NOMEM, ERR_UNSUPPORTED, ERR_DIVERGED, ERR_STATE = range(7)
ERR_NOT_FOUND, ERR_IO = 8, 9
D3Q19, D3Q27 = 19, 27
OP_REGULARIZED, OP_BGK = 0, 1
NEWTONIAN, BINGHAM, POWERLAW = 0, 1, 2
STORE_F32, STORE_F16, STORE_BF16 = 0, 1, 2
LAYOUT_AUTO, LAYOUT_NATURAL, LAYOUT_ZPAIR = 0, 1, 2
(BUILDER_PERIODIC, BUILDER_PLATES_Y, BUILDER_LID_DRIVEN, BUILDER_CLOSED_BOX,
 BUILDER_SQUARE_DUCT, BUILDER_DUCT_YZ, BUILDER_LID_CAVITY_CLOSED,
 BUILDER_PLATES_Y_FREE_SLIP, BUILDER_PLATES_Y_ZOUHE, BUILDER_CIRCULAR_DUCT,
 BUILDER_ANNULAR_DUCT) = range(11)
BC_NULL, BC_VEL_ZOUHE, BC_VEL_BOUNCE_BACK, BC_PRES_ZOUHE, BC_FREE_SLIP, \
    BC_BOUNCE_BACK, BC_INTERP_BOUNCE_BACK, BC_SPECIAL = range(8)
DIRECTIONS = ["N", "S", "W", "E", "F", "B", "NW", "NE", "NF", "NB", "SW", "SE", "SF", "SB",
              "WF", "WB", "EF", "EB", "NWF", "NWB", "NEF", "NEB", "SWF", "SWB", "SEF", "SEB"]
MAP_RHO_IDX_OFFSET, MAP_UZ_IDX_OFFSET, MAP_UY_IDX_OFFSET, MAP_UX_IDX_OFFSET = 0, 3, 6, 9
MAP_GEOMETRY_OFFSET, MAP_DIRECTION_OFFSET, MAP_SCHEME_OFFSET = 12, 13, 18
MAP_IS_USED_OFFSET, MAP_SAVE_POST_COL_OFFSET, MAP_INTERP_BB_OFFSET = 21, 22, 23


class VlbmError(RuntimeError):
    def __init__(self, status, where):
        msg = _lib.vlbm_last_error()
        text = msg.decode() if msg else ""
        super().__init__(f"{where} failed with status {status}: {text}")
        self.status = status


class Config(C.Structure):
    """vlbm_config (include/vlbm.h)."""
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
        c = cls()
        _check(_lib.vlbm_config_default(C.byref(c)), "vlbm_config_default")
        for k, v in kw.items():
            if k in ("ux_bc", "uy_bc", "uz_bc", "rho_bc"):
                arr = getattr(c, k)
                for i, val in enumerate(v):
                    arr[i] = val
            else:
                setattr(c, k, v)
        return c

    def as_dict(self):
        d = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            if name.endswith("_bc"):
                v = list(v)
            elif name == "reserved":
                continue
            d[name] = v
        return d


class IbmConfig(C.Structure):
    """vlbm_ibm_config (include/vlbm.h)."""
    _fields_ = [
        ("max_iterations", C.c_int32), ("stencil", C.c_int32),
        ("thickness", C.c_double), ("movement_alpha", C.c_double),
        ("fluid_density", C.c_double),
        ("gx", C.c_double), ("gy", C.c_double), ("gz", C.c_double),
        ("wall_x", C.c_int32), ("wall_y", C.c_int32), ("wall_z", C.c_int32),
        ("pp_friction", C.c_double), ("pw_friction", C.c_double),
        ("pp_restitution", C.c_double), ("pw_restitution", C.c_double),
        ("particle_young", C.c_double), ("particle_poisson", C.c_double),
        ("wall_young", C.c_double), ("wall_poisson", C.c_double),
        ("mesh_scale", C.c_double), ("breugem", C.c_double),
        ("reserved", C.c_int32 * 8),
    ]

    @classmethod
    def default(cls, **kw):
        c = cls()
        _check(_lib.vlbm_ibm_config_default(C.byref(c)), "vlbm_ibm_config_default")
        for k, v in kw.items():
            setattr(c, k, v)
        return c


class Sphere(C.Structure):
    _fields_ = [
        ("diameter", C.c_double), ("cx", C.c_double), ("cy", C.c_double), ("cz", C.c_double),
        ("vx", C.c_double), ("vy", C.c_double), ("vz", C.c_double),
        ("wx", C.c_double), ("wy", C.c_double), ("wz", C.c_double),
        ("density", C.c_double), ("movable", C.c_int32), ("reserved", C.c_int32),
    ]


class ParticleState(C.Structure):
    _fields_ = [(n, C.c_double * 3) for n in (
        "pos", "vel", "w", "f", "M", "pos_old", "vel_old", "w_old", "f_old", "M_old",
        "w_avg", "w_pos")] + [
        ("I", C.c_double * 6), ("radius", C.c_double), ("volume", C.c_double),
        ("density", C.c_double), ("S", C.c_double),
        ("movable", C.c_int32), ("n_nodes", C.c_int32)]


class Info(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("q", C.c_int32),
        ("storage_bytes", C.c_int32), ("step", C.c_int64), ("n_bc_nodes", C.c_int64),
        ("device_bytes", C.c_int64), ("bytes_per_node_step", C.c_double),
        ("n_particles", C.c_int32), ("n_lagrangian_nodes", C.c_int32),
        ("last_kernel_variant", C.c_int32), ("layout", C.c_int32), ("aa_parity", C.c_int32),
        ("reserved", C.c_int32 * 5),
    ]


class Treat(C.Structure):
    _fields_ = [("step", C.c_int64), ("residual", C.c_double), ("avg_rho", C.c_double),
                ("stop", C.c_int32), ("reserved", C.c_int32)]


class Request(C.Structure):
    _fields_ = [
        ("cfg", Config), ("builder", C.c_int32), ("steps", C.c_uint32),
        ("tag", C.c_uint64), ("n_spheres", C.c_int32),
        ("spheres", C.POINTER(Sphere)), ("ibm", IbmConfig),
    ]


class Completion(C.Structure):
    _fields_ = [
        ("tag", C.c_uint64), ("status", C.c_int),
        ("submit_time_s", C.c_double), ("start_time_s", C.c_double),
        ("finish_time_s", C.c_double), ("mean_ux", C.c_double), ("steps", C.c_uint64),
    ]


class RunConfig(C.Structure):
    """vlbm_run_config (include/vlbm.h): the drop-in driver's configuration,
    read from the reference's pyvisc YAML file."""
    _fields_ = [
        ("cfg", Config), ("ibm", IbmConfig), ("builder", C.c_int32), ("use_ibm", C.c_int32),
        ("precision_double", C.c_int32), ("n_gpus", C.c_int32),
        ("steps", C.c_int64), ("ini_step", C.c_int64), ("macr_save", C.c_int64), ("data_report", C.c_int64),
        ("checkpoint_save", C.c_int64), ("particles_save", C.c_int64),
        ("data_stop", C.c_int32), ("data_save", C.c_int32), ("pop_save", C.c_int32), ("load_checkpoint", C.c_int32),
        ("particles_nodes_save", C.c_int32), ("export_forces", C.c_int32), ("n_spheres", C.c_int32),
        ("reserved0", C.c_int32), ("resid_max", C.c_double), ("u_max", C.c_double),
        ("sim_id", C.c_char * 32), ("path_save", C.c_char * 256), ("load_folder", C.c_char * 256),
        ("reserved", C.c_int32 * 16),
    ]


_P = C.c_void_p
_F32P = C.POINTER(C.c_float)
_U32P = C.POINTER(C.c_uint32)
_F64P = C.POINTER(C.c_double)

_SIGS = {
    "vlbm_config_default": [C.POINTER(Config)],
    "vlbm_ibm_config_default": [C.POINTER(IbmConfig)],
    "vlbm_create": [C.POINTER(Config), C.POINTER(_P)],
    "vlbm_destroy": [_P],
    "vlbm_set_node_map": [_P, _U32P, C.c_size_t],
    "vlbm_set_builder": [_P, C.c_int32],
    "vlbm_build_node_map": [C.c_int, C.c_int, C.c_int, C.c_int, _U32P, C.c_size_t],
    "vlbm_init_equilibrium": [_P, C.c_double, C.c_double, C.c_double, C.c_double],
    "vlbm_step": [_P, C.c_uint32],
    "vlbm_sync": [_P],
    "vlbm_set_stream": [_P, _P],
    "vlbm_get_macroscopics": [_P, _F32P, _F32P, _F32P, _F32P, _F32P],
    "vlbm_get_macroscopics_device": [_P, _P, _P, _P, _P, _P],
    "vlbm_get_populations": [_P, _F32P, C.c_size_t],
    "vlbm_set_populations": [_P, _F32P, C.c_size_t],
    "vlbm_get_forces": [_P, _F32P, C.c_size_t],
    "vlbm_get_info": [_P, C.POINTER(Info)],
    "vlbm_moments_sum": [_P, _F64P],
    "vlbm_moments_sum_noalloc": [_P, _F64P],
    "vlbm_add_spheres": [_P, C.POINTER(IbmConfig), C.POINTER(Sphere), C.c_int32],
    "vlbm_get_particles": [_P, C.POINTER(ParticleState), C.c_int32],
    "vlbm_get_lagrangian_nodes": [_P, _F64P, _F64P, C.c_size_t],
    "vlbm_write_macr_bin": [_P, C.c_char_p, C.c_char_p, C.c_uint32, C.c_int32],
    "vlbm_write_info": [_P, C.c_char_p, C.c_char_p, C.c_uint64, C.c_double, C.c_int32, C.c_int32, C.c_double],
    "vlbm_write_particles_csv": [_P, C.c_char_p, C.c_char_p, C.c_uint32, C.c_int32],
    "vlbm_run_config_parse": [C.c_char_p, C.POINTER(RunConfig), C.POINTER(Sphere), C.c_int32],
    "vlbm_run_config_load": [C.c_char_p, C.POINTER(RunConfig), C.POINTER(Sphere), C.c_int32],
    "vlbm_checkpoint_save": [_P, _P, C.c_size_t, C.POINTER(C.c_size_t)],
    "vlbm_checkpoint_load": [_P, _P, C.c_size_t],
    "vlbm_save_checkpoint": [_P, C.c_char_p, C.c_char_p],
    "vlbm_load_checkpoint": [_P, C.c_char_p, C.c_char_p],
    "vlbm_treat_data": [_P, C.c_double, C.POINTER(Treat), _F64P, C.c_int32],
    "vlbm_server_create": [C.c_int, C.c_size_t, C.c_int32, C.POINTER(_P)],
    "vlbm_server_submit": [_P, C.POINTER(Request)],
    "vlbm_server_pump": [_P, C.c_uint32, C.POINTER(Completion), C.c_int32, C.POINTER(C.c_int32)],
    "vlbm_server_stats": [_P, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                          C.POINTER(C.c_int64), C.POINTER(C.c_double)],
    "vlbm_server_fetch": [_P, C.c_uint64, _F32P, C.c_size_t],
    "vlbm_server_profile": [_P, _F64P, C.c_int32],
    "vlbm_server_set_own_launch_min": [_P, C.c_int64],
    "vlbm_server_destroy": [_P],
    "vlbm_autotune": [_P, C.POINTER(C.c_int32)],
    "vlbm_set_variant": [_P, C.c_int32],
    "vlbm_set_layout": [_P, C.c_int32],
    "vlbm_halo_bytes": [_P, C.POINTER(C.c_size_t)],
    "vlbm_halo_pack": [_P, C.c_int32, C.c_int32, _P],
    "vlbm_halo_unpack": [_P, C.c_int32, C.c_int32, _P],
    "vlbm_halo_pack2": [_P, C.c_int32, C.c_int32, _P, C.c_int32, C.c_int32, _P],
    "vlbm_halo_unpack2": [_P, C.c_int32, C.c_int32, _P, C.c_int32, C.c_int32, _P],
    "vlbm_build_node_map_planes": [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _U32P, C.c_size_t],
}
EXPORTED = sorted(list(_SIGS) + ["vlbm_last_error", "vlbm_abi_version"])

for _name, _args in _SIGS.items():
    try:
        _fn = getattr(_lib, _name)
    except AttributeError:
        continue
    _fn.argtypes = _args
    _fn.restype = C.c_int
_lib.vlbm_last_error.restype = C.c_char_p
_lib.vlbm_last_error.argtypes = []
_lib.vlbm_abi_version.restype = C.c_int
_lib.vlbm_abi_version.argtypes = []


def _check(status, where):
    if status != OK:
        raise VlbmError(status, where)


def lib():
    """The loaded ctypes library (for symbol checks)."""
    return _lib


def lib_path():
    return _LIB_PATH


def _fptr(a):
    return a.ctypes.data_as(_F32P)


def load_run_config(path=None, text=None):
    """Read a pyvisc YAML configuration (file `path` or string `text`):
    returns (RunConfig, [Sphere])."""
    rc = RunConfig()
    fn, arg = (_lib.vlbm_run_config_load, path.encode()) if path is not None else \
        (_lib.vlbm_run_config_parse, text.encode())
    _check(fn(arg, C.byref(rc), None, 0), "vlbm_run_config")
    spheres = (Sphere * max(1, rc.n_spheres))()
    _check(fn(arg, C.byref(rc), spheres, rc.n_spheres), "vlbm_run_config")
    return rc, list(spheres)[:rc.n_spheres]


def driver_path():
    """The drop-in host program built next to the library (driver/vlbm_run.cpp)."""
    return os.path.join(_HERE, "vlbm_run")


def build_node_map(builder, nx, ny, nz):
    """Host restatement of the reference builders, [nz][ny][nx] uint32 words."""
    out = np.zeros(nx * ny * nz, dtype=np.uint32)
    _check(_lib.vlbm_build_node_map(builder, nx, ny, nz, out.ctypes.data_as(_U32P), out.size),
           "vlbm_build_node_map")
    return out


def build_node_map_planes(builder, nx, ny, nz, z_first, n_planes):
    """The builder's words of planes z_first .. z_first + n_planes - 1 (modulo nz)
    of an nx x ny x nz lattice, [n_planes][ny][nx] uint32."""
    out = np.zeros(nx * ny * n_planes, dtype=np.uint32)
    _check(_lib.vlbm_build_node_map_planes(builder, nx, ny, nz, z_first, n_planes, out.ctypes.data_as(_U32P),
                                           out.size), "vlbm_build_node_map_planes")
    return out


class Simulation:
    """One lattice on one GPU (vlbm_sim)."""

    def __init__(self, cfg, node_map=None, builder=None):
        self.cfg = cfg
        h = _P()
        _check(_lib.vlbm_create(C.byref(cfg), C.byref(h)), "vlbm_create")
        self._h = h
        self.n = cfg.nx * cfg.ny * cfg.nz
        if node_map is None:
            # named builder: tables straight from the builder's rules on the faces
            _check(_lib.vlbm_set_builder(self._h, BUILDER_PERIODIC if builder is None else builder),
                   "vlbm_set_builder")
            return
        node_map = np.ascontiguousarray(node_map, dtype=np.uint32).ravel()
        _check(_lib.vlbm_set_node_map(self._h, node_map.ctypes.data_as(_U32P), node_map.size),
               "vlbm_set_node_map")

    def close(self):
        if getattr(self, "_h", None):
            _lib.vlbm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def step(self, n=1):
        _check(_lib.vlbm_step(self._h, n), "vlbm_step")

    def sync(self):
        _check(_lib.vlbm_sync(self._h), "vlbm_sync")

    def set_stream(self, stream_ptr):
        _check(_lib.vlbm_set_stream(self._h, C.c_void_p(stream_ptr)), "vlbm_set_stream")

    def init_equilibrium(self, rho=1.0, ux=0.0, uy=0.0, uz=0.0):
        _check(_lib.vlbm_init_equilibrium(self._h, rho, ux, uy, uz), "vlbm_init_equilibrium")

    def macroscopics(self):
        shape = (self.cfg.nz, self.cfg.ny, self.cfg.nx)
        rho, ux, uy, uz, om = (np.empty(self.n, dtype=np.float32) for _ in range(5))
        _check(_lib.vlbm_get_macroscopics(self._h, _fptr(rho), _fptr(ux), _fptr(uy), _fptr(uz),
                                          _fptr(om)), "vlbm_get_macroscopics")
        return {k: v.reshape(shape) for k, v in
                zip(("rho", "ux", "uy", "uz", "omega"), (rho, ux, uy, uz, om))}

    def macroscopics_device(self, rho, ux, uy, uz, omega=None):
        """Write into device buffers given as integer pointers (e.g. tensor.data_ptr())."""
        _check(_lib.vlbm_get_macroscopics_device(self._h, rho, ux, uy, uz, omega),
               "vlbm_get_macroscopics_device")

    def populations(self):
        q = self.cfg.vel_set
        out = np.empty(q * self.n, dtype=np.float32)
        _check(_lib.vlbm_get_populations(self._h, _fptr(out), out.size), "vlbm_get_populations")
        return out.reshape(q, self.cfg.nz, self.cfg.ny, self.cfg.nx)

    def set_populations(self, pops):
        a = np.ascontiguousarray(pops, dtype=np.float32).ravel()
        _check(_lib.vlbm_set_populations(self._h, _fptr(a), a.size), "vlbm_set_populations")

    def forces(self):
        out = np.empty(3 * self.n, dtype=np.float32)
        _check(_lib.vlbm_get_forces(self._h, _fptr(out), out.size), "vlbm_get_forces")
        return out.reshape(3, self.cfg.nz, self.cfg.ny, self.cfg.nx)

    def moments_sum(self):
        """FP64 (sum rho, sum rho ux, sum rho uy, sum rho uz) of the current state."""
        out = np.zeros(4, dtype=np.float64)
        _check(_lib.vlbm_moments_sum(self._h, out.ctypes.data_as(_F64P)), "vlbm_moments_sum")
        return out

    def info(self):
        i = Info()
        _check(_lib.vlbm_get_info(self._h, C.byref(i)), "vlbm_get_info")
        return i

    def add_spheres(self, ibm_cfg, spheres):
        arr = (Sphere * len(spheres))(*spheres)
        _check(_lib.vlbm_add_spheres(self._h, C.byref(ibm_cfg), arr, len(spheres)), "vlbm_add_spheres")

    def particles(self, n):
        arr = (ParticleState * n)()
        _check(_lib.vlbm_get_particles(self._h, arr, n), "vlbm_get_particles")
        return list(arr)

    def lagrangian_nodes(self):
        n = self.info().n_lagrangian_nodes
        pos = np.empty(3 * n, dtype=np.float64)
        frc = np.empty(3 * n, dtype=np.float64)
        _check(_lib.vlbm_get_lagrangian_nodes(self._h, pos.ctypes.data_as(_F64P),
                                              frc.ctypes.data_as(_F64P), n),
               "vlbm_get_lagrangian_nodes")
        return pos.reshape(3, n), frc.reshape(3, n)

    def write_particles_csv(self, path_files, id_sim, step_label, save_nodes=True):
        _check(_lib.vlbm_write_particles_csv(self._h, path_files.encode(), id_sim.encode(), step_label,
                                             int(save_nodes)), "vlbm_write_particles_csv")

    def write_macr_bin(self, path_files, id_sim, step_label, export_forces=False):
        _check(_lib.vlbm_write_macr_bin(self._h, path_files.encode(), id_sim.encode(),
                                        step_label, int(export_forces)), "vlbm_write_macr_bin")

    def checkpoint(self):
        """The complete state as a uint8 image (vlbm_checkpoint_save)."""
        need = C.c_size_t()
        _check(_lib.vlbm_checkpoint_save(self._h, None, 0, C.byref(need)), "vlbm_checkpoint_save")
        buf = np.empty(need.value, dtype=np.uint8)
        _check(_lib.vlbm_checkpoint_save(self._h, buf.ctypes.data_as(_P), buf.size, C.byref(need)),
               "vlbm_checkpoint_save")
        return buf

    def restore(self, image):
        """Continue from an image written by checkpoint() (vlbm_checkpoint_load)."""
        a = np.ascontiguousarray(image, dtype=np.uint8)
        _check(_lib.vlbm_checkpoint_load(self._h, a.ctypes.data_as(_P), a.size), "vlbm_checkpoint_load")

    def save_checkpoint(self, path_files, id_sim):
        _check(_lib.vlbm_save_checkpoint(self._h, path_files.encode(), id_sim.encode()), "vlbm_save_checkpoint")

    def load_checkpoint(self, path_files, id_sim):
        _check(_lib.vlbm_load_checkpoint(self._h, path_files.encode(), id_sim.encode()), "vlbm_load_checkpoint")

    def treat_data(self, resid_max=1e-5):
        """Report-step residual, mean density, per-plane mean uz and stop flag (vlbm_treat_data)."""
        t = Treat()
        prof = np.empty(self.cfg.ny, dtype=np.float64)
        _check(_lib.vlbm_treat_data(self._h, resid_max, C.byref(t), prof.ctypes.data_as(_F64P), prof.size),
               "vlbm_treat_data")
        return {"step": t.step, "residual": t.residual, "avg_rho": t.avg_rho, "stop": bool(t.stop),
                "avg_uz_plane_xz": prof}

    def write_info(self, path_files, id_sim, total_steps, time_elapsed_s, report_steps=0, save_steps=0,
                   u_max=0.1):
        _check(_lib.vlbm_write_info(self._h, path_files.encode(), id_sim.encode(), total_steps, time_elapsed_s,
                                    report_steps, save_steps, u_max), "vlbm_write_info")

    def autotune(self):
        v = C.c_int32()
        _check(_lib.vlbm_autotune(self._h, C.byref(v)), "vlbm_autotune")
        return v.value

    def set_variant(self, v):
        _check(_lib.vlbm_set_variant(self._h, v), "vlbm_set_variant")

    def set_layout(self, layout):
        _check(_lib.vlbm_set_layout(self._h, layout), "vlbm_set_layout")

    def aa_parity(self):
        """1 when the next step is the in-place scheme's odd (neighbour) step."""
        return self.info().aa_parity

    def halo_bytes(self):
        n = C.c_size_t()
        _check(_lib.vlbm_halo_bytes(self._h, C.byref(n)), "vlbm_halo_bytes")
        return n.value

    def halo_pack(self, z, dz, dst):
        """Populations with c_z == dz of plane z into the device tensor dst (halo_bytes bytes)."""
        _check(_lib.vlbm_halo_pack(self._h, z, dz, C.c_void_p(dst.data_ptr())), "vlbm_halo_pack")

    def halo_unpack(self, z, dz, src):
        _check(_lib.vlbm_halo_unpack(self._h, z, dz, C.c_void_p(src.data_ptr())), "vlbm_halo_unpack")

    def halo_pack2(self, m0, m1):
        """Two messages in one launch; each m is (z, dz, tensor)."""
        _check(_lib.vlbm_halo_pack2(self._h, m0[0], m0[1], C.c_void_p(m0[2].data_ptr()),
                                    m1[0], m1[1], C.c_void_p(m1[2].data_ptr())), "vlbm_halo_pack2")

    def halo_unpack2(self, m0, m1):
        _check(_lib.vlbm_halo_unpack2(self._h, m0[0], m0[1], C.c_void_p(m0[2].data_ptr()),
                                      m1[0], m1[1], C.c_void_p(m1[2].data_ptr())), "vlbm_halo_unpack2")


class Server:
    """Continuous-batching serving loop (vlbm_server)."""

    def __init__(self, device=0, hbm_budget_bytes=8 << 30, max_resident=64):
        h = _P()
        _check(_lib.vlbm_server_create(device, hbm_budget_bytes, max_resident, C.byref(h)),
               "vlbm_server_create")
        self._h = h
        self._keep = []

    def submit(self, cfg, builder, steps, tag, spheres=(), ibm_cfg=None):
        r = Request()
        r.cfg = cfg
        r.builder = builder
        r.steps = steps
        r.tag = tag
        r.n_spheres = len(spheres)
        if spheres:
            arr = (Sphere * len(spheres))(*spheres)
            self._keep.append(arr)
            r.spheres = arr
        r.ibm = ibm_cfg if ibm_cfg is not None else IbmConfig.default()
        _check(_lib.vlbm_server_submit(self._h, C.byref(r)), "vlbm_server_submit")

    def pump(self, steps=1, max_out=1024):
        out = (Completion * max_out)()
        n = C.c_int32()
        _check(_lib.vlbm_server_pump(self._h, steps, out, max_out, C.byref(n)), "vlbm_server_pump")
        return [out[i] for i in range(n.value)]

    def stats(self):
        r, q, b, lu = C.c_int32(), C.c_int32(), C.c_int64(), C.c_double()
        _check(_lib.vlbm_server_stats(self._h, C.byref(r), C.byref(q), C.byref(b), C.byref(lu)),
               "vlbm_server_stats")
        return {"resident": r.value, "queued": q.value, "bytes": b.value, "lattice_updates": lu.value}

    def profile(self):
        """Host seconds per phase of the serving loop, launch counters and the
        device bytes of the memory cache (live, cached)."""
        out = (C.c_double * 16)()
        _check(_lib.vlbm_server_profile(self._h, out, 16), "vlbm_server_profile")
        return dict(zip(("admit_s", "rebuild_s", "enqueue_s", "wait_s", "readout_s", "batch_steps",
                         "direct_launches", "graph_launches", "graph_captures", "capture_s",
                         "device_live_bytes", "device_cached_bytes", "admit_create_s", "admit_tables_s",
                         "admit_spheres_s", "admit_stream_s"), list(out)))

    def set_own_launch_min(self, nodes):
        """Lattices of at least `nodes` nodes get their own launch (-1: default rule)."""
        _check(_lib.vlbm_server_set_own_launch_min(self._h, nodes), "vlbm_server_set_own_launch_min")

    def fetch(self, tag, n):
        out = np.empty(n, dtype=np.float32)
        _check(_lib.vlbm_server_fetch(self._h, tag, _fptr(out), n), "vlbm_server_fetch")
        return out

    def close(self):
        if getattr(self, "_h", None):
            _lib.vlbm_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
