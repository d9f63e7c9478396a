"""The C-ABI library loads and exports every function include/vlbm.h declares."""
import os
import re
import subprocess

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    text = open(os.path.join(REPO, "include", "vlbm.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(vlbm_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_core_entry_points():
    names = declared()
    for n in ("vlbm_create", "vlbm_step", "vlbm_get_macroscopics", "vlbm_set_node_map", "vlbm_destroy"):
        assert n in names


def test_library_exports_every_declared_symbol(vlbm):
    out = subprocess.run(["nm", "-D", "--defined-only", vlbm.lib_path()], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (vlbm_\w+)", out))
    missing = [n for n in declared() if n not in exported]
    assert not missing, missing


def test_binding_covers_header(vlbm):
    assert sorted(vlbm.EXPORTED) == declared()


def test_config_defaults_match_reference_var_h(vlbm):
    c = vlbm.Config.default()
    assert (c.nx, c.ny, c.nz) == (128, 128, 384)      # var.h:95-100
    assert c.vel_set == 19 and abs(c.tau - 0.6) < 1e-15 and c.rho0 == 1.0
    assert list(c.ux_bc)[:2] == [0.0, 0.1]            # var.h:114
    assert abs(c.eta_p - 0.3) < 1e-15 and abs(c.yield_stress - 1e-4) < 1e-18  # nnf.h:20-21
    assert vlbm.lib().vlbm_abi_version() == 2


def test_invalid_config_is_rejected_without_gpu(vlbm):
    c = vlbm.Config.default(tau=0.4)
    import ctypes
    h = ctypes.c_void_p()
    st = vlbm.lib().vlbm_create(ctypes.byref(c), ctypes.byref(h))
    assert st == vlbm.ERR_INVALID
    assert b"tau" in vlbm.lib().vlbm_last_error()


def test_checkpoint_calls_reject_null_arguments_without_gpu(vlbm):
    import ctypes
    L = vlbm.lib()
    need = ctypes.c_size_t()
    assert L.vlbm_checkpoint_save(None, None, 0, ctypes.byref(need)) == vlbm.ERR_INVALID
    assert L.vlbm_checkpoint_load(None, None, 0) == vlbm.ERR_INVALID
    assert L.vlbm_save_checkpoint(None, None, None) == vlbm.ERR_INVALID
    assert L.vlbm_load_checkpoint(None, b"/nonexistent", b"x") == vlbm.ERR_INVALID
