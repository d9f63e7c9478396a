"""The drop-in run configuration: pyvisc's YAML (pyvisc/schemes.py:53-74) read by
vlbm_run_config_parse, without a GPU."""
import ctypes

import pytest

BASE = """\
# a pyvisc configuration: a list whose first item is used (conf_handler.py:20)
- sim_id: 7
  precision: single
  steps: 3000
  NX: 48
  NY: 24
  NZ: 16
  FX: 2e-6
  FY: 0
  FZ: 0
  tau: 0.9
  vel_set: D3Q27
  use_ibm: false
  non_newtonian_model: null
  path_save: results
  macr_save: 1000
  data_report: 500
  data_stop: false
  data_save: true
  pop_save: false
  ini_step: 0
  n_gpus: 1
  resid_max: 1e-5
"""


def parse(vlbm, text, max_spheres=0):
    rc = vlbm.RunConfig()
    sph = (vlbm.Sphere * max(1, max_spheres))()
    st = vlbm.lib().vlbm_run_config_parse(text.encode(), ctypes.byref(rc), sph, max_spheres)
    return st, rc, list(sph)[:max_spheres]


def test_scheme_keys_map_onto_the_configuration(vlbm):
    st, rc, _ = parse(vlbm, BASE)
    assert st == vlbm.OK, vlbm.lib().vlbm_last_error()
    c = rc.cfg
    assert (c.nx, c.ny, c.nz, c.vel_set) == (48, 24, 16, 27)
    assert c.tau == 0.9 and c.fx == 2e-6 and c.fy == 0 and c.rheology == vlbm.NEWTONIAN
    assert rc.sim_id == b"007"                     # var.h.j2: '%03d' % sim_id
    assert rc.path_save == b"results"
    assert (rc.steps, rc.macr_save, rc.data_report, rc.ini_step) == (3000, 1000, 500, 0)
    assert (rc.data_stop, rc.data_save, rc.pop_save, rc.n_gpus) == (0, 1, 0, 1)
    assert rc.resid_max == 1e-5 and rc.use_ibm == 0
    assert rc.builder == vlbm.BUILDER_CLOSED_BOX   # the builder compiled by default
    assert list(c.ux_bc)[:2] == [0.0, 0.1]          # var.h:114 with U_MAX = 0.1


def test_bare_mapping_and_defaults(vlbm):
    text = "\n".join(line[2:] for line in BASE.splitlines() if line.startswith("  ") or line.startswith("- "))
    text = text.replace("data_save: true", "")
    text = "\n".join(l for l in text.splitlines() if not l.startswith(("FY", "FZ", "ini_step", "n_gpus")))
    st, rc, _ = parse(vlbm, text)
    assert st == vlbm.OK, vlbm.lib().vlbm_last_error()
    assert rc.data_save == 0 and rc.cfg.fy == 0 and rc.n_gpus == 1


@pytest.mark.parametrize("key", ["precision", "NX", "tau", "vel_set", "use_ibm", "sim_id", "path_save", "steps",
                                 "macr_save", "data_report"])
def test_required_keys(vlbm, key):
    lines = BASE.splitlines()
    k = next(i for i, l in enumerate(lines) if l.lstrip("- ").startswith(key + ":"))
    if lines[k].startswith("- "):      # keep the list item's marker on the next key
        lines[k + 1] = "- " + lines[k + 1][2:]
    text = "\n".join(lines[:k] + lines[k + 1:])
    st, _, _ = parse(vlbm, text)
    assert st == vlbm.ERR_INVALID
    assert key.encode() in vlbm.lib().vlbm_last_error() and b"field required" in vlbm.lib().vlbm_last_error()


@pytest.mark.parametrize("key,value,status,msg", [
    ("tau", "abc", 1, b"valid float"), ("NX", "12.5", 1, b"valid integer"), ("vel_set", "D2Q9", 1, b"permitted"),
    ("use_ibm", "maybe", 1, b"boolean"), ("non_newtonian_model", "CASSON", 1, b"BINGHAM"),
    ("precision", "double", 4, b"precision"), ("n_gpus", "2", 4, b"n_gpus"), ("precision", "half", 1, b"permitted"),
])
def test_rejected_values(vlbm, key, value, status, msg):
    text = "\n".join((f"  {key}: {value}" if l.strip().startswith(key + ":") else l) for l in BASE.splitlines())
    st, _, _ = parse(vlbm, text)
    assert st == status
    assert msg in vlbm.lib().vlbm_last_error()


def test_extension_keys_and_spheres(vlbm):
    text = BASE.replace("  non_newtonian_model: null", """\
  non_newtonian_model: "BINGHAM"   # quoted scalars work too
  eta_p: 0.1
  yield_stress: 2e-5
  builder: plates_y
  storage: f16
  collision: bgk
  rho_0: 1.0
  u_max: 0.05
  uz_bc: [0, 0.02, -0.02]
  checkpoint_save: 2000
  ibm:
    max_iterations: 3
    gz: -1e-5
    wall_x: true
    particles_save: 100
    particle_density: 1.5
    spheres:
      - diameter: 8
        center: [10.5, 12, 8]
      - diameter: 6
        center: [30, 12, 8.25]
        velocity: [0.001, 0, 0]
        movable: false""").replace("use_ibm: false", "use_ibm: true")
    st, rc, sph = parse(vlbm, text, 4)
    assert st == vlbm.OK, vlbm.lib().vlbm_last_error()
    c = rc.cfg
    assert c.rheology == vlbm.BINGHAM and c.eta_p == 0.1 and c.yield_stress == 2e-5
    assert rc.builder == vlbm.BUILDER_PLATES_Y and c.storage == vlbm.STORE_F16 and c.collision == vlbm.OP_BGK
    assert list(c.uz_bc)[:3] == [0, 0.02, -0.02] and list(c.ux_bc)[:2] == [0, 0.05]
    assert rc.checkpoint_save == 2000 and rc.particles_save == 100
    assert rc.ibm.max_iterations == 3 and rc.ibm.gz == -1e-5 and rc.ibm.wall_x == 1
    assert rc.n_spheres == 2
    assert (sph[0].diameter, sph[0].cx, sph[0].cy, sph[0].cz, sph[0].density, sph[0].movable) == (8, 10.5, 12, 8, 1.5, 1)
    assert (sph[1].vx, sph[1].movable, sph[1].cz) == (0.001, 0, 8.25)


def test_malformed_yaml(vlbm):
    for bad in ("- sim_id: 1\n   NX: 4\n  NY: 4\n", "- [1, 2\n", "- a: 1\n  a: 2\n", ""):
        st, _, _ = parse(vlbm, bad)
        assert st == vlbm.ERR_INVALID, bad


def test_loader_reads_files_and_reports_missing(vlbm, tmp_path):
    p = tmp_path / "conf.yaml"
    p.write_text(BASE)
    rc, spheres = vlbm.load_run_config(path=str(p))
    assert rc.cfg.nx == 48 and spheres == []
    with pytest.raises(vlbm.VlbmError) as e:
        vlbm.load_run_config(path=str(tmp_path / "missing.yaml"))
    assert e.value.status == vlbm.ERR_NOT_FOUND


def test_driver_is_built_and_prints_usage(vlbm):
    import os
    import subprocess
    exe = vlbm.driver_path()
    assert os.path.exists(exe)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "usage" in r.stderr
