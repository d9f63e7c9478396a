"""The drop-in host program (viscoplastic-lbm_b200/driver/vlbm_run.cpp): the
reference's YAML in, the reference's files out.

Each test writes a pyvisc configuration, runs `vlbm_run -c conf.yaml`, reads
every .bin back as fileTreat.readFileMacr3D does (raw float32 [NZ][NY][NX],
src/Post Processing/fileTreat.py:146-168) and compares it with the same
simulation run through the Python binding, checking the names getVarFilename
gives (lbmReport.cpp:55-83) and the label conventions of main.cu: a save at
step s holds the state after s steps, the final save (labelled N_STEPS) the
state after N_STEPS - 1 steps."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CONF = """\
- sim_id: 12
  precision: single
  steps: 300
  NX: 24
  NY: 16
  NZ: 8
  FX: 1e-5
  tau: 0.8
  vel_set: D3Q19
  use_ibm: false
  non_newtonian_model: BINGHAM
  eta_p: 0.1
  yield_stress: 1e-6
  builder: plates_y
  path_save: {path}
  macr_save: 100
  data_report: 150
  data_save: true
"""


def run_driver(vlbm, tmp_path, text):
    conf = tmp_path / "conf.yaml"
    conf.write_text(text)
    r = subprocess.run([vlbm.driver_path(), "-c", str(conf)], capture_output=True, text=True, timeout=600,
                       cwd=str(tmp_path))
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r.stdout


def read_bin(path, shape):
    a = np.fromfile(path, dtype="<f4")
    assert a.size == np.prod(shape), path
    return a.reshape(shape)


def test_driver_writes_the_reference_files(vlbm, tmp_path):
    out = tmp_path / "out"
    stdout = run_driver(vlbm, tmp_path, CONF.format(path=str(out)))
    d = out / "012"
    names = sorted(p.name for p in d.iterdir())
    fields = ["rho", "ux", "uy", "uz", "omega"]
    want = sorted([f"012_{v}{s}.bin" for v in fields for s in ("000100", "000200", "000300")]
                  + ["012_info.txt", "012_avgUz000150.csv"])
    assert names == want, names
    assert "TREATED DATA" in stdout and "Step: 150" in stdout
    rc, _ = vlbm.load_run_config(path=str(tmp_path / "conf.yaml"))
    shape = (8, 16, 24)
    sim = vlbm.Simulation(rc.cfg, builder=rc.builder)
    done = 0
    for label, steps in ((100, 100), (200, 200), (300, 299)):
        sim.step(steps - done)
        done = steps
        m = sim.macroscopics()
        for v in fields:
            np.testing.assert_array_equal(read_bin(d / f"012_{v}{label:06d}.bin", shape), m[v], err_msg=f"{v} {label}")
    sim.close()
    info = (d / "012_info.txt").read_text()
    assert "Nsteps: 300" in info.replace("  ", " ") or "300" in info
    csv = (d / "012_avgUz000150.csv").read_text().splitlines()
    assert csv[0] == "y\tavg uz" and len(csv) == 17


def test_driver_stops_on_the_data_condition(vlbm, tmp_path):
    """DATA_STOP with a residual bound that the first report meets: the run stops
    at step data_report and its final save carries that label (main.cu:477-483)."""
    out = tmp_path / "out"
    text = CONF.format(path=str(out)).replace("data_save: true", "data_save: false\n  data_stop: true\n  resid_max: 2.0")
    stdout = run_driver(vlbm, tmp_path, text)
    assert "Stopping because of LBM" in stdout
    names = sorted(p.name for p in (out / "012").iterdir() if p.name.startswith("012_rho"))
    assert names == ["012_rho000100.bin", "012_rho000150.bin"]


def test_driver_checkpoint_and_resume(vlbm, tmp_path):
    """CHECKPOINT_SAVE writes the image; load_checkpoint continues from its step
    and ends in the same state as one uninterrupted run."""
    out = tmp_path / "out"
    first = CONF.format(path=str(out)).replace("steps: 300", "steps: 120").replace("data_report: 150", "data_report: 0")
    first += "  checkpoint_save: 1000\n"
    run_driver(vlbm, tmp_path, first)
    assert (out / "012" / "checkpoint" / "0_state.bin").exists()
    second = CONF.format(path=str(out)).replace("data_report: 150", "data_report: 0").replace("sim_id: 12", "sim_id: 12")
    second += f"  load_checkpoint: true\n  checkpoint_folder: {out}\n"
    run_driver(vlbm, tmp_path, second)
    rc, _ = vlbm.load_run_config(path=str(tmp_path / "conf.yaml"))
    sim = vlbm.Simulation(rc.cfg, builder=rc.builder)
    sim.step(299)
    m = sim.macroscopics()
    sim.close()
    np.testing.assert_array_equal(read_bin(out / "012" / "012_ux000300.bin", (8, 16, 24)), m["ux"])


def test_driver_with_spheres_writes_particle_files(vlbm, tmp_path):
    out = tmp_path / "out"
    text = CONF.format(path=str(out)).replace("use_ibm: false", "use_ibm: true").replace(
        "builder: plates_y", "builder: closed_box").replace("data_report: 150", "data_report: 0")
    text += """  ibm:
    max_iterations: 2
    gz: -1e-5
    particles_save: 100
    spheres:
      - diameter: 6
        center: [12, 8, 4]
        density: 1.5
"""
    text = text.replace("NZ: 8", "NZ: 10").replace("center: [12, 8, 4]", "center: [12, 8, 5]")
    run_driver(vlbm, tmp_path, text)
    d = out / "012"
    for s in ("0000000", "000100", "000200", "000300"):
        assert (d / f"012_pCenters{s}.csv").exists(), s
        assert (d / f"012_pNodes{s}.csv").exists(), s
    rows = (d / "012_pCenters000300.csv").read_text().splitlines()
    head = rows[0].split(",")
    assert head[:5] == ["p_number", "step", "pos_x", "pos_y", "pos_z"] and head[-1] == "semi3z" and len(head) == 36
    vals = rows[1].split(",")
    assert vals[0] == "0" and vals[1] == "300"
    rc, spheres = vlbm.load_run_config(path=str(tmp_path / "conf.yaml"))
    sim = vlbm.Simulation(rc.cfg, builder=rc.builder)
    sim.add_spheres(rc.ibm, spheres)
    sim.step(300)
    p = sim.particles(1)[0]
    nodes = sim.info().n_lagrangian_nodes
    sim.close()
    np.testing.assert_allclose([float(v) for v in vals[2:5]], list(p.pos), rtol=1e-6)
    assert len((d / "012_pNodes000300.csv").read_text().splitlines()) == nodes + 1
