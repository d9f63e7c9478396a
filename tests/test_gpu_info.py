"""Run-information file (saveSimInfo / getSimInfoString, lbmReport.cpp:174-386)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def parse(path):
    out = {}
    for line in open(path):
        if ":" in line and not line.startswith("-"):
            k, v = line.split(":", 1)
            out[k.strip()] = v.strip()
    return out


def test_info_file_keys_and_values(vlbm, tmp_path):
    cfg = vlbm.Config.default(nx=24, ny=20, nz=16, rheology=vlbm.BINGHAM, eta_p=0.1, yield_stress=1e-6,
                              fx=1e-5, storage=vlbm.STORE_F16)
    sim = vlbm.Simulation(cfg, builder=vlbm.BUILDER_CLOSED_BOX)
    sim.add_spheres(vlbm.IbmConfig.default(max_iterations=2, gz=-1e-5),
                    [vlbm.Sphere(diameter=6, cx=12.0, cy=10.0, cz=8.0, density=1.5, movable=1)])
    sim.step(10)
    sim.sync()
    sim.write_info(str(tmp_path), "007", 1000, 0.5, report_steps=100, save_steps=500, u_max=0.05)
    f = tmp_path / "007" / "007_info.txt"
    text = f.read_text()
    d = parse(f)
    assert text.startswith("---------------------------- SIMULATION INFORMATION")
    assert d["Simulation ID"] == "007" and d["Velocity set"] == "D3Q19" and d["Precision"] == "float"
    assert (d["NX"], d["NY"], d["NZ"], d["NZ_TOTAL"]) == ("24", "20", "16", "16")
    assert d["FX"] == "1.000000e-05" and d["Umax"] == "5.000000e-02"
    assert d["Report steps"] == "100" and d["Save steps"] == "500" and d["Nsteps"] == "1000"
    assert float(d["MLUPS"]) == pytest.approx(1000 * 24 * 20 * 16 / 1e6 / 0.5, abs=0.05)
    assert d["Time elapsed"] == "0.500 (s)"
    assert d["Population storage"] == "float16 deviations"
    assert d["Model"] == "Bingham" and float(d["Plastic omega"]) == pytest.approx(1 / 0.8, rel=1e-6)
    assert d["Number of particles"] == "1" and d["IBM iterations"] == "2" and d["Stencil size"] == "4"
    assert "CUDA INFORMATION" in text and d["compute capability"] == "10.0"


def read_macr(path, nx, ny, nz):
    """Raw little-endian float32 [NZ][NY][NX], as fileTreat.readFileMacr3D reads it
    (src/Post Processing/fileTreat.py:146-168)."""
    a = np.fromfile(path, dtype="<f4")
    assert a.size == nx * ny * nz, (path, a.size)
    return a.reshape(nz, ny, nx)


@pytest.mark.parametrize("rheology", [0, 2])
def test_macr_bin_names_and_contents(vlbm, tmp_path, rheology):
    """vlbm_write_macr_bin: getVarFilename's names (lbmReport.cpp:55-83; step 0 has
    seven digits, later steps six) and the fields of vlbm_get_macroscopics."""
    nx, ny, nz = 20, 12, 8
    kw = dict(n_index=0.7, k_consistency=0.05) if rheology == 2 else {}
    cfg = vlbm.Config.default(nx=nx, ny=ny, nz=nz, rheology=rheology, fx=2e-5, fz=-1e-5, **kw)
    sim = vlbm.Simulation(cfg, builder=vlbm.BUILDER_PLATES_Y)
    sim.write_macr_bin(str(tmp_path), "042", 0)
    sim.step(37)
    sim.sync()
    sim.write_macr_bin(str(tmp_path), "042", 37)
    m = sim.macroscopics()
    sim.close()
    names = ["rho", "ux", "uy", "uz"] + (["omega"] if rheology else [])
    got = sorted(p.name for p in (tmp_path / "042").iterdir())
    want = sorted([f"042_{v}0000000.bin" for v in names] + [f"042_{v}000037.bin" for v in names])
    assert got == want
    for v in names:
        a = read_macr(tmp_path / "042" / f"042_{v}000037.bin", nx, ny, nz)
        np.testing.assert_array_equal(a, m[v])
    r0 = read_macr(tmp_path / "042" / "042_rho0000000.bin", nx, ny, nz)
    np.testing.assert_array_equal(r0, np.ones_like(r0))
    assert np.abs(m["ux"]).max() > 0


def test_macr_bin_step_field(vlbm, tmp_path):
    """Step fields of getVarFilename for steps of one to seven digits."""
    cfg = vlbm.Config.default(nx=4, ny=4, nz=4)
    sim = vlbm.Simulation(cfg)
    cases = {1: "000001", 99: "000099", 12345: "012345", 100000: "100000", 999999: "999999",
             1234567: "1234567"}
    for step, field in cases.items():
        sim.write_macr_bin(str(tmp_path), "s", step)
        assert (tmp_path / "s" / f"s_rho{field}.bin").exists(), step
    sim.close()
