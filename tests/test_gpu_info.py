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
