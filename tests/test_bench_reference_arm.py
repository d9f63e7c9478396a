"""`bench.py --impl reference` (the CPU arm the driver times beside the GPU arm)
runs without a GPU and prints one JSON line with the contract's keys."""
import json
import os
import subprocess
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_json_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "3"],
                       cwd=REPO, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "MLUPS" and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["config"]["workload"] == "d3q19_regularized_bingham_channel_256x128x64"


def test_reference_arm_maps_no_product_library():
    """The reference arm loads the oracle only: after it ran, the process maps
    oracle/liboracle.so and neither libvlbm.so nor torch's CUDA libraries."""
    code = (
        "import sys, io, contextlib; sys.argv=['bench.py','--impl','reference','--steps','1','--warmup','3'];"
        "sys.path.insert(0, '.'); import bench; buf = io.StringIO()\n"
        "with contextlib.redirect_stdout(buf): bench.main()\n"
        "maps = open('/proc/self/maps').read(); print('VLBM', 'libvlbm.so' in maps);"
        "print('ORACLE', 'liboracle.so' in maps); print('TORCH', 'torch' in sys.modules)")
    r = subprocess.run([sys.executable, "-c", code], cwd=REPO, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    out = r.stdout.split()
    assert out[out.index("VLBM") + 1] == "False"
    assert out[out.index("ORACLE") + 1] == "True"
    assert out[out.index("TORCH") + 1] == "False"


def test_oracle_plates_map_matches_builder_restatement():
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import numpy as np
    import oracle
    for size in [(6, 5, 4), (3, 9, 2), (1, 4, 1)]:
        np.testing.assert_array_equal(oracle.plates_y_map(*size), oracle.reference_builder_map("plates_y", *size))


def test_oracle_config_layout_matches_header():
    """oracle.Config mirrors vlbm_config field for field (the oracle reads it as one)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    sys.path.insert(0, os.path.join(REPO, "viscoplastic-lbm_b200"))
    import ctypes
    import oracle
    import vlbm
    assert ctypes.sizeof(oracle.Config) == ctypes.sizeof(vlbm.Config)
    assert [f[0] for f in oracle.Config._fields_] == [f[0] for f in vlbm.Config._fields_]
    for (n, t), (n2, t2) in zip(oracle.Config._fields_, vlbm.Config._fields_):
        assert getattr(oracle.Config, n).offset == getattr(vlbm.Config, n2).offset
    a, b = oracle.Config.default(), vlbm.Config.default()
    for n, _ in oracle.Config._fields_:
        va, vb = getattr(a, n), getattr(b, n)
        if n.endswith("_bc") or n == "reserved":
            assert list(va) == list(vb), n
        else:
            assert va == vb, n
