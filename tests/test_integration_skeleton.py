"""The C++ driver skeleton of INTEGRATION.md compiles against include/vlbm.h
and links against libvlbm.so (no GPU needed: it is built, not run)."""
import os
import re
import shutil
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(REPO, "viscoplastic-lbm_b200", "libvlbm.so")


def test_integration_cpp_skeleton_builds(tmp_path):
    text = open(os.path.join(REPO, "INTEGRATION.md")).read()
    blocks = re.findall(r"```cpp\n(.*?)```", text, flags=re.S)
    assert len(blocks) == 1, "one C++ skeleton expected"
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    if not os.path.exists(LIB):
        pytest.skip("libvlbm.so not built")
    src = tmp_path / "skeleton.cpp"
    src.write_text(blocks[0])
    exe = tmp_path / "skeleton"
    r = subprocess.run([gxx, "-std=c++17", "-Wall", "-Werror", str(src), "-I", os.path.join(REPO, "include"),
                        "-L", os.path.dirname(LIB), "-lvlbm", "-Wl,-rpath," + os.path.dirname(LIB), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
