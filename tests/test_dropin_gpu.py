"""The reference drivers' call pattern, compiled against the cuStinger-compatible headers."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def build_driver(tmp_path):
    exe = str(tmp_path / "dropin_driver")
    lib = os.path.join(ROOT, "custingeralg_b200")
    cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O2", "-I",
           os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", "dropin_driver.cu"), "-o", exe,
           "-L", lib, "-lcustinger_tc", "-ltcgen", "-Xlinker", "-rpath", "-Xlinker", lib]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return exe


@pytest.mark.parametrize("scale,edges", [(10, 100), (14, 2000)])
def test_reference_call_pattern(tmp_path, scale, edges):
    exe = build_driver(tmp_path)
    r = subprocess.run([exe, str(scale), str(edges)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "dropin driver ok" in r.stdout
