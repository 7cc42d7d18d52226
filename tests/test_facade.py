"""The C++ facade (include/baas_b200.hpp): compiled with g++ against the C ABI library, driven
like the reference's Schedule::Scheduler, results checked against the oracle bit for bit
(tests/cpp/facade_check.cpp)."""
import subprocess
from pathlib import Path

import pytest

from baas_b200 import build

ROOT = Path(__file__).resolve().parents[1]


def _compile(tmp_path):
    lib = build.build_lib()
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "oracle"], check=True)
    exe = tmp_path / "facade_check"
    cuda = Path("/usr/local/cuda")
    cmd = ["/usr/bin/g++", "-std=c++17", "-O2", str(ROOT / "tests" / "cpp" / "facade_check.cpp"),
           f"-I{ROOT / 'include'}", f"-I{ROOT / 'oracle'}", f"-I{cuda / 'include'}",
           f"-L{lib.parent}", "-lbaas_b200", f"-Wl,-rpath,{lib.parent}",
           f"-L{ROOT / 'oracle' / '_lib'}", "-lbaas_oracle", f"-Wl,-rpath,{ROOT / 'oracle' / '_lib'}",
           f"-L{cuda / 'lib64'}", "-lcudart", "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_facade_compiles_and_analyses(tmp_path):
    exe = _compile(tmp_path)
    r = subprocess.run([str(exe), "--analysis-only"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.startswith("OK analysis"), r.stdout + r.stderr


@pytest.mark.gpu
def test_facade_on_gpu(tmp_path):
    exe = _compile(tmp_path)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.startswith("OK gpu"), r.stdout + r.stderr
