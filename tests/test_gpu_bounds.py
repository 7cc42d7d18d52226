"""The bounds-checked build (python -m baas_b200.build --debug-bounds, loaded with BAAS_LIB=bounds):
its kernels check every index they read through in the cluster walk (small.cuh) and the level
walk (staged.cuh) and report a failed check as a status instead of touching memory outside an
array. Run in a child process (this one has the ordinary library loaded) on the systems those
walks take: every call returns OK and the results equal the oracle's."""
import os
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
CHILD = r"""
import numpy as np, torch
from baas_b200 import (KERNEL_ICCG, PREC_FP32_FACTORS, PREC_FP64, WALK_LEVELS, WALK_SMALL, DeviceCSR, Schedule, gen,
                       _native)
from oracle.oracle import Port
assert _native.lib_path().name == "libbaas_b200_bounds.so"
A = gen.knn_stiffness(nodes=1500, k=12, seed=6)
dA = DeviceCSR.from_host(A)
b = gen.uniform_rhs(A.n, 3)
xo, ito, _ = Port.pcg(A, b, tol=1e-10)
want, _ = Port.ic0(A)
Lo = gen.CSR(A.n, A.rowptr, A.colidx, want).lower()
for walk, cs in ((WALK_SMALL, 1), (WALK_SMALL, 8), (WALK_LEVELS, 0)):
    s = Schedule(A, kind=KERNEL_ICCG, nthread=8, walk=walk, small_cluster=cs)
    lu = dA.values.clone()
    s.ic0(dA, lu)
    assert np.array_equal(lu.cpu().numpy(), want)
    y = torch.zeros(A.n, dtype=torch.float64, device="cuda")
    s.forward(DeviceCSR.from_host(Lo), torch.from_numpy(b).cuda(), y)
    assert np.array_equal(y.cpu().numpy(), Port.lower_solve(Lo, b))
    for prec in (PREC_FP64, PREC_FP32_FACTORS):
        x = torch.zeros(A.n, dtype=torch.float64, device="cuda")
        it, rel = s.iccg(dA, torch.from_numpy(b).cuda(), x, tol=1e-10, precision=prec)
        assert rel < 1e-10 and np.linalg.norm(x.cpu().numpy() - xo) / np.linalg.norm(xo) < 1e-9
print("OK bounds")
"""


def test_bounds_checked_build_runs_clean():
    lib = ROOT / "baas_b200" / "_lib" / "libbaas_b200_bounds.so"
    assert lib.exists(), "build it with python -m baas_b200.build --debug-bounds (__graft_entry__.build does)"
    env = dict(os.environ, BAAS_LIB="bounds", PYTHONPATH=str(ROOT))
    r = subprocess.run([sys.executable, "-c", CHILD], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "OK bounds" in r.stdout, r.stdout[-2000:] + r.stderr[-2000:]
