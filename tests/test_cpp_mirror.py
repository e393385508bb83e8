"""The C++ mirror of the reference classes (include/mlods.hpp) compiles
against the C ABI and, driven like scene::projectPoints (ten one-iteration
project calls on the in-place buffer) and scene::projectPointsOnCPU
(projectCPU per query, serially and from 16 host threads at once on one tree,
bit-identical), agrees with the FP64 oracle."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
from mlodsurfaces_b200 import synth
from mlodsurfaces_b200.apss import Kernel
from mlodsurfaces_b200._capi import LIB_PATH
from conftest import TOL_DIAG, rel_err

ROOT = Path(__file__).resolve().parents[1]


def compile_mirror(tmp: Path) -> Path:
    exe = tmp / "mirror_main"
    cmd = ["g++", "-std=c++17", "-O2", f"-I{ROOT / 'include'}", str(ROOT / "tests" / "cpp" / "mirror_main.cpp"),
           "-o", str(exe), f"-L{LIB_PATH.parent}", "-lmlods", f"-Wl,-rpath,{LIB_PATH.parent}", "-pthread"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_mirror_header_compiles(tmp_path):
    compile_mirror(tmp_path)


@pytest.mark.gpu
def test_mirror_projects_like_the_reference_protocol(tmp_path):
    exe = compile_mirror(tmp_path)
    pts, nrm = synth.torus(20000, seed=51)
    pts = synth.make_tie_free(pts)
    q = synth.perturbed_queries(pts, 0.01, seed=52)[:200]
    for name, arr in (("p", pts), ("n", nrm), ("q", q)):
        arr.astype(np.float32).tofile(tmp_path / f"{name}.bin")
    sigma_rel = 0.04  # in units of the box radius, as the -s CLI option
    res = subprocess.run([str(exe), str(tmp_path / "p.bin"), str(tmp_path / "n.bin"), str(tmp_path / "q.bin"),
                          str(tmp_path / "gpu.bin"), str(tmp_path / "cpu.bin"), str(sigma_rel),
                          str(tmp_path / "sphere.bin")],
                         capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    gpu = np.fromfile(tmp_path / "gpu.bin", np.float32).reshape(-1, 3)
    cpu = np.fromfile(tmp_path / "cpu.bin", np.float32).reshape(-1, 3)
    diag = synth.bbox_diag(pts)
    bb, BB = pts.min(0), pts.max(0)
    d = (BB - bb).astype(np.float32)
    radius = float(np.float32(np.sqrt(np.float32(np.float32(d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]))) / 2)
    k = Kernel()
    k.type = Kernel.GAUSSIAN
    k.sigma = float(np.float32(sigma_rel) * np.float32(radius))
    ot = oracle.OracleTree(pts, nrm, 12)
    g64, _ = ot.project_mlod(q, 10, k, rule=0, cutoff=3.0)
    c64, _ = ot.project_mlod(q, 10, k, rule=1, cutoff=3.0)
    assert rel_err(gpu, g64, diag).max() < TOL_DIAG
    assert rel_err(cpu, c64, diag).max() < TOL_DIAG
    # APSSOctree::cpuSphere against the reference's own (CPUUtils.cpp:638-663)
    u = np.fromfile(tmp_path / "sphere.bin", np.float32).reshape(-1, 5)
    ref_u = oracle.RefTree(pts, nrm, 12).cpu_sphere(q, k, 20)
    assert np.allclose(u, ref_u, rtol=2e-3, atol=2e-3 * np.abs(ref_u).max(axis=0))
