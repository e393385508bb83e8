"""Generates tests/golden/golden_small.npz from the reference's own CPU code.

Run in a checkout where the reference sources are available (the reference
shim oracle/_ref/libmlods_ref.so is built from them by oracle/Makefile):

    python tests/golden/make_golden.py

The fixture holds a small seeded torus, the reference octree's topology in
breadth-first order, and the reference's projections (APSSOctree::projectCPU)
in MLoD, global, kNN and ball modes for three kernels, plus kd-tree kNN sets.
The GPU tests compare against it on machines that have no reference sources.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from mlodsurfaces_b200 import synth  # noqa: E402
from mlodsurfaces_b200.apss import Kernel  # noqa: E402

OUT = Path(__file__).resolve().parent / "golden_small.npz"


def kernels(diag: float, radius: float):
    kg = Kernel()
    kg.type = Kernel.GAUSSIAN
    kg.sigma = 0.02 * diag
    km = Kernel()
    km.type = Kernel.GAUSSIAN_MULTIPLE
    km.beginningSigma = 0.02
    km.factor = 2.0
    km.nbOfComputedSigmas = 4
    km.updateSigmas(True, radius)
    ks = Kernel()
    ks.type = Kernel.SINGULAR
    ks.exponent = 4.0
    ks.constant_shift = 1e-3
    return {"gauss": kg, "multi": km, "singular": ks}


def main() -> None:
    oracle.build(with_ref=True)
    pts, nrm = synth.torus(4000, seed=11)
    pts = synth.make_tie_free(pts)
    q = synth.perturbed_queries(pts, 0.01, seed=12)[:300]
    rt = oracle.RefTree(pts, nrm, 12, seed=0)
    ex = rt.export()
    diag = synth.bbox_diag(pts)
    bb, BB = pts.min(0), pts.max(0)
    d = (BB - bb).astype(np.float32)
    radius = float(np.float32(np.sqrt(np.float32(np.float32(d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]))) / 2)
    out = {
        "pts": pts, "nrm": nrm, "q": q, "diag": np.float64(diag), "radius": np.float64(radius),
        "depth_ref": np.int32(rt.depth),
    }
    for k in ["depth", "parent", "first_child", "n_children", "next_brother", "leaf_off", "leaf_cnt", "perm"]:
        out["tree_" + k] = ex[k]
    out["tree_stats"] = ex["stats"]
    out["tree_area"] = ex["area"]
    ks = kernels(diag, radius)
    for name, k in ks.items():
        out[f"k_{name}_type"] = np.int32(k.type)
        out[f"k_{name}_sigma"] = np.float32(k.sigma)
        out[f"k_{name}_exponent"] = np.float32(k.exponent)
        out[f"k_{name}_shift"] = np.float32(k.constant_shift)
        out[f"k_{name}_sigmas"] = np.asarray(k.sigmas, np.float32)
        p, n, _ = rt.project(q, 10, k, cutoff=3.0, mode=0)
        out[f"mlod_{name}_p"], out[f"mlod_{name}_n"] = p, n
    kg = ks["gauss"]
    p, n, _ = rt.project(q[:100], 2, kg, mode=1)
    out["global_gauss_p"], out["global_gauss_n"] = p, n
    p, n, _ = rt.project(q, 3, kg, mode=2, k=32)
    out["knn32_gauss_p"], out["knn32_gauss_n"] = p, n
    p, n, _ = rt.project(q, 3, kg, mode=3, ball_r=0.05 * diag)
    out["ball_gauss_p"], out["ball_gauss_n"] = p, n
    out["ball_r"] = np.float32(0.05 * diag)
    idx, d2 = oracle.ref_kdtree_knn(pts, q, 32)
    out["kd_knn32_idx"], out["kd_knn32_d2"] = idx, d2
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes)")


if __name__ == "__main__":
    main()
