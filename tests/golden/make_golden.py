"""Generate the committed golden vectors under tests/golden/.

Runs in the build container, where the reference tree exists, by executing the
reference's own CPU code compiled from source into oracle/_ref/libtdp_ref.so
(see oracle/Makefile), next to the FP64 oracle (oracle/liboracle.so):

  tridist_golden.npz   triangle pairs (analytic known-answer cases + seeded
                       random families) with the reference's FP32 TriDist
                       (computing_cpu.cpp:403-439) and the oracle's FP64 distance
  meshdist_golden.npz  voxel pairs (seeded triangle clusters with Hausdorff
                       pairs) with the reference's MeshDist (computing_cpu.cpp:441-481)
                       and the oracle's FP64 restatement

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
OUT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "tests"))
from oracle_bind import oracle, reference  # noqa: E402


def kat_pairs():
    """Analytic triangle pairs with known distances (float32-exact coordinates)."""
    cases = []  # (S, T, exact distance)
    base = np.array([[0, 0, 0], [4, 0, 0], [0, 4, 0]], np.float64)
    # parallel offset: T above S's interior
    cases.append((base, base + [0.5, 0.5, 3.0], 3.0))
    # crossing (T pierces S)
    cases.append((base, np.array([[1, 1, -1], [1, 1, 1], [2, 1, 1]], np.float64), 0.0))
    # vertex-face: T's vertex hovers over S's interior at height 2
    cases.append((base, np.array([[1, 1, 2], [1, 1, 7], [3, 1, 7]], np.float64), 2.0))
    # edge-edge skew: S's edge on x axis, T's edge parallel to y at z=5 over x=2
    cases.append((base, np.array([[2, -3, 5], [2, -1, 5], [2, -2, 9]], np.float64),
                  float(np.sqrt(1 + 25))))
    # shared vertex
    cases.append((base, np.array([[0, 0, 0], [-3, 0, 1], [0, -3, 1]], np.float64), 0.0))
    # degenerate sliver (collinear T) above S's edge
    cases.append((base, np.array([[1, -2, 0], [2, -2, 0], [3, -2, 0]], np.float64), 2.0))
    # coplanar disjoint
    cases.append((base, base + [10, 0, 0], 6.0))
    # vertex-vertex
    cases.append((base, np.array([[-3, -4, 0], [-6, -4, 0], [-3, -8, 0]], np.float64), 5.0))
    S = np.stack([c[0].reshape(9) for c in cases]).astype(np.float32)
    T = np.stack([c[1].reshape(9) for c in cases]).astype(np.float32)
    d = np.array([c[2] for c in cases], np.float64)
    return S, T, d


def random_pairs(rng, n, scale, offset):
    S = (rng.normal(size=(n, 9)) * scale).astype(np.float32)
    T = (rng.normal(size=(n, 9)) * scale + offset).astype(np.float32)
    return S, T


def voxel_cluster(rng, n, center, spread, size):
    c = center + rng.normal(size=(n, 3)) * spread
    tri = (c[:, None, :] + rng.normal(size=(n, 3, 3)) * size).reshape(n, 9).astype(np.float32)
    hd = np.abs(rng.normal(size=(n, 2)) * 0.2).astype(np.float32)
    return tri, hd


def main():
    O, R = oracle(), reference()
    if R is None:
        raise SystemExit("oracle/_ref/libtdp_ref.so is missing: run `make -C oracle ref` in the build container")
    rng = np.random.default_rng(20260001)
    fam = {}
    S, T, d = kat_pairs()
    fam["kat"] = (S, T)
    fam["near"] = random_pairs(rng, 1500, 1.0, 0.5)
    fam["far"] = random_pairs(rng, 1500, 1.0, 5.0)
    fam["overlap"] = random_pairs(rng, 1500, 1.0, 0.0)
    fam["wide"] = random_pairs(rng, 1500, 30.0, 100.0)
    out = {"kat_exact": d}
    for k, (S, T) in fam.items():
        out[f"{k}_S"] = S
        out[f"{k}_T"] = T
        out[f"{k}_ref32"] = R.tri_dist_batch(S, T)
        out[f"{k}_oracle64"] = O.tri_dist_batch(S.astype(np.float64), T.astype(np.float64))[0]
    np.savez_compressed(OUT / "tridist_golden.npz", **out)

    rows = []
    tris, hds = [], []
    off = 0
    vp = []
    for k in range(24):
        n1, n2 = int(rng.integers(1, 40)), int(rng.integers(1, 40))
        gap = float(rng.uniform(0.0, 20.0))
        t1, h1 = voxel_cluster(rng, n1, np.zeros(3), 2.0, 1.0)
        t2, h2 = voxel_cluster(rng, n2, np.array([gap, 0.3, -0.2]), 2.0, 1.0)
        tris += [t1, t2]
        hds += [h1, h2]
        vp.append((off, n1, off + n1, n2))
        off += n1 + n2
    tri = np.concatenate(tris)
    hd = np.concatenate(hds)
    osz = np.array(vp, np.uint64)
    ref = np.stack([R.mesh_dist(tri[o1:o1 + n1], tri[o2:o2 + n2], hd[o1:o1 + n1], hd[o2:o2 + n2])
                    for o1, n1, o2, n2 in vp])
    ora = np.stack([O.voxel_pair(tri[o1:o1 + n1], hd[o1:o1 + n1], tri[o2:o2 + n2], hd[o2:o2 + n2])
                    for o1, n1, o2, n2 in vp])
    np.savez_compressed(OUT / "meshdist_golden.npz", tri=tri, hd=hd, offset_size=osz, ref32=ref, oracle64=ora)
    print("wrote", OUT / "tridist_golden.npz", OUT / "meshdist_golden.npz")


if __name__ == "__main__":
    main()
