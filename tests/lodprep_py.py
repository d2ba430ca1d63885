"""Pure-Python restatement of the LOD preparation rule (test infrastructure,
small meshes only), written the way the GPU kernels run it rather than the way
the C++ oracle does: the decimation keeps a refused-edge flag per facet slot
and takes the smallest key over all candidate slots each round (no priority
queue, no versions).  Agreeing with the oracle's priority-queue decimation on
the same meshes pins that the two formulations are the same rule.

The rule itself is stated in oracle/lodprep_oracle.cpp and
3dpipe_b200/csrc/prep_kernels.cu.  Arithmetic follows the same expression
order: Python floats are IEEE doubles, float32 steps use numpy float32 scalars.
"""
from __future__ import annotations

import math
import struct

import numpy as np

PCT = (20, 40, 60, 80)


def _d2(P, a, b):
    dx, dy, dz = P[a][0] - P[b][0], P[a][1] - P[b][1], P[a][2] - P[b][2]
    return dx * dx + dy * dy + dz * dz


def _turns(P, f, u, v):
    def normal(t):
        p0, p1, p2 = P[t[0]], P[t[1]], P[t[2]]
        a = (p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2])
        b = (p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2])
        return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])

    def dot(a, b):
        return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]

    n0 = normal(f)
    n1 = normal([v if x == u else x for x in f])
    a0, a1 = math.sqrt(dot(n0, n0)), math.sqrt(dot(n1, n1))
    return a1 < 1e-12 * (a0 + 1e-300) or dot(n0, n1) < 0.3 * a0 * a1


def decimate(P, F):
    """{20: faces, 40: ..., 60: ..., 80: ...} (lists of vertex triples, index order)"""
    m = len(F)
    F = [list(f) for f in F]
    live = [True] * m
    refused = [[False] * 3 for _ in range(m)]
    alive = m
    out = {}
    li = 3
    while li >= 0:
        target = m * PCT[li] // 100
        best = None
        if alive > target:
            for f in range(m):
                if not live[f]:
                    continue
                for j in range(3):
                    if refused[f][j]:
                        continue
                    x, y = F[f][j], F[f][(j + 1) % 3]
                    a, b = min(x, y), max(x, y)
                    key = (_d2(P, a, b), a, b)
                    if best is None or key < best:
                        best = key
        if alive <= target or best is None:
            out[PCT[li]] = [tuple(F[f]) for f in range(m) if live[f]]
            li -= 1
            continue
        _, u, v = best
        faces_u = [f for f in range(m) if live[f] and u in F[f]]
        faces_v = [f for f in range(m) if live[f] and v in F[f]]
        both = [f for f in faces_u if v in F[f]]
        third = [next(x for x in F[f] if x != u and x != v) for f in both]

        def nbrs(w):
            return {x for f in range(m) if live[f] and w in F[f] for x in F[f] if x != w}

        link = (len(third) == 2 and third[0] != third[1] and len(nbrs(u) & nbrs(v)) == 2
                and len(nbrs(third[0])) > 3 and len(nbrs(third[1])) > 3)
        mode = None
        if link and not any(_turns(P, F[f], u, v) for f in faces_u if v not in F[f]):
            mode = (u, v)
        elif link and not any(_turns(P, F[f], v, u) for f in faces_v if u not in F[f]):
            mode = (v, u)
        if mode is None:
            for f in both:
                for j in range(3):
                    if {F[f][j], F[f][(j + 1) % 3]} == {u, v}:
                        refused[f][j] = True
            continue
        r, k = mode
        for f in range(m):
            if not live[f] or (r not in F[f] and k not in F[f]):
                continue
            if r in F[f] and k in F[f]:
                live[f] = False
                alive -= 1
                continue
            F[f] = [k if x == r else x for x in F[f]]
            for j in range(3):
                if k in (F[f][j], F[f][(j + 1) % 3]):
                    refused[f][j] = False
    return out


def _nearest(p, pts):
    g, best = 0, math.inf
    for s, c in enumerate(pts):
        d = _d2([p, c], 0, 1)
        if d < best:
            best, g = d, s
    return g, best


def prepare_object(Pf, F, voxel_size):
    """RAW bytes of one object (zero bounds) under the preparation rule"""
    Pf = np.asarray(Pf, np.float32)
    P = [tuple(float(x) for x in p) for p in Pf]
    F = [tuple(int(x) for x in f) for f in F]
    m, n = len(F), len(P)
    dec = decimate(P, F)
    lods = [dec[20], dec[40], dec[60], dec[80], F]
    nseed = m // voxel_size + 1
    seeds, dmin, cur = [], [math.inf] * n, 0
    for _ in range(nseed):
        seeds.append(P[cur])
        far = 0
        for i in range(n):
            dmin[i] = min(dmin[i], math.sqrt(_d2(P, i, cur)))
            if dmin[i] > dmin[far]:
                far = i
        cur = far
    for _ in range(2):
        acc = [[0.0, 0.0, 0.0] for _ in range(nseed)]
        cnt = [0] * nseed
        for i in range(n):
            g, _ = _nearest(P[i], seeds)
            acc[g] = [acc[g][0] + P[i][0], acc[g][1] + P[i][1], acc[g][2] + P[i][2]]
            cnt[g] += 1
        for s in range(nseed):
            if cnt[s]:
                r = 1.0 / cnt[s]
                seeds[s] = (acc[s][0] * r, acc[s][1] * r, acc[s][2] * r)
    best_d, best_f = [math.inf] * nseed, [-1] * nseed
    for f, t in enumerate(F):
        a, b, c = P[t[0]], P[t[1]], P[t[2]]
        q = tuple(((a[k] + b[k]) + c[k]) * (1.0 / 3.0) for k in range(3))
        g, d = _nearest(q, seeds)
        if d < best_d[g]:
            best_d[g], best_f[g] = d, f
    core0 = [F[best_f[s]][0] for s in range(nseed) if best_f[s] >= 0]
    got = [0] * len(core0)
    for t in F:
        got[_nearest(P[t[0]], [P[c] for c in core0])[0]] += 1
    core = [c for c, k in zip(core0, got) if k]
    cp = [P[c] for c in core]
    byvox = [[[t for t in lod if _nearest(P[t[0]], cp)[0] == v] for v in range(len(core))] for lod in lods]
    body, offs, box = bytearray(), [], []
    lo = [[math.inf] * 3 for _ in core]
    hi = [[-math.inf] * 3 for _ in core]
    for li in range(5):
        for v in range(len(core)):
            offs.append((li, v, len(body), len(byvox[li][v])))
            for t in byvox[li][v]:
                for x in t:
                    for k in range(3):
                        q = Pf[x][k]
                        body += struct.pack("<f", q)
                        lo[v][k] = q if q < lo[v][k] else lo[v][k]
                        hi[v][k] = q if hi[v][k] < q else hi[v][k]
            body += b"\0" * (8 * len(byvox[li][v]))
    rec = bytearray(struct.pack("<Q", len(body))) + body + struct.pack("<Q", len(core)) + b"\0" * 40
    table = {(li, v): (o, c) for li, v, o, c in offs}
    for v, c in enumerate(core):
        rec += struct.pack("<6f", *lo[v], *hi[v]) + struct.pack("<3f", *Pf[c])
        for li in range(5):
            rec += struct.pack("<QQ", *table[(li, v)])
    blo, bhi = Pf.min(axis=0), Pf.max(axis=0)
    cen = np.float32(0.5) * (blo + bhi)
    bi, bd = 0, np.float32(np.inf)
    for i in range(n):
        dx, dy, dz = Pf[i] - cen
        d = dx * dx + dy * dy + dz * dz
        if d < bd:
            bd, bi = d, i
    rec += struct.pack("<3f", *Pf[bi])
    return bytes(rec)


def prepare(meshes, voxel_size=100):
    """[(vertices, facets), ...] -> RAW tile bytes with zero bounds"""
    return b"\x01" + b"".join(prepare_object(v, f, voxel_size) for v, f in meshes)
