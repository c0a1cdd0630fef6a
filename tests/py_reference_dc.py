"""Second, independent restatement of the reference's CPU dual contouring, in plain Python
loops over the reference's own data structures (TEST INFRASTRUCTURE ONLY, small grids).

It exists to check the C oracle (``oracle/dc_oracle.cpp``), which is organised for speed
(owner-cell driven, OpenMP) and uses a cyclic-Jacobi eigen-solver. This file instead walks
the reference's steps one by one and uses LAPACK's SVD (numpy), so the two restatements
share no code and no solver:

* grid positions GV = float(o + float(i) * v)              src/cpp/dc_backend.cpp:58-68
* cells, strict-sign activity, corner order                 src/cpp/contouring.cpp:210-271,
                                                            src/cpp/Cell.cpp:57-77
* Hermite samples, t = fa / (fa - fb + 1e-16), trilinear
  gradient normals                                          src/cpp/Cell.cpp:80-212
* 4-cell normal averaging over grid edges                   src/cpp/hermite_update.cpp:34-91,
                                                            171-438
* QEF: pinv of A^T A (singular values > 0.01) about the
  centroid                                                  src/cpp/Cell.cpp:284-361, 586-600
* faces X, Y, Z edges, winding from central-difference
  gradients                                                 src/cpp/contouring.cpp:141-207,
                                                            486-741
"""
import math

import numpy as np

# Corner order and edge list of a cell (Cell.h:9-30): corner c -> (dx, dy, dz).
CORNERS = ((0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1))
EDGE_PAIRS = ((0, 1), (1, 2), (2, 3), (3, 0), (4, 5), (5, 6), (6, 7), (7, 4), (0, 4), (1, 5), (2, 6), (3, 7))
# The two cell faces beside each edge, as directions 0:+X 1:-X 2:+Y 3:-Y 4:+Z 5:-Z (Cell.cpp:26-45).
EDGE_FACES = ((3, 5), (0, 5), (2, 5), (1, 5), (3, 4), (0, 4), (2, 4), (1, 4), (1, 3), (0, 3), (0, 2), (1, 2))
DIRS = ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1))


def _normalized(v):
    n = math.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])
    return [v[0] / n, v[1] / n, v[2] / n] if n > 0.0 else list(v)


class _Cell:
    __slots__ = ("ix", "iy", "iz", "pos", "sdf", "has_vertex", "hp", "hn", "vertex")


def _trilinear_gradient(sdf, pos, p):
    x0, x1 = pos[0][0], pos[1][0]
    y0, y1 = pos[0][1], pos[3][1]
    z0, z1 = pos[0][2], pos[4][2]
    dx, dy, dz = x1 - x0, y1 - y0, z1 - z0
    u = v = w = 0.5
    if abs(dx) > 1e-12:
        u = (p[0] - x0) / dx
    if abs(dy) > 1e-12:
        v = (p[1] - y0) / dy
    if abs(dz) > 1e-12:
        w = (p[2] - z0) / dz
    u, v, w = (min(1.0, max(0.0, q)) for q in (u, v, w))
    s000, s100, s110, s010, s001, s101, s111, s011 = sdf
    du = ((s100 - s000) * (1 - v) * (1 - w) + (s110 - s010) * v * (1 - w) +
          (s101 - s001) * (1 - v) * w + (s111 - s011) * v * w)
    dv = ((s010 - s000) * (1 - u) * (1 - w) + (s110 - s100) * u * (1 - w) +
          (s011 - s001) * (1 - u) * w + (s111 - s101) * u * w)
    dw = ((s001 - s000) * (1 - u) * (1 - v) + (s101 - s100) * u * (1 - v) +
          (s011 - s010) * (1 - u) * v + (s111 - s110) * u * v)
    return [du / dx if abs(dx) > 1e-12 else 0.0, dv / dy if abs(dy) > 1e-12 else 0.0,
            dw / dz if abs(dz) > 1e-12 else 0.0]


def extract(values, dims, spacing, origin, svd_threshold=0.01):
    """Returns (V float64 (nv,3), F int32 (nf,4), cells int64 (nv,)) like the oracle."""
    nx, ny, nz = dims
    S = np.asarray(values, np.float32).reshape(-1).astype(np.float64)
    axes = [(np.float32(origin[a]) + np.arange(d, dtype=np.float32) * np.float32(spacing[a])).astype(np.float64)
            for a, d in enumerate(dims)]
    cx, cy, cz = nx - 1, ny - 1, nz - 1

    def sval(i, j, k):
        return S[i + nx * (j + ny * k)]

    def gpos(i, j, k):
        return (axes[0][i], axes[1][j], axes[2][k])

    def cidx(i, j, k):
        return i + cx * (j + cy * k)

    # cells in k, j, i order with Hermite data (contouring.cpp:210-271)
    cells = []
    for k in range(cz):
        for j in range(cy):
            for i in range(cx):
                c = _Cell()
                c.ix, c.iy, c.iz = i, j, k
                c.pos = [gpos(i + d[0], j + d[1], k + d[2]) for d in CORNERS]
                c.sdf = [sval(i + d[0], j + d[1], k + d[2]) for d in CORNERS]
                c.has_vertex = any(s < 0 for s in c.sdf) and any(s > 0 for s in c.sdf)
                c.hp, c.hn = {}, {}
                if c.has_vertex:
                    for e, (a, b) in enumerate(EDGE_PAIRS):
                        fa, fb = c.sdf[a], c.sdf[b]
                        if fa * fb > 0.0:
                            continue
                        t = fa / (fa - fb + 1e-16)
                        p = [(1.0 - t) * c.pos[a][q] + t * c.pos[b][q] for q in range(3)]
                        c.hp[e] = p
                        c.hn[e] = _normalized(_trilinear_gradient(c.sdf, c.pos, p))
                cells.append(c)

    def local_edge(c, p0, p1):
        d0 = (p0[0] - c.ix, p0[1] - c.iy, p0[2] - c.iz)
        d1 = (p1[0] - c.ix, p1[1] - c.iy, p1[2] - c.iz)
        for e, (a, b) in enumerate(EDGE_PAIRS):
            if (CORNERS[a] == d0 and CORNERS[b] == d1) or (CORNERS[b] == d0 and CORNERS[a] == d1):
                return e
        return -1

    def inside(i, j, k):
        return 0 < i < nx - 1 and 0 < j < ny - 1 and 0 < k < nz - 1

    # 4-cell normal averaging (hermite_update.cpp:171-438)
    groups = []
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                for d, ok in (((1, 0, 0), i < nx - 1), ((0, 1, 0), j < ny - 1), ((0, 0, 1), k < nz - 1)):
                    if not ok:
                        continue
                    p0, p1 = (i, j, k), (i + d[0], j + d[1], k + d[2])
                    if not inside(*p0) and not inside(*p1):
                        continue
                    owner = cells[cidx(i, j, k)]
                    e = local_edge(owner, p0, p1)
                    if e < 0 or e not in owner.hp:
                        continue
                    f1, f2 = EDGE_FACES[e]
                    n1 = (i + DIRS[f1][0], j + DIRS[f1][1], k + DIRS[f1][2])
                    n2 = (i + DIRS[f2][0], j + DIRS[f2][1], k + DIRS[f2][2])
                    n3 = (n1[0] + DIRS[f2][0], n1[1] + DIRS[f2][1], n1[2] + DIRS[f2][2])
                    four = [owner, cells[cidx(*n1)], cells[cidx(*n2)], cells[cidx(*n3)]]
                    if not all(c.has_vertex for c in four):
                        continue
                    groups.append([(c, local_edge(c, p0, p1)) for c in four])
    for g in groups:
        acc = [0.0, 0.0, 0.0]
        for c, e in g:
            n = c.hn[e]
            if math.sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]) > 0:
                acc = [acc[q] + n[q] for q in range(3)]
        acc = _normalized(acc)
        for c, e in g:
            c.hn[e] = list(acc)

    # QEF per active cell (Cell.cpp:284-361)
    for c in cells:
        if not c.has_vertex:
            continue
        keys = sorted(c.hp)
        A = np.array([_normalized(c.hn[e]) for e in keys], np.float64)
        P = np.array([c.hp[e] for e in keys], np.float64)
        b = (A * P).sum(1)
        ata = A.T @ A
        atb = A.T @ b
        U, sv, Vt = np.linalg.svd(ata)
        sinv = np.where(sv > svd_threshold, 1.0 / np.where(sv > svd_threshold, sv, 1.0), 0.0)
        pinv = Vt.T @ np.diag(sinv) @ U.T
        centroid = P.sum(0) / len(keys)
        c.vertex = centroid + pinv @ (atb - ata @ centroid)

    # vertices in linear cell order, then faces (contouring.cpp:486-741)
    vidx = {}
    V, cell_ids = [], []
    for ci, c in enumerate(cells):
        if c.has_vertex:
            vidx[ci] = len(V)
            V.append(c.vertex)
            cell_ids.append(ci)

    def grad_at(i, j, k):
        im, ip = max(i - 1, 0), min(i + 1, nx - 1)
        jm, jp = max(j - 1, 0), min(j + 1, ny - 1)
        km, kp = max(k - 1, 0), min(k + 1, nz - 1)
        g = [0.0, 0.0, 0.0]
        dx = axes[0][ip] - axes[0][im]
        dy = axes[1][jp] - axes[1][jm]
        dz = axes[2][kp] - axes[2][km]
        if abs(dx) > 1e-12:
            g[0] = (sval(ip, j, k) - sval(im, j, k)) / dx
        if abs(dy) > 1e-12:
            g[1] = (sval(i, jp, k) - sval(i, jm, k)) / dy
        if abs(dz) > 1e-12:
            g[2] = (sval(i, j, kp) - sval(i, j, km)) / dz
        return _normalized(g)

    def vert(i, j, k):
        if 0 <= i < cx and 0 <= j < cy and 0 <= k < cz:
            return vidx.get(cidx(i, j, k), -1)
        return -1

    F = []

    def emit(p0, p1, quad):
        if not sval(*p0) * sval(*p1) < 0.0:
            return
        q = [vert(*c) for c in quad]
        if min(q) < 0:
            return
        g0, g1 = grad_at(*p0), grad_at(*p1)
        gn = np.array(g0) + np.array(g1)
        pa, pb, pc, pd = (V[x] for x in q)
        qn = np.cross(pb - pa, pd - pa)
        if qn @ qn < 1e-24:
            qn = np.cross(pc - pa, pd - pa)
        if gn @ gn > 0 and qn @ qn > 0 and qn @ gn < 0.0:
            q[1], q[3] = q[3], q[1]
        F.append(q)

    for i in range(cx):
        for j in range(1, cy):
            for k in range(1, cz):
                emit((i, j, k), (i + 1, j, k), ((i, j - 1, k - 1), (i, j, k - 1), (i, j, k), (i, j - 1, k)))
    for i in range(1, cx):
        for j in range(cy):
            for k in range(1, cz):
                emit((i, j, k), (i, j + 1, k), ((i - 1, j, k - 1), (i, j, k - 1), (i, j, k), (i - 1, j, k)))
    for i in range(1, cx):
        for j in range(1, cy):
            for k in range(cz):
                emit((i, j, k), (i, j, k + 1), ((i - 1, j - 1, k), (i, j - 1, k), (i, j, k), (i - 1, j, k)))
    return (np.array(V, np.float64).reshape(-1, 3), np.array(F, np.int32).reshape(-1, 4),
            np.array(cell_ids, np.int64))
