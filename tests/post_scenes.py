"""Quad meshes for the mesh post-pass tests (postprocess_mesh, src/cpp/dc_backend.cpp:127-558).

Dual-contouring meshes of small analytic grids (the CPU oracle extracts them, so no GPU is
needed) and hand-built meshes for the cases the reference's code branches on: welded
duplicates, degenerate faces, non-manifold edges, boundary vertices on two loops, loops longer
than 4096 vertices, ties between components. Every scene is a function of its name only.
"""
import numpy as np

FLAGS = ((1, 1), (1, 0), (0, 1), (0, 0))


def _grid(res, fn, lo=-0.5, hi=0.5):
    ax = np.linspace(lo, hi, res, dtype=np.float64)
    z, y, x = np.meshgrid(ax, ax, ax, indexing="ij")
    sp = (hi - lo) / (res - 1)
    return fn(x, y, z).astype(np.float32).ravel(), (res, res, res), (sp, sp, sp), (lo, lo, lo)


def _dc(vals, dims, sp, org):
    import oracle as O
    r = O.dc_extract(vals, dims, sp, org)
    return r["V"].astype(np.float32), r["F"].astype(np.int32)


def cut_sphere(res=40):
    """A sphere larger than the grid: six open caps' holes."""
    return _dc(*_grid(res, lambda x, y, z: np.sqrt(x * x + y * y + z * z) - 0.6))


def floaters(res=48):
    """A sphere and two small ones apart from it."""
    def f(x, y, z):
        a = np.sqrt(x * x + y * y + z * z) - 0.25
        b = np.sqrt((x - 0.38) ** 2 + (y - 0.38) ** 2 + (z - 0.38) ** 2) - 0.06
        c = np.sqrt((x + 0.4) ** 2 + (y - 0.4) ** 2 + z * z) - 0.05
        return np.minimum(np.minimum(a, b), c)
    return _dc(*_grid(res, f))


def wavy_plane(res=32):
    """An open sheet across the grid: one boundary loop around it."""
    return _dc(*_grid(res, lambda x, y, z: z - 0.1 + 0.05 * np.sin(7 * x)))


def noise(res=20, seed=0):
    """White noise: many components, non-manifold edges, loops of every length."""
    vals = np.random.default_rng(seed).standard_normal(res ** 3).astype(np.float32)
    return _dc(vals, (res, res, res), (0.05,) * 3, (0.0,) * 3)


def open_box_and_cut_spheres(res=56):
    """Several shapes cut by the grid's faces and each other."""
    def f(x, y, z):
        a = np.sqrt((x - 0.3) ** 2 + y * y + z * z) - 0.35
        b = np.maximum(np.abs(x + 0.25), np.maximum(np.abs(y), np.abs(z - 0.3))) - 0.3
        c = np.sqrt(x * x + (y + 0.45) ** 2 + (z + 0.45) ** 2) - 0.2
        return np.minimum(np.minimum(a, b), c)
    return _dc(*_grid(res, f))


def split_quads(seed=1):
    """Every face with its own four vertex copies (some moved by less than the weld step):
    the weld must put the mesh back together."""
    V, F = cut_sphere(24)
    rng = np.random.default_rng(seed)
    V2 = V[F.reshape(-1)].copy()
    diag = float(np.linalg.norm(V.max(0) - V.min(0)))
    jitter = rng.uniform(-0.2, 0.2, V2.shape).astype(np.float32) * np.float32(diag * 1e-5)
    pick = rng.random(V2.shape[0]) < 0.3
    V2[pick] += jitter[pick]
    F2 = np.arange(V2.shape[0], dtype=np.int32).reshape(-1, 4)
    return V2, F2


def degenerate_faces():
    """A 6x6 sheet of quads with repeated indices: (a,a,b,c) stays, (a,a,b,b) goes, and
    coincident vertices that the weld merges turn faces degenerate."""
    n = 7
    g = np.stack(np.meshgrid(np.arange(n), np.arange(n), indexing="ij"), -1).reshape(-1, 2).astype(np.float32)
    V = np.concatenate([g, np.zeros((g.shape[0], 1), np.float32)], 1) * np.float32(0.1)
    F = []
    for i in range(n - 1):
        for j in range(n - 1):
            a, b, c, d = i * n + j, (i + 1) * n + j, (i + 1) * n + j + 1, i * n + j + 1
            F.append((a, b, c, d))
    F = np.array(F, np.int32)
    extra = np.array([(0, 0, 1, 8), (2, 2, 3, 3), (10, 11, 11, 10), (20, 21, 22, 20)], np.int32)
    dup = V[[5, 6]]                     # coincident copies of vertices 5 and 6
    V = np.concatenate([V, dup])
    m = V.shape[0]
    extra2 = np.array([(5, m - 2, 6, m - 1), (5, 12, m - 2, 13)], np.int32)
    return V, np.concatenate([F, extra, extra2])


def nonmanifold_fan():
    """A closed cube plus three flaps on one of its edges (an edge with five uses)."""
    c = np.array([[x, y, z] for z in (0, 1) for y in (0, 1) for x in (0, 1)], np.float32)
    F = np.array([(0, 2, 3, 1), (4, 5, 7, 6), (0, 1, 5, 4), (2, 6, 7, 3), (0, 4, 6, 2), (1, 3, 7, 5)], np.int32)
    flaps = np.array([[0.5, -1, 0], [0.5, -1, 1], [-1, 0.5, 0], [-1, 0.5, 1], [1.5, -0.5, 0], [1.5, -0.5, 1]], np.float32)
    V = np.concatenate([c, flaps])
    F2 = np.array([(0, 4, 9, 8), (4, 0, 10, 11), (0, 4, 13, 12)], np.int32)
    return V, np.concatenate([F, F2])


def figure_eight():
    """A 9x5 sheet with two 1-cell holes whose corners touch: a boundary vertex with two
    outgoing edges (the walks split off a sub-loop)."""
    nx, ny = 9, 5
    V = np.array([[i * 0.1, j * 0.1, 0.0] for j in range(ny) for i in range(nx)], np.float32)
    holes = {(3, 1), (4, 2)}
    F = [(j * nx + i, j * nx + i + 1, (j + 1) * nx + i + 1, (j + 1) * nx + i)
         for j in range(ny - 1) for i in range(nx - 1) if (i, j) not in holes]
    return V, np.array(F, np.int32)


def tube(segments, rings=3, radius=1.0):
    """An open tube: two boundary loops of `segments` vertices (filled only up to 4096)."""
    t = np.arange(segments) * (2 * np.pi / segments)
    V = np.concatenate([np.stack([radius * np.cos(t), radius * np.sin(t), np.full(segments, 0.01 * r)], 1)
                        for r in range(rings)]).astype(np.float32)
    F = [(r * segments + k, r * segments + (k + 1) % segments, (r + 1) * segments + (k + 1) % segments,
          (r + 1) * segments + k) for r in range(rings - 1) for k in range(segments)]
    return V, np.array(F, np.int32)


def tied_components():
    """Two disjoint open sheets with the same number of faces: the first one is kept."""
    V1, F1 = figure_eight()
    V2 = V1 + np.float32([0, 0, 1])
    return np.concatenate([V1, V2]), np.concatenate([F1, F1 + V1.shape[0]])


def single_triangle():
    return np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32), np.array([(0, 1, 2, 2)], np.int32)


SMALL = {
    "cut_sphere": lambda: cut_sphere(24),
    "floaters": lambda: floaters(32),
    "wavy_plane": lambda: wavy_plane(20),
    "noise": lambda: noise(12),
    "split_quads": split_quads,
    "degenerate_faces": degenerate_faces,
    "nonmanifold_fan": nonmanifold_fan,
    "figure_eight": figure_eight,
    "tube_64": lambda: tube(64),
    "tied_components": tied_components,
    "single_triangle": single_triangle,
}

LARGE = {
    "cut_sphere_40": lambda: cut_sphere(40),
    "floaters_48": lambda: floaters(48),
    "noise_20": lambda: noise(20),
    "shapes_56": open_box_and_cut_spheres,
    "tube_4096": lambda: tube(4096),
    "tube_4097": lambda: tube(4097),
}
