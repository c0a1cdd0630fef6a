"""Seeded synthetic SDF grids for the benchmark workloads and the tests.

Every generator returns a :class:`contouring_b200.grid.DenseSdfGrid`-compatible tuple
``(values, dims, spacing, origin)`` where ``values`` is a float32 tensor of ``nx*ny*nz``
entries laid out x-fastest (``i + nx*(j + ny*k)``), the layout of the reference's
``DenseSdfGrid::values`` (include/dc_backend.h:13-21).

Grid point positions are computed in float32 as ``origin + float(i) * spacing``, the
way the reference's CPU backend builds its position matrix (src/cpp/dc_backend.cpp:63-65);
analytic distances are evaluated in float64 from those positions and rounded to float32.
Large grids are produced slab by slab on whatever device is passed in.
"""
import math

import numpy as np
import torch


def _axis(n, lo, step, device):
    o = torch.tensor(lo, dtype=torch.float32)
    v = torch.tensor(step, dtype=torch.float32)
    return (o + torch.arange(n, dtype=torch.float32) * v).to(device)


def _grid_params(res, lo, hi):
    step = float(np.float32((hi - lo) / (res - 1)))
    return (res, res, res), (step, step, step), (float(np.float32(lo)),) * 3


def _eval_slabs(dims, spacing, origin, fn, device, slab_points=1 << 26, planes=None):
    """Evaluate fn (FP64 points -> FP64 values) at the grid points, slab by slab, cast to
    float32. ``planes`` = (k0, k1) limits the evaluation to z planes k0..k1-1 (the same
    values as the full grid has there)."""
    nx, ny, nz = dims
    xs = _axis(nx, origin[0], spacing[0], device).double()
    ys = _axis(ny, origin[1], spacing[1], device).double()
    zs = _axis(nz, origin[2], spacing[2], device).double()
    if planes is not None:
        zs = zs[planes[0]:planes[1]]
        nz = zs.numel()
    out = torch.empty(nx * ny * nz, dtype=torch.float32, device=device)
    per = max(1, slab_points // (nx * ny))
    for k0 in range(0, nz, per):
        k1 = min(nz, k0 + per)
        Z, Y, X = torch.meshgrid(zs[k0:k1], ys, xs, indexing="ij")
        p = torch.stack([X, Y, Z], dim=-1)
        out[k0 * nx * ny:k1 * nx * ny] = fn(p).reshape(-1).to(torch.float32)
    return out


def sphere(res=128, radius=0.35, lo=-0.5, hi=0.5, device="cpu"):
    """Sphere of ``radius`` at the origin sampled at the corners of a res^3 grid on [lo,hi]^3."""
    dims, spacing, origin = _grid_params(res, lo, hi)
    vals = _eval_slabs(dims, spacing, origin, lambda p: p.norm(dim=-1) - radius, device)
    return vals, dims, spacing, origin


def _rand_rotation(rng):
    q = rng.normal(size=4)
    q = q / np.linalg.norm(q)
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


def csg_scene(seed=0, n_boxes=16, n_cyl=8, n_holes=4):
    """Primitive list of the sharp-feature CSG scene: a union of rotated boxes and capped
    cylinders minus spheres, every parameter drawn from one seeded generator."""
    rng = np.random.default_rng(seed)
    prims = []
    for _ in range(n_boxes):
        prims.append(("box", rng.uniform(-0.3, 0.3, 3), _rand_rotation(rng), rng.uniform(0.05, 0.2, 3)))
    for _ in range(n_cyl):
        c = rng.uniform(-0.3, 0.3, 3)
        R = _rand_rotation(rng)
        r = rng.uniform(0.03, 0.1)
        h = rng.uniform(0.1, 0.4)
        prims.append(("cyl", c, R, np.array([r, 0.5 * h])))
    holes = [(rng.uniform(-0.3, 0.3, 3), rng.uniform(0.05, 0.15)) for _ in range(n_holes)]
    return prims, holes


def _csg_fn(prims, holes, device):
    def fn(p):
        d = None
        for kind, c, R, par in prims:
            ct = torch.tensor(c, dtype=torch.float64, device=device)
            Rt = torch.tensor(R, dtype=torch.float64, device=device)
            q = (p - ct) @ Rt  # world -> local: R^T (p - c), row-vector form
            if kind == "box":
                h = torch.tensor(par, dtype=torch.float64, device=device)
                a = q.abs() - h
                outside = a.clamp(min=0).norm(dim=-1)
                inside = a.max(dim=-1).values.clamp(max=0)
                di = outside + inside
            else:
                r, hh = float(par[0]), float(par[1])
                dx = torch.sqrt(q[..., 0] ** 2 + q[..., 2] ** 2) - r
                dy = q[..., 1].abs() - hh
                di = torch.minimum(torch.maximum(dx, dy), torch.zeros_like(dx)) + torch.sqrt(
                    dx.clamp(min=0) ** 2 + dy.clamp(min=0) ** 2)
            d = di if d is None else torch.minimum(d, di)
        for c, r in holes:
            ct = torch.tensor(c, dtype=torch.float64, device=device)
            ds = (p - ct).norm(dim=-1) - r
            d = torch.maximum(d, -ds)
        return d
    return fn


def csg(res=1024, seed=0, lo=-0.5, hi=0.5, device="cpu", planes=None):
    """Sharp-feature CSG: 16 boxes (half-extents U(0.05,0.2)) and 8 capped cylinders
    (radius U(0.03,0.1), height U(0.1,0.4)) under random rotations with centres
    U(-0.3,0.3)^3, minus 4 spheres of radius U(0.05,0.15); exact CSG min/max distances.
    ``planes`` = (k0, k1) returns only z planes k0..k1-1 of the res^3 grid; dims then
    report those planes while spacing and origin stay the full grid's."""
    dims, spacing, origin = _grid_params(res, lo, hi)
    prims, holes = csg_scene(seed)
    vals = _eval_slabs(dims, spacing, origin, _csg_fn(prims, holes, device), device,
                       slab_points=1 << 24, planes=planes)
    if planes is not None:
        dims = (dims[0], dims[1], vals.numel() // (dims[0] * dims[1]))
    return vals, dims, spacing, origin


# ---- the reference's own generators (dc_cli.cpp:49-118, dc_tests.cpp:14-215), in float32 ----

def csg_batch(n=256, seed=0, resolutions=(32, 48, 64, 96, 128, 192), lo=-0.5, hi=0.5, device="cpu"):
    """n seeded CSG shapes at uneven resolutions: shape s draws its resolution uniformly from
    ``resolutions`` and a random mix of 1-16 boxes, 0-8 capped cylinders and 0-4 subtracted
    spheres with the distributions of ``csg``. Returns [(values, dims, spacing, origin)]."""
    rng = np.random.default_rng(seed)
    out = []
    for s in range(n):
        res = int(rng.choice(resolutions))
        nb, nc, nh = int(rng.integers(1, 17)), int(rng.integers(0, 9)), int(rng.integers(0, 5))
        prims, holes = csg_scene(int(rng.integers(0, 2 ** 31)), nb, nc, nh)
        dims, spacing, origin = _grid_params(res, lo, hi)
        vals = _eval_slabs(dims, spacing, origin, _csg_fn(prims, holes, device), device, slab_points=1 << 24)
        out.append((vals, dims, spacing, origin))
    return out


def _cli_axes(res):
    v = np.float32(2.0) / np.float32(res - 1)
    o = np.float32(-1.0)
    ax = (o + np.arange(res, dtype=np.float32) * v).astype(np.float32)
    return ax, (float(v),) * 3, (float(o),) * 3


def cli_sphere(res, radius=0.5):
    """``generate_sphere`` (dc_cli.cpp:49-71): float sqrt(x^2+y^2+z^2) - r on [-1,1]^3."""
    ax, sp, org = _cli_axes(res)
    Z, Y, X = np.meshgrid(ax, ax, ax, indexing="ij")
    d = np.sqrt((X * X + Y * Y) + Z * Z).astype(np.float32) - np.float32(radius)
    return torch.from_numpy(d.reshape(-1).astype(np.float32)), (res,) * 3, sp, org


def cli_box(res, half=0.5):
    """``generate_box`` (dc_cli.cpp:73-97): max(|x|-h, |y|-h, |z|-h) in float."""
    ax, sp, org = _cli_axes(res)
    Z, Y, X = np.meshgrid(ax, ax, ax, indexing="ij")
    h = np.float32(half)
    d = np.maximum(np.abs(X) - h, np.maximum(np.abs(Y) - h, np.abs(Z) - h))
    return torch.from_numpy(d.reshape(-1).astype(np.float32)), (res,) * 3, sp, org


def cli_plane(res):
    """``generate_plane`` (dc_cli.cpp:99-118): value = z."""
    ax, sp, org = _cli_axes(res)
    Z, Y, X = np.meshgrid(ax, ax, ax, indexing="ij")
    return torch.from_numpy(Z.reshape(-1).astype(np.float32).copy()), (res,) * 3, sp, org


def thin_gap(res=32):
    """Two spheres of radius 0.25 at x=+-0.2 (dc_tests.cpp:131-169), float arithmetic."""
    ax, sp, org = _cli_axes(res)
    Z, Y, X = np.meshgrid(ax, ax, ax, indexing="ij")
    a, b, r = np.float32(0.2), np.float32(0.25), np.float32(0.25)
    d1 = np.sqrt(((X - a) * (X - a) + Y * Y) + Z * Z).astype(np.float32) - r
    d2 = np.sqrt(((X + a) * (X + a) + Y * Y) + Z * Z).astype(np.float32) - b
    return torch.from_numpy(np.minimum(d1, d2).reshape(-1).astype(np.float32)), (res,) * 3, sp, org


def thin_shell(res=48, radius=0.3, half_width=0.3, seed=0):
    """A spherical shell thinner than a cell, |r - radius| - half_width * h (h the spacing,
    half_width < 0.5): where the shell falls between two grid points both are positive, small
    and have opposed gradients — the sparse backends' thin edges, and cells whose samples
    split into two vertices. A seeded shift of the centre (within a cell) varies the cut."""
    lo, hi = -0.5, 0.5
    dims, sp, org = _grid_params(res, lo, hi)
    c = np.random.default_rng(seed).uniform(-0.5, 0.5, 3) * sp[0]
    ax = _axis(res, lo, sp[0], "cpu").numpy().astype(np.float64)
    Z, Y, X = np.meshgrid(ax, ax, ax, indexing="ij")
    r = np.sqrt((X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2)
    v = np.abs(r - radius) - half_width * sp[0]
    return torch.from_numpy(v.reshape(-1).astype(np.float32)), dims, sp, org


def constant(res, value):
    """Constant grid (dc_tests.cpp:171-215 use +1 and -1 on 16^3)."""
    _, sp, org = _cli_axes(res)
    return torch.full((res ** 3,), float(value), dtype=torch.float32), (res,) * 3, sp, org


def noise(dims, seed=0, scale=1.0, zero_frac=0.0):
    """Uniform random values in [-scale, scale]; optionally a fraction of exact zeros
    (zeros count as crossings for Hermite data but not for activity or faces)."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = dims
    v = rng.uniform(-scale, scale, nx * ny * nz).astype(np.float32)
    if zero_frac > 0:
        v[rng.random(v.size) < zero_frac] = 0.0
    return torch.from_numpy(v), tuple(dims), (0.1, 0.1, 0.1), (-1.0, -1.0, -1.0)


def rbf_sphere(res=128, radius=0.3, n_rbf=64, seed=0, lo=-0.5, hi=0.5, device="cpu"):
    """Sphere of radius 0.3 perturbed by a sum of Gaussian RBFs a*exp(-|x-c|^2/w^2),
    a ~ U(-0.03,0.03), w ~ U(0.03,0.08), seeded centres in U(-0.4,0.4)^3."""
    rng = np.random.default_rng(seed)
    cs = rng.uniform(-0.4, 0.4, (n_rbf, 3))
    amp = rng.uniform(-0.03, 0.03, n_rbf)
    wid = rng.uniform(0.03, 0.08, n_rbf)
    dims, spacing, origin = _grid_params(res, lo, hi)

    def fn(p):
        d = p.norm(dim=-1) - radius
        for c, a, w in zip(cs, amp, wid):
            ct = torch.tensor(c, dtype=torch.float64, device=p.device)
            d = d + a * torch.exp(-((p - ct) ** 2).sum(-1) / (w * w))
        return d
    vals = _eval_slabs(dims, spacing, origin, fn, device)
    return vals, dims, spacing, origin


def rbf_sphere_points(n=50000, radius=0.3, n_rbf=64, seed=1):
    """n points on a second perturbed sphere: directions uniform on the sphere, radius
    0.3 + sum_q a_q exp(-|0.3 u - c_q|^2 / w_q^2) with the RBF parameters of
    ``rbf_sphere(seed=seed)``. float64 (n, 3)."""
    rng = np.random.default_rng(seed)
    cs = rng.uniform(-0.4, 0.4, (n_rbf, 3))
    amp = rng.uniform(-0.03, 0.03, n_rbf)
    wid = rng.uniform(0.03, 0.08, n_rbf)
    u = np.random.default_rng(seed + 1000).normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    q = radius * u
    r = radius + (amp[None] * np.exp(-((q[:, None, :] - cs[None]) ** 2).sum(-1) / (wid[None] ** 2))).sum(1)
    return u * r[:, None]


def ternary(dims, seed=0):
    """Values drawn from {-1, 0, +1}: maximal ties and exact zeros."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = dims
    v = rng.integers(-1, 2, nx * ny * nz).astype(np.float32)
    return torch.from_numpy(v), tuple(dims), (0.05, 0.05, 0.05), (0.0, 0.0, 0.0)


def sphere_with_zero_shell(res=40, radius=0.3):
    """Sphere SDF with every grid point within 0.2 cell widths of the surface set to 0."""
    vals, dims, spacing, origin = sphere(res, radius)
    v = vals.clone()
    v[v.abs() < 0.2 * spacing[0]] = 0.0
    return v, dims, spacing, origin


# ---- triangle meshes for the mesh -> SDF conversion -------------------------------------

def icosphere(subdiv=4):
    """Unit icosphere: the icosahedron (vertices (0,+-1,+-p), (+-1,+-p,0), (+-p,0,+-1), p the
    golden ratio, faces = the 20 mutually adjacent vertex triples, wound outward), each
    triangle split into 4 at its edge midpoints ``subdiv`` times, vertices projected onto the
    sphere. Returns float64 vertices (10*4^s + 2, 3) and int64 faces (20*4^s, 3)."""
    p = (1.0 + 5 ** 0.5) / 2.0
    V = []
    for a in (-1.0, 1.0):
        for b in (-p, p):
            V += [(0.0, a, b), (a, b, 0.0), (b, 0.0, a)]
    V = np.array(V, np.float64)
    d = np.linalg.norm(V[:, None] - V[None], axis=-1)
    adj = np.isclose(d, 2.0)
    F = []
    for i in range(12):
        for j in range(i + 1, 12):
            for k in range(j + 1, 12):
                if adj[i, j] and adj[j, k] and adj[i, k]:
                    tri = [i, j, k]
                    if np.dot(np.cross(V[j] - V[i], V[k] - V[i]), V[i] + V[j] + V[k]) < 0:
                        tri = [i, k, j]
                    F.append(tri)
    V = V / np.linalg.norm(V, axis=1, keepdims=True)
    F = np.array(F, np.int64)
    for _ in range(subdiv):
        mid = {}
        verts = list(V)

        def midpoint(a, b):
            key = (a, b) if a < b else (b, a)
            if key not in mid:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                mid[key] = len(verts) - 1
            return mid[key]
        nf = []
        for a, b, c in F.tolist():
            ab, bc, ca = midpoint(a, b), midpoint(b, c), midpoint(c, a)
            nf += [[a, ab, ca], [b, bc, ab], [c, ca, bc], [ab, bc, ca]]
        V, F = np.array(verts), np.array(nf, np.int64)
    return V, F


def icosphere_scene(n_spheres=32, subdiv=4, seed=0, noise=0.002):
    """Union (concatenation) of ``n_spheres`` icospheres: radius U(0.05,0.2), centre
    U(-0.3,0.3)^3, every vertex displaced along its normal by N(0, noise). Returns float32
    vertices (n, 3) and int32 triangles (m, 3); 32 spheres of subdivision 4 give 81,984
    vertices and 163,840 triangles."""
    rng = np.random.default_rng(seed)
    U, T = icosphere(subdiv)
    centres = rng.uniform(-0.3, 0.3, (n_spheres, 3))
    radii = rng.uniform(0.05, 0.2, n_spheres)
    Vs, Fs = [], []
    for s in range(n_spheres):
        r = radii[s] + rng.normal(0.0, noise, len(U))
        Vs.append(centres[s] + r[:, None] * U)
        Fs.append(T + s * len(U))
    return np.concatenate(Vs).astype(np.float32), np.concatenate(Fs).astype(np.int32)


def mesh_grid(V, res):
    """Grid of res^3 points over the mesh bounding box grown by 8% of its diagonal, in float
    arithmetic like the CLI's OBJ import (dc_cli.cpp:160-187). Returns dims, spacing, origin."""
    V = np.asarray(V, np.float32)
    lo = V.min(axis=0).astype(np.float32)
    hi = V.max(axis=0).astype(np.float32)
    e = (hi - lo).astype(np.float32)
    diag = np.float32(np.sqrt(np.float32(np.float32(e[0] * e[0] + e[1] * e[1]) + e[2] * e[2])))
    pad = np.float32(diag * np.float32(0.08)) if diag > 0 else np.float32(0.1)
    lo = (lo - pad).astype(np.float32)
    hi = (hi + pad).astype(np.float32)
    sp = ((hi - lo) / np.float32(res - 1)).astype(np.float32)
    return (res, res, res), tuple(float(x) for x in sp), tuple(float(x) for x in lo)
