"""The FP64 reference adjoint (oracle/dc_adjoint_oracle.cpp) pinned on the CPU: its per-cell
vertex run with double is the FP64 oracle's vertex bit for bit, and its dual-number
Jacobian equals FP64 central finite differences of that vertex."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def grid48():
    import oracle as O
    from contouring_b200 import synth
    from dc_compare import grid_axes
    vals, dims, sp, org = synth.rbf_sphere(48)
    vals = vals.numpy()
    r = O.dc_extract(vals, dims, sp, org)
    return vals, dims, sp, org, grid_axes(dims, sp, org), r


def test_cell_vertices_equal_the_oracle(grid48):
    import oracle as O
    vals, dims, sp, org, ax, r = grid48
    V = O.cell_vertices(vals, dims, ax, r["cells"])
    assert np.array_equal(V, r["V"])
    Vj, _ = O.cell_jacobians(vals, dims, ax, r["cells"])
    assert np.abs(Vj - V).max() <= 1e-15


def test_jacobian_matches_central_differences(grid48):
    import oracle as O
    vals, dims, sp, org, ax, r = grid48
    cells = r["cells"]
    _, J = O.cell_jacobians(vals, dims, ax, cells)
    nx, ny, nz = dims
    cx, cy = nx - 1, ny - 1
    vd = vals.astype(np.float64)
    rng = np.random.default_rng(0)
    h = 1e-6
    worst, scale, n = 0.0, 0.0, 0
    while n < 300:
        q = int(rng.integers(len(cells)))
        c = cells[q]
        i, j, k = c % cx, (c // cx) % cy, c // (cx * cy)
        s = int(rng.integers(64))
        gi, gj, gk = i - 1 + s % 4, j - 1 + (s // 4) % 4, k - 1 + s // 16
        if not (0 <= gi < nx and 0 <= gj < ny and 0 <= gk < nz):
            continue
        p = gi + nx * (gj + ny * gk)
        if abs(vd[p]) < 10 * h:
            continue
        base = vd[p]
        vd[p] = base + h
        vp = O.cell_vertices(vd, dims, ax, [c])[0]
        vd[p] = base - h
        vm = O.cell_vertices(vd, dims, ax, [c])[0]
        vd[p] = base
        fd = (vp - vm) / (2 * h)
        worst = max(worst, float(np.abs(fd - J[q, :, s]).max()))
        scale = max(scale, float(np.abs(fd).max()))
        n += 1
    assert worst <= 1e-5 * scale, (worst, scale)


def test_vjp_is_the_sum_over_cells(grid48):
    import oracle as O
    vals, dims, sp, org, ax, r = grid48
    cells = r["cells"]
    g = np.random.default_rng(1).normal(size=(len(cells), 3))
    total = O.vertex_vjp(vals, dims, ax, cells, g)
    half = (O.vertex_vjp(vals, dims, ax, cells[::2], g[::2]) + O.vertex_vjp(vals, dims, ax, cells[1::2], g[1::2]))
    assert np.allclose(total, half, rtol=1e-12, atol=1e-12)
    far = np.abs(vals) > 4 * sp[0] * np.sqrt(3)
    assert np.all(total[far] == 0.0)
