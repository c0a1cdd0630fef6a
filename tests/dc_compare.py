"""Shared helpers: run the B200 engine and the CPU oracle on one grid and compare.

Parity bar (the engine vs the FP64 restatement of the reference CPU backend):
  * active-cell set, vertex numbering and the quad list (order and winding): bit-exact;
  * vertex positions: |v_b200 - v_oracle| <= VERTEX_TOL cell widths on every axis.
"""
import numpy as np

VERTEX_TOL = 1e-4   # in cell widths, per axis


def run_engine(backend, grid_tuple):
    from contouring_b200 import DenseSdfGrid
    g = DenseSdfGrid.from_tuple(grid_tuple)
    mesh, stats = backend.extract(g)
    cells = backend.active_cells()
    V = mesh.vertices.reshape(-1, 3)
    F = mesh.faces.reshape(-1, 4)
    return V, F, cells, stats


def run_oracle(grid_tuple, threads=0):
    import oracle as O
    values, dims, spacing, origin = grid_tuple
    if hasattr(values, "detach"):
        values = values.detach().cpu().numpy()
    return O.dc_extract(values, dims, spacing, origin, threads=threads)


def compare(backend, grid_tuple, label=""):
    """Return a dict of parity metrics; raise AssertionError with details on a mismatch."""
    V, F, cells, stats = run_engine(backend, grid_tuple)
    ref = run_oracle(grid_tuple)
    _, dims, spacing, _ = grid_tuple
    assert stats.vertex_count == len(ref["V"]), "%s: vertex count %d vs oracle %d" % (
        label, stats.vertex_count, len(ref["V"]))
    assert np.array_equal(cells, ref["cells"]), "%s: active-cell set differs" % label
    h = np.array(spacing, np.float64)
    err = np.abs(V.astype(np.float64) - ref["V"]) / h if len(V) else np.zeros((0, 3))
    max_err = float(err.max()) if len(V) else 0.0
    rms_err = float(np.sqrt((err ** 2).mean())) if len(V) else 0.0
    assert stats.face_count == len(ref["F"]), "%s: face count %d vs oracle %d" % (
        label, stats.face_count, len(ref["F"]))
    if not np.array_equal(F, ref["F"]):
        bad = np.nonzero((F != ref["F"]).any(1))[0]
        raise AssertionError("%s: %d quads differ (first %s: b200 %s oracle %s)" % (
            label, len(bad), bad[0], F[bad[0]].tolist(), ref["F"][bad[0]].tolist()))
    assert max_err <= VERTEX_TOL, "%s: max vertex error %.3g cell widths (worst vertex %d)" % (
        label, max_err, int(err.max(1).argmax()))
    return {"label": label, "nv": int(stats.vertex_count), "nf": int(stats.face_count),
            "max_err": max_err, "rms_err": rms_err, "escalated": int(stats.escalated_fp64_cells),
            "winding_fp64": int(stats.winding_fp64_faces), "rank_hist": list(stats.rank_hist)}


def grid_axes(dims, spacing, origin):
    """Float grid-point coordinates o + float(i) * v per axis (widened to FP64)."""
    return [(np.float32(origin[a]) + np.arange(dims[a], dtype=np.float32) * np.float32(spacing[a])).astype(np.float64)
            for a in range(3)]


def window_parity(vals_zyx, dims, spacing, origin, V, F, cells, n_windows, win, margin, seed=7):
    """Check a whole-grid engine result (V, F, cells) against the oracle run on cubic windows
    of the grid (with the whole grid's float point positions). Cells and faces at least
    ``margin`` cells inside a window depend only on data inside it, so for those the engine
    must match exactly (active set, numbering, quads, winding) and within VERTEX_TOL (vertices).
    Returns (worst vertex error in cell widths, interior faces compared)."""
    import oracle as O
    nx, ny, nz = dims
    cx, cy = nx - 1, ny - 1
    ax = grid_axes(dims, spacing, origin)
    V = np.asarray(V, np.float64)
    fkey = F[:, 2].astype(np.int64) * (1 << 31) + F[:, 0]
    order = np.argsort(fkey)
    fkey_sorted = fkey[order]
    rng = np.random.default_rng(seed)
    centers = cells[rng.choice(len(cells), n_windows, replace=False)]
    worst, nfaces = 0.0, 0
    gi, gj, gk = cells % cx, (cells // cx) % cy, cells // (cx * cy)
    for c in centers:
        ci, cj, ck = c % cx, (c // cx) % cy, c // (cx * cy)
        i0 = int(np.clip(ci - win // 2, 0, nx - win))
        j0 = int(np.clip(cj - win // 2, 0, ny - win))
        k0 = int(np.clip(ck - win // 2, 0, nz - win))
        sub = np.ascontiguousarray(vals_zyx[k0:k0 + win, j0:j0 + win, i0:i0 + win])
        r = O.dc_extract_positions(sub, (win, win, win), ax[0][i0:i0 + win], ax[1][j0:j0 + win],
                                   ax[2][k0:k0 + win], threads=0)
        wc = win - 1
        la, lb, lc = r["cells"] % wc, (r["cells"] // wc) % wc, r["cells"] // (wc * wc)
        glob = (i0 + la) + cx * ((j0 + lb) + cy * (k0 + lc))
        interior = ((la >= margin) & (la < wc - margin) & (lb >= margin) & (lb < wc - margin) &
                    (lc >= margin) & (lc < wc - margin))
        in_block = ((gi >= i0 + margin) & (gi < i0 + wc - margin) & (gj >= j0 + margin) & (gj < j0 + wc - margin) &
                    (gk >= k0 + margin) & (gk < k0 + wc - margin))
        assert np.array_equal(np.sort(glob[interior]), cells[in_block]), "active set differs in window %s" % ((i0, j0, k0),)
        gidx = np.searchsorted(cells, glob)
        err = np.abs(V[gidx[interior]] - r["V"][interior]) / np.array(spacing)
        if err.size:
            worst = max(worst, float(err.max()))
        ok = interior[r["F"]].all(axis=1)
        Fw = gidx[r["F"][ok]]
        nfaces += len(Fw)
        key = Fw[:, 2].astype(np.int64) * (1 << 31) + Fw[:, 0]
        pos = np.searchsorted(fkey_sorted, key)
        assert np.all(pos < len(fkey_sorted)) and np.all(fkey_sorted[np.minimum(pos, len(fkey_sorted) - 1)] == key), \
            "a window face is missing from the engine output"
        assert np.array_equal(F[order[pos]], Fw), "a window face differs (winding) in window %s" % ((i0, j0, k0),)
    assert worst <= VERTEX_TOL, "max vertex error %.3g cell widths" % worst
    return worst, nfaces
