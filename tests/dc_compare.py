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
