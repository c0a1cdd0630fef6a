"""Single-grid z-slab pipeline: a handle whose buffers come from an earlier extraction marks
the grid slab by slab (runs of the mark's z-chunks) on the caller's stream while a second stream
scans each marked slab's segments, writes its ranks and cell list and solves its cells' FP32
vertices; faces follow once every slab is done. A fresh handle's first call runs the one-pass
pipeline (mark, host count, buffers sized to it, the rest). Both must give the same mesh bit for
bit: the per-cell arithmetic is the same and the slabs only change when it runs. A grid with more
active cells than the earlier buffers hold is finished on the exact path; NaN values anywhere a
slab's stencils reach must still send every cell to the FP64 path before the slab is solved.
"""
import numpy as np
import pytest

from dc_compare import VERTEX_TOL

pytestmark = pytest.mark.gpu


def _fresh(grid, tri=False):
    """The one-pass pipeline: the first call on a new handle."""
    from contouring_b200 import B200DualContouringBackend, DenseSdfGrid
    be = B200DualContouringBackend(0)
    be.options.emit_triangles = tri
    try:
        mesh, st = be.extract(DenseSdfGrid.from_tuple(grid))
        return mesh.vertices.copy(), mesh.faces.copy(), be.active_cells(), st
    finally:
        be.close()


def _warm(grid, warm_with, tri=False):
    """The slab pipeline: the call after an extraction of `warm_with` on the same handle."""
    from contouring_b200 import B200DualContouringBackend, DenseSdfGrid
    be = B200DualContouringBackend(0)
    be.options.emit_triangles = tri
    try:
        be.extract(DenseSdfGrid.from_tuple(warm_with))
        mesh, st = be.extract(DenseSdfGrid.from_tuple(grid))
        first = (mesh.vertices.copy(), mesh.faces.copy(), be.active_cells(), st)
        mesh, st = be.extract(DenseSdfGrid.from_tuple(grid))      # and once more on its own buffers
        second = (mesh.vertices.copy(), mesh.faces.copy(), be.active_cells(), st)
        return first, second
    finally:
        be.close()


def _same(a, b, name):
    Va, Fa, Ca, sa = a
    Vb, Fb, Cb, sb = b
    assert np.array_equal(Ca, Cb), "%s: active cells differ" % name
    assert np.array_equal(Fa, Fb), "%s: faces differ (%d vs %d)" % (name, Fa.size, Fb.size)
    assert np.array_equal(Va, Vb, equal_nan=True), "%s: vertices differ" % name
    assert sa.vertex_count == sb.vertex_count and sa.face_count == sb.face_count


def _cases():
    from contouring_b200 import synth
    return {
        "csg96": lambda: synth.csg(96, seed=4),
        "csg160_seed3": lambda: synth.csg(160, seed=3),
        "sphere128_r035": lambda: synth.sphere(128, 0.35),
        "noise_ragged": lambda: synth.noise((33, 7, 141), seed=9),
        "noise_zeros": lambda: synth.noise((24, 19, 71), seed=3, zero_frac=0.5),
        "ternary": lambda: synth.ternary((21, 22, 93), seed=4),
        "thin_gap64": lambda: synth.thin_gap(64),
    }


@pytest.mark.parametrize("name", list(_cases().keys()))
def test_slab_pipeline_equals_one_pass(name):
    from contouring_b200 import synth
    grid = _cases()[name]()
    ref = _fresh(grid)
    # buffers from a larger grid: every cell fits, the slab path runs to the end
    first, second = _warm(grid, synth.csg(192, seed=1))
    _same(first, ref, name)
    _same(second, ref, name)


@pytest.mark.parametrize("tri", [False, True])
def test_slab_pipeline_overflow_finishes_on_the_exact_path(tri):
    """Buffers from a small sphere, then a CSG grid with far more active cells: the slabs past
    the capacity are cut short and the exact path runs the rest; the next call fits."""
    from contouring_b200 import synth
    grid = synth.csg(160, seed=2)
    ref = _fresh(grid, tri)
    first, second = _warm(grid, synth.sphere(24, 0.3), tri)
    _same(first, ref, "overflow")
    _same(second, ref, "refit")


def test_slab_pipeline_triangles():
    from contouring_b200 import synth
    grid = synth.csg(128, seed=5)
    ref = _fresh(grid, True)
    first, second = _warm(grid, synth.csg(160, seed=1), True)
    _same(first, ref, "triangles")
    _same(second, ref, "triangles")


@pytest.mark.parametrize("where", ["slab_boundary", "spread"])
def test_slab_pipeline_nan_values_match_oracle(where):
    """NaN values in a grid run as slabs: each slab's cells are solved only after every value
    their stencils read has been checked, so the NaN vertices and the quads equal the oracle's
    (the reference CPU backend propagates NaN through zero-weighted trilinear terms)."""
    import oracle as O
    from contouring_b200 import B200DualContouringBackend, DenseSdfGrid, synth
    vals, dims, sp, org = synth.csg(48, seed=0)
    v = vals.numpy().copy()
    nx, ny, nz = dims
    rng = np.random.default_rng(11)
    if where == "spread":
        v[rng.choice(v.size, 40, replace=False)] = np.nan
    else:
        # NaN points near the surface on the point planes just past z-chunk ends (chunks of 8
        # cell planes on a grid this small)
        for kp in (9, 17, 25, 33):
            plane = v[kp * nx * ny:(kp + 1) * nx * ny].reshape(ny, nx)
            js, is_ = np.nonzero(np.abs(plane) < 2 * sp[0])
            pick = rng.choice(len(js), min(6, len(js)), replace=False)
            plane[js[pick], is_[pick]] = np.nan
    be = B200DualContouringBackend(0)
    try:
        be.extract(DenseSdfGrid.from_tuple(synth.csg(64, seed=1)))
        mesh, st = be.extract(DenseSdfGrid(*dims, *sp, *org, values=v))
        cells = be.active_cells()
    finally:
        be.close()
    ref = O.dc_extract(v, dims, sp, org)
    V = mesh.vertices.reshape(-1, 3).astype(np.float64)
    F = mesh.faces.reshape(-1, 4)
    assert np.array_equal(cells, ref["cells"])
    nan_rows = np.isnan(V).any(1)
    assert nan_rows.any() and np.array_equal(nan_rows, np.isnan(ref["V"]).any(1))
    assert (np.abs(V[~nan_rows] - ref["V"][~nan_rows]) / np.asarray(sp)).max() <= VERTEX_TOL
    assert np.array_equal(F, ref["F"])
