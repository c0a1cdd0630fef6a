"""Extraction on the buffers of an earlier call: once a handle holds per-cell buffers, the
kernels after the mark are launched at once with the active count read on the device, instead
of waiting on the host for the count. A fresh handle's first call sizes its buffers from the
count. Both must give the same mesh bit for bit; a grid with more active cells than the
earlier buffers hold (the kernels past the mark then do nothing) is run again with buffers
for its count, also for triangles and for batches."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(be, grid):
    from contouring_b200 import DenseSdfGrid
    mesh, st = be.extract(DenseSdfGrid.from_tuple(grid))
    return mesh.vertices.copy(), mesh.faces.copy(), be.active_cells(), st


def _fresh(grid, tri=False):
    from contouring_b200 import B200DualContouringBackend
    be = B200DualContouringBackend(0)
    be.options.emit_triangles = tri
    try:
        return _run(be, grid)
    finally:
        be.close()


def _after(grid, first, tri=False):
    """The call after an extraction of `first` on the same handle, then once more."""
    from contouring_b200 import B200DualContouringBackend
    be = B200DualContouringBackend(0)
    be.options.emit_triangles = tri
    try:
        _run(be, first)
        return _run(be, grid), _run(be, grid)
    finally:
        be.close()


def _same(a, b, name):
    Va, Fa, Ca, sa = a
    Vb, Fb, Cb, sb = b
    assert np.array_equal(Ca, Cb), "%s: active cells differ" % name
    assert np.array_equal(Fa, Fb), "%s: faces differ" % name
    assert np.array_equal(Va, Vb, equal_nan=True), "%s: vertices differ" % name
    assert sa.vertex_count == sb.vertex_count and sa.face_count == sb.face_count


@pytest.mark.parametrize("name", ["csg96", "sphere128_r035", "noise_ragged", "noise_zeros", "thin_gap64"])
def test_reused_buffers_equal_a_fresh_handle(name):
    from contouring_b200 import synth
    grid = {"csg96": lambda: synth.csg(96, seed=4), "sphere128_r035": lambda: synth.sphere(128, 0.35),
            "noise_ragged": lambda: synth.noise((33, 7, 141), seed=9),
            "noise_zeros": lambda: synth.noise((24, 19, 71), seed=3, zero_frac=0.5),
            "thin_gap64": lambda: synth.thin_gap(64)}[name]()
    ref = _fresh(grid)
    first, second = _after(grid, synth.csg(160, seed=1))
    _same(first, ref, name)
    _same(second, ref, name)


@pytest.mark.parametrize("tri", [False, True])
def test_more_cells_than_the_buffers_run_again(tri):
    from contouring_b200 import synth
    grid = synth.csg(160, seed=2)
    ref = _fresh(grid, tri)
    first, second = _after(grid, synth.sphere(24, 0.3), tri)
    _same(first, ref, "overflow")
    _same(second, ref, "refit")


def test_batch_after_a_smaller_batch():
    import torch
    from contouring_b200 import B200DualContouringBackend, synth
    small = synth.csg_batch(8, seed=1, device="cuda")
    big = synth.csg_batch(24, seed=2, device="cuda")
    fresh = B200DualContouringBackend(0)
    warm = B200DualContouringBackend(0)
    try:
        ref, _ = fresh.extract_batch(big)
        ref = [(V.clone(), F.clone()) for V, F in ref]
        warm.extract_batch(small)
        for _ in range(2):
            got, _ = warm.extract_batch(big)
            for (Va, Fa), (Vb, Fb) in zip(ref, got):
                assert torch.equal(Va, Vb) and torch.equal(Fa, Fb)
    finally:
        fresh.close()
        warm.close()
