"""Batched extraction (dcb_extract_batch_device): every grid's part of a batch equals its
own single-grid extraction bit for bit (same kernels, same arithmetic per cell), and so the
oracle; mixed sizes, the scalar and the float4 mark paths, empty grids and triangles."""
import numpy as np
import pytest

from dc_compare import VERTEX_TOL

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def backend():
    from contouring_b200 import B200DualContouringBackend
    b = B200DualContouringBackend(0)
    yield b
    b.close()


def _mixed():
    from contouring_b200 import synth
    cases = [synth.csg(64, seed=1), synth.noise((37, 21, 30), seed=5), synth.constant(16, 1.0),
             synth.sphere(48, 0.3), synth.noise((2, 2, 2), seed=9), synth.noise((17, 23, 9), seed=2, zero_frac=0.3),
             synth.csg(96, seed=4), synth.cli_plane(17), synth.ternary((21, 22, 23), seed=4), synth.thin_gap(32)]
    return [(v.cuda(), d, s, o) for v, d, s, o in cases]


def _single(backend, g):
    V, F, st = backend.extract_tensor(*g)
    return V.cpu().numpy(), F.cpu().numpy(), backend.active_cells()


@pytest.mark.parametrize("tri", [False, True])
def test_batch_parts_equal_single_extractions(backend, tri):
    grids = _mixed()
    backend.options.emit_triangles = tri
    try:
        meshes, st = backend.extract_batch(grids)
        cells = backend.active_cells()
        singles = [_single(backend, g) for g in grids]
    finally:
        backend.options.emit_triangles = False
    assert len(meshes) == len(grids)
    off = 0
    for (V, F), (V1, F1, c1) in zip(meshes, singles):
        assert np.array_equal(V.cpu().numpy(), V1)
        assert np.array_equal(F.cpu().numpy(), F1)
        assert np.array_equal(cells[off:off + len(V1)], c1)
        off += len(V1)
    assert st.vertex_count == off and st.face_count == sum(len(F1) for _, F1, _ in singles)


def test_batch_matches_oracle(backend):
    import oracle as O
    grids = _mixed()
    meshes, _ = backend.extract_batch(grids)
    for (V, F), (vals, dims, sp, org) in zip(meshes, grids):
        ref = O.dc_extract(vals.cpu().numpy(), dims, sp, org)
        assert np.array_equal(F.cpu().numpy(), ref["F"])
        if len(ref["V"]):
            assert (np.abs(V.cpu().numpy().astype(np.float64) - ref["V"]) / np.array(sp)).max() <= VERTEX_TOL


def test_benchmark_batch(backend):
    """The 256-shape batch of uneven resolutions {32..192}^3: every part equals its single
    extraction; the batch is deterministic."""
    import torch
    from contouring_b200 import synth
    grids = [(v, d, s, o) for v, d, s, o in synth.csg_batch(256, seed=0, device="cuda")]
    meshes, st = backend.extract_batch(grids)
    parts = [(V.cpu().numpy(), F.cpu().numpy()) for V, F in meshes]
    meshes2, _ = backend.extract_batch(grids)
    for (V, F), (V2, F2) in zip(parts, meshes2):
        assert np.array_equal(V, V2.cpu().numpy()) and np.array_equal(F, F2.cpu().numpy())
    rng = np.random.default_rng(0)
    for b in rng.choice(len(grids), 24, replace=False):
        V1, F1, _ = _single(backend, grids[b])
        assert np.array_equal(parts[b][0], V1) and np.array_equal(parts[b][1], F1)
    print("batch: %d grids, %d cells, %d vertices, %d faces, %.2f ms" % (
        len(grids), st.total_cells, st.vertex_count, st.face_count, st.total_ms))


def test_autotune_keeps_the_results(backend):
    """The mark tile autotuner picks one of its candidate tilings and the extraction's output
    does not change with it."""
    import torch
    from contouring_b200 import synth
    grids = synth.csg_batch(24, seed=5, device="cuda")
    before, _ = backend.extract_batch(grids)
    before = [(V.clone(), F.clone()) for V, F in before]
    waves, narrow, ms = backend.autotune_mark(grids)
    assert waves in (1, 2, 4, 8) and narrow in (0, 256, 512, 1024) and ms > 0
    after, _ = backend.extract_batch(grids)
    for (Va, Fa), (Vb, Fb) in zip(before, after):
        assert torch.equal(Va, Vb) and torch.equal(Fa, Fb)
    print("autotuned mark tiling: %d waves, 256-cell tiles up to %d cells wide, %.3f ms" % (waves, narrow, ms))


def test_cell_autotune_keeps_the_results():
    """The vertex/face autotuner picks a register cap and launch widths among its candidates;
    batches and single extractions afterwards give the same quads and vertices within the
    parity tolerance (the register caps are separately compiled kernels, whose multiply-adds
    may round differently in the last bit)."""
    import torch
    from contouring_b200 import B200DualContouringBackend, synth
    be = B200DualContouringBackend(0)
    try:
        grids = synth.csg_batch(24, seed=6, device="cuda")
        single = grids[0]
        before, _ = be.extract_batch(grids)
        before = [(V.clone(), F.clone()) for V, F in before]
        V1, F1, _ = be.extract_tensor(*single)
        V1, F1 = V1.clone(), F1.clone()
        m, q, f, ms = be.autotune_cells(grids)
        assert m in (4, 5, 6) and q in (8, 16, 32) and f in (8, 16, 32) and ms > 0
        after, _ = be.extract_batch(grids)
        for (Va, Fa), (Vb, Fb), (_, _, sp, _) in zip(before, after, grids):
            assert torch.equal(Fa, Fb)
            assert float((Va - Vb).abs().max()) <= VERTEX_TOL * min(sp)
        V2, F2, _ = be.extract_tensor(*single)
        assert torch.equal(F1, F2)
        assert float((V1 - V2).abs().max()) <= VERTEX_TOL * min(single[2])
        print("autotuned cell kernels: vertex cap %d blocks/SM, width %d, faces width %d; %.3f ms" % (m, q, f, ms))
    finally:
        be.close()


# ---- the batch captured in a CUDA graph (dcb_batch_graph_*) -----------------------------------

def _same(meshes_a, meshes_b):
    assert len(meshes_a) == len(meshes_b)
    for (Va, Fa), (Vb, Fb) in zip(meshes_a, meshes_b):
        assert np.array_equal(Va.cpu().numpy(), Vb.cpu().numpy())
        assert np.array_equal(Fa.cpu().numpy(), Fb.cpu().numpy())


def test_graph_replays_equal_eager_batches(backend):
    """The captured pipeline gives the eager batch's meshes bit for bit, replay after replay,
    and follows new values written into the same grid buffers."""
    import torch
    grids = _mixed()
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        eager, st = backend.extract_batch(grids)
        eager = [(V.clone(), F.clone()) for V, F in eager]
        backend.batch_graph_create(grids, headroom=0.5)
        for _ in range(3):
            backend.batch_graph_launch()
        got, gst = backend.batch_graph_meshes()
        _same(got, eager)
        assert gst.vertex_count == st.vertex_count and gst.face_count == st.face_count
        # new values in the same buffers (fewer active cells: a smaller sphere)
        from contouring_b200 import synth
        v, d, sp, o = synth.sphere(48, 0.2)
        grids[3][0].copy_(v.cuda())
        backend.batch_graph_launch()
        got2, _ = backend.batch_graph_meshes()
        ref, _ = backend.extract_batch(grids)            # an eager call: invalidates the graph
        _same(got2, ref)
        from contouring_b200 import DcbError
        with pytest.raises(DcbError):
            backend.batch_graph_launch()
        backend.batch_graph_destroy()
    torch.cuda.synchronize()


def test_graph_capacity_overflow_is_reported(backend):
    import torch
    from contouring_b200 import DcbError, synth
    grids = [(synth.sphere(40, 0.2)[0].cuda(), (40, 40, 40), synth.sphere(40, 0.2)[2], synth.sphere(40, 0.2)[3])]
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        backend.batch_graph_create(grids, headroom=0.0)          # capacity = active cells + 1024
        noise = synth.noise((40, 40, 40), seed=3)[0]            # far more active cells
        grids[0][0].copy_(noise.cuda())
        backend.batch_graph_launch()
        with pytest.raises(DcbError):
            backend.batch_graph_finish()
        backend.batch_graph_destroy()
    torch.cuda.synchronize()
