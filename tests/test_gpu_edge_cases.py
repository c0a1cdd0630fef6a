"""Edge cases of the refinement, the adjoint and the tile autotuner: grids without a surface,
the smallest grids, ragged tiny grids in a batch."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def backend():
    from contouring_b200 import B200DualContouringBackend
    b = B200DualContouringBackend(0)
    yield b
    b.close()


def _ours(backend, vals, dims, sp, org, **kw):
    from contouring_b200 import ContouringMethod, ContouringOptions
    o = ContouringOptions()
    o.method = ContouringMethod.Ours
    for k, v in kw.items():
        setattr(o, k, v)
    old = backend.options
    backend.options = o
    try:
        return backend.extract_tensor(vals.cuda(), dims, sp, org)
    finally:
        backend.options = old


@pytest.mark.parametrize("value", [1.0, -1.0, 0.0])
def test_refinement_without_surface(backend, value):
    from contouring_b200 import synth
    vals, dims, sp, org = synth.constant(12, value)
    V, F, st = _ours(backend, vals, dims, sp, org, outer_iters=3)
    assert V.shape[0] == 0 and F.shape[0] == 0


def test_refinement_smallest_grid(backend):
    """A 2x2x2 grid: one cell, no interior grid edge, hence no quads and no face points."""
    import torch
    import oracle as O
    vals = torch.tensor([-1, 1, 1, 1, 1, 1, 1, 1], dtype=torch.float32)
    dims, sp, org = (2, 2, 2), (1.0, 1.0, 1.0), (0.0, 0.0, 0.0)
    V, F, st = _ours(backend, vals, dims, sp, org, outer_iters=2)
    r = O.ours(vals.numpy(), dims, sp, org, outer_iters=2)
    assert V.shape == (1, 3) and F.shape[0] == 0
    assert np.abs(V.cpu().numpy().astype(np.float64) - r["V"]).max() <= 1e-6


def test_adjoint_without_vertices(backend):
    import torch
    from contouring_b200 import synth
    vals, dims, sp, org = synth.constant(10, 1.0)
    d = vals.cuda()
    V, F, st = backend.extract_tensor(d, dims, sp, org)
    assert V.shape[0] == 0
    g = backend.backward_tensor(d, dims, sp, org, torch.zeros((0, 3), device="cuda"))
    assert g.shape == (d.numel(),) and int(torch.count_nonzero(g)) == 0


def test_autotune_tiny_and_empty_grids(backend):
    import torch
    from contouring_b200 import synth
    grids = [(synth.sphere(6)[0].cuda(),) + synth.sphere(6)[1:], (synth.constant(5, 1.0)[0].cuda(),) + synth.constant(5, 1.0)[1:],
             (synth.sphere(40)[0].cuda(),) + synth.sphere(40)[1:]]
    before, _ = backend.extract_batch(grids)
    before = [(V.clone(), F.clone()) for V, F in before]
    waves, narrow, ms = backend.autotune_mark(grids)
    after, _ = backend.extract_batch(grids)
    for (Va, Fa), (Vb, Fb) in zip(before, after):
        assert torch.equal(Va, Vb) and torch.equal(Fa, Fb)
    assert after[1][0].shape[0] == 0
