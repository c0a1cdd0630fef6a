"""Size-independent properties of the extraction on the full 1024^3 sharp-feature CSG grid,
where the oracle would take minutes: symmetries of the algorithm that hold for the reference
CPU backend's arithmetic and so for the engine's.

* Negating every value keeps every active cell and every vertex (the normal equations see each
  normal twice, so its sign cancels; only lerp_t's +1e-16, Cell.cpp:49-52, can move a sample by
  ~1e-16) and reverses every quad's winding: the orientation test is the sign of
  dot(quad normal, gradient sum), and the gradients negate exactly (contouring.cpp:624-641).
  A quad whose normal vanishes keeps its order in both (no orientation to reverse).
* Scaling every value by 4 keeps every sign, lerp parameter and normal direction, so the same
  cells, quads and windings, and the vertices up to lerp_t's +1e-16."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def csg1024():
    import torch
    from contouring_b200 import B200DualContouringBackend, synth
    vals, dims, sp, org = synth.csg(1024, seed=0, device="cuda")
    be = B200DualContouringBackend(0)
    V, F, _ = be.extract_tensor(vals, dims, sp, org)
    base = (V.cpu().numpy(), F.cpu().numpy(), be.active_cells())
    yield be, vals, dims, sp, org, base
    be.close()
    del vals
    torch.cuda.empty_cache()


def _close(V0, V1, sp):
    """Vertices equal up to a float rounding of each coordinate (an escalated cell's double
    lerp parameter carries the +1e-16 term, which can move its rounding by one ulp)."""
    d = np.abs(V0.astype(np.float64) - V1)
    return bool((d <= 2.5e-7 * np.abs(V0) + 1e-6 * min(sp)).all())


def _run(be, vals, dims, sp, org):
    V, F, _ = be.extract_tensor(vals, dims, sp, org)
    return V.cpu().numpy(), F.cpu().numpy(), be.active_cells()


def test_negated_grid_flips_every_quad(csg1024):
    be, vals, dims, sp, org, (V0, F0, C0) = csg1024
    vals.neg_()
    try:
        V1, F1, C1 = _run(be, vals, dims, sp, org)
    finally:
        vals.neg_()
    assert len(F0) > 6_000_000
    assert np.array_equal(C0, C1)
    assert _close(V0, V1, sp)
    flipped = F0[:, [0, 3, 2, 1]]
    same = (F1 == flipped).all(axis=1)
    if not same.all():
        # only quads without an orientation may keep their order: a vanishing quad normal
        rest = np.flatnonzero(~same)
        assert (F1[rest] == F0[rest]).all()
        P = V0.astype(np.float64)
        q = F0[rest]
        n = np.cross(P[q[:, 1]] - P[q[:, 0]], P[q[:, 3]] - P[q[:, 0]])
        n2 = np.cross(P[q[:, 2]] - P[q[:, 0]], P[q[:, 3]] - P[q[:, 0]])
        assert (np.minimum(np.einsum("ij,ij->i", n, n), np.einsum("ij,ij->i", n2, n2)) < 1e-20).all()


def test_power_of_two_scale_keeps_the_mesh(csg1024):
    import torch
    be, vals, dims, sp, org, (V0, F0, C0) = csg1024
    vals.mul_(torch.tensor(4.0, device=vals.device))
    try:
        V1, F1, C1 = _run(be, vals, dims, sp, org)
    finally:
        vals.mul_(torch.tensor(0.25, device=vals.device))
    assert np.array_equal(C0, C1)
    assert np.array_equal(F0, F1)
    assert _close(V0, V1, sp)


def test_negated_batch_flips_every_quad():
    """The same symmetry through the batched path (one pass of every kernel over 64 ragged
    grids of 32^3..192^3): per grid, identical vertices up to a float rounding and every quad
    reversed."""
    import torch
    from contouring_b200 import B200DualContouringBackend, synth
    grids = synth.csg_batch(64, seed=3, device="cuda")
    be = B200DualContouringBackend(0)
    try:
        a, _ = be.extract_batch(grids)
        a = [(V.cpu().numpy(), F.cpu().numpy()) for V, F in a]
        for v, _, _, _ in grids:
            v.neg_()
        b, _ = be.extract_batch(grids)
        b = [(V.cpu().numpy(), F.cpu().numpy()) for V, F in b]
    finally:
        be.close()
    nq = 0
    for (V0, F0), (V1, F1), (_, _, sp, _) in zip(a, b, grids):
        assert _close(V0, V1, sp)
        assert np.array_equal(F1, F0[:, [0, 3, 2, 1]])
        nq += len(F0)
    assert nq > 100_000
    torch.cuda.synchronize()
