"""The outer/inner vertex refinement (ContouringMethod.Ours) on the GPU against its FP64 CPU
restatement (oracle/ours_oracle.cpp): same quads, vertices within VERTEX_TOL cell widths, on
small grids (the oracle finds closest points by brute force) with a few outer iterations; the
full default run (100 outer x 100 inner iterations) at 64^3 for its invariants."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

VERTEX_TOL = 1e-5          # cell widths; the engine's output is float, the oracle's FP64


@pytest.fixture(scope="module")
def backend():
    from contouring_b200 import B200DualContouringBackend
    b = B200DualContouringBackend(0)
    yield b
    b.close()


def _grid(name):
    from contouring_b200 import synth
    if name == "sphere32":
        return synth.sphere(32, radius=0.35)
    if name == "rbf32":
        return synth.rbf_sphere(32)
    if name == "csg32":
        return synth.csg(32, seed=3)
    if name == "ragged":
        v, dims, sp, org = synth.rbf_sphere(36, seed=2)
        g = v.numpy().reshape(36, 36, 36)[1:33, 3:36, 0:29]
        import torch
        return torch.from_numpy(np.ascontiguousarray(g).reshape(-1)), (29, 33, 32), sp, org
    raise KeyError(name)


def _run(backend, vals, dims, sp, org, **kw):
    from contouring_b200 import ContouringMethod, ContouringOptions
    o = ContouringOptions()
    o.method = ContouringMethod.Ours
    for k, v in kw.items():
        setattr(o, k, v)
    old = backend.options
    backend.options = o
    try:
        V, F, st = backend.extract_tensor(vals.cuda(), dims, sp, org)
    finally:
        backend.options = old
    return V.cpu().numpy(), F.cpu().numpy(), st


def _compare(V, F, r, sp, label):
    assert np.array_equal(F, r["F"]), "%s: quads differ" % label
    err = np.abs(V.astype(np.float64) - r["V"]) / np.array(sp)
    frac = np.mean(err.max(1) <= VERTEX_TOL)
    print("%s: vertices %d, quads %d, max err %.3g cell widths, within tol %.5f" % (
        label, len(V), len(F), err.max(), frac))
    assert err.max() <= VERTEX_TOL


@pytest.mark.parametrize("name,outer", [("sphere32", 3), ("rbf32", 3), ("csg32", 2), ("ragged", 2)])
def test_matches_oracle(backend, name, outer):
    import oracle as O
    vals, dims, sp, org = _grid(name)
    V, F, st = _run(backend, vals, dims, sp, org, outer_iters=outer)
    r = O.ours(vals.numpy(), dims, sp, org, outer_iters=outer)
    _compare(V, F, r, sp, name)


def test_outer_zero_gives_centroids(backend):
    import oracle as O
    vals, dims, sp, org = _grid("sphere32")
    V, F, st = _run(backend, vals, dims, sp, org, outer_iters=0)
    _compare(V, F, O.ours(vals.numpy(), dims, sp, org, outer_iters=0), sp, "outer0")


def test_random_fill_matches(backend):
    """A batch larger than the near-surface points: the rest is filled with seeded random
    grid points, the same ones in the engine and the oracle."""
    import oracle as O
    vals, dims, sp, org = _grid("sphere32")
    nband = int(np.sum(np.abs(vals.numpy().astype(np.float64)) < 3 * np.sqrt(3) * sp[0]))
    kw = dict(outer_iters=2, batch_size=nband + 3000, seed=1234)
    V, F, st = _run(backend, vals, dims, sp, org, **kw)
    _compare(V, F, O.ours(vals.numpy(), dims, sp, org, **kw), sp, "fill")


def test_options_without_hermite_update(backend):
    import oracle as O
    vals, dims, sp, org = _grid("rbf32")
    kw = dict(outer_iters=3, inner_iters=20, hermite_update=False, mu=0.05, dc_weight=0.05, svd_threshold=0.05)
    V, F, st = _run(backend, vals, dims, sp, org, **kw)
    _compare(V, F, O.ours(vals.numpy(), dims, sp, org, **kw), sp, "no-hermite-update")


def test_default_run_64(backend):
    """100 outer x 100 inner iterations at 64^3: finite vertices near the surface, the sphere's
    radial error no worse than the dual-contouring start, the same quad topology."""
    import time
    import torch
    from contouring_b200 import synth
    vals, dims, sp, org = synth.sphere(64, radius=0.35)
    Vd, Fd, _ = backend.extract_tensor(vals.cuda(), dims, sp, org)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    V, F, st = _run(backend, vals, dims, sp, org)
    ms = (time.perf_counter() - t0) * 1e3
    Vd = Vd.cpu().numpy()
    assert np.isfinite(V).all() and len(V) == len(Vd)
    assert np.array_equal(np.sort(np.sort(F, 1), 0), np.sort(np.sort(Fd.cpu().numpy(), 1), 0))
    e_dc = np.abs(np.linalg.norm(Vd, axis=1) - 0.35)
    e_ours = np.abs(np.linalg.norm(V, axis=1) - 0.35)
    print("64^3, 100x100 iterations: %.1f ms; radial error DC mean %.3g max %.3g, refined mean %.3g max %.3g" % (
        ms, e_dc.mean(), e_dc.max(), e_ours.mean(), e_ours.max()))
    assert e_ours.mean() <= e_dc.mean() * 1.05
    assert e_ours.max() <= 2 * sp[0]


def test_triangles(backend):
    import oracle as O
    vals, dims, sp, org = _grid("sphere32")
    V, F, st = _run(backend, vals, dims, sp, org, outer_iters=2, emit_triangles=True)
    r = O.ours(vals.numpy(), dims, sp, org, outer_iters=2)
    assert F.shape == (2 * len(r["F"]), 3)
    assert np.array_equal(F, O.triangulate(r["V"], r["F"]))
